// my_structs.h -- the .bin file header.
//
// 1380 bytes, 4-byte packing, the field order of ATUS-2's generic_header
// (include/my_structs.h:40-72): a .bin file is this header followed by the
// grid values (complex128 interleaved, x slowest).
#pragma once

#pragma pack(push, 4)
struct generic_header {
  long long nself;
  long long nDatatyp;
  long long nself_and_data;
  long long nDims;
  long long nDimX;
  long long nDimY;
  long long nDimZ;
  int bAtom;
  int bComplex;
  double t;
  double xMin, xMax, yMin, yMax, zMin, zMax;
  double dx, dy, dz;
  double dkx, dky, dkz;
  double dt;
  int ks;
  int fs;
  int nFuture[99];
  double dFuture[100];
};
#pragma pack(pop)

static_assert(sizeof(generic_header) == 1380, "generic_header must be 1380 bytes");
