// my_structs.h (drop-in) -- the .bin header and the small shared types of
// ATUS-2's include/my_structs.h: generic_header (1380 bytes, 4-byte packing,
// include/my_structs.h:40-72), the grid-dimension macros, the TEF function
// type and zernike_polynomial (my_structs.h:30-38), under the same names so
// that programs written for ATUS-2 compile unchanged.
#ifndef ATUS_DROPIN_MY_STRUCTS_H
#define ATUS_DROPIN_MY_STRUCTS_H

#include "../host/my_structs.h"

#define DIM1D 1
#define DIM2D 2
#define DIM3D 3

typedef double (*TEF)(const double, const double);

struct zernike_polynomial {
  int n;
  int m;
  double alpha;
};

#endif
