// CRT_shared.h (drop-in) -- grid bookkeeping shared by the solver templates,
// with the members and accessors of ATUS-2's CRT_shared (include/
// CRT_shared.h:39-188): the header of the input file, point counts, index
// shifts, volume elements, the StepFunction type and a log file.
#ifndef ATUS_DROPIN_CRT_SHARED_H
#define ATUS_DROPIN_CRT_SHARED_H

#include <array>
#include <cassert>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <string>

#include "CPoint.h"
#include "atus_gpu.h"
#include "ParameterHandler.h"
#include "fftw3.h"
#include "my_structs.h"

/// A step of a sequence: called with the solver object and the sequence item.
typedef void (*StepFunction)(void *, sequence_item &);

class CRT_shared {
 public:
  CRT_shared()
      : m_no_of_pts(0), m_no_of_pts_red(0), m_shift_x(0), m_shift_y(0), m_shift_z(0), m_ar(0), m_ar_k(0) {
    m_header = {};
    m_log.open("log.txt");
    m_log << std::scientific;
    m_log << std::setprecision(10);
  }
  virtual ~CRT_shared() {}

  double &Get_t() { return m_header.t; }
  const double &Get_dt() const { return m_header.dt; }
  const double &Get_dx() const { return m_header.dx; }
  const double &Get_dy() const { return m_header.dy; }
  const double &Get_dz() const { return m_header.dz; }
  const double &Get_dkx() const { return m_header.dkx; }
  const double &Get_dky() const { return m_header.dky; }
  const double &Get_dkz() const { return m_header.dkz; }
  long long &Get_dimX() { return m_header.nDimX; }
  long long &Get_dimY() { return m_header.nDimY; }
  long long &Get_dimZ() { return m_header.nDimZ; }
  const int &Get_No_Points() const { return m_no_of_pts; }

  /// New time step: the kinetic phases are rebuilt (Init()).
  void Set_dt(const double dt) {
    m_header.dt = dt;
    Init();
  }
  std::ofstream m_log;

 protected:
  // CRT_shared::Read_header (include/CRT_shared.h:131-172)
  void Read_header(const std::string &filename, const int dim) {
    std::ifstream f(filename, std::ifstream::binary);
    if (!f.is_open()) throw std::string("Could not open file " + filename + ".\n");
    f.read(reinterpret_cast<char *>(&m_header), sizeof(generic_header));
    f.close();
    set_geometry(dim);
  }
  // point counts, shifts and volume elements of m_header's grid
  void set_geometry(const int dim) {
    switch (dim) {
      case 1:
        m_ar = m_header.dx;
        m_ar_k = m_header.dkx;
        m_no_of_pts = (int)m_header.nDimX;
        m_shift_x = (int)(m_header.nDimX / 2);
        m_no_of_pts_red = m_shift_x + 1;
        m_header.nDimY = 1;
        m_header.nDimZ = 1;
        break;
      case 2:
        m_ar = m_header.dx * m_header.dy;
        m_ar_k = m_header.dkx * m_header.dky;
        m_no_of_pts = (int)(m_header.nDimX * m_header.nDimY);
        m_shift_x = (int)(m_header.nDimX / 2);
        m_shift_y = (int)(m_header.nDimY / 2);
        m_no_of_pts_red = (int)(m_header.nDimX * (m_shift_y + 1));
        m_header.nDimZ = 1;
        break;
      case 3:
        m_ar = m_header.dx * m_header.dy * m_header.dz;
        m_ar_k = m_header.dkx * m_header.dky * m_header.dkz;
        m_no_of_pts = (int)(m_header.nDimX * m_header.nDimY * m_header.nDimZ);
        m_shift_x = (int)(m_header.nDimX / 2);
        m_shift_y = (int)(m_header.nDimY / 2);
        m_shift_z = (int)(m_header.nDimZ / 2);
        m_no_of_pts_red = (int)(m_header.nDimX * m_header.nDimY * (m_shift_z + 1));
        break;
    }
  }
  // the grid of m_header in the C ABI's form
  atus_grid abi_grid(const int dim) const {
    atus_grid g{};
    g.dim = dim;
    g.n[0] = m_header.nDimX;
    g.n[1] = dim >= 2 ? m_header.nDimY : 1;
    g.n[2] = dim >= 3 ? m_header.nDimZ : 1;
    g.d[0] = m_header.dx;
    g.d[1] = m_header.dy;
    g.d[2] = m_header.dz;
    g.dk[0] = m_header.dkx;
    g.dk[1] = m_header.dky;
    g.dk[2] = m_header.dkz;
    g.t = m_header.t;
    return g;
  }

  generic_header m_header;
  int m_no_of_pts;
  int m_no_of_pts_red;
  int m_shift_x;
  int m_shift_y;
  int m_shift_z;
  double m_ar;
  double m_ar_k;
  virtual void Init() = 0;
};

// Throws the reference's error type (std::string) for a failed ABI call.
inline void atus_check(atus_ctx *ctx, int r, const char *what) {
  if (r != ATUS_OK)
    throw std::string(std::string("GPU error in ") + what + ": " + (ctx ? atus_last_error(ctx) : "no context") +
                      " (code " + std::to_string(r) + ")");
}

// Precision of the solver contexts: ATUS_PRECISION=mixed selects complex64
// fields with FP64 phase arguments (the fast form), anything else FP64 (the
// drop-in form, results as the reference's).
inline int atus_precision_from_env() {
  const char *p = std::getenv("ATUS_PRECISION");
  return (p && std::string(p) == "mixed") ? ATUS_PREC_MIXED : ATUS_PREC_FP64;
}

#endif
