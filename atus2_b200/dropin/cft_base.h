// cft_base.h (drop-in) -- the field type T of ATUS-2's solver templates
// (source/libs/lib_myutils/cft_base.h:38-263), backed by the GPU.
//
// A field is one component of a GPU context (atus_ctx, include/atus_gpu.h)
// plus a host mirror with the reference's layout (interleaved complex128,
// x slowest), the array Getp2In() returns.  Which copy is current is tracked
// per field:
//   * Getp2In() / Getp2Out() bring the mirror up to date (one download when
//     the device copy is newer) and then count the device copy as stale,
//     because the caller may write through the pointer;
//   * every GPU operation on the context first uploads the fields whose
//     device copy is stale (push()), and afterwards marks the mirrors stale
//     (device_changed());
//   * host_view() reads the mirror without making the device copy stale (file
//     output).
// Step functions call Getp2In() from every thread of an OpenMP parallel
// region (bragg.cpp:196-197 does), so bringing the mirror up to date is done
// once, under a lock: a second thread must not download over the first
// thread's updates.
// ft(isign) is cft_Nd::ft on the GPU: the unnormalised transform over all
// axes with FFTW's sign convention, then the reference's scale, in place.  A
// field constructed by a program (not by a solver) gets a one-component GPU
// context of its own on its first ft().  Only complex, in-place fields
// (the solvers' use) are supported; SetFix(true) (centred ordering) is
// accepted for Get_k but ft() refuses it.
#ifndef ATUS_DROPIN_CFT_BASE_H
#define ATUS_DROPIN_CFT_BASE_H

#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <mutex>
#include <string>

#include "CPoint.h"
#include "atus_gpu.h"
#include "fftw3.h"
#include "my_structs.h"

namespace Fourier {

enum TYPE { REAL, COMPLEX };

template <int dim>
class cft_base {
 public:
  cft_base(const generic_header &header, bool inplace = true, bool fix = false, TYPE t = COMPLEX)
      : m_bInplace(inplace), m_bfix(fix), m_type(t) {
    if (header.nDims != dim) {
      std::cerr << "Critical error: header.nDims does not match template parameter dim" << std::endl;
      throw std::string("header.nDims does not match template parameter dim");
    }
    if (!inplace || t != COMPLEX) throw std::string("GPU fields are complex and transformed in place");
    m_header = header;
    m_dim_x = (int)header.nDimX;
    m_dim_y = dim >= 2 ? (int)header.nDimY : 1;
    m_dim_z = dim >= 3 ? (int)header.nDimZ : 1;
    m_shift_x = m_dim_x / 2;
    m_shift_y = m_dim_y / 2;
    m_shift_z = m_dim_z / 2;
    m_dim = (int64_t)m_dim_x * m_dim_y * m_dim_z;
    m_dim_fs = m_dim;
    m_red_dim = m_dim;
    m_dx = header.dx;
    m_dy = header.dy;
    m_dz = header.dz;
    m_dkx = header.dkx;
    m_dky = header.dky;
    m_dkz = header.dkz;
    m_in = fftw_alloc_complex(m_dim);
    if (!m_in) throw std::string("host mirror allocation failed");
    std::memset(m_in, 0, sizeof(fftw_complex) * m_dim);
    m_out = m_in;
    m_in_real = nullptr;
  }
  cft_base(const cft_base &) = delete;
  cft_base &operator=(const cft_base &) = delete;
  virtual ~cft_base() {
    if (m_own_ctx) atus_destroy(m_own_ctx);
    fftw_free(m_in);
  }

  void SetFix(bool b) { m_bfix = b; }

  virtual void ft(int isign) {
    if (m_bfix) throw std::string("ft: centred (fixed) ordering is not supported on the GPU");
    if (!m_ctx) own_context();
    push();
    check(atus_ft(m_ctx, m_comp, isign), "ft");
    m_isign = isign;
    device_changed();
  }
  virtual CPoint<dim> Get_k(const int64_t l) = 0;
  virtual CPoint<dim> Get_x(const int64_t l) = 0;

  double *Getp2InReal() { return m_in_real; }
  fftw_complex *Getp2In() {
    std::lock_guard<std::mutex> lock(m_sync);
    if (m_host_stale && m_ctx) {
      check(atus_download_psi(m_ctx, m_comp, &m_in[0][0]), "download");
      m_host_stale = false;
    }
    m_dev_stale = true;
    return m_in;
  }
  fftw_complex *Getp2Out() { return Getp2In(); }

  int Get_Dim_X() { return m_dim_x; }
  int Get_Dim_Y() { return m_dim_y; }
  int Get_Dim_Z() { return m_dim_z; }
  int64_t Get_red_Dim() { return m_red_dim; }
  int64_t Get_Dim_RS() { return m_dim; }
  int64_t Get_Dim_FS() { return m_dim_fs; }

  // the field and its header as a .bin file (cft_base::save, real space only)
  void save(const std::string &filename, bool rs = true) {
    if (!rs) throw std::string("save: Fourier-space output is not supported");
    generic_header h = m_header;
    h.nDatatyp = sizeof(fftw_complex);
    h.bComplex = true;
    h.fs = 0;
    std::ofstream ofs(filename, std::ofstream::binary);
    ofs.write(reinterpret_cast<const char *>(&h), sizeof(generic_header));
    ofs.write(reinterpret_cast<const char *>(host_view()), sizeof(fftw_complex) * m_dim);
  }

  // ---- GPU binding (used by the solver templates)
  // Makes this field component `comp` of `ctx`; the mirror's contents are
  // uploaded before the next GPU operation.
  void atus_bind(atus_ctx *ctx, int comp) {
    m_ctx = ctx;
    m_comp = comp;
    m_dev_stale = true;
    m_host_stale = false;
  }
  atus_ctx *atus_context() const { return m_ctx; }
  // upload the mirror if the program may have changed it
  void push() {
    std::lock_guard<std::mutex> lock(m_sync);
    if (m_dev_stale && m_ctx) {
      check(atus_upload_psi(m_ctx, m_comp, &m_in[0][0]), "upload");
      m_dev_stale = false;
    }
  }
  // the device copy changed: the mirror is stale
  void device_changed() { m_host_stale = true; }
  // the mirror, current, read-only use (the device copy stays valid)
  const fftw_complex *host_view() {
    pull();
    return m_in;
  }
  // the mirror was overwritten wholesale (a file read): upload before use
  void host_changed() {
    m_host_stale = false;
    m_dev_stale = true;
  }

 protected:
  void pull() {
    std::lock_guard<std::mutex> lock(m_sync);
    if (m_host_stale && m_ctx) {
      check(atus_download_psi(m_ctx, m_comp, &m_in[0][0]), "download");
      m_host_stale = false;
    }
  }
  void check(int r, const char *what) {
    if (r != ATUS_OK)
      throw std::string(std::string("GPU error in ") + what + ": " + (m_ctx ? atus_last_error(m_ctx) : "no context") +
                        " (code " + std::to_string(r) + ")");
  }
  void own_context() {
    atus_grid g{};
    g.dim = dim;
    g.n[0] = m_dim_x;
    g.n[1] = m_dim_y;
    g.n[2] = m_dim_z;
    g.d[0] = m_dx;
    g.d[1] = m_dy;
    g.d[2] = m_dz;
    g.dk[0] = m_dkx;
    g.dk[1] = m_dky;
    g.dk[2] = m_dkz;
    g.t = m_header.t;
    atus_ctx *c = nullptr;
    const int r = atus_create(&g, 1, ATUS_PREC_FP64, &c);
    if (r != ATUS_OK) throw std::string("atus_create failed (code " + std::to_string(r) + ")");
    m_own_ctx = c;
    atus_bind(c, 0);
  }

  int m_dim_x, m_dim_y, m_dim_z;
  int m_shift_x, m_shift_y, m_shift_z;
  int64_t m_red_dim, m_dim, m_dim_fs;
  int m_isign = 0;
  bool m_bInplace, m_bfix;
  TYPE m_type;
  double m_dx, m_dy, m_dz, m_dkx, m_dky, m_dkz;
  double *m_in_real;
  fftw_complex *m_in;
  fftw_complex *m_out;
  generic_header m_header;

 private:
  atus_ctx *m_ctx = nullptr;
  atus_ctx *m_own_ctx = nullptr;
  int m_comp = 0;
  std::mutex m_sync;
  bool m_dev_stale = true, m_host_stale = false;
};

// k of index i on an axis of n points: wrapped (k = dk ((i + n/2) mod n - n/2),
// SetFix(false), the solvers' setting) or centred (dk (i - n/2))
inline double cft_k(int64_t i, int n, int shift, double dk, bool fix) {
  if (!fix) i = (i + shift) % n;
  return dk * double(i - shift);
}

}  // namespace Fourier

#endif
