// cft_3d.h (drop-in) -- the 3D field class of ATUS-2
// (source/libs/lib_myutils/cft_3d.h) on the GPU: see cft_base.h.  Get_x and
// Get_k follow cft_3d.cpp:120-166: x_i = (i - N/2) dx, k from the wrapped index unless
// SetFix(true).
#ifndef ATUS_DROPIN_CFT_3D_H
#define ATUS_DROPIN_CFT_3D_H

#include "cft_base.h"

namespace Fourier {

class cft_3d : public cft_base<3> {
 public:
  explicit cft_3d(const generic_header &header, bool inplace = true, bool fix = false)
      : cft_base<3>(header, inplace, fix) {}

  CPoint<3> Get_x(const int64_t l) override {
    CPoint<3> r;
    const int64_t i = l / m_dim_y / m_dim_z;
    const int64_t j = (l - i * m_dim_y * m_dim_z) / m_dim_z;
    const int64_t k = l - i * m_dim_y * m_dim_z - j * m_dim_z;
    r[0] = double(i - m_shift_x) * m_dx;
    r[1] = double(j - m_shift_y) * m_dy;
    r[2] = double(k - m_shift_z) * m_dz;
    return r;
  }
  CPoint<3> Get_k(const int64_t l) override {
    CPoint<3> r;
    const int64_t i = l / m_dim_y / m_dim_z;
    const int64_t j = (l - i * m_dim_y * m_dim_z) / m_dim_z;
    const int64_t k = l - i * m_dim_y * m_dim_z - j * m_dim_z;
    r[0] = cft_k(i, m_dim_x, m_shift_x, m_dkx, m_bfix);
    r[1] = cft_k(j, m_dim_y, m_shift_y, m_dky, m_bfix);
    r[2] = cft_k(k, m_dim_z, m_shift_z, m_dkz, m_bfix);
    return r;
  }
};

}  // namespace Fourier

#endif
