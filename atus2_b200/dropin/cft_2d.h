// cft_2d.h (drop-in) -- the 2D field class of ATUS-2
// (source/libs/lib_myutils/cft_2d.h) on the GPU: see cft_base.h.  Get_x and
// Get_k follow cft_2d.cpp:81-120: x_i = (i - N/2) dx, k from the wrapped index unless
// SetFix(true).
#ifndef ATUS_DROPIN_CFT_2D_H
#define ATUS_DROPIN_CFT_2D_H

#include "cft_base.h"

namespace Fourier {

class cft_2d : public cft_base<2> {
 public:
  explicit cft_2d(const generic_header &header, bool inplace = true, bool fix = false)
      : cft_base<2>(header, inplace, fix) {}

  CPoint<2> Get_x(const int64_t l) override {
    CPoint<2> r;
    const int64_t i = l / m_dim_y, j = l % m_dim_y;
    r[0] = double(i - m_shift_x) * m_dx;
    r[1] = double(j - m_shift_y) * m_dy;
    return r;
  }
  CPoint<2> Get_k(const int64_t l) override {
    CPoint<2> r;
    const int64_t i = l / m_dim_y, j = l % m_dim_y;
    r[0] = cft_k(i, m_dim_x, m_shift_x, m_dkx, m_bfix);
    r[1] = cft_k(j, m_dim_y, m_shift_y, m_dky, m_bfix);
    return r;
  }
};

}  // namespace Fourier

#endif
