// cft_1d.h (drop-in) -- the 1D field class of ATUS-2
// (source/libs/lib_myutils/cft_1d.h) on the GPU: see cft_base.h.  Get_x and
// Get_k follow cft_1d.cpp:85-110: x_i = (i - N/2) dx, k from the wrapped index unless
// SetFix(true).
#ifndef ATUS_DROPIN_CFT_1D_H
#define ATUS_DROPIN_CFT_1D_H

#include "cft_base.h"

namespace Fourier {

class cft_1d : public cft_base<1> {
 public:
  explicit cft_1d(const generic_header &header, bool inplace = true, bool fix = false)
      : cft_base<1>(header, inplace, fix) {}

  CPoint<1> Get_x(const int64_t l) override {
    CPoint<1> r;
    const int64_t i = l;
    r[0] = double(i - m_shift_x) * m_dx;
    return r;
  }
  CPoint<1> Get_k(const int64_t l) override {
    CPoint<1> r;
    const int64_t i = l;
    r[0] = cft_k(i, m_dim_x, m_shift_x, m_dkx, m_bfix);
    return r;
  }
};

}  // namespace Fourier

#endif
