// CRT_Base_2.h (drop-in) -- two species of no_int_states/2 internal states
// each, with the interface of ATUS-2's template <class T, int dim, int
// no_int_states> class CRT_Base_2 (include/CRT_Base_2.h:40-105): as
// CRT_Base, plus Alpha_2 for the components [no_int_states/2, no_int_states)
// (their kinetic phases use m_alpha2, include/CRT_Base_2.h:194-221).  Built
// on the drop-in CRT_Base, so the GPU binding, the fused blocks and the host
// step fallback are the same.
#ifndef ATUS_DROPIN_CRT_BASE_2_H
#define ATUS_DROPIN_CRT_BASE_2_H

#include "CRT_Base.h"

template <class T, int dim, int no_int_states>
class CRT_Base_2 : public CRT_Base<T, dim, no_int_states> {
 public:
  // constructor (include/CRT_Base_2.h:107-135): Alpha_2 is read after the
  // kinetic phases are first built, as Alpha_1 is
  CRT_Base_2(ParameterHandler *params) : CRT_Base<T, dim, no_int_states>(params) {
    for (int i = 0; i < dim; i++) m_alpha2[i] = this->m_params->Get_VConstant("Alpha_2", i);
    double a[3] = {0, 0, 0};
    for (int i = 0; i < dim; i++) a[i] = m_alpha2[i];
    for (int c = no_int_states / 2; c < no_int_states; c++)
      atus_check(this->m_gpu, atus_set_alpha(this->m_gpu, c, a), "set_alpha");
  }
  virtual ~CRT_Base_2() {}

  void Save(double *data, std::string filename, const int = 0) { CRT_Base<T, dim, no_int_states>::Save(data, filename); }
  void Save(fftw_complex *data, std::string filename, const int = 0) {
    CRT_Base<T, dim, no_int_states>::Save(data, filename);
  }

 protected:
  CPoint<dim> m_alpha2;
};

#endif
