// fftw3.h (drop-in) -- the part of FFTW's API that ATUS-2 programs touch
// themselves, for programs built against libatus_gpu.so.  The transforms run
// on the GPU (the field classes of cft_base.h); FFTW itself is not used, so
// the thread set-up calls are no-ops and the allocators are the C heap with
// the alignment FFTW guarantees.  Call sites in the reference: the programs'
// main() (rt_solver.cpp:158-160, bragg.cpp:397-399, sob_solver.cpp:177-179)
// and the field allocation of cft_base.h:52-84.
#ifndef ATUS_DROPIN_FFTW3_H
#define ATUS_DROPIN_FFTW3_H

#include <cstddef>
#include <cstdlib>

typedef double fftw_complex[2];
typedef struct atus_no_fftw_plan *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE (0U)

inline int fftw_init_threads() { return 1; }
inline void fftw_plan_with_nthreads(int) {}
inline void fftw_cleanup_threads() {}
inline void fftw_cleanup() {}
inline void fftw_destroy_plan(fftw_plan) {}

inline void *fftw_malloc(size_t n) {
  void *p = nullptr;
  if (posix_memalign(&p, 64, n ? n : 64) != 0) return nullptr;
  return p;
}
inline void fftw_free(void *p) { free(p); }
inline fftw_complex *fftw_alloc_complex(size_t n) { return static_cast<fftw_complex *>(fftw_malloc(n * sizeof(fftw_complex))); }
inline double *fftw_alloc_real(size_t n) { return static_cast<double *>(fftw_malloc(n * sizeof(double))); }

#endif
