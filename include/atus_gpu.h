/*
 * atus_gpu.h -- C ABI of libatus_gpu.so, the B200 (sm_100a) split-step
 * Gross-Pitaevskii engine behind the ATUS-2 solver classes.
 *
 * Plain C: no CUDA, no C++ and no torch types cross this boundary.  Every call
 * returns ATUS_OK (0) or a negative ATUS_E* code; atus_last_error() gives the
 * message of the last failure on a context.  A context is used by one host
 * thread at a time.  Host buffers are borrowed for the duration of the call.
 *
 * Each entry point replaces one piece of the reference's FFTW/OpenMP path
 * (paths relative to the ATUS-2 source tree):
 *
 *   atus_create / atus_destroy      CRT_Base ctor+dtor, Allocate, LoadFiles
 *                                   (include/CRT_Base.h:138-240); the header
 *                                   fields used are those of Read_header
 *                                   (include/CRT_shared.h:131-172)
 *   atus_set_alpha, atus_set_dt     Alpha_1/Alpha_2 and CRT_Base::Init / Set_dt
 *                                   (include/CRT_Base.h:171-174, 252-274;
 *                                   CRT_Base_2.h:194-221; CRT_shared.h:117-121)
 *   atus_set_gs                     GS_i matrix (include/CRT_Base.h:161-169)
 *   atus_set_potential              Init_Potential + Setup_Potential
 *                                   (include/CRT_Base.h:276-298)
 *   atus_set_laser                  CRT_Base_IF::UpdateParams members
 *                                   (include/CRT_Base_IF.h:65-77, 144-168)
 *   atus_upload_psi/atus_download_psi  m_fields[c]->Getp2In() contents
 *                                   (source/libs/lib_myutils/cft_base.h:175)
 *   atus_snapshot/_read             Save_Phi / Append_Phi of run_sequence written from a
 *                                   snapshot (include/CRT_Base.h:606-641)
 *   atus_ft                         cft_Nd::ft (source/libs/lib_myutils/cft_3d.cpp:58-74)
 *   atus_ft_step                    Do_FT_Step_full / Do_FT_Step_half
 *                                   (include/CRT_Base.h:336-392)
 *   atus_nl_step                    Do_NL_Step (include/CRT_Base.h:396-441),
 *                                   CRT_Base_IF::Do_NL_Step (CRT_Base_IF.h:380-419),
 *                                   Bragg_single::Do_Bragg_ad
 *                                   (source/interferometry/src/bragg.cpp:185-304)
 *   atus_strang_block(_rabi)        the inner loop of run_sequence,
 *                                   half,(V,full)^(Nk-1),V,half
 *                                   (include/CRT_Base.h:776-786,
 *                                   CRT_Base_IF.h:779-789), fused on the GPU
 *   atus_particle_number            Get_Particle_Number (include/CRT_Base.h:586-599)
 *   atus_expval_position/momentum   Expval_Position / Expval_Momentum
 *                                   (include/CRT_Base.h:480-580)
 *   atus_setup_momentum             Setup_Momentum (include/CRT_Base.h:448-473)
 *   atus_rabi_integrals             compute_rabi_integrals (CRT_Base_IF.h:207-281)
 *   atus_sob_*                      CSOB_Base (include/CSOB_Base.h:96-543)
 *   atus_particle_number_noalloc    no counterpart in the reference (see its
 *                                   declaration below)
 *   atus_clone                      no counterpart in the reference: a copy of a
 *                                   context's state (the scans of a phase scan side by side)
 *   atus_embed                      no counterpart in the reference: seeding the
 *                                   Sobolev descent from a smaller grid
 *   atus_guess_*                    no counterpart in the reference: a learned
 *                                   initial state for CSOB_Base::run (the
 *                                   reference starts from a muParser guess,
 *                                   sob_solver.cpp:117-137)
 *   atus_batch_*                    many bragg runs at once: per instance the
 *                                   Strang loop of CRT_Base_IF::run_sequence
 *                                   (CRT_Base_IF.h:779-789) with the bragg_ad
 *                                   step (bragg.cpp:185-304) and the AMP_T
 *                                   pulse (CRT_Base_IF.h:170-198)
 */
#ifndef ATUS_GPU_H
#define ATUS_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define ATUS_API __attribute__((visibility("default")))
#else
#define ATUS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define ATUS_OK 0
#define ATUS_E_ARG (-1)         /* invalid argument */
#define ATUS_E_UNSUPPORTED (-2) /* grid or mode this build does not handle */
#define ATUS_E_CUDA (-3)        /* CUDA runtime error */
#define ATUS_E_STATE (-4)       /* call not valid in the current state */
#define ATUS_E_NOMEM (-5)       /* device allocation failed */
#define ATUS_E_LIMIT (-6)       /* input larger than a fixed, documented limit */

#define ATUS_PREC_FP64 0  /* complex128 fields, FP64 FFTs: the drop-in */
#define ATUS_PREC_MIXED 1 /* complex64 fields and FFTs, FP64 phase arguments */

/* Potential-step kinds (the XML sequence tag that selects them). */
#define ATUS_STEP_NL 0       /* "freeprop" of CRT_Base: V + g|psi|^2 */
#define ATUS_STEP_NL_IF 1    /* "freeprop" of CRT_Base_IF: g|psi|^2 + beta.x - DeltaL */
#define ATUS_STEP_BRAGG_AD 2 /* "bragg_ad": analytic 2x2 Bragg exponential */
#define ATUS_STEP_DOUBLE_BRAGG_AD 3 /* "bragg_ad" of double_bragg: three-level exponential,
                                       Bragg_double::Do_Double_Bragg_ad (double_bragg.cpp:100-258) */
#define ATUS_STEP_NL_IF_2 4  /* "freeprop" of CRT_Base_IF_2 (two species, include/CRT_Base_IF_2.h:
                                378-416): g|psi|^2 + beta_s x - DeltaL, beta_s of the component's
                                species (atus_set_laser / atus_set_laser2) */
#define ATUS_STEP_BRAGG_DS_AD 5 /* "bragg_ad" of bragg_ds: a 2x2 Bragg exponential per species,
                                   components (0,1) and (2,3), Bragg_single::Do_Bragg_ad
                                   (bragg_ds.cpp:111-322) */
#define ATUS_STEP_NUMERICAL_BRAGG 6 /* "bragg" of CRT_Base_IF: n-state (n = 2, 3) Bragg exponential,
                                       CRT_Base_IF::Numerical_Bragg (include/CRT_Base_IF.h:426-526);
                                       F is not used (the reference has no envelope here) */
#define ATUS_STEP_NUMERICAL_RAMAN 7 /* "raman" of CRT_Base_IF: three-state Raman exponential,
                                       CRT_Base_IF::Numerical_Raman (include/CRT_Base_IF.h:533-632);
                                       F is not used */

#define ATUS_MAX_COMP 4

typedef struct atus_ctx atus_ctx;

/* The grid part of the 1380-byte generic_header (include/my_structs.h:40-72). */
typedef struct {
  int dim;          /* nDims */
  int64_t n[3];     /* nDimX, nDimY, nDimZ (unused axes: 1) */
  double d[3];      /* dx, dy, dz */
  double dk[3];     /* dkx, dky, dkz */
  double t;         /* header time */
} atus_grid;

/* CRT_Base_IF laser members; arrays sized as in the reference. */
typedef struct {
  double beta[3];
  double DeltaL[ATUS_MAX_COMP];
  double Amp[2];
  double laser_k[2];
  double laser_dk[2];
  double laser_domh[2];
  double phase[2];
  double chirp_rate[2];
  double chirp;
} atus_laser;

/* ------------------------------------------------------------ context */
/* Axis lengths: powers of two, 2..8192 per axis in 2D and 3D; a 1D grid up to
 * 2^26 points (above 8192 the transforms run four-step over an n1 x n2 view;
 * the Sobolev descent keeps the 8192 limit).  Else ATUS_E_UNSUPPORTED. */
ATUS_API int atus_create(const atus_grid *grid, int ncomp, int precision, atus_ctx **out);
ATUS_API void atus_destroy(atus_ctx *ctx);
/* A new context with the state of src: grid, precision, fields, potentials,
 * kinetic phases as src holds them, alpha, g, lasers, pulse windows, time and
 * dt, on a stream of its own.  No counterpart in the reference: the chirp /
 * phase scan of CRT_Base_IF::run_sequence (include/CRT_Base_IF.h:755-921)
 * reruns a sequence from one start state per scan; clones let the scans of
 * a phase scan run side by side. */
ATUS_API int atus_clone(const atus_ctx *src, atus_ctx **out);
ATUS_API const char *atus_last_error(const atus_ctx *ctx);
/* Kernels run on this CUDA stream (a cudaStream_t; NULL = the context's own). */
ATUS_API int atus_set_stream(atus_ctx *ctx, void *stream);
ATUS_API int atus_synchronize(atus_ctx *ctx);
/* Number of kernels this context has launched so far. */
ATUS_API int atus_launch_count(const atus_ctx *ctx, int64_t *out);

/* ------------------------------------------------------------ parameters */
ATUS_API int atus_set_alpha(atus_ctx *ctx, int comp, const double *alpha /* dim */);
/* Stores dt and rebuilds the kinetic phases from the alpha values set so far
 * (CRT_Base::Init semantics: later atus_set_alpha calls take effect at the
 * next atus_set_dt). */
ATUS_API int atus_set_dt(atus_ctx *ctx, double dt);
ATUS_API int atus_get_dt(const atus_ctx *ctx, double *dt);
ATUS_API int atus_set_time(atus_ctx *ctx, double t);
ATUS_API int atus_get_time(const atus_ctx *ctx, double *t);
ATUS_API int atus_set_gs(atus_ctx *ctx, const double *gs /* ncomp*ncomp, row i = GS_(i+1) */);
/* V: N doubles in grid order, or NULL to drop the potential of comp. */
ATUS_API int atus_set_potential(atus_ctx *ctx, int comp, const double *V);
ATUS_API int atus_set_laser(atus_ctx *ctx, const atus_laser *laser);
/* The second species of the two-species programs (CRT_Base_IF_2::UpdateParams,
 * include/CRT_Base_IF_2.h:80-113: Beta_2, Amp_2, laser_k_2, laser_dk_2,
 * laser_domh_2 and the members phase2, chirp_rate2); element 0 of each array is
 * used.  DeltaL of all four components stays with atus_set_laser. */
ATUS_API int atus_set_laser2(atus_ctx *ctx, const atus_laser *laser2);
/* Pulse windows of ATUS_STEP_BRAGG_DS_AD (bragg_ds.cpp:114-127): with t1 = t +
 * dt/2 at the potential step, species s couples while t1 - t_start <=
 * duration[s] and only takes its phases afterwards.  t_start is the sequence's
 * start time (seq.time = Get_t(), include/CRT_Base_IF_2.h:466).  Default: no
 * window (duration = +inf). */
ATUS_API int atus_set_pulse_windows(atus_ctx *ctx, double t_start, const double *duration /* 2 */);
/* on = 1: FP64 contexts take the bragg_ad step in the eigenvalue-free form
 * U = e^{-i dt m}[cos(r dt) - i sin(r dt)/r (H - m)] (complex64 contexts always
 * do).  No counterpart in the reference: its eigen-form (bragg.cpp:254-277)
 * divides by (V11 - E)^2 + Omega^2, loses unitarity once |Omega| is below the
 * spacing of V11 and divides by zero once Omega^2 underflows -- the tails of a
 * Gaussian pulse reach both.  Default 0: the reference's form, bit for bit. */
ATUS_API int atus_set_bragg_stable(atus_ctx *ctx, int on);

/* No counterpart in the reference.  Bounded waits of the TMA-fed strided
 * passes: a tile copy not complete after wait_rounds rounds of
 * mbarrier.try_wait (default 2^22) ends the pass, and the call that ran it
 * (a block, step, transform, spectral reduction or descent; else the next
 * atus_synchronize) returns ATUS_E_CUDA ("a TMA tile copy did not complete
 * ...") instead of hanging; the context stays usable (its fields are then
 * undefined).
 * drop_copies = 1 issues no tile copies, so every wait runs out with nothing
 * in flight: a test hook for that error path, 0 in normal use.  ATUS_E_ARG
 * for wait_rounds < 1 or drop_copies not 0 or 1. */
ATUS_API int atus_set_wait_limits(atus_ctx *ctx, int64_t wait_rounds, int drop_copies);

/* ------------------------------------------------------------ fields */
/* Interleaved complex128, N values, grid order (the .bin payload). */
ATUS_API int atus_upload_psi(atus_ctx *ctx, int comp, const double *psi);
ATUS_API int atus_download_psi(atus_ctx *ctx, int comp, double *psi);
/* Device pointer of component comp (complex128 or complex64 per precision). */
ATUS_API int atus_device_psi(atus_ctx *ctx, int comp, void **dptr);
/* Output without stalling the steps (Save_Phi / Append_Phi of run_sequence,
 * include/CRT_Base.h:606-641, written from a snapshot).  atus_snapshot
 * copies every component into a device staging buffer of the context
 * (complex128), ordered after the steps enqueued before, and returns at once;
 * the steps enqueued next run while the snapshot is read.  The first call
 * allocates the staging buffer (ncomp x N x 16 bytes); a snapshot waits on the
 * device for the reads of the one before.
 * atus_snapshot_read copies component comp of the last snapshot into host_dst
 * (N complex128 values) on a copy stream of the context and returns when it
 * is there.  It may be called from other host threads (one per component)
 * while the context's own thread goes on with other calls; the caller makes
 * sure the reads of one snapshot finish before it takes the next. */
ATUS_API int atus_snapshot(atus_ctx *ctx);
ATUS_API int atus_snapshot_read(atus_ctx *ctx, int comp, double *host_dst);
/* cft_Nd::ft(isign) on component comp, in place (source/libs/lib_myutils/
 * cft_1d.cpp:61-77, cft_2d.cpp:58-74, cft_3d.cpp:58-74): the transform over
 * every axis with FFTW's sign convention (isign -1 forward, +1 backward),
 * natural (unshifted) order, then the scale (dx/sqrt(2 pi))^dim after a
 * forward and (dk/sqrt(2 pi))^dim after a backward transform. */
ATUS_API int atus_ft(atus_ctx *ctx, int comp, int isign);

/* ------------------------------------------------------------ steps */
ATUS_API int atus_ft_step(atus_ctx *ctx, int half);
/* F: pulse amplitude AMP_T(t + dt/2) for ATUS_STEP_BRAGG_AD (1 without AMP_T). */
ATUS_API int atus_nl_step(atus_ctx *ctx, int kind, double F);
/* nk Strang steps: half, (V, full)^(nk-1), V, half.  F[j] is the pulse
 * amplitude of the j-th potential step (NULL: all 1). */
ATUS_API int atus_strang_block(atus_ctx *ctx, int nk, int kind, const double *F);
/* atus_strang_block with the Rabi sums of the block's final state:
 * compute_rabi_integrals (include/CRT_Base_IF.h:207-281; both species of
 * CRT_Base_IF_2, include/CRT_Base_IF_2.h:115-210) of components comps[c]
 * (c < ncomp_r <= 2) for the centres k0[(c*n + m)*dim ..] (m < n, ncomp_r*n <=
 * 8), radius thr, into out[c*n + m].  Where the block's last kinetic pass is
 * the register-staged x pass (2D / 3D, 32 <= nx <= 256) the sums are taken
 * inside it (every axis is in k-space there and |psi^|^2 does not see the
 * kinetic phase); otherwise by a separate transform and reduction as
 * atus_rabi_integrals_comp does. */
ATUS_API int atus_strang_block_rabi(atus_ctx *ctx, int nk, int kind, const double *F, int ncomp_r, const int *comps,
                                    const double *k0, int n, double thr, double *out);

/* ------------------------------------------------------------ measurement */
/* Device time of the fused passes that make up one Strang step of `kind`,
 * each launched `reps` times back to back on the context's stream and timed
 * with CUDA events there.  ms[i] receives the average duration of one launch
 * of pass i, launches_per_step[i] how often one Strang step launches it, and
 * bytes[i] the field bytes one launch reads and writes (the algorithmic
 * traffic).  *npass receives the number of pass kinds (<= 8).  The passes
 * run out of the Strang schedule on the context's fields; the fields and the
 * time are saved before (a temporary device copy of the fields) and restored
 * after, so the context's state is unchanged. */
ATUS_API int atus_profile_passes(atus_ctx *ctx, int kind, int reps, double *ms, double *launches_per_step,
                                 double *bytes, int *npass);

/* ------------------------------------------------------------ observables */
ATUS_API int atus_particle_number(atus_ctx *ctx, int comp, double *out);
/* Particle number  ar * sum_l |psi_l|^2  of one field in device memory, with
 * no allocation of any kind.  No counterpart in the reference: it is the
 * reduction of atus_particle_number for callers that cannot allocate device
 * memory -- a host framework whose caching allocator or fixed pool owns the
 * device memory (a foreign cudaMalloc would fragment it or fail), or a time
 * step that cannot take cudaFree's device-wide synchronisation.  It needs no
 * context; its partial sums live in a fixed device array inside the library.
 *
 *   psi_dev    npts complex values (complex128 for ATUS_PREC_FP64, complex64
 *              for ATUS_PREC_MIXED), device memory of the current device
 *   ar         volume element (dx, dx*dy or dx*dy*dz)
 *   out_dev    one double in device memory, written on `stream`
 *   stream     cudaStream_t, NULL for the legacy default stream
 *
 * npts is limited to ATUS_NOALLOC_MAX_POINTS (2^27 points: one partial sum
 * per 32768 points in a 32 KB array); larger fields return ATUS_E_LIMIT and
 * launch nothing.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture.  The address is kept per device together
 * with the id of the CUDA context it belongs to: after cudaDeviceReset, or
 * under another context, the next call looks it up again (so make that call,
 * too, outside a capture).  All calls on a device share the array, so
 * calls whose kernels overlap on the GPU (other streams, other host threads)
 * race and may return wrong sums: order them on one stream.  The result
 * equals atus_particle_number's to rounding (another summation order). */
#define ATUS_NOALLOC_MAX_POINTS 134217728LL
ATUS_API int atus_particle_number_noalloc(const void *psi_dev, int64_t npts, int precision, double ar,
                                          double *out_dev, void *stream);
ATUS_API int atus_expval_position(atus_ctx *ctx, int comp, double *out /* dim */);
ATUS_API int atus_expval_momentum(atus_ctx *ctx, int comp, double *out /* dim */);
ATUS_API int atus_setup_momentum(atus_ctx *ctx, int comp, const double *p /* dim */);
/* n momentum points k0 (n*dim), threshold thr: m_ar_k * sum |psi0^(k)|^2 per ball. */
ATUS_API int atus_rabi_integrals(atus_ctx *ctx, const double *k0, int n, double thr, double *out);
/* The same on component comp: the second species' sums of
 * CRT_Base_IF_2::compute_rabi_integrals (include/CRT_Base_IF_2.h:115-210) use
 * component no_int_states/2. */
ATUS_API int atus_rabi_integrals_comp(atus_ctx *ctx, int comp, const double *k0, int n, double thr, double *out);

/* ------------------------------------------------------------ Sobolev gradient */
/* Component comp_s of a context on a smaller grid with the same spacing,
 * centred in component comp_d of a larger one (index offset (n_dst - n_src)/2
 * per axis), zero elsewhere; both FP64.  No counterpart in the reference: it
 * carries a ground state solved on a box that just holds the condensate into
 * the full box, as the start of the Sobolev descent there. */
ATUS_API int atus_embed(atus_ctx *src, int comp_s, atus_ctx *dst, int comp_d);
/* Ground-state descent of CSOB_Base on the context's grid: alpha per
 * component (Alpha_i[0] on every axis), gs already scaled by sqrt(N_i N_j),
 * fixed stepsize.  The potential comes from atus_set_potential and the start
 * from atus_upload_psi. */
ATUS_API int atus_sob_init(atus_ctx *ctx, const double *alpha /* ncomp */, double stepsize);
ATUS_API int atus_sob_renormalize(atus_ctx *ctx);
/* n_iter iterations of CSOB_Base::run's loop body; res/N receive the values of
 * the last one (N: ncomp entries). */
ATUS_API int atus_sob_iterate(atus_ctx *ctx, int n_iter, double *res, double *N);
/* CSOB_Base::run: renormalise, iterate until res <= epsilon (at most
 * max_iter); iterations taken in *iters. */
ATUS_API int atus_sob_run(atus_ctx *ctx, double epsilon, int max_iter, int *iters, double *res);
/* mu_i = m_ar * sum[-Re(psi* Lap psi) + (V + sum_j g_ij |psi_j|^2) |psi_i|^2] */
ATUS_API int atus_sob_mu(atus_ctx *ctx, double *mu /* ncomp */);

/* ------------------------------------------------------------ learned guess
 * A small MLP (3 inputs, two tanh layers of 64, 64 linear outputs) maps the
 * scaled parameters of a ground-state problem to the coefficients of the
 * state in the 64 products phi_a(x/lx) phi_b(y/ly) phi_c(z/lz) of even
 * Hermite functions (a, b, c in {0, 2, 4, 6}; coefficient 16 a' + 4 b' + c'
 * with a' = a/2 ...).  Training and inference run in hand-written FP64
 * kernels.  Parameter vector: W1[64][3], b1[64], W2[64][64], b2[64],
 * W3[64][64], b3[64]. */
#define ATUS_GUESS_NIN 3
#define ATUS_GUESS_NOUT 64
#define ATUS_GUESS_NPARAM 8576
/* Glorot-uniform weights, zero biases, from a seeded splitmix64 stream. */
ATUS_API int atus_guess_init(uint64_t seed, double *params);
/* Mean squared error over B samples (X: B x 3, Y: B x 64) and its gradient. */
ATUS_API int atus_guess_grad(const double *params, const double *X, const double *Y, int B, double *loss,
                             double *grad);
/* Full-batch Adam (beta 0.9 / 0.999) for `epochs` steps; params updated in
 * place; loss_history (may be NULL) gets the loss before each step. */
ATUS_API int atus_guess_train(double *params, const double *X, const double *Y, int B, int epochs, double lr,
                              double *loss_history);
ATUS_API int atus_guess_predict(const double *params, const double *X, int B, double *coef /* B x 64 */);
/* Writes sum coef * phi phi phi (real) into component comp of a 3D FP64
 * context; scale = the three basis lengths (lx, ly, lz). */
ATUS_API int atus_guess_decode(atus_ctx *ctx, int comp, const double *coef, const double *scale);

/* ------------------------------------------------------------ batched sweep
 * Independent two-component bragg_ad instances (1D lengths 1024..16384, square
 * 2D grids 64^2..512^2; powers of two), all advanced by one CUDA-graph launch
 * per Strang block: 1D instances by one persistent kernel per length with the
 * instance resident in shared memory, 2D instances by batched passes over all
 * instances of a size.  atus_batch_tune picks, per size class, the kernel
 * variant (threads per CTA and resident components for 1D; register-staged or
 * shared-memory tile passes for 2D) from timed probe runs on copies of the
 * fields.  Each instance computes what a context with the same parameters
 * computes with atus_strang_block(ATUS_STEP_BRAGG_AD) and F[j] =
 * AMP_T(t1_j) = exp(-(t1_j - tc)^2 / (2 sigma^2)), t1_j = t0 + dt (j + 1). */
typedef struct atus_batch atus_batch;
typedef struct {
  atus_grid grid;      /* dim 1 or 2, n, d, dk, t (2D: n[0] == n[1]) */
  double alpha;        /* kinetic coefficient on every axis */
  double gs[4];        /* g11, g12, g21, g22 */
  atus_laser laser;    /* bragg_ad laser members */
  double pulse_tc;     /* AMP_T centre */
  double pulse_sigma;  /* AMP_T width; <= 0: AMP_T = 1 */
  int bragg_stable;    /* FP64 batches: the eigenvalue-free form (atus_set_bragg_stable) */
} atus_batch_instance;
ATUS_API int atus_batch_create(const atus_batch_instance *inst, int count, int precision, double dt,
                               atus_batch **out);
ATUS_API void atus_batch_destroy(atus_batch *b);
ATUS_API const char *atus_batch_last_error(const atus_batch *b);
/* Interleaved complex128 host buffers of the instance's grid size. */
ATUS_API int atus_batch_upload_psi(atus_batch *b, int inst, int comp, const double *psi);
ATUS_API int atus_batch_download_psi(atus_batch *b, int inst, int comp, double *psi);
ATUS_API int atus_batch_get_time(const atus_batch *b, int inst, double *t);
/* Autotuner: probe_steps Strang steps per candidate and size class. */
ATUS_API int atus_batch_tune(atus_batch *b, int probe_steps);
/* One Strang block of nk steps for every instance (one graph launch); *ms
 * (may be NULL) receives its device time. */
ATUS_API int atus_batch_run(atus_batch *b, int nk, double *ms);
/* Human-readable schedule (size classes, chosen variants, probe times). */
ATUS_API int atus_batch_schedule(const atus_batch *b, char *buf, int len);

#ifdef __cplusplus
}
#endif
#endif
