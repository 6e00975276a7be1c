// pipe.cuh -- the real-space half of a 3D Strang step as one plane pipeline.
//
// The potential step of a 3D grid needs the fields in real space along y and
// z: IFFT_y, then per z-pencil IFFT_z -> potential step -> FFT_z, then FFT_y.
// All three stages stay inside one x-plane (fixed x index), so they can run
// plane by plane while the plane is still in L2: with P planes and a lag of L
// slots, slot s holds the IFFT_y tiles of plane s, the z tiles of plane s - L
// and the FFT_y tiles of plane s - 2L.  CTAs take work items in that order
// from one atomic counter; before a z tile of plane p starts, every IFFT_y
// tile of p has finished (a per-plane completion counter), and likewise FFT_y
// waits for the z tiles.  Items only wait for items handed out earlier, to
// CTAs that are running, so the pipeline always progresses.  About 2L + 3
// planes are in flight (26 MB for 256^3 two-component complex128), far below
// the 126 MB L2, so HBM sees one read and one write of the fields instead of
// three of each.
//
// Each wait is bounded: after PIPE_SPIN_LIMIT polls the CTA records an error
// in the queue, skips the item and carries on, and the host reports the
// failure after the launch (no hang).
#pragma once
#include "pass2.cuh"

namespace atus {

constexpr int PIPE_MAX_PLANES = 8192;
constexpr unsigned PIPE_SPIN_LIMIT = 1u << 21;  // polls of 64 ns sleep each: >= 0.13 s

// Device-resident state of a context's pipeline.  done[] counts finished
// items per plane over all launches; launch e (1, 2, ...) waits for e * nA
// IFFT_y items and e * nB z items of a plane.
struct PipeQueue {
  unsigned long long next;  // items handed out in this launch (zeroed before it)
  unsigned int err;         // 1: a wait gave up
  unsigned int pad;
  unsigned int done[2][PIPE_MAX_PLANES];
};

struct PipeArgs {
  PassArgs pa, pb, pc;   // IFFT_y (per component), z (IFFT, potential, FFT), FFT_y
  PipeQueue *q;
  unsigned int epoch;
  int P, L;              // planes, lag in slots
  int nA, nB;            // items of a plane: IFFT_y (= FFT_y), z
  int tpcA;              // IFFT_y tiles per component of a plane
  int n1, n2;            // y and z lengths
  long long total;       // items of the launch
};

template <typename R, int N, int TC>
struct PipeCfg {
  using CT = P2Cfg<R, N, 1>;
  using CZ = P2Cfg<R, N, TC>;
  static_assert(CT::smem == CZ::smem, "both stages share one exchange layout");
  static constexpr size_t smem = CT::smem;
};

template <typename R, int N, int TC>
__global__ void __launch_bounds__(Tile2<R>::NT, (sizeof(R) == 8 ? 512 : 768) / Tile2<R>::NT) pipe_kernel(PipeArgs a) {
  using CT = P2Cfg<R, N, 1>;
  using CZ = P2Cfg<R, N, TC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_om[CZ::B], s_ec[CZ::B], s_es[CZ::B];
  __shared__ long long s_w;
  __shared__ int s_skip;
  const int tid = threadIdx.x;
  p2_setup<R, N, 1, M2_INV>(a.pa, smem_raw);  // twiddle rows (same N for y and z)
  const int per_slot = 2 * a.nA + a.nB;
  for (;;) {
    if (tid == 0) s_w = (long long)atomicAdd(&a.q->next, 1ULL);
    __syncthreads();
    const long long w = s_w;
    if (w >= a.total) break;
    const int slot = (int)(w / per_slot), r = (int)(w % per_slot);
    int phase, p, t;
    if (r < a.nA) { phase = 0; p = slot; t = r; }
    else if (r < a.nA + a.nB) { phase = 1; p = slot - a.L; t = r - a.nA; }
    else { phase = 2; p = slot - 2 * a.L; t = r - a.nA - a.nB; }
    if (p < 0 || p >= a.P) {
      __syncthreads();  // every thread has read s_w before it is rewritten
      continue;
    }
    if (tid == 0) {
      int skip = 0;
      if (phase > 0) {
        const unsigned target = a.epoch * (unsigned)(phase == 1 ? a.nA : a.nB);
        const volatile unsigned *cnt = &a.q->done[phase - 1][p];
        unsigned polls = 0;
        while (*cnt < target) {
          if (++polls > PIPE_SPIN_LIMIT) {
            atomicExch(&a.q->err, 1u);
            skip = 1;
            break;
          }
          __nanosleep(64);
        }
        __threadfence();
      }
      s_skip = skip;
    }
    __syncthreads();
    if (!s_skip) {
      const int64_t plane = (int64_t)p * a.n1 * a.n2;
      TileGeo g;
      if (phase == 1) {
        const int y0 = t * CZ::B;
        g.base0 = plane + (int64_t)y0 * a.n2;
        g.pstride = a.n2;
        g.nb = (a.n1 - y0) < CZ::B ? (a.n1 - y0) : CZ::B;
        g.comp0 = 0;
        p2_item<R, N, TC, M2_NL, false, true>(a.pb, g, smem_raw, false, s_om, s_ec, s_es);
      } else {
        const int z0 = (t % a.tpcA) * CT::B;
        g.base0 = plane + z0;
        g.pstride = 1;
        g.nb = (a.n2 - z0) < CT::B ? (a.n2 - z0) : CT::B;
        g.comp0 = t / a.tpcA;
        if (phase == 0) p2_item<R, N, 1, M2_INV, true, true>(a.pa, g, smem_raw, false, s_om, s_ec, s_es);
        else p2_item<R, N, 1, M2_FWD, true, true>(a.pc, g, smem_raw, false, s_om, s_ec, s_es);
      }
    }
    __syncthreads();  // the tile's stores are issued (and s_w, s_skip are read)
    if (phase < 2 && tid == 0) {
      __threadfence();
      atomicAdd(&a.q->done[phase][p], 1u);
    }
  }
}

}  // namespace atus
