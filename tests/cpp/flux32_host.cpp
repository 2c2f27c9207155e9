// Host build of the FP32-mode deposit (csrst_b200/csrc/flux32.cuh) for the
// CPU test of its construction: the same source as the CUDA kernels, with
// the device qualifiers and the two round-to-nearest conversions defined for
// the host.  Exposes one call over n moves, accumulating into dense patches.
#include <math.h>
#include <stdint.h>

#define __device__
#define __forceinline__ inline
static inline long long __double2ll_rn(double x) { return llrint(x); }
static inline long long __float2ll_rn(float x) { return llrintf(x); }

#include "../../csrst_b200/csrc/flux32.cuh"

namespace {

template <int ORDER, int COMP>
int run(const int *c0, const float *a0, const float *a1, const int *c1, const float *b0, const float *b1,
        const float *q, long n, double scale, int i0, int j0, int ni, int nj, long long *F, long long *drho,
        bool fast_ok) {
  using SH = csrst::Flux32Shape<ORDER>;
  int bad = 0;
  for (long k = 0; k < n; ++k) {
    const int ci = c0[k] & 0xffff, cj = (int)((unsigned)c0[k] >> 16);
    const int ni_ = c1[k] & 0xffff, nj_ = (int)((unsigned)c1[k] >> 16);
    const double K = (double)q[k] * scale;
    const long long Ki = llrint(K);
    auto put = [&](long long *dst, int i, int j, long long v) {
      i += ci - i0; j += cj - j0;
      if (i >= 0 && j >= 0 && i < ni && j < nj) dst[(long)j * ni + i] += v;
      else if (v) bad |= 2;
    };
    auto sink = [&](int i, int j, long long v) { put(F, i, j, v); };
    const int dx = ni_ - ci + csrst::base_index<ORDER>(b0[k]) - csrst::base_index<ORDER>(a0[k]);
    const bool fast = fast_ok && (unsigned)dx <= 1u &&
                      nj_ - cj + csrst::base_index<ORDER>(b1[k]) == csrst::base_index<ORDER>(a1[k]);
    const bool ok = fast ? csrst::flux_particle<ORDER, COMP, true>(a0[k], a1[k], ni_ - ci, nj_ - cj, b0[k], b1[k], K,
                                                                   Ki, sink)
                         : csrst::flux_particle<ORDER, COMP, false>(a0[k], a1[k], ni_ - ci, nj_ - cj, b0[k], b1[k],
                                                                    K, Ki, sink);
    if (!ok) {
      bad |= 1;
      continue;
    }
    if (drho)
      for (int e = 0; e < 2; ++e) {
        double wx[SH::S], wy[SH::S];
        long long R[SH::S], Q[SH::S];
        const int I = (e ? ni_ - ci : 0) + csrst::charge_weights<ORDER>(e ? b0[k] : a0[k], wx);
        const int J = (e ? nj_ - cj : 0) + csrst::charge_weights<ORDER>(e ? b1[k] : a1[k], wy);
        csrst::quantise<ORDER>(wy, K, Ki, R);
        for (int r = 0; r < SH::S; ++r) {
          csrst::quantise<ORDER>(wx, (double)R[r], R[r], Q);
          for (int c = 0; c < SH::S; ++c) put(drho, I + SH::OFF + c, J + SH::OFF + r, e ? Q[c] : -Q[c]);
        }
      }
  }
  return bad;
}

}  // namespace

// fast: take the compact form for the moves that allow it (as the push does)
extern "C" int flux32_host(int order, int comp, const int *c0, const float *a0, const float *a1, const int *c1,
                           const float *b0, const float *b1, const float *q, long n, double scale, int i0, int j0,
                           int ni, int nj, long long *F, long long *drho, int fast) {
  if (order == 0) return comp ? run<0, 1>(c0, a0, a1, c1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, fast != 0)
                              : run<0, 0>(c0, a0, a1, c1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, fast != 0);
  if (order == 1) return comp ? run<1, 1>(c0, a0, a1, c1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, fast != 0)
                              : run<1, 0>(c0, a0, a1, c1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, fast != 0);
  return comp ? run<2, 1>(c0, a0, a1, c1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, fast != 0)
              : run<2, 0>(c0, a0, a1, c1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, fast != 0);
}
