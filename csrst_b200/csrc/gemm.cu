// BF16 tensor-core GEMM on the 5th-generation tensor cores (tcgen05) for the
// surrogate network: C[M, N] = A[M, K] . B[N, K]^T with FP32 accumulation, both
// operands K-major (rows contiguous along K), batched, over one or two K
// segments into one accumulator.
//
// Persistent and warp-specialised: one CTA of 576 threads per SM walks the
// 128 x BN output tiles (batch, row tile, column tile) in a fixed stride.
//   - warp 0 (one lane) copies the A and B tiles of 64 K-columns with TMA
//     (128-byte swizzle; 3-D tensor maps over (K, rows, batch) for batched
//     operands, rows past the matrix read as zero) into a ring of stages, each
//     stage completing on its `full` mbarrier;
//   - warp 1 (one lane) issues four tcgen05.mma (M = 128, N = BN, K = 16) per
//     stage into one of the FP32 accumulators in tensor memory (TMEM), commits
//     them to the stage's `empty` mbarrier, which hands the stage back to the
//     copies, and at the end of a tile to the accumulator's `acc_full`
//     mbarrier;
//   - warps 2..17 (the epilogue) read the accumulator with tcgen05.ld (warp w
//     may read TMEM lanes 32 (w % 4) .. + 31, i.e. rows; the four warps of a
//     row quarter take one 32-column chunk each, of the same tile when BN is
//     128, else of 2 or 4 tiles in turn, with 4 or 8 accumulators of BN
//     columns in the 256 TMEM columns), hand it back through
//     `acc_empty` after their read, add the biases and write FP32 and/or BF16
//     outputs through affine index maps: as 16-byte runs through a 32 x 33
//     staging block in shared memory where the map allows (below), else
//     element by element, a warp storing whole columns of its 32 rows (lanes
//     on consecutive rows, straight from the registers) or, through the
//     staging block, whole rows, whichever puts a warp's 32 stores next to
//     each other under the map.  Sixteen epilogue warps, four per scheduler,
//     hide the latency of each warp's dependent steps.
// With two or more accumulators the epilogue of one tile overlaps the copies and
// products of the next, and the copies run up to a ring ahead of the
// products, so the kernel streams its operands and outputs at once.
//
// Waits on mbarriers are bounded (a launch parameter, csrst_gemm_set_wait_limit):
// a wait that gives up sets *err = 1 and a shared flag that ends the other
// roles' loops at their next wait.  Before the TMEM is freed, the copy warp
// waits for every copy it issued and the MMA warp for every product it
// issued (with the default bound; *err = 2 if even that gives up), so nothing
// still writes into TMEM or shared memory the CTA no longer owns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/csrst.h"
#include "gemm_maps.h"
#include "tma.cuh"

namespace csrst {
namespace {

constexpr int kBM = 128, kBK = 64;
constexpr int kEpiWarps = 16, kThreads = 64 + 32 * kEpiWarps;
constexpr long long kSpin = 1ll << 24;  // default mbarrier polls before a wait gives up

template <int BN>
struct Cfg {
  static constexpr int A_BYTES = kBM * kBK * 2;               // 16 KB, 128 rows of 128 B
  static constexpr int B_BYTES = BN * kBK * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;             // multiples of 1024 B: swizzle atoms stay aligned
  static constexpr int STAGES = BN == 128 ? 4 : 6;
  static constexpr int EPI = kEpiWarps * 32 * 33 * 4;         // per-warp 32 x 33 FP32 staging blocks
  static constexpr int SMEM = STAGES * STAGE + EPI + 1024;    // + alignment slack
  static constexpr int TMEM_COLS = 256;                       // NACC accumulators of BN columns
  static constexpr int NACC = TMEM_COLS / BN;                 // 2, 4 or 8
  static constexpr int CHUNKS = BN / 32;                      // 32-column pieces of a tile
  static constexpr int TG = 4 / CHUNKS;                       // epilogue groups working on different tiles
};

// Shared-memory matrix descriptor of a K-major operand tile with 128-byte
// swizzle (the layout a TMA copy with CU_TENSOR_MAP_SWIZZLE_128B writes):
// rows 128 B apart, 8-row atoms 1024 B apart (SBO), LBO unused (1),
// descriptor version 1, layout type 2.  Stepping K by 16 elements adds 32 B
// to the start address inside the atom.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// The same for an MN-major A tile (rows contiguous along M) with 128-byte
// swizzle, as two TMA boxes of 64 M x 64 K write it: each 64-row chunk holds
// the tile's 64 K rows of 128 B (8-row atoms 1024 B apart: SBO), the second
// chunk 8192 B after the first (LBO).  Stepping K by 16 rows adds 2048 B.
__device__ __forceinline__ uint64_t sw128_mn_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(8192 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, B
// K-major, A K-major or MN-major (bit 15), M = 128, N = BN.
template <int BN>
__device__ __forceinline__ uint32_t instr_desc(bool a_mn = false) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn ? 1u << 15 : 0u) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// Arrives on `bar` once every tensor-core operation this thread issued before
// it has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Starts the load of 32 accumulator columns (TMEM lanes of this warp, one row
// per lane) into v; the registers hold the values only after tmem_wait(v).
__device__ __forceinline__ void tmem_ld32(uint32_t ta, uint32_t *v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(ta));
}

// Waits for this thread's TMEM loads; v is named so that no use of it moves
// above the wait.
__device__ __forceinline__ void tmem_wait(uint32_t *v) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                 "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),
                 "+r"(v[15]), "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]),
                 "+r"(v[22]), "+r"(v[23]), "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]),
                 "+r"(v[29]), "+r"(v[30]), "+r"(v[31])
               :
               : "memory");
}

// GELU, erf form: 0.5 x (1 + erf(x / sqrt 2)), with erf from the rational
// approximation of C. Hastings (Abramowitz & Stegun 7.1.28):
//   1 - erf(u) = (1 + a1 u + a2 u^2 + ... + a6 u^6)^-16,  u >= 0,
// absolute error at most 3e-7.  With r = that power, 1 + erf(x / sqrt 2) is
// r for x < 0 and 2 - r for x >= 0, so GELU is 0.5 x r or x - 0.5 x r: one
// reciprocal and no cancellation on the negative side.
__device__ __forceinline__ float gelu(float x) {
  const float u = fabsf(x) * 0.70710678118654752f;
  float p = fmaf(u, 0.0000430638f, 0.0002765672f);
  p = fmaf(u, p, 0.0001520143f);
  p = fmaf(u, p, 0.0092705272f);
  p = fmaf(u, p, 0.0422820123f);
  p = fmaf(u, p, 0.0705230784f);
  p = fmaf(u, p, 1.0f);
  p *= p;
  p *= p;
  p *= p;
  p *= p;
  const float h = 0.5f * x * __fdividef(1.0f, p);
  return x < 0.0f ? h : x - h;
}

// Bounded wait of one thread that also gives up when another role has
// failed (the shared flag, read every 64 polls).  Returns false on either;
// a wait that ran out of polls raises the flag and sets *err = 1.
__device__ __forceinline__ bool wait_role(uint64_t *bar, uint32_t parity, long long spin, volatile int *fail,
                                          int *err) {
  if (spin > 0 && mbar_test(bar, parity)) return true;
  for (long long k = 1; k < spin; ++k) {
    if (mbar_try(bar, parity)) return true;
    if ((k & 63) == 0 && *fail) return false;
  }
  *fail = 1;
  atomicExch(err, 1);
  return false;
}

// One K segment of a product: A[M, Kseg] and B[N, Kseg], K-major, batch
// strides sA / sB, nk tiles of 64 K-columns.  A product runs over the K
// tiles of its first segment and then of its second (nk = 0 when absent):
// C = A1 B1^T + A2 B2^T in one accumulator.
struct Seg {
  const __nv_bfloat16 *A;
  long long lda, sA;
  const __nv_bfloat16 *B;
  long long ldb, sB;
  int nk;
  int amn;  // A is MN-major: element (m, k) of a batch at A[k * lda + m]
};


// Everything one launch reads: the operand tensor maps (A1, B1, A2, B2;
// 3-D over (K, rows, batch) where the operand has a batch stride, else
// 2-D), the epilogue, the tile grid, the sweep orders of the two maps and
// their vector forms (vec: every output of the launch has one and there is
// no residual or accumulation).
struct alignas(64) GemmArgs {
  CUtensorMap map[4];
  csrst_gemm_epilogue ep;
  int *err;
  long long spin;
  long long ntiles;
  int nk1, nk2, M, N, tilesM, tilesN;
  int rank3[4];
  int amn[2];                 // per segment: A MN-major (two 64-row TMA boxes per stage)
  int o_mfast, t_mfast;
  int vec;
  RunShape rs[4];             // pre, out32, out16 (primary map), out16t (second map)
  long long del[2][2][32];    // [map][rows, columns][i or j]
};

// Row and column parts of an output map's index: z*sb + (m/md)*s0 + (m%md)*s1
// and (n/nd)*t0 + (n%nd)*t1.
__device__ __forceinline__ long long row_part(long long zb, int m, int md, long long s0, long long s1) {
  return zb + (long long)(m / md) * s0 + (long long)(m % md) * s1;
}
__device__ __forceinline__ long long col_part(int n, int nd, long long t0, long long t1) {
  return (long long)(n / nd) * t0 + (long long)(n % nd) * t1;
}

// One element under the primary map: residual, pre-activation, activation,
// FP32 and BF16 outputs; returns the value the second map copies.
__device__ __forceinline__ float finish(const csrst_gemm_epilogue &ep, long long o, float x) {
  if (ep.res) x += ep.res[o];
  if (ep.pre) ep.pre[o] = x;
  if (ep.act == 1) x = gelu(x);
  if (ep.out32) ep.out32[o] = ep.accumulate ? ep.out32[o] + x : x;
  if (ep.out16) reinterpret_cast<__nv_bfloat16 *>(ep.out16)[o] = __float2bfloat16(x);
  return x;
}

// Writes one 32-row x 32-column piece of a tile held by a warp (lane = row
// mrow + lane, x[j] = column ncol + j, biases added) through both output
// maps.  Under a map whose consecutive rows are neighbours the warp stores a
// column per instruction straight from the registers; otherwise the piece
// goes through the warp's staging block st[32][33] (conflict-free both ways)
// and the warp stores a row per instruction.
__device__ __forceinline__ void store_piece(const GemmArgs &a, float (&x)[32], float *st, int lane, int mrow, int ncol,
                                            long long orow, long long trow, long long ocol, long long tcol) {
  const csrst_gemm_epilogue &ep = a.ep;
  const bool mok = mrow + lane < a.M, nok = ncol + lane < a.N;
  if (a.o_mfast) {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const long long oc = __shfl_sync(0xffffffffu, ocol, j);
      if (mok && ncol + j < a.N) x[j] = finish(ep, orow + oc, x[j]);
    }
  } else {
#pragma unroll
    for (int j = 0; j < 32; ++j) st[lane * 33 + j] = x[j];
    __syncwarp();
#pragma unroll 4
    for (int i = 0; i < 32; ++i) {
      const long long ori = __shfl_sync(0xffffffffu, orow, i);
      if (mrow + i < a.M && nok) st[i * 33 + lane] = finish(ep, ori + ocol, st[i * 33 + lane]);
    }
    __syncwarp();
    if (ep.out16t && a.t_mfast) {
#pragma unroll
      for (int j = 0; j < 32; ++j) x[j] = st[lane * 33 + j];
    }
  }
  if (ep.out16t) {
    __nv_bfloat16 *t16 = reinterpret_cast<__nv_bfloat16 *>(ep.out16t);
    if (a.t_mfast) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const long long tc = __shfl_sync(0xffffffffu, tcol, j);
        if (mok && ncol + j < a.N) t16[trow + tc] = __float2bfloat16(x[j]);
      }
    } else {
      if (a.o_mfast) {
#pragma unroll
        for (int j = 0; j < 32; ++j) st[lane * 33 + j] = x[j];
        __syncwarp();
      }
#pragma unroll 4
      for (int i = 0; i < 32; ++i) {
        const long long tri = __shfl_sync(0xffffffffu, trow, i);
        if (mrow + i < a.M && nok) t16[tri + tcol] = __float2bfloat16(st[i * 33 + lane]);
      }
    }
  }
  __syncwarp();  // the staging block is free for the next piece
}

// Row and column offsets of element t of a run of shape S, and the run's
// extent in rows (RI) and columns (RJ).
template <int S, int L>
struct Run {
  static constexpr int RI = S == 0 ? 1 : S == 1 ? L : S == 2 ? L / 2 : 2;
  static constexpr int RJ = S == 0 ? L : S == 1 ? 1 : S == 2 ? 2 : L / 2;
  static __device__ __forceinline__ int di(int t) { return S == 0 ? 0 : S == 1 ? t : S == 2 ? t >> 1 : t & 1; }
  static __device__ __forceinline__ int dj(int t) { return S == 0 ? t : S == 1 ? 0 : S == 2 ? t & 1 : t >> 1; }
};

__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&h);
}

// Writes a staged piece st[32][33] (final values) as runs of shape S: the
// warp's 32 lanes take 32 runs per store, 1024 / L runs in all.
template <int S, int L>
__device__ __forceinline__ void store_runs(const float *st, const long long *rdel, const long long *cdel, void *out,
                                           long long base, int lane, int fast_j) {
  using R = Run<S, L>;
  constexpr int NI = 32 / R::RI, NJ = 32 / R::RJ;
#pragma unroll
  for (int k = 0; k < NI * NJ / 32; ++k) {
    const int r = k * 32 + lane;
    const int oi = (fast_j ? r / NJ : r % NI) * R::RI, oj = (fast_j ? r % NJ : r / NI) * R::RJ;
    float v[L];
#pragma unroll
    for (int t = 0; t < L; ++t) v[t] = st[(oi + R::di(t)) * 33 + oj + R::dj(t)];
    const long long o = base + rdel[oi] + cdel[oj];
    if constexpr (L == 8) {
      *reinterpret_cast<uint4 *>(reinterpret_cast<__nv_bfloat16 *>(out) + o) =
          make_uint4(bf16x2(v[0], v[1]), bf16x2(v[2], v[3]), bf16x2(v[4], v[5]), bf16x2(v[6], v[7]));
    } else {
      *reinterpret_cast<float4 *>(reinterpret_cast<float *>(out) + o) = make_float4(v[0], v[1], v[2], v[3]);
    }
  }
}

template <int L>
__device__ __forceinline__ void store_vec(const RunShape &rs, const float *st, const long long *rdel,
                                          const long long *cdel, void *out, long long base, int lane) {
  switch (rs.shape) {
    case 0: store_runs<0, L>(st, rdel, cdel, out, base, lane, rs.fast_j); break;
    case 1: store_runs<1, L>(st, rdel, cdel, out, base, lane, rs.fast_j); break;
    case 2: store_runs<2, L>(st, rdel, cdel, out, base, lane, rs.fast_j); break;
    default: store_runs<3, L>(st, rdel, cdel, out, base, lane, rs.fast_j); break;
  }
}

// A whole 32 x 32 piece (lane = row, x[j] = column j, biases added) through
// the vector forms: the pre-activation, then the activation, then the FP32
// and BF16 copies, each from the warp's staging block.  obase / tbase: the
// piece's base index under the primary and the second map.
__device__ __forceinline__ void store_piece_vec(const GemmArgs &a, const long long (*del)[2][32], float (&x)[32],
                                                float *st, int lane, long long obase, long long tbase) {
  const csrst_gemm_epilogue &ep = a.ep;
  if (ep.pre) {
#pragma unroll
    for (int j = 0; j < 32; ++j) st[lane * 33 + j] = x[j];
    __syncwarp();
    store_vec<4>(a.rs[0], st, del[0][0], del[0][1], ep.pre, obase, lane);
    __syncwarp();
  }
  if (ep.act == 1) {
#pragma unroll
    for (int j = 0; j < 32; ++j) x[j] = gelu(x[j]);
  }
#pragma unroll
  for (int j = 0; j < 32; ++j) st[lane * 33 + j] = x[j];
  __syncwarp();
  if (ep.out32) store_vec<4>(a.rs[1], st, del[0][0], del[0][1], ep.out32, obase, lane);
  if (ep.out16) store_vec<8>(a.rs[2], st, del[0][0], del[0][1], ep.out16, obase, lane);
  if (ep.out16t) store_vec<8>(a.rs[3], st, del[1][0], del[1][1], ep.out16t, tbase, lane);
  __syncwarp();  // the staging block is free for the next piece
}

template <int BN>
__global__ void __launch_bounds__(kThreads, 1) k_gemm(const __grid_constant__ GemmArgs a) {
  using G = Cfg<BN>;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t full[G::STAGES], empty[G::STAGES], acc_full[G::NACC], acc_empty[G::NACC], drain, never;
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  __shared__ long long s_del[2][2][32];  // the maps' row and column offsets over a piece
  uint8_t *base = smem + ((1024 - (smem_u32(smem) & 1023)) & 1023);
  float *epi = reinterpret_cast<float *>(base + G::STAGES * G::STAGE);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int *fail = &s_fail;
  // spin < 0: the epilogue's first wait is on `never`, which nothing
  // completes, with -spin polls (the stuck wait the error path is tested with)
  const bool stuck = a.spin < 0;
  const long long spin = stuck ? -a.spin : a.spin;

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(G::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < G::STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < G::NACC; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 32 * 4 * G::CHUNKS);  // the warps that read one tile
    }
    mbar_init(&drain, 1);
    mbar_init(&never, 1);
    mbar_init_fence();
    s_fail = 0;
  }
  for (int k = threadIdx.x; k < 128; k += kThreads) (&s_del[0][0][0])[k] = (&a.del[0][0][0])[k];
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const int nk = a.nk1 + a.nk2;

  if (warp == 0) {
    // ---- copies ----
    if (lane == 0) {
      long long it = 0;  // stage fills issued
      bool ok = true;
      for (long long t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x) {
        const long long r = t / a.tilesN;
        const int n0 = (int)(t % a.tilesN) * BN, m0 = (int)(r % a.tilesM) * kBM, z = (int)(r / a.tilesM);
        for (int kt = 0; kt < nk; ++kt) {
          const int s = (int)(it % G::STAGES);
          if (!wait_role(&empty[s], (uint32_t)((it / G::STAGES) & 1) ^ 1u, spin, fail, a.err)) {
            ok = false;
            break;
          }
          uint8_t *sa = base + s * G::STAGE, *sb = sa + G::A_BYTES;
          mbar_expect_tx(&full[s], G::STAGE);
          const int seg = kt < a.nk1 ? 0 : 1, k0 = (kt < a.nk1 ? kt : kt - a.nk1) * kBK;
          const int ia = 2 * seg, ib = ia + 1;
          if (a.amn[seg]) {  // (M, K) boxes of 64 x 64: the tile's two row chunks
            for (int h = 0; h < 2; ++h) {
              if (a.rank3[ia]) tma_load_3d(sa + h * 8192, &a.map[ia], m0 + 64 * h, k0, z, &full[s]);
              else tma_load_2d(sa + h * 8192, &a.map[ia], m0 + 64 * h, k0, &full[s]);
            }
          } else if (a.rank3[ia]) {
            tma_load_3d(sa, &a.map[ia], k0, m0, z, &full[s]);
          } else {
            tma_load_2d(sa, &a.map[ia], k0, m0, &full[s]);
          }
          if (a.rank3[ib]) tma_load_3d(sb, &a.map[ib], k0, n0, z, &full[s]);
          else tma_load_2d(sb, &a.map[ib], k0, n0, &full[s]);
          ++it;
        }
      }
      // every fill issued has landed before the CTA ends (fills older than
      // the last STAGES were consumed by the products, so they had landed)
      for (long long i = it > G::STAGES ? it - G::STAGES : 0; i < it; ++i)
        if (!mbar_wait(&full[i % G::STAGES], (uint32_t)((i / G::STAGES) & 1), kSpin)) atomicExch(a.err, 2);
    }
  } else if (warp == 1) {
    // ---- products ----
    if (lane == 0) {
      long long it = 0;
      int lt = 0;
      bool ok = true, issued = false;
      for (long long t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x, ++lt) {
        const int b = lt % G::NACC;
        if (!wait_role(&acc_empty[b], (uint32_t)((lt / G::NACC) & 1) ^ 1u, spin, fail, a.err)) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t d = tmem + (uint32_t)(b * BN);
        for (int kt = 0; kt < nk; ++kt) {
          const int s = (int)(it % G::STAGES);
          if (!wait_role(&full[s], (uint32_t)((it / G::STAGES) & 1), spin, fail, a.err)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t a0 = smem_u32(base + s * G::STAGE), b0 = a0 + G::A_BYTES;
          const bool amn = a.amn[kt < a.nk1 ? 0 : 1];
          const uint32_t idesc = instr_desc<BN>(amn);
#pragma unroll
          for (int kk = 0; kk < kBK / 16; ++kk)
            mma_bf16(d, amn ? sw128_mn_desc(a0 + kk * 2048) : sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32),
                     idesc, (kt > 0 || kk > 0) ? 1u : 0u);
          mma_commit(&empty[s]);
          issued = true;
          ++it;
        }
        if (ok) mma_commit(&acc_full[b]);
      }
      // every product issued has completed before the TMEM is freed
      if (issued) {
        mma_commit(&drain);
        if (!mbar_wait(&drain, 0, kSpin)) atomicExch(a.err, 2);
      }
    }
  } else {
    // ---- epilogue: warp (q, h) owns rows 32q .. 32q + 31 and chunk h % CHUNKS (32 columns) of the
    // tiles of group h / CHUNKS: with fewer than four chunks a tile, the groups take turns by tile ----
    const int e = warp - 2, q = warp & 3, h = e >> 2, g = h / G::CHUNKS, c = h % G::CHUNKS;
    float *st = epi + e * 32 * 33;
    const csrst_gemm_epilogue &ep = a.ep;
    int lt = 0;
    bool first = true;
    for (long long t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++lt) {
      if (lt % G::TG != g) continue;
      const int b = lt % G::NACC;
      int ok = 1;
      if (lane == 0)
        ok = stuck && first ? wait_role(&never, 0, spin, fail, a.err)
                            : wait_role(&acc_full[b], (uint32_t)((lt / G::NACC) & 1), spin, fail, a.err);
      first = false;
      if (!__shfl_sync(0xffffffffu, ok, 0)) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * BN + c * 32), v);
      tmem_wait(v);
      asm volatile("tcgen05.fence::before_thread_sync;");
      mbar_arrive(&acc_empty[b]);  // this warp's read of the accumulator is done: hand it back
      const long long r = t / a.tilesN;
      const int n0 = (int)(t % a.tilesN) * BN, m0 = (int)(r % a.tilesM) * kBM, z = (int)(r / a.tilesM);
      const int mrow = m0 + 32 * q, m = mrow + lane;
      const int ncol = n0 + c * 32, n = ncol + lane;
      const long long orow = row_part((long long)z * ep.sb, m, ep.md, ep.sm0, ep.sm1);
      const long long trow = ep.out16t ? row_part((long long)z * ep.tb, m, ep.tmd, ep.tm0, ep.tm1) : 0;
      const long long ocol = col_part(n, ep.nd, ep.sn0, ep.sn1);
      const long long tcol = ep.out16t ? col_part(n, ep.tnd, ep.tn0, ep.tn1) : 0;
      const float bm = (ep.bias_m && m < a.M) ? ep.bias_m[m] : 0.0f;
      float x[32];
      if (ep.bias) {
        const float bc = n < a.N ? ep.bias[n] : 0.0f;
#pragma unroll
        for (int j = 0; j < 32; ++j) x[j] = ep.alpha * __uint_as_float(v[j]) + __shfl_sync(0xffffffffu, bc, j) + bm;
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) x[j] = ep.alpha * __uint_as_float(v[j]) + bm;
      }
      if (a.vec && mrow + 32 <= a.M && ncol + 32 <= a.N)
        store_piece_vec(a, s_del, x, st, lane, __shfl_sync(0xffffffffu, orow, 0) + __shfl_sync(0xffffffffu, ocol, 0),
                        __shfl_sync(0xffffffffu, trow, 0) + __shfl_sync(0xffffffffu, tcol, 0));
      else
        store_piece(a, x, st, lane, mrow, ncol, orow, trow, ocol, tcol);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(G::TMEM_COLS));
  }
}

// Fills the launch's vector forms; a.vec = 1 when every output has one and
// the epilogue has no residual or accumulation (read-modify-write outputs
// keep the element-wise path).
void vector_forms(GemmArgs &a, int M, int N, int batch) {
  const csrst_gemm_epilogue &ep = a.ep;
  a.vec = 0;
  const MapDesc om{ep.md, ep.nd, ep.sb, ep.sm0, ep.sm1, ep.sn0, ep.sn1};
  const MapDesc tm{ep.tmd, ep.tnd, ep.tb, ep.tm0, ep.tm1, ep.tn0, ep.tn1};
  if (ep.res || ep.accumulate || !piece_offsets(om, a.del[0][0], a.del[0][1]) ||
      (ep.out16t && !piece_offsets(tm, a.del[1][0], a.del[1][1])))
    return;
  bool ok = true;
  const auto want = [&](int k, const void *p, int L, int mp) {
    if (!p) return;
    a.rs[k] = run_shape(a.del[mp][0], a.del[mp][1], L);
    ok = ok && a.rs[k].shape >= 0 && bases_aligned(mp ? tm : om, M, N, batch, p, L);
  };
  want(0, ep.pre, 4, 0);
  want(1, ep.out32, 4, 0);
  want(2, ep.out16, 8, 0);
  want(3, ep.out16t, 8, 1);
  a.vec = ok;
}

// Polls an mbarrier wait makes before it gives up (csrst_gemm_set_wait_limit).
long long g_wait_polls = kSpin;

// Tensor map of a K-major BF16 operand: K x rows (x batch when it has a
// batch stride), rows ld elements apart, box 64 x box_rows (x 1), 128-byte
// swizzle; rows past `rows` read as zero.
// mn: the operand is MN-major (K rows of `rows` contiguous elements, ld
// apart): rows x K (x batch), box 64 x 64.
bool encode_operand(CUtensorMap *m, int *rank3, const __nv_bfloat16 *p, int K, long long rows, long long ld,
                    long long stride, int batch, int box_rows, bool mn = false) {
  const EncodeTiled enc = tensor_map_encoder();
  if (!enc) return false;
  *rank3 = batch > 1 && stride != 0;
  const cuuint64_t dims[3] = {(cuuint64_t)(mn ? rows : K), (cuuint64_t)(mn ? K : rows), (cuuint64_t)batch};
  const cuuint64_t strides[2] = {(cuuint64_t)ld * 2, (cuuint64_t)stride * 2};
  const cuuint32_t box[3] = {(cuuint32_t)kBK, (cuuint32_t)(mn ? 64 : box_rows), 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, *rank3 ? 3 : 2, const_cast<__nv_bfloat16 *>(p), dims, strides,
             box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN>
int launch_gemm(const Seg &g0, const Seg &g1, int M, int N, int batch, const csrst_gemm_epilogue &ep, int *err,
                cudaStream_t s) {
  using G = Cfg<BN>;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                cudaSuccess)
    return CSRST_E_CUDA;
  static unsigned long long attr = 0;  // devices the shared-memory size was set on
  if (dev < 64 && !(attr >> dev & 1ull)) {
    if (cudaFuncSetAttribute(k_gemm<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM) != cudaSuccess)
      return CSRST_E_CUDA;
    attr |= 1ull << dev;
  }
  GemmArgs a{};
  a.ep = ep;
  a.err = err;
  a.spin = g_wait_polls;
  a.nk1 = g0.nk;
  a.nk2 = g1.nk;
  a.M = M;
  a.N = N;
  a.tilesM = (M + kBM - 1) / kBM;
  a.tilesN = (N + BN - 1) / BN;
  a.ntiles = (long long)batch * a.tilesM * a.tilesN;
  a.amn[0] = g0.amn;
  a.amn[1] = g1.amn;
  if (!encode_operand(&a.map[0], &a.rank3[0], g0.A, g0.nk * kBK, M, g0.lda, g0.sA, batch, kBM, g0.amn) ||
      !encode_operand(&a.map[1], &a.rank3[1], g0.B, g0.nk * kBK, N, g0.ldb, g0.sB, batch, BN))
    return CSRST_E_ARG;
  if (g1.nk && (!encode_operand(&a.map[2], &a.rank3[2], g1.A, g1.nk * kBK, M, g1.lda, g1.sA, batch, kBM, g1.amn) ||
                !encode_operand(&a.map[3], &a.rank3[3], g1.B, g1.nk * kBK, N, g1.ldb, g1.sB, batch, BN)))
    return CSRST_E_ARG;
  const int o_bytes = (ep.out32 || ep.res || ep.pre) ? 4 : 2;
  a.o_mfast = rows_fast(ep.md, ep.nd, ep.sm0, ep.sm1, ep.sn0, ep.sn1, o_bytes);
  a.t_mfast = ep.out16t ? rows_fast(ep.tmd, ep.tnd, ep.tm0, ep.tm1, ep.tn0, ep.tn1, 2) : 0;
  vector_forms(a, M, N, batch);
  const long long grid = a.ntiles < sms ? a.ntiles : sms;
  k_gemm<BN><<<(unsigned)grid, kThreads, G::SMEM, s>>>(a);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

bool seg_ok(const void *A, long long lda, long long sa, const void *B, long long ldb, long long sb, int K) {
  return A && B && K > 0 && K % kBK == 0 && lda % 8 == 0 && ldb % 8 == 0 && lda >= K && ldb >= K &&
         !((uintptr_t)A & 15) && !((uintptr_t)B & 15) && sa >= 0 && sb >= 0 && sa % 8 == 0 && sb % 8 == 0;
}

int gemm_dispatch(const Seg &g0, const Seg &g1, int M, int N, int batch, const csrst_gemm_epilogue *ep, int *err,
                  void *stream) {
  if (!ep || !err || M <= 0 || N <= 0 || batch <= 0 || N % 16 != 0 || ep->md <= 0 || ep->nd <= 0 ||
      (ep->out16t && (ep->tmd <= 0 || ep->tnd <= 0)))
    return CSRST_E_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (N % 128 == 0) return launch_gemm<128>(g0, g1, M, N, batch, *ep, err, s);
  if (N % 64 == 0) return launch_gemm<64>(g0, g1, M, N, batch, *ep, err, s);
  return launch_gemm<32>(g0, g1, M, N, batch, *ep, err, s);
}

}  // namespace
}  // namespace csrst

extern "C" int csrst_gemm_set_wait_limit(long long polls) {
  csrst::g_wait_polls = polls != 0 ? polls : csrst::kSpin;
  return CSRST_OK;
}

extern "C" int csrst_gemm_bf16(const void *A, long long lda, long long stride_a, const void *B, long long ldb,
                               long long stride_b, int M, int N, int K, int batch, const csrst_gemm_epilogue *ep,
                               int *err, void *stream) {
  using namespace csrst;
  if (!seg_ok(A, lda, stride_a, B, ldb, stride_b, K)) return CSRST_E_ARG;
  const Seg g0{static_cast<const __nv_bfloat16 *>(A), lda, stride_a, static_cast<const __nv_bfloat16 *>(B), ldb,
               stride_b, K / kBK, 0};
  const Seg g1{nullptr, 0, 0, nullptr, 0, 0, 0, 0};
  return gemm_dispatch(g0, g1, M, N, batch, ep, err, stream);
}

extern "C" int csrst_gemm_bf16_ex(const void *A, long long lda, long long stride_a, int a_mn_major, const void *B,
                                  long long ldb, long long stride_b, int M, int N, int K, int batch,
                                  const csrst_gemm_epilogue *ep, int *err, void *stream) {
  using namespace csrst;
  if (!a_mn_major) return csrst_gemm_bf16(A, lda, stride_a, B, ldb, stride_b, M, N, K, batch, ep, err, stream);
  // MN-major A: K rows of M elements, lda apart (the rules of seg_ok with M for K on A)
  if (!(A && B && K > 0 && K % kBK == 0 && lda % 8 == 0 && ldb % 8 == 0 && lda >= M && ldb >= K &&
        !((uintptr_t)A & 15) && !((uintptr_t)B & 15) && stride_a >= 0 && stride_b >= 0 && stride_a % 8 == 0 &&
        stride_b % 8 == 0))
    return CSRST_E_ARG;
  const Seg g0{static_cast<const __nv_bfloat16 *>(A), lda, stride_a, static_cast<const __nv_bfloat16 *>(B), ldb,
               stride_b, K / kBK, 1};
  const Seg g1{nullptr, 0, 0, nullptr, 0, 0, 0, 0};
  return gemm_dispatch(g0, g1, M, N, batch, ep, err, stream);
}

extern "C" int csrst_gemm_bf16_dual(const void *A1, long long lda1, long long stride_a1, const void *B1,
                                    long long ldb1, long long stride_b1, int K1, const void *A2, long long lda2,
                                    long long stride_a2, const void *B2, long long ldb2, long long stride_b2, int K2,
                                    int M, int N, int batch, const csrst_gemm_epilogue *ep, int *err, void *stream) {
  using namespace csrst;
  if (!seg_ok(A1, lda1, stride_a1, B1, ldb1, stride_b1, K1) || !seg_ok(A2, lda2, stride_a2, B2, ldb2, stride_b2, K2))
    return CSRST_E_ARG;
  const Seg g0{static_cast<const __nv_bfloat16 *>(A1), lda1, stride_a1, static_cast<const __nv_bfloat16 *>(B1), ldb1,
               stride_b1, K1 / kBK, 0};
  const Seg g1{static_cast<const __nv_bfloat16 *>(A2), lda2, stride_a2, static_cast<const __nv_bfloat16 *>(B2), ldb2,
               stride_b2, K2 / kBK, 0};
  return gemm_dispatch(g0, g1, M, N, batch, ep, err, stream);
}
