// BF16 tensor-core GEMM on the 5th-generation tensor cores (tcgen05) for the
// surrogate network: C[M, N] = A[M, K] . B[N, K]^T with FP32 accumulation, both
// operands K-major (rows contiguous along K), batched over blockIdx.z.
//
// One CTA of 128 threads computes a 128 x BN tile:
//   - the A and B tiles of 64 K-columns are copied to shared memory with
//     cp.async in two stages, in the tensor core's canonical K-major layout
//     without swizzle: 8-row x 16-byte core matrices, the 8-row groups 128 B
//     apart (SBO) and the 8-element K chunks a whole tile column apart (LBO);
//   - one thread issues four tcgen05.mma (M = 128, N = BN, K = 16 each) per
//     stage into an FP32 accumulator in tensor memory (TMEM) and commits them
//     to the stage's mbarrier, which frees the stage for the next copy;
//   - the epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM
//     lanes 32w .. 32w + 31, i.e. rows) into an FP32 staging tile in the
//     freed operand stages, then writes FP32 and/or BF16 outputs through
//     affine index maps (transposed and mode-major layouts come out
//     directly), each swept in the order - along rows or along columns -
//     that puts a warp's stores next to each other under its map.
// Waits on mbarriers are bounded (a launch parameter, csrst_gemm_set_wait_limit):
// a wait that gives up sets *err and skips the epilogue; the kernel then waits,
// with the default bound, for the tensor-core work it has issued and for its
// copies in flight before it frees the TMEM and returns, so that nothing
// still writes into TMEM or shared memory it no longer owns.
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/csrst.h"
#include "tma.cuh"

namespace csrst {
namespace {

constexpr int kBM = 128, kBK = 64, kThreads = 128;
constexpr long long kSpin = 1ll << 24;  // default mbarrier polls before a wait gives up

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Shared-memory matrix descriptor, K-major, no swizzle (version 1 for sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version
  return d;                // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = BN.
template <int BN>
__device__ __forceinline__ uint32_t instr_desc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

// Copies rows [r0, r0 + R) x K-columns [k0, k0 + 64) of a K-major matrix into
// the canonical layout: element (r, k) at ((k / 8) * (R / 8) + r / 8) * 128 +
// (r % 8) * 16 + (k % 8) * 2 bytes.  Rows at or beyond `rows` are zero.
template <int R>
__device__ __forceinline__ void load_tile(uint8_t *dst, const __nv_bfloat16 *src, long long ld, int r0, int rows,
                                          int k0) {
  constexpr int chunks = R * (kBK / 8);  // 16-byte pieces
#pragma unroll
  for (int c = threadIdx.x; c < chunks; c += kThreads) {
    const int r = c % 8 + 8 * ((c / 8) % (R / 8));  // row: 8 consecutive threads take one core matrix column
    const int kc = c / R;                           // K chunk
    uint8_t *d = dst + ((kc * (R / 8) + r / 8) * 128 + (r % 8) * 16);
    if (r0 + r < rows) {
      cp_async16(d, src + (long long)(r0 + r) * ld + k0 + kc * 8);
    } else {
      *reinterpret_cast<uint4 *>(d) = make_uint4(0, 0, 0, 0);
    }
  }
}

// Affine output index of tile element (m, n) of batch z under a map.
__device__ __forceinline__ long long map_index(long long zb, int m, int n, int md, int nd, long long s0, long long s1,
                                               long long t0, long long t1) {
  return zb + (long long)(m / md) * s0 + (long long)(m % md) * s1 + (long long)(n / nd) * t0 +
         (long long)(n % nd) * t1;
}

// Visits the tile's (row, column) pairs in groups of eight per thread, so
// that the 32 lanes of a warp take consecutive columns (m_fast == 0) or
// consecutive rows (m_fast == 1): the order in which the output map puts
// neighbouring lanes next to each other.  A group's reads of global memory
// (residual, accumulated output) are all issued before its first store.
constexpr int kGroup = 8;
template <int BN, class F>
__device__ __forceinline__ void tile_order(int m_fast, F &&f) {
  int rr[kGroup], cc[kGroup];
  if (m_fast) {
    for (int c = 0; c < BN; c += kGroup) {
#pragma unroll
      for (int j = 0; j < kGroup; ++j) rr[j] = threadIdx.x, cc[j] = c + j;
      f(rr, cc);
    }
  } else {
    constexpr int kRows = kThreads / BN;  // rows per sweep of the block
    const int c = threadIdx.x % BN;
    for (int r = threadIdx.x / BN; r < kBM; r += kGroup * kRows) {
#pragma unroll
      for (int j = 0; j < kGroup; ++j) rr[j] = r + j * kRows, cc[j] = c;
      f(rr, cc);
    }
  }
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
};

template <int BN>
__global__ void __launch_bounds__(kThreads) k_gemm(Seg g0, Seg g1, int M, int N, csrst_gemm_epilogue ep, int *err,
                                                   int o_mfast, int t_mfast, long long spin) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar[3];  // MMA commits of the two stages; bar[2]: nothing arrives on it
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail, s_last;  // a wait gave up; the last MMA commit issued
  constexpr int kA = kBM * kBK * 2, kB = BN * kBK * 2, kStage = kA + kB;
  uint8_t *base = smem + ((1024 - (smem_u32(smem) & 1023)) & 1023);
  const int z = blockIdx.z, m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN;
  g0.A += (long long)z * g0.sA;
  g0.B += (long long)z * g0.sB;
  if (g1.nk) {
    g1.A += (long long)z * g1.sA;
    g1.B += (long long)z * g1.sB;
  }
  // copies K tile kt (of either segment) into a stage
  auto load_k = [&](uint8_t *stage, int kt) {
    const Seg &g = kt < g0.nk ? g0 : g1;
    const int k0 = (kt < g0.nk ? kt : kt - g0.nk) * kBK;
    load_tile<kBM>(stage, g.A, g.lda, m0, M, k0);
    load_tile<BN>(stage + kBM * kBK * 2, g.B, g.ldb, n0, N, k0);
  };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == 0) {  // TMEM: BN FP32 columns x 128 lanes
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
    s_last = -1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const int nk = g0.nk + g1.nk;
  // spin < 0: the first wait in the loop is on bar[2], which nothing
  // completes, with -spin polls (the stuck wait the error path is tested with)
  const bool stuck = spin < 0;
  if (stuck) spin = -spin;

  load_k(base, 0);
  cp_async_commit();
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt & 1;
    if (kt + 1 < nk) {
      const int s1 = (kt + 1) & 1;
      if (kt >= 1) {  // the MMAs of tile kt - 1 still read stage s1
        uint64_t *wb = stuck && kt == 1 ? &bar[2] : &bar[s1];
        if (threadIdx.x == 0 && !mbar_wait(wb, stuck && kt == 1 ? 0u : ((kt - 1) >> 1) & 1, spin)) {
          s_fail = 1;
          s_last = kt - 1;
        }
        __syncthreads();
        if (s_fail) break;
      }
      load_k(base + s1 * kStage, kt + 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // copies visible to the tensor core
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = smem_u32(base + s * kStage), b0 = a0 + kA;
#pragma unroll
      for (int kk = 0; kk < kBK / 16; ++kk) {
        // K = 16 is two 8-element chunks: advance by two chunk strides (LBO)
        const uint64_t da = smem_desc(a0 + kk * 2 * (kBM / 8) * 128, (kBM / 8) * 128, 128);
        const uint64_t db = smem_desc(b0 + kk * 2 * (BN / 8) * 128, (BN / 8) * 128, 128);
        mma_bf16(tmem, da, db, instr_desc<BN>(), (kt > 0 || kk > 0) ? 1u : 0u);
      }
      mma_commit(&bar[s]);
    }
  }
  // the last commit covers every MMA issued before it
  if (threadIdx.x == 0 && !s_fail && nk > 0 && !mbar_wait(&bar[(nk - 1) & 1], ((nk - 1) >> 1) & 1, spin)) {
    s_fail = 1;
    s_last = nk - 1;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (s_fail) {
    // the MMAs issued so far complete in order: wait for the last commit with
    // the default bound before the TMEM they write is freed
    if (threadIdx.x == 0) {
      atomicExch(err, 1);
      if (s_last >= 0 && !mbar_wait(&bar[s_last & 1], (s_last >> 1) & 1, kSpin)) atomicExch(err, 2);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
  } else {
    // The MMAs have completed and every copy has landed: the operand stages
    // become an FP32 staging tile [128][BN + 1] (the +1 keeps both row- and
    // column-wise sweeps free of bank conflicts).
    constexpr int LD = BN + 1;
    float *tile = reinterpret_cast<float *>(base);
    const int r = warp * 32 + lane;
    for (int c0 = 0; c0 < BN; c0 += 16) {
      uint32_t v[16];
      const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(ta));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 16; ++j) tile[r * LD + c0 + j] = __uint_as_float(v[j]);
    }
    // Each map's address is a row part plus a column part: both computed once
    // per tile (128 + BN divisions instead of two per element).
    __shared__ long long s_row[2][kBM], s_col[2][BN];
    {
      const int m = m0 + threadIdx.x;
      s_row[0][threadIdx.x] = (long long)z * ep.sb + map_index(0, m, 0, ep.md, ep.nd, ep.sm0, ep.sm1, 0, 0);
      if (ep.out16t)
        s_row[1][threadIdx.x] = (long long)z * ep.tb + map_index(0, m, 0, ep.tmd, ep.tnd, ep.tm0, ep.tm1, 0, 0);
      if (threadIdx.x < BN) {
        const int n = n0 + threadIdx.x;
        s_col[0][threadIdx.x] = map_index(0, 0, n, 1, ep.nd, 0, 0, ep.sn0, ep.sn1);
        if (ep.out16t) s_col[1][threadIdx.x] = map_index(0, 0, n, 1, ep.tnd, 0, 0, ep.tn0, ep.tn1);
      }
    }
    __syncthreads();
    // outputs through the primary map, in the order that map makes contiguous
    tile_order<BN>(o_mfast, [&](const int *rr, const int *cc) {
      long long o[kGroup];
      bool ok[kGroup];
      float rv[kGroup], ov[kGroup];
#pragma unroll
      for (int j = 0; j < kGroup; ++j) {
        ok[j] = m0 + rr[j] < M && n0 + cc[j] < N;
        o[j] = s_row[0][rr[j]] + s_col[0][cc[j]];
      }
#pragma unroll
      for (int j = 0; j < kGroup; ++j) {
        rv[j] = (ok[j] && ep.res) ? ep.res[o[j]] : 0.0f;
        ov[j] = (ok[j] && ep.out32 && ep.accumulate) ? ep.out32[o[j]] : 0.0f;
      }
#pragma unroll
      for (int j = 0; j < kGroup; ++j) {
        if (!ok[j]) continue;
        float x = ep.alpha * tile[rr[j] * LD + cc[j]];
        if (ep.bias) x += ep.bias[n0 + cc[j]];
        if (ep.bias_m) x += ep.bias_m[m0 + rr[j]];
        if (ep.res) x += rv[j];
        if (ep.pre) ep.pre[o[j]] = x;
        if (ep.act == 1) x = gelu(x);
        if (ep.out32) ep.out32[o[j]] = ep.accumulate ? ov[j] + x : x;
        if (ep.out16) reinterpret_cast<__nv_bfloat16 *>(ep.out16)[o[j]] = __float2bfloat16(x);
        tile[rr[j] * LD + cc[j]] = x;
      }
    });
    if (ep.out16t) {  // the second BF16 copy through its own map and order
      __syncthreads();
      tile_order<BN>(t_mfast, [&](const int *rr, const int *cc) {
#pragma unroll
        for (int j = 0; j < kGroup; ++j) {
          if (m0 + rr[j] >= M || n0 + cc[j] >= N) continue;
          reinterpret_cast<__nv_bfloat16 *>(ep.out16t)[s_row[1][rr[j]] + s_col[1][cc[j]]] =
              __float2bfloat16(tile[rr[j] * LD + cc[j]]);
        }
      });
    }
  }
  cp_async_wait<0>();  // nothing still landing in shared memory (an early exit leaves copies in flight)
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

// 32-byte sectors one warp's 32 stores touch under a map when its lanes take
// 32 consecutive rows (m_fast) or 32 consecutive columns of a tile at the
// origin, for elements of `bytes` bytes.
int warp_sectors(int md, int nd, long long sm0, long long sm1, long long sn0, long long sn1, int m_fast,
                 int bytes) {
  long long sec[32];
  int k = 0;
  for (int i = 0; i < 32; ++i) {
    const int m = m_fast ? i : 0, n = m_fast ? 0 : i;
    const long long a = ((long long)(m / md) * sm0 + (long long)(m % md) * sm1 + (long long)(n / nd) * sn0 +
                         (long long)(n % nd) * sn1) * bytes;
    const long long s = a >= 0 ? a / 32 : -((-a + 31) / 32);
    bool seen = false;
    for (int j = 0; j < k; ++j) seen |= sec[j] == s;
    if (!seen) sec[k++] = s;
  }
  return k;
}

// 1 when a warp's stores touch fewer sectors with its lanes on consecutive
// rows than on consecutive columns: the epilogue then sweeps the tile by rows.
int rows_fast(int md, int nd, long long sm0, long long sm1, long long sn0, long long sn1, int bytes) {
  return warp_sectors(md, nd, sm0, sm1, sn0, sn1, 1, bytes) < warp_sectors(md, nd, sm0, sm1, sn0, sn1, 0, bytes);
}

// Polls an mbarrier wait makes before it gives up (csrst_gemm_set_wait_limit).
long long g_wait_polls = kSpin;

template <int BN>
int launch_gemm(const Seg &g0, const Seg &g1, int M, int N, int batch, const csrst_gemm_epilogue &ep, int *err,
                cudaStream_t s) {
  // operand stages, or the FP32 staging tile of the epilogue if larger, plus alignment slack
  const int stages = 2 * (kBM * kBK * 2 + BN * kBK * 2), staging = kBM * (BN + 1) * 4;
  const int smem = (stages > staging ? stages : staging) + 1024;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_gemm<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return CSRST_E_CUDA;
    attr = true;
  }
  dim3 grid((N + BN - 1) / BN, (M + kBM - 1) / kBM, batch);
  const int o_bytes = (ep.out32 || ep.res || ep.pre) ? 4 : 2;
  const int o_mfast = rows_fast(ep.md, ep.nd, ep.sm0, ep.sm1, ep.sn0, ep.sn1, o_bytes);
  const int t_mfast = ep.out16t ? rows_fast(ep.tmd, ep.tnd, ep.tm0, ep.tm1, ep.tn0, ep.tn1, 2) : 0;
  k_gemm<BN><<<grid, kThreads, smem, s>>>(g0, g1, M, N, ep, err, o_mfast, t_mfast, g_wait_polls);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

bool seg_ok(const void *A, long long lda, long long sa, const void *B, long long ldb, long long sb, int K) {
  return A && B && K > 0 && K % kBK == 0 && lda % 8 == 0 && ldb % 8 == 0 && lda >= K && ldb >= K &&
         !((uintptr_t)A & 15) && !((uintptr_t)B & 15) && sa % 8 == 0 && sb % 8 == 0;
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
               stride_b, K / kBK};
  const Seg g1{nullptr, 0, 0, nullptr, 0, 0, 0};
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
               stride_b1, K1 / kBK};
  const Seg g1{static_cast<const __nv_bfloat16 *>(A2), lda2, stride_a2, static_cast<const __nv_bfloat16 *>(B2), ldb2,
               stride_b2, K2 / kBK};
  return gemm_dispatch(g0, g1, M, N, batch, ep, err, stream);
}
