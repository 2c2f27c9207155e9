// Host-side choice of the GEMM epilogue's store order (csrc/gemm.cu): for
// each output map, the sweep order of the element-wise path and the vector
// form of the 16-byte-run path.  Plain C++ (no CUDA types), so that the CPU
// tests compile it as it is.
#pragma once

#include <stdint.h>

#include <initializer_list>

namespace csrst {

// Vector stores.  Where an output map, restricted to a 32 x 32 piece of a
// tile that starts on multiples of 32, is index = base + rdel[i] + cdel[j]
// (row and column divisors that divide 32 or are multiples of it), the
// piece is written as runs of 16 bytes (L = 8 BF16 or 4 FP32 elements at
// consecutive indices), one per lane and store.  A run's elements lie, from
// its origin (i0, j0), at
//   shape 0: (i0, j0 + t)                      L columns of a row
//   shape 1: (i0 + t, j0)                      L rows of a column
//   shape 2: (i0 + t / 2, j0 + t % 2)          column pairs over L/2 rows
//   shape 3: (i0 + t % 2, j0 + t / 2)          row pairs over L/2 columns
// (the host finds the shape a map allows, checks every run of the piece and
// the 16-byte alignment of every piece's base, and orders the lanes along
// i or j, whichever keeps a warp's runs on fewer sectors).
struct RunShape {
  int shape;   // 0..3, or -1: the map has no vector form
  int fast_j;  // lanes take consecutive run origins along j (else along i)
};

// 32-byte sectors one warp's 32 stores touch under a map when its lanes take
// 32 consecutive rows (m_fast) or 32 consecutive columns of a tile at the
// origin, for elements of `bytes` bytes.
inline int warp_sectors(int md, int nd, long long sm0, long long sm1, long long sn0, long long sn1, int m_fast,
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
// rows than on consecutive columns: the epilogue then stores by columns.
inline int rows_fast(int md, int nd, long long sm0, long long sm1, long long sn0, long long sn1, int bytes) {
  return warp_sectors(md, nd, sm0, sm1, sn0, sn1, 1, bytes) < warp_sectors(md, nd, sm0, sm1, sn0, sn1, 0, bytes);
}

// An output map as the host checks it.
struct MapDesc {
  int md, nd;
  long long sb, s0, s1, t0, t1;  // batch; rows m/md, m%md; columns n/nd, n%nd
};

// Row and column offsets of a map over a 32 x 32 piece that starts on
// multiples of 32: the same for every such piece when each divisor divides
// 32 or is a multiple of it (false otherwise).
inline bool piece_offsets(const MapDesc &d, long long *rdel, long long *cdel) {
  if (!(32 % d.md == 0 || d.md % 32 == 0) || !(32 % d.nd == 0 || d.nd % 32 == 0)) return false;
  for (int i = 0; i < 32; ++i) {
    rdel[i] = (long long)(i / d.md) * d.s0 + (long long)(i % d.md) * d.s1;
    cdel[i] = (long long)(i / d.nd) * d.t0 + (long long)(i % d.nd) * d.t1;
  }
  return true;
}

inline long long mod_pos(long long a, long long m) { return ((a % m) + m) % m; }

// Every piece's base index a multiple of L (16 bytes) and the output 16-byte
// aligned.  A piece starts at row 32p: its row part advances by (32 / md) s0
// per piece when md divides 32, else by 32 s1 within a block of md rows and
// by s0 between blocks; the same for columns.
inline bool bases_aligned(const MapDesc &d, int M, int N, int batch, const void *p, int L) {
  if ((uintptr_t)p % 16 || (batch > 1 && mod_pos(d.sb, L))) return false;
  if (d.md <= 32 ? mod_pos((32 / d.md) * d.s0, L) : (mod_pos(32 * d.s1, L) || (M > d.md && mod_pos(d.s0, L))))
    return false;
  if (d.nd <= 32 ? mod_pos((32 / d.nd) * d.t0, L) : (mod_pos(32 * d.t1, L) || (N > d.nd && mod_pos(d.t0, L))))
    return false;
  return true;
}

// The first run shape (0..3) whose every run over the piece covers L
// consecutive indices from a multiple of L, and the lane order that keeps a
// warp's first 32 runs on fewer 32-byte sectors; shape -1 if none.
inline RunShape run_shape(const long long *rdel, const long long *cdel, int L) {
  for (int S = 0; S < 4; ++S) {
    const int ri = S == 0 ? 1 : S == 1 ? L : S == 2 ? L / 2 : 2, rj = S == 0 ? L : S == 1 ? 1 : S == 2 ? 2 : L / 2;
    bool ok = true;
    for (int oi = 0; oi < 32 && ok; oi += ri)
      for (int oj = 0; oj < 32 && ok; oj += rj) {
        const long long o = rdel[oi] + cdel[oj];
        ok = mod_pos(o, L) == 0;
        for (int t = 0; t < L && ok; ++t) {
          const int i = oi + (S == 0 ? 0 : S == 1 ? t : S == 2 ? t / 2 : t % 2);
          const int j = oj + (S == 0 ? t : S == 1 ? 0 : S == 2 ? t % 2 : t / 2);
          ok = rdel[i] + cdel[j] == o + t;
        }
      }
    if (!ok) continue;
    const int ni = 32 / ri, nj = 32 / rj;
    int best = 1 << 30, fast = 1;
    for (int f = 1; f >= 0; --f) {
      int cost = 0;
      for (const int unit : {32, 128}) {  // sectors, then 128-byte lines as the tie-break
        long long seen_at[32];
        int k = 0;
        for (int r = 0; r < 32; ++r) {
          const int oi = (f ? r / nj : r % ni) * ri, oj = (f ? r % nj : r / ni) * rj;
          const long long b = (rdel[oi] + cdel[oj]) * (16 / L);
          const long long s = (b - mod_pos(b, unit)) / unit;
          bool seen = false;
          for (int q = 0; q < k; ++q) seen |= seen_at[q] == s;
          if (!seen) seen_at[k++] = s;
        }
        cost = cost * 64 + k;
      }
      if (cost < best) best = cost, fast = f;
    }
    return RunShape{S, fast};
  }
  return RunShape{-1, 0};
}

}  // namespace csrst
