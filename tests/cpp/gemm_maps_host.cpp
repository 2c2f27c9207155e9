// Host build of the GEMM epilogue's store-order choice (csrst_b200/csrc/
// gemm_maps.h) for its CPU test: the same header, exposed over a C ABI.
#include "../../csrst_b200/csrc/gemm_maps.h"

// Vector form of a map for runs of L elements (shape 0..3 or -1; *fast_j the
// lane order), or -2 when the map is not a sum of row and column offsets over
// a 32 x 32 piece.  rdel / cdel receive the offsets (32 each).
extern "C" int gm_run_shape(int md, int nd, long long s0, long long s1, long long t0, long long t1, int L,
                            int *fast_j, long long *rdel, long long *cdel) {
  const csrst::MapDesc d{md, nd, 0, s0, s1, t0, t1};
  if (!csrst::piece_offsets(d, rdel, cdel)) return -2;
  const csrst::RunShape r = csrst::run_shape(rdel, cdel, L);
  *fast_j = r.fast_j;
  return r.shape;
}

extern "C" int gm_bases_aligned(int md, int nd, long long sb, long long s0, long long s1, long long t0, long long t1,
                                int M, int N, int batch, unsigned long long addr, int L) {
  const csrst::MapDesc d{md, nd, sb, s0, s1, t0, t1};
  return csrst::bases_aligned(d, M, N, batch, reinterpret_cast<const void *>(addr), L) ? 1 : 0;
}

extern "C" int gm_rows_fast(int md, int nd, long long s0, long long s1, long long t0, long long t1, int bytes) {
  return csrst::rows_fast(md, nd, s0, s1, t0, t1, bytes);
}
