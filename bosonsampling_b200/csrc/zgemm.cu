// Grouped complex128 GEMM for the contraction-shaped steps of the BS update
// (the Theta block products, V = T Y / sigma, W = V^H C).
//
// FP64 has no tcgen05 kind on sm_100a, so this is a SIMT DFMA kernel: 64 x 64 output
// tile per CTA, K staged through shared memory 16 complex at a time with a register
// prefetch of the next slab, 4 x 4 complex accumulators per thread.  A thread owns
// rows ty + 16 i and columns tx + 16 j so shared-memory reads are conflict-free
// broadcasts and global stores are 256-byte coalesced rows.  All groups of one
// update go in one launch; a CTA finds its group by binary search over tile_start.
#include "common.cuh"
#include "kernels.h"

namespace {

constexpr int TM = 64, TN = 64, TK = 16, NT = 256;

__device__ __forceinline__ double2 ld2(const cplx* p) {
  return __ldg(reinterpret_cast<const double2*>(p));
}

__global__ __launch_bounds__(NT) void zgemm_grouped_kernel(const cplx* __restrict__ A,
                                                           const cplx* __restrict__ B,
                                                           cplx* __restrict__ C,
                                                           const double* __restrict__ scale,
                                                           const GemmGroup* __restrict__ groups,
                                                           int n_groups) {
  __shared__ double2 As[TK][TM + 1];
  __shared__ double2 Bs[TK][TN + 1];
  __shared__ GemmGroup g;
  const int tid = threadIdx.x;
  if (tid == 0) {
    int lo = 0, hi = n_groups - 1;
    const int t = blockIdx.x;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (groups[mid].tile_start <= t) lo = mid; else hi = mid - 1;
    }
    g = groups[lo];
  }
  __syncthreads();
  const int tile = blockIdx.x - g.tile_start;
  const int m0 = (tile / g.tiles_n) * TM;
  const int n0 = (tile % g.tiles_n) * TN;
  const int M = g.M, N = g.N, K = g.K;
  const cplx* a = A + g.a_off;
  const cplx* b = B + g.b_off;
  const double* ks = g.ks_off >= 0 ? scale + g.ks_off : nullptr;

  // global -> register staging coordinates (4 complex per thread per operand)
  // opA == 0: A[m][k] row-major, thread loads row ra, k = ka..ka+3
  // opA == 1: A stored [k][m], thread loads k = ka2, m = ma2..ma2+3 (conjugated)
  const int ra = tid >> 2, ka = (tid & 3) * 4;
  const int ka2 = tid >> 4, ma2 = (tid & 15) * 4;
  const int kb = tid >> 4, nb = (tid & 15) * 4;      // opB == 0: B[k][n]
  const int nb2 = tid >> 2, kb2 = (tid & 3) * 4;     // opB == 1: B stored [n][k]

  double2 ra_reg[4], rb_reg[4];

  auto load_a = [&](int k0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int m, k;
      if (g.opA == 0) { m = m0 + ra; k = k0 + ka + i; } else { m = m0 + ma2 + i; k = k0 + ka2; }
      double2 v = make_double2(0.0, 0.0);
      if (m < M && k < K) {
        v = (g.opA == 0) ? ld2(a + (int64_t)m * g.lda + k) : ld2(a + (int64_t)k * g.lda + m);
        if (g.opA == 1) v.y = -v.y;
        if (ks) { double s = __ldg(ks + k); v.x *= s; v.y *= s; }
      }
      ra_reg[i] = v;
    }
  };
  auto load_b = [&](int k0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int n, k;
      if (g.opB == 0) { k = k0 + kb; n = n0 + nb + i; } else { n = n0 + nb2; k = k0 + kb2 + i; }
      double2 v = make_double2(0.0, 0.0);
      if (n < N && k < K) {
        v = (g.opB == 0) ? ld2(b + (int64_t)k * g.ldb + n) : ld2(b + (int64_t)n * g.ldb + k);
        if (g.opB == 1) v.y = -v.y;
      }
      rb_reg[i] = v;
    }
  };
  auto store_ab = [&]() {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (g.opA == 0) As[ka + i][ra] = ra_reg[i]; else As[ka2][ma2 + i] = ra_reg[i];
      if (g.opB == 0) Bs[kb][nb + i] = rb_reg[i]; else Bs[kb2 + i][nb2] = rb_reg[i];
    }
  };

  const int ty = tid >> 4, tx = tid & 15;
  cplx acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = cmake(0.0, 0.0);

  load_a(0);
  load_b(0);
  for (int k0 = 0; k0 < K; k0 += TK) {
    __syncthreads();
    store_ab();
    __syncthreads();
    if (k0 + TK < K) { load_a(k0 + TK); load_b(k0 + TK); }
#pragma unroll 4
    for (int kk = 0; kk < TK; ++kk) {
      cplx av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        double2 t = As[kk][ty + 16 * i];
        av[i] = cmake(t.x, t.y);
        double2 u = Bs[kk][tx + 16 * i];
        bv[i] = cmake(u.x, u.y);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cfma(acc[i][j], av[i], bv[j]);
    }
  }

  const double* rs = g.rs_off >= 0 ? scale + g.rs_off : nullptr;
  const double* cs = g.cs_off >= 0 ? scale + g.cs_off : nullptr;
  cplx* c = C + g.c_off;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
    const double rsv = rs ? rs[m] : 1.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx + 16 * j;
      if (n >= N) continue;
      double f = rsv * (cs ? cs[n] : 1.0);
      cplx v = cscale(acc[i][j], f);
      cplx* p = c + (int64_t)m * g.ldc + n;
      if (g.beta) v = cadd(v, ldc(p));
      stc(p, v);
    }
  }
}

}  // namespace

int zgemm_tile_m() { return TM; }
int zgemm_tile_n() { return TN; }

cudaError_t launch_zgemm_grouped(const void* a, const void* b, void* c, const double* scale,
                                 const GemmGroup* groups_dev, int n_groups, int total_tiles,
                                 cudaStream_t s) {
  if (total_tiles <= 0 || n_groups <= 0) return cudaSuccess;
  zgemm_grouped_kernel<<<total_tiles, NT, 0, s>>>(
      reinterpret_cast<const cplx*>(a), reinterpret_cast<const cplx*>(b),
      reinterpret_cast<cplx*>(c), scale, groups_dev, n_groups);
  return cudaGetLastError();
}
