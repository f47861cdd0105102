// Trace and single-mode photon-number marginals of the MPO, in FP64.
//
// Generalises summary.Probability (src/summary.py:11-26): the trace keeps, on every
// bond, only entries whose ket and bra charges agree (and Lambda > 0), and contracts
// the Gamma chain.  Right environments R_b (b = n..0) and left environments L_b
// (b = 0..n) are masked matrix-vector products; the marginal of mode i is
//     P_i(k) = sum_{a, j : c0(a) - c0(j) = k} L_i[a] Gamma_i[a, j] R_{i+1}[j].
// All reductions run in a fixed order (no floating-point atomics), so results are
// bit-reproducible from run to run.
#include "common.cuh"
#include "kernels.h"

namespace {

__device__ __forceinline__ bool diag_ok(int2 c, double lam, int d) {
  return c.x < d && c.x == c.y && lam > 0.0;
}

__global__ void env_init_kernel(int d, int chi, const int2* __restrict__ cb,
                                const double* __restrict__ lam, cplx* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < chi; i += gridDim.x * blockDim.x)
    v[i] = diag_ok(cb[i], lam[i], d) ? cmake(1.0, 0.0) : cmake(0.0, 0.0);
}

// r_out[a] = mask_b(a) * sum_j gamma[a][j] r_next[j]   (one warp per row)
__global__ void env_right_kernel(int d, int chi, const cplx* __restrict__ g,
                                 const int2* __restrict__ cb, const double* __restrict__ lam,
                                 const cplx* __restrict__ rn, cplx* __restrict__ ro, int rows,
                                 int cols) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= chi) return;
  const int a = warp;
  cplx acc = cmake(0.0, 0.0);
  if (a < rows && diag_ok(cb[a], lam[a], d)) {
    for (int j = lane; j < cols; j += 32) cfma(acc, ldc(g + (int64_t)a * chi + j), ldc(rn + j));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  if (lane == 0) ro[a] = acc;
}

// l_out[j] = mask_{b+1}(j) * sum_a l_cur[a] gamma[a][j]; columns split over the
// x-dimension, rows over 8 thread rows per block reduced in shared memory
__global__ void env_left_kernel(int d, int chi, const cplx* __restrict__ g,
                                const int2* __restrict__ cn, const double* __restrict__ lamn,
                                const cplx* __restrict__ lc, cplx* __restrict__ lo, int rows,
                                int cols) {
  __shared__ double2 part[8][33];
  const int j = blockIdx.x * 32 + threadIdx.x;
  cplx acc = cmake(0.0, 0.0);
  if (j < cols) {
    for (int a = threadIdx.y; a < rows; a += 8) cfma(acc, ldc(lc + a), ldc(g + (int64_t)a * chi + j));
  }
  part[threadIdx.y][threadIdx.x] = make_double2(acc.x, acc.y);
  __syncthreads();
  if (threadIdx.y == 0 && j < chi) {
    cplx s = cmake(0.0, 0.0);
    for (int y = 0; y < 8; ++y) s = cadd(s, cmake(part[y][threadIdx.x].x, part[y][threadIdx.x].y));
    lo[j] = (j < cols && diag_ok(cn[j], lamn[j], d)) ? s : cmake(0.0, 0.0);
  }
}

// part[site][chunk][k] = sum over rows of the chunk; one CTA per (site, chunk)
constexpr int MNT = 256;
__global__ __launch_bounds__(MNT) void marginal_kernel(int n, int d, int chi,
                                                        const cplx* __restrict__ gamma,
                                                        const int2* __restrict__ charge,
                                                        const cplx* __restrict__ envl,
                                                        const cplx* __restrict__ envr,
                                                        const int* __restrict__ dims,
                                                        int chunk_rows, cplx* __restrict__ part) {
  __shared__ double2 red[MNT / 32][BSMPO_MAX_D];
  const int site = blockIdx.y, chunk = blockIdx.x;
  const int nchunk = gridDim.x;
  const int rows = dims[site], cols = dims[site + 1];
  const cplx* g = gamma + (int64_t)site * chi * chi;
  const int2* ca = charge + (int64_t)site * chi;
  const int2* cj = charge + (int64_t)(site + 1) * chi;
  const cplx* L = envl + (int64_t)site * chi;
  const cplx* R = envr + (int64_t)(site + 1) * chi;
  cplx acc[BSMPO_MAX_D];
#pragma unroll
  for (int k = 0; k < BSMPO_MAX_D; ++k) acc[k] = cmake(0.0, 0.0);
  const int r0 = chunk * chunk_rows, r1 = min(rows, r0 + chunk_rows);
  for (int a = r0; a < r1; ++a) {
    const cplx la = ldc(L + a);
    if (la.x == 0.0 && la.y == 0.0) continue;
    const int ka = ca[a].x;
    for (int j = threadIdx.x; j < cols; j += MNT) {
      const int k = ka - cj[j].x;
      if (k < 0 || k >= d) continue;
      const cplx v = cmul(cmul(la, ldc(g + (int64_t)a * chi + j)), ldc(R + j));
#pragma unroll
      for (int kk = 0; kk < BSMPO_MAX_D; ++kk)
        if (kk == k) acc[kk] = cadd(acc[kk], v);
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < BSMPO_MAX_D; ++k) {
    double x = acc[k].x, y = acc[k].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, o);
      y += __shfl_xor_sync(0xffffffffu, y, o);
    }
    if (lane == 0) red[wid][k] = make_double2(x, y);
  }
  __syncthreads();
  if (threadIdx.x < d) {
    cplx s = cmake(0.0, 0.0);
    for (int w = 0; w < MNT / 32; ++w)
      s = cadd(s, cmake(red[w][threadIdx.x].x, red[w][threadIdx.x].y));
    part[((int64_t)site * nchunk + chunk) * d + threadIdx.x] = s;
  }
}

__global__ void marginal_reduce_kernel(int n, int d, int nchunk, const cplx* __restrict__ part,
                                       cplx* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * d) return;
  const int site = e / d, k = e % d;
  cplx s = cmake(0.0, 0.0);
  for (int c = 0; c < nchunk; ++c) s = cadd(s, part[((int64_t)site * nchunk + c) * d + k]);
  out[e] = s;
}

__global__ void sum_vector_kernel(const cplx* __restrict__ v, int len, cplx* __restrict__ out) {
  __shared__ double2 red[256];
  cplx acc = cmake(0.0, 0.0);
  for (int i = threadIdx.x; i < len; i += 256) acc = cadd(acc, v[i]);
  red[threadIdx.x] = make_double2(acc.x, acc.y);
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[threadIdx.x].x += red[threadIdx.x + s].x;
      red[threadIdx.x].y += red[threadIdx.x + s].y;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = cmake(red[0].x, red[0].y);
}

}  // namespace

cudaError_t launch_env_init(int d, int chi, const int* charge_b, const double* lam_b, void* v,
                            cudaStream_t s) {
  env_init_kernel<<<ceil_div(chi, 256), 256, 0, s>>>(d, chi, reinterpret_cast<const int2*>(charge_b),
                                                     lam_b, reinterpret_cast<cplx*>(v));
  return cudaGetLastError();
}

cudaError_t launch_env_right_step(int d, int chi, const void* gamma_b, const int* charge_b,
                                  const double* lam_b, const void* r_next, void* r_out, int rows,
                                  int cols, cudaStream_t s) {
  env_right_kernel<<<ceil_div(chi * 32, 256), 256, 0, s>>>(
      d, chi, reinterpret_cast<const cplx*>(gamma_b), reinterpret_cast<const int2*>(charge_b),
      lam_b, reinterpret_cast<const cplx*>(r_next), reinterpret_cast<cplx*>(r_out), rows, cols);
  return cudaGetLastError();
}

cudaError_t launch_env_left_step(int d, int chi, const void* gamma_b, const int* charge_next,
                                 const double* lam_next, const void* l_cur, void* l_out, int rows,
                                 int cols, cudaStream_t s) {
  dim3 block(32, 8);
  env_left_kernel<<<ceil_div(chi, 32), block, 0, s>>>(
      d, chi, reinterpret_cast<const cplx*>(gamma_b), reinterpret_cast<const int2*>(charge_next),
      lam_next, reinterpret_cast<const cplx*>(l_cur), reinterpret_cast<cplx*>(l_out), rows, cols);
  return cudaGetLastError();
}

cudaError_t launch_marginals(int n, int d, int chi, const void* gamma, const int* charge,
                             const void* env_l, const void* env_r, const int* dims, void* part,
                             int chunk_rows, void* out, cudaStream_t s) {
  const int nchunk = ceil_div(chi, chunk_rows);
  dim3 grid(nchunk, n);
  marginal_kernel<<<grid, MNT, 0, s>>>(n, d, chi, reinterpret_cast<const cplx*>(gamma),
                                       reinterpret_cast<const int2*>(charge),
                                       reinterpret_cast<const cplx*>(env_l),
                                       reinterpret_cast<const cplx*>(env_r), dims, chunk_rows,
                                       reinterpret_cast<cplx*>(part));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  marginal_reduce_kernel<<<ceil_div(n * d, 128), 128, 0, s>>>(
      n, d, nchunk, reinterpret_cast<const cplx*>(part), reinterpret_cast<cplx*>(out));
  return cudaGetLastError();
}

cudaError_t launch_sum_vector(const void* v, int len, void* out, cudaStream_t s) {
  sum_vector_kernel<<<1, 256, 0, s>>>(reinterpret_cast<const cplx*>(v), len,
                                      reinterpret_cast<cplx*>(out));
  return cudaGetLastError();
}
