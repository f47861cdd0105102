// Standalone single-sector contraction: the drop-in for cuda_kernels.update_MPO
// (src/cuda_kernels.py:101-127) and its kernel (src/update_MPO_kernel.cu:193-733).
//
//   C[l][r] = sum_c Glc[l][c] Gcr[c][r] U(cl0-cc0, cc0-cr0, cl0-q0(c)) conj U(cl1-cc1, cc1-cr1, cl1-q1(c))
//
// with each charge taken per row / column / centre entry (so no x8 alignment
// padding or centre-charge change list is needed) and the term zero unless every U
// index lies in [0, d).  FP64, 16 x 16 output tile per CTA, centre index staged
// through shared memory 16 at a time.  The whole-BS path (bsmpo_bs_update) does not
// use these kernels; it contracts charge blocks as GEMMs instead.
#include "common.cuh"
#include "kernels.h"

namespace {

constexpr int CT = 16;

__global__ void contract_sector_kernel(int d, int cc0, int cc1, const cplx* __restrict__ u,
                                       const cplx* __restrict__ glc, const cplx* __restrict__ gcr,
                                       const int2* __restrict__ cl, const int2* __restrict__ cc,
                                       const int2* __restrict__ cr, int len_l, int len_c,
                                       int len_r, cplx* __restrict__ out) {
  __shared__ cplx us[BSMPO_MAX_D * BSMPO_MAX_D * BSMPO_MAX_D];
  __shared__ cplx ga[CT][CT + 1], gb[CT][CT + 1];
  __shared__ int2 qc[CT];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * CT + tx;
  const int d3 = d * d * d;
  for (int i = tid; i < d3; i += CT * CT) us[i] = u[i];
  const int l = blockIdx.y * CT + ty, r = blockIdx.x * CT + tx;
  const int2 a = l < len_l ? cl[l] : make_int2(d, d);
  const int2 b = r < len_r ? cr[r] : make_int2(d, d);
  const bool row_ok = a.x < d && a.y < d && a.x >= cc0 && a.y >= cc1;
  const bool col_ok = b.x < d && b.y < d && b.x <= cc0 && b.y <= cc1;
  cplx acc = cmake(0.0, 0.0);
  for (int c0 = 0; c0 < len_c; c0 += CT) {
    __syncthreads();
    {
      const int lr = blockIdx.y * CT + ty, cc_ = c0 + tx;
      ga[ty][tx] = (lr < len_l && cc_ < len_c) ? ldc(glc + (int64_t)lr * len_c + cc_) : cmake(0.0, 0.0);
      const int cr_ = c0 + ty, rc = blockIdx.x * CT + tx;
      gb[ty][tx] = (cr_ < len_c && rc < len_r) ? ldc(gcr + (int64_t)cr_ * len_r + rc) : cmake(0.0, 0.0);
      if (ty == 0) qc[tx] = (c0 + tx < len_c) ? cc[c0 + tx] : make_int2(d, d);
    }
    __syncthreads();
    if (!(row_ok && col_ok)) continue;
    for (int j = 0; j < CT; ++j) {
      const int2 q = qc[j];
      if (q.x >= d || q.y >= d) continue;
      if (!(a.x >= q.x && q.x >= b.x && a.y >= q.y && q.y >= b.y)) continue;
      const cplx u0 = us[((a.x - cc0) * d + (cc0 - b.x)) * d + (a.x - q.x)];
      const cplx u1 = us[((a.y - cc1) * d + (cc1 - b.y)) * d + (a.y - q.y)];
      const cplx w = cmulc(u0, u1);
      cfma(acc, w, cmul(ga[ty][j], gb[j][tx]));
    }
  }
  if (l < len_l && r < len_r) out[(int64_t)l * len_r + r] = acc;
}

// The pure-state (MPS) variant: the drop-in for cuda_kernels.update_MPS
// (src/cuda_kernels.py:72-90) and its kernel (src/update_kernel.cu:193-769), one charge
// per bond index:
//   T[l][r] = LL[l] LR[r] sum_c LC[c] Glc[l][c] Gcr[c][r] U(cl - tau, tau - cr, cl - q(c)),
// the term zero unless cl >= q(c) >= cr and every U index lies in [0, d).  The reference
// reloads LC in tiles of 256 centre indices and, on its last partial tile, from offset 0
// (src/update_kernel.cu:632-638) -- a quirk for k > 256; here LC[c] is read per index.
__global__ void contract_mps_kernel(int d, int tau, const cplx* __restrict__ u,
                                    const cplx* __restrict__ glc, const cplx* __restrict__ gcr,
                                    const double* __restrict__ ll, const double* __restrict__ lc,
                                    const double* __restrict__ lr, const int* __restrict__ cl,
                                    const int* __restrict__ cc, const int* __restrict__ cr, int len_l,
                                    int len_c, int len_r, cplx* __restrict__ out) {
  __shared__ cplx us[BSMPO_MAX_D * BSMPO_MAX_D * BSMPO_MAX_D];
  __shared__ cplx ga[CT][CT + 1], gb[CT][CT + 1];
  __shared__ int qc[CT];
  __shared__ double lcs[CT];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * CT + tx;
  const int d3 = d * d * d;
  for (int i = tid; i < d3; i += CT * CT) us[i] = u[i];
  const int l = blockIdx.y * CT + ty, r = blockIdx.x * CT + tx;
  const int a = l < len_l ? cl[l] : -1;
  const int b = r < len_r ? cr[r] : -1;
  const bool ok = a >= 0 && b >= 0 && a - tau >= 0 && a - tau < d && tau - b >= 0 && tau - b < d;
  cplx acc = cmake(0.0, 0.0);
  for (int c0 = 0; c0 < len_c; c0 += CT) {
    __syncthreads();
    {
      const int lrow = blockIdx.y * CT + ty, ccol = c0 + tx;
      ga[ty][tx] = (lrow < len_l && ccol < len_c) ? ldc(glc + (int64_t)lrow * len_c + ccol) : cmake(0.0, 0.0);
      const int crow = c0 + ty, rc = blockIdx.x * CT + tx;
      gb[ty][tx] = (crow < len_c && rc < len_r) ? ldc(gcr + (int64_t)crow * len_r + rc) : cmake(0.0, 0.0);
      if (ty == 0) {
        qc[tx] = (c0 + tx < len_c) ? cc[c0 + tx] : -1;
        lcs[tx] = (c0 + tx < len_c) ? lc[c0 + tx] : 0.0;
      }
    }
    __syncthreads();
    if (!ok) continue;
    for (int j = 0; j < CT; ++j) {
      const int q = qc[j];
      if (q < 0 || !(a >= q && q >= b) || a - q >= d) continue;
      const cplx w = cscale(us[((a - tau) * d + (tau - b)) * d + (a - q)], lcs[j]);
      cfma(acc, w, cmul(ga[ty][j], gb[j][tx]));
    }
  }
  if (l < len_l && r < len_r) out[(int64_t)l * len_r + r] = ok ? cscale(acc, ll[l] * lr[r]) : cmake(0.0, 0.0);
}

}  // namespace

cudaError_t launch_contract_mps(int d, int tau, const void* u, const void* glc, const void* gcr,
                                const double* ll, const double* lc, const double* lr, const int* cl,
                                const int* cc, const int* cr, int len_l, int len_c, int len_r, void* t,
                                cudaStream_t s) {
  if (len_l <= 0 || len_r <= 0) return cudaSuccess;
  dim3 grid(ceil_div(len_r, CT), ceil_div(len_l, CT));
  dim3 block(CT, CT);
  contract_mps_kernel<<<grid, block, 0, s>>>(d, tau, reinterpret_cast<const cplx*>(u),
                                             reinterpret_cast<const cplx*>(glc), reinterpret_cast<const cplx*>(gcr),
                                             ll, lc, lr, cl, cc, cr, len_l, len_c, len_r, reinterpret_cast<cplx*>(t));
  return cudaGetLastError();
}

cudaError_t launch_contract_sector(int d, int cc0, int cc1, const void* u, const void* glc,
                                   const void* gcr, const int* cl, const int* cc, const int* cr,
                                   int len_l, int len_c, int len_r, void* c, cudaStream_t s) {
  if (len_l <= 0 || len_r <= 0) return cudaSuccess;
  dim3 grid(ceil_div(len_r, CT), ceil_div(len_l, CT));
  dim3 block(CT, CT);
  contract_sector_kernel<<<grid, block, 0, s>>>(
      d, cc0, cc1, reinterpret_cast<const cplx*>(u), reinterpret_cast<const cplx*>(glc),
      reinterpret_cast<const cplx*>(gcr), reinterpret_cast<const int2*>(cl),
      reinterpret_cast<const int2*>(cc), reinterpret_cast<const int2*>(cr), len_l, len_c, len_r,
      reinterpret_cast<cplx*>(c));
  return cudaGetLastError();
}
