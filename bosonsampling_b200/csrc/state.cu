// Product-state MPO fill on the device (the filling of the reference's Initialize,
// src/MPO.py:56-109, for arbitrary per-mode density matrices).
//
// Gamma[site][i][j] = rho_site[a0 - b0][a1 - b1] where (a0, a1) is the charge of slot i
// of bond `site` and (b0, b1) the charge of slot j of bond site + 1, when both slots are
// occupied and the occupation differences lie in [0, d); every other entry is 0.  One
// thread per entry, grid-stride over all n chi^2 entries: a streaming write of the whole
// state at HBM rate.
#include "common.cuh"
#include "kernels.h"

#include <algorithm>

namespace {

constexpr int PF_NT = 256;

__global__ __launch_bounds__(PF_NT) void product_fill_kernel(int n, int d, int chi,
                                                            const int2* __restrict__ charge,
                                                            const cplx* __restrict__ rho,
                                                            cplx* __restrict__ gamma) {
  const int64_t chi2 = (int64_t)chi * chi;
  const int64_t total = (int64_t)n * chi2;
  for (int64_t e = (int64_t)blockIdx.x * PF_NT + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * PF_NT) {
    const int site = (int)(e / chi2);
    const int64_t r = e - (int64_t)site * chi2;
    const int i = (int)(r / chi), j = (int)(r % chi);
    const int2 a = charge[(int64_t)site * chi + i];
    const int2 b = charge[(int64_t)(site + 1) * chi + j];
    cplx v = cmake(0.0, 0.0);
    const int o0 = a.x - b.x, o1 = a.y - b.y;
    if (a.x < d && b.x < d && o0 >= 0 && o0 < d && o1 >= 0 && o1 < d)
      v = rho[((int64_t)site * d + o0) * d + o1];
    stc(gamma + e, v);
  }
}

}  // namespace

cudaError_t launch_product_fill(int n, int d, int chi, const int* charge, const void* rho,
                                void* gamma, cudaStream_t s) {
  const int64_t total = (int64_t)n * chi * chi;
  const int blocks = (int)std::min<int64_t>((total + PF_NT - 1) / PF_NT, 148 * 16);
  product_fill_kernel<<<blocks, PF_NT, 0, s>>>(n, d, chi, reinterpret_cast<const int2*>(charge),
                                               reinterpret_cast<const cplx*>(rho),
                                               reinterpret_cast<cplx*>(gamma));
  return cudaGetLastError();
}
