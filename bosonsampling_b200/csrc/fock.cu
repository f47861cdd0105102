// Two-mode Fock beam-splitter tensor, U[n][m][l] = <l, n+m-l| M |n, m>.
//
// Same amplitude as the reference's `unitary` kernel (src/u_kernel.cu:37-71) and
// CPU Rand_BS_MPS (src/MPO.py:6-18), but evaluated with integer powers and exact
// binomials in FP64 instead of the reference's log-domain lgamma/log/exp: no NaN at
// |r| = 0 or |t| = 0 (the reason for the reference's host branch,
// src/cuda_kernels.py:20-33) and exact zeros where the amplitude vanishes.
// One thread per (gate, n, m, l); the whole mesh's tensors are built in one launch.
#include "common.cuh"
#include "kernels.h"

namespace {

BSMPO_DEV cplx cpow_int(cplx z, int e) {
  cplx r = cmake(1.0, 0.0);
  for (int i = 0; i < e; ++i) r = cmul(r, z);
  return r;
}

BSMPO_DEV double fact(int n) {
  double f = 1.0;
  for (int i = 2; i <= n; ++i) f *= (double)i;
  return f;
}

BSMPO_DEV double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double b = 1.0;
  for (int i = 1; i <= k; ++i) b = b * (double)(n - k + i) / (double)i;
  return b;
}

// m4: per gate 8 doubles (re, im of M00, M01, M10, M11), creation-operator map
// a+ -> M00 a+ + M10 b+, b+ -> M01 a+ + M11 b+.
__global__ void fock_tensor_kernel(int d, int n_gates, const double* __restrict__ m4,
                                   cplx* __restrict__ u) {
  const int d3 = d * d * d;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= n_gates * d3) return;
  const int g = tid / d3;
  const int e = tid % d3;
  const int n = e / (d * d), m = (e / d) % d, l = e % d;
  const double* M = m4 + 8 * g;
  const cplx m00 = cmake(M[0], M[1]), m01 = cmake(M[2], M[3]);
  const cplx m10 = cmake(M[4], M[5]), m11 = cmake(M[6], M[7]);
  cplx acc = cmake(0.0, 0.0);
  const int o = n + m - l;
  if (o >= 0 && o < d) {
    const int klo = l - m > 0 ? l - m : 0;
    const int khi = l < n ? l : n;
    for (int k = klo; k <= khi; ++k) {
      const double c = binom(n, k) * binom(m, l - k);
      cplx t = cmul(cmul(cpow_int(m00, k), cpow_int(m10, n - k)),
                    cmul(cpow_int(m01, l - k), cpow_int(m11, m - l + k)));
      acc = cadd(acc, cscale(t, c));
    }
    acc = cscale(acc, sqrt(fact(l) * fact(o) / (fact(n) * fact(m))));
  }
  u[tid] = acc;
}

}  // namespace

cudaError_t launch_fock_tensor(int d, int n_gates, const double* m4_dev, void* u_dev,
                               cudaStream_t s) {
  const int total = n_gates * d * d * d;
  if (total == 0) return cudaSuccess;
  fock_tensor_kernel<<<ceil_div(total, 128), 128, 0, s>>>(d, n_gates, m4_dev,
                                                          reinterpret_cast<cplx*>(u_dev));
  return cudaGetLastError();
}

namespace {
__global__ void fock_single_kernel(int d, M8 m, cplx* __restrict__ uc, double* __restrict__ ur,
                                   double* __restrict__ ui) {
  const int d3 = d * d * d;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d3) return;
  const int n = e / (d * d), mm = (e / d) % d, l = e % d;
  const cplx m00 = cmake(m.v[0], m.v[1]), m01 = cmake(m.v[2], m.v[3]);
  const cplx m10 = cmake(m.v[4], m.v[5]), m11 = cmake(m.v[6], m.v[7]);
  cplx acc = cmake(0.0, 0.0);
  const int o = n + mm - l;
  if (o >= 0 && o < d) {
    const int klo = l - mm > 0 ? l - mm : 0;
    const int khi = l < n ? l : n;
    for (int k = klo; k <= khi; ++k) {
      const double c = binom(n, k) * binom(mm, l - k);
      cplx t = cmul(cmul(cpow_int(m00, k), cpow_int(m10, n - k)),
                    cmul(cpow_int(m01, l - k), cpow_int(m11, mm - l + k)));
      acc = cadd(acc, cscale(t, c));
    }
    acc = cscale(acc, sqrt(fact(l) * fact(o) / (fact(n) * fact(mm))));
  }
  if (uc) {
    uc[e] = acc;
  } else {
    ur[e] = acc.x;
    ui[e] = acc.y;
  }
}
}  // namespace

cudaError_t launch_fock_tensor_single(int d, M8 m, void* u_re_or_cplx, double* u_im,
                                      cudaStream_t s) {
  const int d3 = d * d * d;
  if (u_im) {
    fock_single_kernel<<<ceil_div(d3, 128), 128, 0, s>>>(d, m, nullptr,
                                                          reinterpret_cast<double*>(u_re_or_cplx),
                                                          u_im);
  } else {
    fock_single_kernel<<<ceil_div(d3, 128), 128, 0, s>>>(d, m, reinterpret_cast<cplx*>(u_re_or_cplx),
                                                          nullptr, nullptr);
  }
  return cudaGetLastError();
}
