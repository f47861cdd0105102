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

// Gradient of a loss with respect to the angles of every gate T(theta, phi) =
// [[e^{i phi} cos, -sin], [e^{i phi} sin, cos]] (the mesh's beam splitter, tensor of
// M = T^T), given the gradient ubar of its tensor U[n][m][l] (pairing Re sum conj(ubar) dU):
//   dL/dtheta = Re sum_e conj(ubar_e) sum_xy dU_e/dM_xy dM_xy/dtheta, likewise for phi,
// with dU/dM_xy from the polynomial form of U (d z^p = p z^(p-1) dz).  One CTA per gate,
// one thread per tensor entry, a fixed-order reduction over the entries.
namespace {
constexpr int FG_NT = BSMPO_MAX_D * BSMPO_MAX_D * BSMPO_MAX_D;   // 512

BSMPO_DEV cplx dpow(cplx z, int p, cplx dz) {   // d(z^p) = p z^(p-1) dz
  return p > 0 ? cscale(cmul(cpow_int(z, p - 1), dz), (double)p) : cmake(0.0, 0.0);
}

__global__ void __launch_bounds__(FG_NT) fock_angle_grad_kernel(int d, const double* __restrict__ m4,
                                                                const double* __restrict__ dm4,
                                                                const cplx* __restrict__ ubar,
                                                                double* __restrict__ grad) {
  __shared__ double red[2][FG_NT];
  const int g = blockIdx.x, e = threadIdx.x, d3 = d * d * d;
  const double* M = m4 + 8 * g;
  const cplx z[4] = {cmake(M[0], M[1]), cmake(M[2], M[3]), cmake(M[4], M[5]), cmake(M[6], M[7])};  // 00 01 10 11
  double gt = 0.0, gp = 0.0;
  if (e < d3) {
    const int n = e / (d * d), m = (e / d) % d, l = e % d;
    const int o = n + m - l;
    if (o >= 0 && o < d) {
      const double norm = sqrt(fact(l) * fact(o) / (fact(n) * fact(m)));
      const cplx ub = ubar[(size_t)g * d3 + e];
      for (int dir = 0; dir < 2; ++dir) {
        const double* D = dm4 + 16 * g + 8 * dir;
        const cplx dz[4] = {cmake(D[0], D[1]), cmake(D[2], D[3]), cmake(D[4], D[5]), cmake(D[6], D[7])};
        cplx acc = cmake(0.0, 0.0);
        const int klo = l - m > 0 ? l - m : 0;
        const int khi = l < n ? l : n;
        for (int k = klo; k <= khi; ++k) {
          // exponents of M00, M10, M01, M11
          const int p00 = k, p10 = n - k, p01 = l - k, p11 = m - l + k;
          const cplx f00 = cpow_int(z[0], p00), f10 = cpow_int(z[2], p10);
          const cplx f01 = cpow_int(z[1], p01), f11 = cpow_int(z[3], p11);
          cplx t = cmul(cmul(dpow(z[0], p00, dz[0]), f10), cmul(f01, f11));
          t = cadd(t, cmul(cmul(f00, dpow(z[2], p10, dz[2])), cmul(f01, f11)));
          t = cadd(t, cmul(cmul(f00, f10), cmul(dpow(z[1], p01, dz[1]), f11)));
          t = cadd(t, cmul(cmul(f00, f10), cmul(f01, dpow(z[3], p11, dz[3]))));
          acc = cadd(acc, cscale(t, binom(n, k) * binom(m, l - k)));
        }
        acc = cscale(acc, norm);
        const double v = ub.x * acc.x + ub.y * acc.y;   // Re conj(ubar) dU
        if (dir == 0) gt = v; else gp = v;
      }
    }
  }
  red[0][e] = gt;
  red[1][e] = gp;
  __syncthreads();
  for (int s = FG_NT / 2; s > 0; s >>= 1) {
    if (e < s) {
      red[0][e] += red[0][e + s];
      red[1][e] += red[1][e + s];
    }
    __syncthreads();
  }
  if (e == 0) {
    grad[2 * g] = red[0][0];
    grad[2 * g + 1] = red[1][0];
  }
}
}  // namespace

cudaError_t launch_fock_angle_grad(int d, int n_gates, const double* m4_dev, const double* dm4_dev,
                                   const void* ubar_dev, double* grad_dev, cudaStream_t s) {
  if (n_gates <= 0) return cudaSuccess;
  fock_angle_grad_kernel<<<n_gates, FG_NT, 0, s>>>(d, m4_dev, dm4_dev, reinterpret_cast<const cplx*>(ubar_dev),
                                                    grad_dev);
  return cudaGetLastError();
}
