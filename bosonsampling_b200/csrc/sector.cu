// Charge-sector kernels of the BS update: gate mix, top-chi selection, vector
// extraction and the scatter into the new site tensors.
//
// Block structure (the reference's, src/MPO.py:182-254 and src/mpo_sort.py): bond
// entries are sorted by (ket, bra) charge, so every charge block is a contiguous
// range; sector cc = (cc0, cc1) uses left blocks a >= cc and right blocks b <= cc.
// The contraction is split into Theta_q = Glc[a, q] Gcr[q, b] (one GEMM per valid
// charge triple, zgemm.cu) and this mix,
//     C_cc[a, b] = sum_q U(a0-cc0, cc0-b0, a0-q0) conj U(a1-cc1, cc1-b1, a1-q1) Theta_q[a, b],
// which is the reference's block product (src/MPO.py:254) with the sum over centre
// charges reassociated: each triple product is formed once instead of once per sector.
#include "common.cuh"
#include "kernels.h"

#include <algorithm>

namespace {

constexpr int MIX_NT = 256;

template <int MD>
__global__ __launch_bounds__(MIX_NT) void mix_kernel(const UpdateTables* __restrict__ tab,
                                                     const int* __restrict__ tidx,
                                                     const ThetaDesc* __restrict__ td,
                                                     const SectorDesc* __restrict__ sd,
                                                     const MixPair* __restrict__ pairs, int n_pairs,
                                                     const cplx* __restrict__ u3,
                                                     const cplx* __restrict__ theta,
                                                     const double* __restrict__ lam_r,
                                                     cplx* __restrict__ cbuf,
                                                     cplx* __restrict__ abuf) {
  __shared__ MixPair P;
  __shared__ cplx u0s[MD][MD], u1s[MD][MD];
  __shared__ int64_t qbase[MD][MD];
  __shared__ int qld[MD][MD];
  __shared__ int64_t cb[MD][MD], ab[MD][MD];
  __shared__ int cn[MD][MD], ck[MD][MD], cleft[MD][MD], crow[MD][MD], ccol[MD][MD], crt[MD][MD];
  const int tid = threadIdx.x;
  const int d = tab->d;
  if (tid == 0) {
    int lo = 0, hi = n_pairs - 1;
    const int t = blockIdx.x;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (pairs[mid].tile_start <= t) lo = mid; else hi = mid - 1;
    }
    P = pairs[lo];
  }
  __syncthreads();
  const int D0 = P.a0 - P.b0 + 1, D1 = P.a1 - P.b1 + 1;
  // per-box tables: index i0 <-> charge b0 + i0, i1 <-> b1 + i1
  if (tid < MD * MD) {
    const int i0 = tid / MD, i1 = tid % MD;
    // u0s[ic][iq] = U[a0-cc0][cc0-b0][a0-q0] with cc0 = b0+ic, q0 = b0+iq (same for 1)
    if (i0 < D0 && i1 < D0) {
      const int n0 = (D0 - 1) - i0, m0 = i0, l0 = (D0 - 1) - i1;
      u0s[i0][i1] = u3[(n0 * d + m0) * d + l0];
    } else {
      u0s[i0][i1] = cmake(0.0, 0.0);
    }
    if (i0 < D1 && i1 < D1) {
      const int n1 = (D1 - 1) - i0, m1 = i0, l1 = (D1 - 1) - i1;
      u1s[i0][i1] = u3[(n1 * d + m1) * d + l1];
    } else {
      u1s[i0][i1] = cmake(0.0, 0.0);
    }
    // Theta source of centre charge q = (b0 + i0, b1 + i1)
    qbase[i0][i1] = -1;
    qld[i0][i1] = 0;
    if (i0 < D0 && i1 < D1) {
      const int q0 = P.b0 + i0, q1 = P.b1 + i1;
      const int ti = tidx[((q0 * d + q1) * d + P.a0) * d + P.b0];
      if (ti >= 0) {
        const ThetaDesc T = td[ti];
        // rows of group start at left block (a0, q1); columns at right block (b0, 0)
        const int lr0 = P.row0 - tab->offL[P.a0 * d + q1];
        const int lc0 = P.col0 - tab->offR[P.b0 * d];
        qbase[i0][i1] = T.off + (int64_t)lr0 * T.ncol + lc0;
        qld[i0][i1] = T.ncol;
      }
    }
    // destination sector cc = (b0 + i0, b1 + i1)
    cb[i0][i1] = -1;
    if (i0 < D0 && i1 < D1) {
      const int cc0 = P.b0 + i0, cc1 = P.b1 + i1;
      const int s = tab->sidx[cc0 * d + cc1];
      if (s >= 0) {
        const SectorDesc& S = sd[s];
        cb[i0][i1] = S.c_off;
        ab[i0][i1] = S.a_off;
        cn[i0][i1] = S.n;
        ck[i0][i1] = S.k;
        cleft[i0][i1] = S.left;
        crt[i0][i1] = S.rows_tot;
        crow[i0][i1] = S.row_start[P.a0] + (P.row0 - tab->offL[P.a0 * d + cc1]);
        ccol[i0][i1] = S.col_start[P.b0] + (P.col0 - tab->offR[P.b0 * d]);
      }
    }
  }
  __syncthreads();
  const int le = (blockIdx.x - P.tile_start) * MIX_NT + tid;
  if (le >= P.nrow * P.ncol) return;
  const int lr = le / P.ncol, lc = le % P.ncol;
  const double lam = lam_r[P.col0 + lc];

  cplx th[MD][MD];
#pragma unroll
  for (int i0 = 0; i0 < MD; ++i0)
#pragma unroll
    for (int i1 = 0; i1 < MD; ++i1) {
      th[i0][i1] = cmake(0.0, 0.0);
      if (i0 < D0 && i1 < D1 && qbase[i0][i1] >= 0)
        th[i0][i1] = ldc(theta + qbase[i0][i1] + (int64_t)lr * qld[i0][i1] + lc);
    }
  // X[c0][q1] = sum_q0 u0[c0][q0] th[q0][q1]
  cplx X[MD][MD];
#pragma unroll
  for (int c0 = 0; c0 < MD; ++c0)
#pragma unroll
    for (int q1 = 0; q1 < MD; ++q1) {
      cplx acc = cmake(0.0, 0.0);
#pragma unroll
      for (int q0 = 0; q0 < MD; ++q0) cfma(acc, u0s[c0][q0], th[q0][q1]);
      X[c0][q1] = acc;
    }
#pragma unroll
  for (int c0 = 0; c0 < MD; ++c0) {
    if (c0 >= D0) continue;
#pragma unroll
    for (int c1 = 0; c1 < MD; ++c1) {
      if (c1 >= D1 || cb[c0][c1] < 0) continue;
      cplx acc = cmake(0.0, 0.0);
#pragma unroll
      for (int q1 = 0; q1 < MD; ++q1) ccfma(acc, u1s[c1][q1], X[c0][q1]);
      const int row = crow[c0][c1] + lr, col = ccol[c0][c1] + lc;
      stc(cbuf + cb[c0][c1] + (int64_t)row * cn[c0][c1] + col, acc);
      if (!cleft[c0][c1]) {
        stc(abuf + ab[c0][c1] + (int64_t)row * ck[c0][c1] + col, cscale(acc, lam));
      } else {
        stc(abuf + ab[c0][c1] + (int64_t)col * ck[c0][c1] + row, cscale(cconj(acc), lam));
      }
    }
  }
}

__global__ void identity_rows_kernel(const SectorDesc* __restrict__ sd, cplx* __restrict__ abuf) {
  const SectorDesc& S = sd[blockIdx.y];
  if (!S.left) return;
  const int m = S.m;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m * m; e += gridDim.x * blockDim.x) {
    const int i = e / m, j = e % m;
    stc(abuf + S.a_off + (int64_t)(S.n + i) * S.k + j, cmake(i == j ? 1.0 : 0.0, 0.0));
  }
}

// ------------------------------------------------------------------ selection
__device__ __forceinline__ int count_gt(const double* key, int k, double v) {
  // keys sorted descending: number of entries > v
  int lo = 0, hi = k;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (key[mid] > v) lo = mid + 1; else hi = mid;
  }
  return lo;
}
__device__ __forceinline__ int count_ge(const double* key, int k, double v) {
  int lo = 0, hi = k;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (key[mid] >= v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

constexpr int SEL_NT = 128;

template <typename T>
__device__ T block_sum(T v, T* red) {
  const int tid = threadIdx.x;
  red[tid] = v;
  __syncthreads();
  for (int s = SEL_NT / 2; s > 0; s >>= 1) {
    if (tid < s) red[tid] = red[tid] + red[tid + s];
    __syncthreads();
  }
  T r = red[0];
  __syncthreads();
  return r;
}

__global__ __launch_bounds__(SEL_NT) void select_kernel(const UpdateTables* __restrict__ tab,
                                                        SectorDesc* __restrict__ sd, int ns,
                                                        const double* __restrict__ sig,
                                                        double* __restrict__ keys, double cutoff,
                                                        int chi, int* __restrict__ kept_out,
                                                        double* __restrict__ trunc_out) {
  __shared__ double redd[SEL_NT];
  __shared__ long long redi[SEL_NT];
  __shared__ int kept_s[BSMPO_MAX_Q];
  const int tid = threadIdx.x;
  const int s = tid;
  const bool own = s < ns;
  int k = 0;
  int64_t off = 0;
  if (own) { k = sd[s].k; off = sd[s].s_off; }
  // keys: singular values made equal within ket/bra-swapped sector pairs
  if (own) {
    const int p = tab->pair_of[s];
    int kp = 0;
    int64_t poff = 0;
    if (p >= 0 && p != s) { kp = sd[p].k; poff = sd[p].s_off; }
    for (int i = 0; i < k; ++i) {
      double v = sig[off + i];
      if (i < kp) v = fmax(v, sig[poff + i]);
      keys[off + i] = v;
    }
  }
  __syncthreads();
  // largest singular value of the update
  double smax = (own && k > 0) ? sig[off] : 0.0;
  redd[tid] = smax;
  __syncthreads();
  for (int w = SEL_NT / 2; w > 0; w >>= 1) {
    if (tid < w) redd[tid] = fmax(redd[tid], redd[tid + w]);
    __syncthreads();
  }
  smax = redd[0];
  __syncthreads();
  const double thr = fmax(cutoff * smax, 0.0);
  const double* key = keys + off;
  const long long ncand = block_sum<long long>(own ? count_gt(key, k, thr) : 0, redi);
  int kept = 0;
  if (ncand <= chi) {
    if (own) kept = count_gt(key, k, thr);
  } else {
    // v* = chi-th largest candidate key: largest v with #(key >= v) >= chi
    unsigned long long lo = (unsigned long long)__double_as_longlong(thr) + 1ull;
    unsigned long long hi = (unsigned long long)__double_as_longlong(smax);
    while (lo < hi) {
      unsigned long long mid = lo + (hi - lo + 1) / 2;
      double v = __longlong_as_double((long long)mid);
      long long c = block_sum<long long>(own ? count_ge(key, k, v) : 0, redi);
      if (c >= chi) lo = mid; else hi = mid - 1;
    }
    const double vstar = __longlong_as_double((long long)lo);
    const int gt = own ? count_gt(key, k, vstar) : 0;
    const int ge = own ? count_ge(key, k, vstar) : 0;
    const long long ngt = block_sum<long long>(gt, redi);
    if (own) kept_s[s] = ge - gt;   // tied entries
    __syncthreads();
    if (tid == 0) {
      long long need = chi - ngt;
      for (int i = 0; i < ns; ++i) {
        int take = (int)min((long long)kept_s[i], need > 0 ? need : 0ll);
        kept_s[i] = take;
        need -= take;
      }
    }
    __syncthreads();
    if (own) kept = gt + kept_s[s];
    __syncthreads();
  }
  // a kept vector needs its own singular value > 0 (the key may come from the partner)
  if (own) kept = min(kept, count_gt(sig + off, k, 0.0));
  if (own) kept_s[s] = kept;
  __syncthreads();
  // a cut inside a degenerate swapped pair keeps neither member
  if (own) {
    const int p = tab->pair_of[s];
    if (p >= 0 && p != s) kept = min(kept, kept_s[p]);
  }
  __syncthreads();
  if (own) kept_s[s] = kept;
  __syncthreads();
  // truncation weight: discarded sigma^2 (fixed-order per sector, then tree sum)
  double tw = 0.0;
  if (own)
    for (int i = kept; i < k; ++i) tw += sig[off + i] * sig[off + i];
  tw = block_sum<double>(tw, redd);
  if (tid == 0) {
    int slot = 0;
    for (int i = 0; i < ns; ++i) {
      sd[i].kept = kept_s[i];
      sd[i].slot0 = slot;
      kept_out[i] = kept_s[i];
      slot += kept_s[i];
    }
    kept_out[ns] = slot;
    trunc_out[0] = tw;
  }
}

// conj-free V[l][t] (row-major [m][kept]) for the kept vectors of each sector
__global__ void extract_v_kernel(const SectorDesc* __restrict__ sd, const cplx* __restrict__ abuf,
                                 const double* __restrict__ sig, const int* __restrict__ perm,
                                 cplx* __restrict__ vbuf) {
  const SectorDesc& S = sd[blockIdx.y];
  const int kept = S.kept, m = S.m;
  const int total = kept * m;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int l = e / kept, t = e % kept;
    const int col = perm[S.s_off + t];
    cplx v;
    if (!S.left) {
      v = cscale(ldc(abuf + S.a_off + (int64_t)l * S.k + col), 1.0 / sig[S.s_off + t]);
    } else {
      v = ldc(abuf + S.a_off + (int64_t)(S.n + l) * S.k + col);
    }
    stc(vbuf + S.v_off + (int64_t)l * kept + t, v);
  }
}

constexpr int SC_NT = 256;

__global__ __launch_bounds__(SC_NT) void scatter_kernel(const UpdateTables* __restrict__ tab,
                                                        const SectorDesc* __restrict__ sd, int ns,
                                                        int total_kept,
                                                        const int2* __restrict__ charge_l,
                                                        const int2* __restrict__ charge_r,
                                                        const cplx* __restrict__ vbuf,
                                                        const cplx* __restrict__ wbuf,
                                                        const double* __restrict__ sig,
                                                        cplx* __restrict__ gamma_l,
                                                        cplx* __restrict__ gamma_r,
                                                        double* __restrict__ lam_c,
                                                        int2* __restrict__ charge_c) {
  __shared__ int slot0[BSMPO_MAX_Q + 1];
  __shared__ SectorDesc S[BSMPO_MAX_Q];
  const int tid = threadIdx.x;
  const int d = tab->d, chi = tab->chi;
  for (int i = tid; i < ns; i += SC_NT) {
    S[i] = sd[i];
    slot0[i] = sd[i].slot0;
  }
  if (tid == 0) slot0[ns] = total_kept;
  __syncthreads();
  const int64_t chi2 = (int64_t)chi * chi;
  for (int64_t e = (int64_t)blockIdx.x * SC_NT + tid; e < 2 * chi2 + chi;
       e += (int64_t)gridDim.x * SC_NT) {
    int j, other;
    bool is_l = e < chi2, is_r = !is_l && e < 2 * chi2;
    if (is_l) { other = (int)(e / chi); j = (int)(e % chi); }
    else if (is_r) { j = (int)((e - chi2) / chi); other = (int)((e - chi2) % chi); }
    else { j = (int)(e - 2 * chi2); other = 0; }
    int s = -1, t = 0;
    if (j < total_kept) {
      int lo = 0, hi = ns - 1;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (slot0[mid] <= j) lo = mid; else hi = mid - 1;
      }
      // skip sectors with zero kept vectors sharing the same slot0
      while (lo + 1 < ns && slot0[lo + 1] <= j) ++lo;
      s = lo;
      t = j - slot0[s];
    }
    if (is_l) {
      cplx v = cmake(0.0, 0.0);
      if (s >= 0) {
        const int2 c = charge_l[other];
        const SectorDesc& D = S[s];
        if (c.x < d && c.x >= D.cc0 && c.y >= D.cc1) {
          const int p = D.row_start[c.x] + (other - tab->offL[c.x * d + D.cc1]);
          v = ldc(vbuf + D.v_off + (int64_t)p * D.kept + t);
        }
      }
      stc(gamma_l + e, v);
    } else if (is_r) {
      cplx v = cmake(0.0, 0.0);
      if (s >= 0) {
        const int2 c = charge_r[other];
        const SectorDesc& D = S[s];
        if (c.x < d && c.x <= D.cc0 && c.y <= D.cc1) {
          const int p = D.col_start[c.x] + (other - tab->offR[c.x * d]);
          v = ldc(wbuf + D.w_off + (int64_t)t * D.n + p);
        }
      }
      stc(gamma_r + (e - chi2), v);
    } else {
      if (s >= 0) {
        lam_c[j] = sig[S[s].s_off + t];
        charge_c[j] = make_int2(S[s].cc0, S[s].cc1);
      } else {
        lam_c[j] = 0.0;
        charge_c[j] = make_int2(d, d);
      }
    }
  }
}

__global__ void phase_kernel(int d, int chi, double phi, const int2* __restrict__ cl,
                             const int2* __restrict__ cr, cplx* __restrict__ g) {
  const int64_t chi2 = (int64_t)chi * chi;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < chi2;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(e / chi), j = (int)(e % chi);
    const int2 x = cl[a], y = cr[j];
    if (x.x >= d || y.x >= d) continue;
    const int dn = (x.x - y.x) - (x.y - y.y);
    if (dn == 0) continue;
    double sn, cs;
    sincos(phi * (double)dn, &sn, &cs);
    stc(g + e, cmul(ldc(g + e), cmake(cs, sn)));
  }
}

}  // namespace

cudaError_t launch_mix_d(int d, const UpdateTables* tab_dev, const int* tidx_dev,
                         const ThetaDesc* td_dev, const SectorDesc* sd_dev,
                         const MixPair* pairs_dev, int n_pairs, int total_tiles, const void* u3,
                         const void* theta, const double* lam_r, void* cbuf, void* abuf,
                         cudaStream_t s) {
  if (total_tiles <= 0) return cudaSuccess;
  const cplx* U = reinterpret_cast<const cplx*>(u3);
  const cplx* T = reinterpret_cast<const cplx*>(theta);
  cplx* C = reinterpret_cast<cplx*>(cbuf);
  cplx* A = reinterpret_cast<cplx*>(abuf);
#define BSMPO_MIX(MD)                                                                        \
  mix_kernel<MD><<<total_tiles, MIX_NT, 0, s>>>(tab_dev, tidx_dev, td_dev, sd_dev, pairs_dev, \
                                                n_pairs, U, T, lam_r, C, A)
  switch (d) {
    case 1: case 2: BSMPO_MIX(2); break;
    case 3: BSMPO_MIX(3); break;
    case 4: BSMPO_MIX(4); break;
    case 5: BSMPO_MIX(5); break;
    case 6: BSMPO_MIX(6); break;
    default: BSMPO_MIX(8); break;
  }
#undef BSMPO_MIX
  return cudaGetLastError();
}

cudaError_t launch_identity_rows(const SectorDesc* sd_dev, int n_sectors, int max_elems,
                                 void* abuf, cudaStream_t s) {
  if (n_sectors <= 0 || max_elems <= 0) return cudaSuccess;
  dim3 grid(min(ceil_div(max_elems, 256), 1024), n_sectors);
  identity_rows_kernel<<<grid, 256, 0, s>>>(sd_dev, reinterpret_cast<cplx*>(abuf));
  return cudaGetLastError();
}

cudaError_t launch_select(const UpdateTables* tab_dev, SectorDesc* sd_dev, int n_sectors,
                          const double* sig, double* keys, double cutoff, int chi, int* kept_out,
                          double* trunc_out, cudaStream_t s) {
  select_kernel<<<1, SEL_NT, 0, s>>>(tab_dev, sd_dev, n_sectors, sig, keys, cutoff, chi,
                                     kept_out, trunc_out);
  return cudaGetLastError();
}

cudaError_t launch_extract_v(const SectorDesc* sd_dev, int n_sectors, int max_elems,
                             const void* abuf, const double* sig, const int* perm, void* vbuf,
                             cudaStream_t s) {
  if (n_sectors <= 0 || max_elems <= 0) return cudaSuccess;
  dim3 grid(min(ceil_div(max_elems, 256), 1024), n_sectors);
  extract_v_kernel<<<grid, 256, 0, s>>>(sd_dev, reinterpret_cast<const cplx*>(abuf), sig, perm,
                                        reinterpret_cast<cplx*>(vbuf));
  return cudaGetLastError();
}

cudaError_t launch_scatter(const UpdateTables* tab_dev, const SectorDesc* sd_dev, int n_sectors,
                           int total_kept, int chi, const int* charge_l, const int* charge_r,
                           const void* vbuf, const void* wbuf, const double* sig, void* gamma_l,
                           void* gamma_r, double* lam_c, int* charge_c, cudaStream_t s) {
  const int64_t total = 2 * (int64_t)chi * chi + chi;
  const int blocks = (int)std::min<int64_t>((total + SC_NT - 1) / SC_NT, 148 * 16);
  scatter_kernel<<<blocks, SC_NT, 0, s>>>(
      tab_dev, sd_dev, n_sectors, total_kept, reinterpret_cast<const int2*>(charge_l),
      reinterpret_cast<const int2*>(charge_r), reinterpret_cast<const cplx*>(vbuf),
      reinterpret_cast<const cplx*>(wbuf), sig, reinterpret_cast<cplx*>(gamma_l),
      reinterpret_cast<cplx*>(gamma_r), lam_c, reinterpret_cast<int2*>(charge_c));
  return cudaGetLastError();
}

cudaError_t launch_phase(int d, int chi, double phi, const int* charge_l, const int* charge_r,
                         void* gamma, cudaStream_t s) {
  const int64_t total = (int64_t)chi * chi;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
  phase_kernel<<<blocks, 256, 0, s>>>(d, chi, phi, reinterpret_cast<const int2*>(charge_l),
                                      reinterpret_cast<const int2*>(charge_r),
                                      reinterpret_cast<cplx*>(gamma));
  return cudaGetLastError();
}
