// Blocked one-sided (Hestenes) Jacobi SVD of every sector, in FP64.
//
// Replaces the reference's per-sector cuSOLVER gesvd (src/beam_splitter_parallel/
// Rank.py:123) / LAPACK svd (src/MPO.py:258).  The Jacobi matrix of a sector is
// T = C diag(Lambda_R) when |L| >= |R| (its orthogonalised columns are sigma * V),
// or [T^H; I] when |L| < |R| (the identity rows accumulate V).  Columns are cut in
// blocks of 16; a round pairs the blocks by the circle method, and one CTA per block
// pair is handled by a thread-block cluster of 8 CTAs that split its rows (all
// sectors of the update in one launch):
//   1. each CTA loads its rows of the pair's 32 columns into shared memory and forms
//      a partial 32 x 32 Gram; the partials are summed through distributed shared
//      memory in a fixed order, so every CTA holds the same bit-exact Gram,
//   2. the cluster stops if every pair is orthogonal to `tol` (relative), else
//   3. every CTA runs the same cyclic two-sided Jacobi sweep on that Gram (complex
//      rotations, 16 disjoint pairs per step), accumulating the 32 x 32 unitary Q, and
//   4. applies Q to its own rows, writing them back to global memory.
// A sector is converged after a sweep without rotations; later rounds of it exit
// at once.  One-sided Jacobi keeps high relative accuracy for small singular values.
// Numerical rank: a column whose norm is <= 16 eps sqrt(rows) ||T||_F is rounding
// noise (the null space of a rank-deficient block); it takes part in no rotation and
// its singular value is reported as 0, as is a column below tol times its partner
// in a pair test.  Without this, noise columns never test orthogonal.
#include <cooperative_groups.h>

#include "common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace {

constexpr int JB = 16;        // columns per block
constexpr int JC = 2 * JB;    // columns per block pair
constexpr int JNT = 256;
constexpr int JCL = 8;        // CTAs per cluster: one cluster per block pair
constexpr int RMAX = 256;     // rows per CTA held in shared memory

struct JacSmem {
  double2 tile[RMAX][JC + 1];   // this CTA's rows of the pair's 32 columns
  double2 G[JC][JC + 1];        // full pair Gram (identical in every CTA of the cluster)
  double2 Q[JC][JC + 1];        // accumulated rotation
  double2 Gp[JC][JC + 1];       // this CTA's partial Gram
  double2 Gf[JC][JC + 1];       // this CTA's slice of the reduced Gram (first JC/cs rows)
  int cols[JC];
  JacobiWork W;
  int64_t aoff;
  int k, rows_g, rows_tot, rotate;
  double z2;
};

__global__ __launch_bounds__(JNT) void jacobi_cluster_kernel(const SectorDesc* __restrict__ sd,
                                                             const JacobiWork* __restrict__ work,
                                                             int n_work, int t, cplx* __restrict__ abuf,
                                                             int* __restrict__ rot_count,
                                                             const double* __restrict__ nf2,
                                                             double tol, int max_sweeps) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  JacSmem& S = *reinterpret_cast<JacSmem*>(smem_raw);
  cg::cluster_group cluster = cg::this_cluster();
  const int cr = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const int gc = blockIdx.x / JCL;   // global cluster index
  if (tid == 0) {
    int lo = 0, hi = n_work - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (work[mid].cta_start <= gc) lo = mid; else hi = mid - 1;
    }
    S.W = work[lo];
    const SectorDesc& D = sd[S.W.sector];
    S.k = D.k;
    S.rows_g = D.rows_g;
    S.rows_tot = D.rows_tot;
    S.aoff = D.a_off;
    // numerical-rank floor: columns with |a|^2 <= z2 are exact zeros for the SVD
    const double zf = 16.0 * 2.220446049250313e-16 * sqrt((double)D.rows_g);
    S.z2 = zf * zf * nf2[S.W.sector];
    S.rotate = 0;
  }
  __syncthreads();
  const JacobiWork W = S.W;
  // a cluster serves one sector: JCL / cs block pairs, each split over cs CTAs by rows
  const int cs = W.cs, slot = cr / cs, part = cr % cs;
  const int pair = (gc - W.cta_start) * (JCL / cs) + slot;
  const bool valid = pair < W.npairs;
  const int sweep = t / W.rounds, rr = t % W.rounds;
  // every exit before the first cluster barrier depends on (sector, t) only, so the
  // whole cluster takes it together
  if (sweep >= max_sweeps) return;
  int* cnt = rot_count + 3 * W.sector;
  // the counter of sweep w+1 is cleared during sweep w (nobody else touches it then),
  // before the converged exit so that a converged sector keeps reading zeros
  if (rr == 0 && pair == 0 && part == 0 && tid == 0) cnt[(sweep + 1) % 3] = 0;
  if (sweep >= 1 && cnt[(sweep - 1) % 3] == 0) return;   // converged
  const int nbp = W.nblk + (W.nblk & 1);
  auto blk_at = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + rr) % (nbp - 1); };
  const int bi = valid ? blk_at(pair) : 0, bj = valid ? blk_at(nbp - 1 - pair) : 0;
  const int k = S.k;
  if (tid < JC) {
    const int b = tid < JB ? bi : bj;
    const int c = b * JB + (tid % JB);
    S.cols[tid] = (valid && b < W.nblk && c < k) ? c : -1;
  }
  const int rows_tot = S.rows_tot, rows_g = S.rows_g;
  const int chunk = ((rows_tot + cs - 1) / cs + 15) / 16 * 16;
  const int r0 = part * chunk;
  const int nr = valid ? max(0, min(rows_tot, r0 + chunk) - r0) : 0;
  const int ng = valid ? max(0, min(rows_g, r0 + chunk) - r0) : 0;   // rows in the Gram
  const int sl = JC / cs;          // Gram rows reduced by each CTA of a pair
  const int base = slot * cs;      // first cluster rank of this pair
  cplx* A = abuf + S.aoff;
  __syncthreads();

  // ---- 1. this CTA's rows -> shared memory; partial Gram over its Gram rows
  for (int e = tid; e < nr * JC; e += JNT) {
    const int r = e / JC, c = e % JC;
    double2 v = make_double2(0.0, 0.0);
    if (S.cols[c] >= 0) v = *reinterpret_cast<const double2*>(A + (int64_t)(r0 + r) * k + S.cols[c]);
    S.tile[r][c] = v;
  }
  __syncthreads();
  {
    const int gi0 = 2 * (tid >> 4), gj0 = 2 * (tid & 15);
    cplx a00 = cmake(0, 0), a01 = cmake(0, 0), a10 = cmake(0, 0), a11 = cmake(0, 0);
#pragma unroll 4
    for (int r = 0; r < ng; ++r) {
      const double2 x0 = S.tile[r][gi0], x1 = S.tile[r][gi0 + 1];
      const double2 y0 = S.tile[r][gj0], y1 = S.tile[r][gj0 + 1];
      const cplx c0 = cmake(x0.x, x0.y), c1 = cmake(x1.x, x1.y);
      const cplx d0 = cmake(y0.x, y0.y), d1 = cmake(y1.x, y1.y);
      ccfma(a00, c0, d0);
      ccfma(a01, c0, d1);
      ccfma(a10, c1, d0);
      ccfma(a11, c1, d1);
    }
    S.Gp[gi0][gj0] = make_double2(a00.x, a00.y);
    S.Gp[gi0][gj0 + 1] = make_double2(a01.x, a01.y);
    S.Gp[gi0 + 1][gj0] = make_double2(a10.x, a10.y);
    S.Gp[gi0 + 1][gj0 + 1] = make_double2(a11.x, a11.y);
  }
  cluster.sync();
  // ---- 2. reduce: this CTA sums Gram rows [part*sl, part*sl + sl) over the pair's cs
  //         CTAs, in rank order
  if (valid) {
    for (int e = tid; e < sl * JC; e += JNT) {
      const int r = e / JC, c = e % JC;
      double sx = 0.0, sy = 0.0;
      for (int q = 0; q < cs; ++q) {
        const JacSmem* R = cluster.map_shared_rank(&S, base + q);
        const double2 v = R->Gp[part * sl + r][c];
        sx += v.x;
        sy += v.y;
      }
      S.Gf[r][c] = make_double2(sx, sy);
    }
  }
  cluster.sync();
  // ---- 3. gather the reduced Gram (bit-identical in every CTA of the pair)
  if (valid) {
    for (int e = tid; e < JC * JC; e += JNT) {
      const int r = e / JC, c = e % JC;
      const JacSmem* R = cluster.map_shared_rank(&S, base + r / sl);
      S.G[r][c] = R->Gf[r % sl][c];
    }
  }
  cluster.sync();   // after this no CTA touches another CTA's shared memory
  if (!valid) return;

  // ---- 4. convergence test (relative tolerance on |a_i^H a_j|)
  if (tol <= 0.0) tol = fmax(8.0 * 2.220446049250313e-16, 4.0 * 2.220446049250313e-16 * sqrt((double)rows_g));
  const double t2 = tol * tol, z2 = S.z2;
  for (int e = tid; e < JC * JC; e += JNT) {
    const int i = e / JC, j = e % JC;
    if (j <= i) continue;
    const double dii = S.G[i][i].x, djj = S.G[j][j].x;
    const double2 g = S.G[i][j];
    const double a2 = g.x * g.x + g.y * g.y;
    // a column at the numerical-rank floor, or below tol times its partner, is rounding
    // noise along the partner and is never rotated against it
    if (dii > z2 && djj > z2 && dii > t2 * djj && djj > t2 * dii && a2 > t2 * dii * djj) S.rotate = 1;
  }
  __syncthreads();
  if (!S.rotate) return;
  if (part == 0 && tid == 0) atomicAdd(cnt + sweep % 3, 1);

  // ---- 5. one cyclic Jacobi sweep on the 32 x 32 Gram, accumulating Q
  for (int e = tid; e < JC * JC; e += JNT) S.Q[e / JC][e % JC] = make_double2((e / JC) == (e % JC) ? 1.0 : 0.0, 0.0);
  __syncthreads();
  const int pr = tid >> 4, l16 = tid & 15;
  for (int step = 0; step < JC - 1; ++step) {
    auto idx = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + step) % (JC - 1); };
    int p = idx(pr), q = idx(JC - 1 - pr);
    if (p > q) { int tmp = p; p = q; q = tmp; }
    const double gpp = S.G[p][p].x, gqq = S.G[q][q].x;
    const double2 gpq = S.G[p][q];
    __syncwarp();   // the group's reads precede its writes to columns p, q
    const double a2 = gpq.x * gpq.x + gpq.y * gpq.y;
    double c = 1.0;
    cplx se = cmake(0.0, 0.0);
    const bool act = a2 > 0.0 && gpp > z2 && gqq > z2 && gpp > t2 * gqq && gqq > t2 * gpp &&
                     a2 > t2 * gpp * gqq;
    if (act) {
      // zeta = (g_qq - g_pp) / (2 |g_pq|), t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)),
      // c = 1 / sqrt(1 + t^2), s e^{i alpha} = t c g_pq / |g_pq|
      const double ra = rsqrt(a2);
      const double zeta = 0.5 * (gqq - gpp) * ra;
      const double tt = copysign(1.0, zeta) / (fabs(zeta) + sqrt(fma(zeta, zeta, 1.0)));
      c = rsqrt(fma(tt, tt, 1.0));
      const double sn = tt * c * ra;
      se = cmake(sn * gpq.x, sn * gpq.y);   // s e^{i alpha}
      // column update: G <- G J, Q <- Q J, J = [[c, s e], [-s conj e, c]]
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = l16 + 16 * h;
        const cplx gp_ = cmake(S.G[r][p].x, S.G[r][p].y), gq_ = cmake(S.G[r][q].x, S.G[r][q].y);
        const cplx np_ = csub(cscale(gp_, c), cmulc(gq_, se));
        const cplx nq_ = cadd(cmul(gp_, se), cscale(gq_, c));
        S.G[r][p] = make_double2(np_.x, np_.y);
        S.G[r][q] = make_double2(nq_.x, nq_.y);
        const cplx qp = cmake(S.Q[r][p].x, S.Q[r][p].y), qq = cmake(S.Q[r][q].x, S.Q[r][q].y);
        const cplx mp = csub(cscale(qp, c), cmulc(qq, se));
        const cplx mq = cadd(cmul(qp, se), cscale(qq, c));
        S.Q[r][p] = make_double2(mp.x, mp.y);
        S.Q[r][q] = make_double2(mq.x, mq.y);
      }
    }
    __syncthreads();
    if (act) {
      // row update: G <- J^H G  (row p: c gp - s e gq, row q: s conj(e) gp + c gq)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int cc = l16 + 16 * h;
        const cplx gp_ = cmake(S.G[p][cc].x, S.G[p][cc].y), gq_ = cmake(S.G[q][cc].x, S.G[q][cc].y);
        const cplx np_ = csub(cscale(gp_, c), cmul(se, gq_));
        const cplx nq_ = cadd(cmulc(gp_, se), cscale(gq_, c));
        S.G[p][cc] = make_double2(np_.x, np_.y);
        S.G[q][cc] = make_double2(nq_.x, nq_.y);
      }
    }
    __syncwarp();   // outside the branch: the two groups of a warp may differ in `act`
    if (act && l16 == 0) {
      S.G[p][q] = make_double2(0.0, 0.0);
      S.G[q][p] = make_double2(0.0, 0.0);
      S.G[p][p].y = 0.0;
      S.G[q][q].y = 0.0;
    }
    __syncthreads();
  }

  // ---- 6. apply Q to this CTA's rows, straight to global memory
  {
    const int j0 = 4 * (tid & 7), rg = tid >> 3;
    for (int rb = 0; rb < nr; rb += 64) {
      const int ra = rb + rg, rc2 = rb + rg + 32;
      cplx o0[4], o1[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) { o0[j] = cmake(0, 0); o1[j] = cmake(0, 0); }
      if (ra < nr) {
#pragma unroll 4
        for (int i = 0; i < JC; ++i) {
          const double2 x = S.tile[ra][i];
          const double2 y = S.tile[rc2 < nr ? rc2 : ra][i];
          const cplx cx = cmake(x.x, x.y), cy = cmake(y.x, y.y);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const double2 qv = S.Q[i][j0 + j];
            const cplx cq = cmake(qv.x, qv.y);
            cfma(o0[j], cx, cq);
            cfma(o1[j], cy, cq);
          }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int col = S.cols[j0 + j];
          if (col < 0) continue;
          stc(A + (int64_t)(r0 + ra) * k + col, o0[j]);
          if (rc2 < nr) stc(A + (int64_t)(r0 + rc2) * k + col, o1[j]);
        }
      }
    }
  }
}

// column norms + descending sort (ties by column index), one CTA per sector
constexpr int FNT = 512;

__global__ __launch_bounds__(FNT) void jacobi_finish_kernel(const SectorDesc* __restrict__ sd,
                                                            const cplx* __restrict__ abuf,
                                                            const double* __restrict__ nf2,
                                                            double* __restrict__ sig,
                                                            int* __restrict__ perm) {
  extern __shared__ unsigned char smem_raw[];
  const SectorDesc& S = sd[blockIdx.x];
  const int k = S.k;
  if (k == 0) return;
  int np2 = 1;
  while (np2 < k) np2 <<= 1;
  double* sv = reinterpret_cast<double*>(smem_raw);
  int* si = reinterpret_cast<int*>(sv + np2);
  const cplx* A = abuf + S.a_off;
  const double zf = 16.0 * 2.220446049250313e-16 * sqrt((double)S.rows_g);
  const double z2 = zf * zf * nf2[blockIdx.x];
  for (int j = threadIdx.x; j < np2; j += FNT) {
    double s2 = -1.0;
    if (j < k) {
      s2 = 0.0;
      for (int r = 0; r < S.rows_g; ++r) s2 += cabs2(ldc(A + (int64_t)r * k + j));
      if (s2 <= z2) s2 = 0.0;   // below the numerical-rank floor: an exact zero
    }
    sv[j] = s2 >= 0.0 ? sqrt(s2) : -1.0;
    si[j] = j;
  }
  __syncthreads();
  // bitonic sort: descending value, ascending index
  for (int size = 2; size <= np2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < np2; i += FNT) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const double a = sv[i], b = sv[j];
          const int ia = si[i], ib = si[j];
          // "a before b" in the final order
          const bool a_first = (a > b) || (a == b && ia < ib);
          if (a_first != up) {
            sv[i] = b; sv[j] = a;
            si[i] = ib; si[j] = ia;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int j = threadIdx.x; j < k; j += FNT) {
    sig[S.s_off + j] = sv[j];
    perm[S.s_off + j] = si[j];
  }
}

// ||T_s||_F^2 over the Gram rows, one CTA per sector, fixed-order reduction
constexpr int NNT = 256;
__global__ __launch_bounds__(NNT) void sector_norm_kernel(const SectorDesc* __restrict__ sd,
                                                          const cplx* __restrict__ abuf,
                                                          double* __restrict__ nf2) {
  __shared__ double red[NNT];
  const SectorDesc& S = sd[blockIdx.x];
  const int64_t total = (int64_t)S.rows_g * S.k;
  const cplx* A = abuf + S.a_off;
  double acc = 0.0;
  for (int64_t e = threadIdx.x; e < total; e += NNT) acc += cabs2(ldc(A + e));
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = NNT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) nf2[blockIdx.x] = red[0];
}

}  // namespace

int jacobi_block_cols() { return JB; }

cudaError_t launch_sector_norms(const SectorDesc* sd_dev, int n_sectors, const void* abuf,
                                double* nf2, cudaStream_t s) {
  if (n_sectors <= 0) return cudaSuccess;
  sector_norm_kernel<<<n_sectors, NNT, 0, s>>>(sd_dev, reinterpret_cast<const cplx*>(abuf), nf2);
  return cudaGetLastError();
}

cudaError_t launch_jacobi_round(const SectorDesc* sd_dev, const JacobiWork* work_dev, int n_work,
                                int total_clusters, int t, void* abuf, int* rot_count,
                                const double* nf2, double tol, int max_sweeps, cudaStream_t s) {
  if (total_clusters <= 0) return cudaSuccess;
  static bool attr_done = false;
  const int smem = (int)sizeof(JacSmem);
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(jacobi_cluster_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(total_clusters * JCL, 1, 1);
  cfg.blockDim = dim3(JNT, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = JCL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, jacobi_cluster_kernel, sd_dev, work_dev, n_work, t,
                            reinterpret_cast<cplx*>(abuf), rot_count, nf2, tol, max_sweeps);
}

int jacobi_max_rows() { return JCL * RMAX; }
int jacobi_cluster_ctas() { return JCL; }
int jacobi_rows_per_cta() { return RMAX; }

cudaError_t launch_jacobi_finish(const SectorDesc* sd_dev, int n_sectors, int max_k,
                                 const void* abuf, const double* nf2, double* sig, int* perm,
                                 cudaStream_t s) {
  if (n_sectors <= 0) return cudaSuccess;
  int np2 = 1;
  while (np2 < max_k) np2 <<= 1;
  const size_t smem = (size_t)np2 * (sizeof(double) + sizeof(int));
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(jacobi_finish_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  jacobi_finish_kernel<<<n_sectors, FNT, smem, s>>>(sd_dev, reinterpret_cast<const cplx*>(abuf),
                                                    nf2, sig, perm);
  return cudaGetLastError();
}
