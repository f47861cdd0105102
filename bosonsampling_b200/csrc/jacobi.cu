// Blocked one-sided (Hestenes) Jacobi SVD of every sector, in FP64.
//
// Replaces the reference's per-sector cuSOLVER gesvd (src/beam_splitter_parallel/
// Rank.py:123) / LAPACK svd (src/MPO.py:258).  The Jacobi matrix of a sector is
// T = C diag(Lambda_R) when |L| >= |R| (its orthogonalised columns are sigma * V),
// or [T^H; I] when |L| < |R| (the identity rows accumulate V).  Columns are cut in
// blocks of 16; a round pairs the blocks by the circle method, and one CTA per block
// pair (all sectors of the update in one launch):
//   1. forms the 32 x 32 Gram of its columns (rows streamed through shared memory),
//   2. stops if every pair is orthogonal to `tol` (relative), else
//   3. runs one cyclic two-sided Jacobi sweep on that Gram (complex rotations,
//      16 disjoint pairs per step), accumulating the 32 x 32 unitary Q, and
//   4. applies Q to its columns (all stored rows).
// A sector is converged after a sweep without rotations; later rounds of it exit
// at once.  One-sided Jacobi keeps high relative accuracy for small singular values.
#include "common.cuh"
#include "kernels.h"

namespace {

constexpr int JB = 16;        // columns per block
constexpr int JC = 2 * JB;    // columns per block pair
constexpr int JNT = 256;
constexpr int JR = 16;        // rows per streamed chunk

__global__ __launch_bounds__(JNT) void jacobi_round_kernel(const SectorDesc* __restrict__ sd,
                                                           const JacobiWork* __restrict__ work,
                                                           int n_work, int t, cplx* __restrict__ abuf,
                                                           int* __restrict__ rot_count, double tol,
                                                           int max_sweeps) {
  __shared__ double2 G[JC][JC + 1];
  __shared__ double2 Q[JC][JC + 1];
  __shared__ double2 tile[JR][JC + 1];
  __shared__ double rc[JC / 2];
  __shared__ double2 rs[JC / 2];
  __shared__ int cols[JC];
  __shared__ JacobiWork W;
  __shared__ int rotate;
  __shared__ int s_k, s_rows_g, s_rows_tot;
  __shared__ int64_t s_aoff;
  const int tid = threadIdx.x;
  if (tid == 0) {
    int lo = 0, hi = n_work - 1;
    const int b = blockIdx.x;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (work[mid].cta_start <= b) lo = mid; else hi = mid - 1;
    }
    W = work[lo];
    const SectorDesc& S = sd[W.sector];
    s_k = S.k;
    s_rows_g = S.rows_g;
    s_rows_tot = S.rows_tot;
    s_aoff = S.a_off;
    rotate = 0;
  }
  __syncthreads();
  const int pair = blockIdx.x - W.cta_start;
  const int sweep = t / W.rounds, rr = t % W.rounds;
  if (sweep >= max_sweeps) return;
  int* cnt = rot_count + 3 * W.sector;
  // counter of sweep w+1 is cleared during sweep w (nobody else touches it then);
  // done before the converged exit so a converged sector keeps reading zeros
  if (rr == 0 && pair == 0 && tid == 0) cnt[(sweep + 1) % 3] = 0;
  if (sweep >= 1 && cnt[(sweep - 1) % 3] == 0) return;   // converged
  const int nbp = W.nblk + (W.nblk & 1);
  auto blk_at = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + rr) % (nbp - 1); };
  const int bi = blk_at(pair), bj = blk_at(nbp - 1 - pair);
  const int k = s_k;
  if (tid < JC) {
    const int b = tid < JB ? bi : bj;
    const int c = b * JB + (tid % JB);
    cols[tid] = (b < W.nblk && c < k) ? c : -1;
  }
  __syncthreads();
  cplx* A = abuf + s_aoff;

  // ---- 1. Gram of the pair's columns over rows [0, rows_g)
  const int gi = tid >> 3, gj0 = (tid & 7) * 4;
  cplx acc[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) acc[j] = cmake(0.0, 0.0);
  const int rows_g = s_rows_g;
  for (int r0 = 0; r0 < rows_g; r0 += JR) {
#pragma unroll
    for (int i = 0; i < (JR * JC) / JNT; ++i) {
      const int e = tid + JNT * i;
      const int r = e / JC, c = e % JC;
      double2 v = make_double2(0.0, 0.0);
      if (r0 + r < rows_g && cols[c] >= 0)
        v = *reinterpret_cast<const double2*>(A + (int64_t)(r0 + r) * k + cols[c]);
      tile[r][c] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int r = 0; r < JR; ++r) {
      const double2 a = tile[r][gi];
      const cplx ac = cmake(a.x, a.y);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double2 b = tile[r][gj0 + j];
        ccfma(acc[j], ac, cmake(b.x, b.y));
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) G[gi][gj0 + j] = make_double2(acc[j].x, acc[j].y);
  __syncthreads();

  // ---- 2. convergence test of this pair (relative tolerance on |a_i^H a_j|)
  if (tol <= 0.0) tol = fmax(8.0 * 2.220446049250313e-16, 4.0 * 2.220446049250313e-16 * sqrt((double)rows_g));
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int gj = gj0 + j;
    if (gj <= gi) continue;
    const double dii = G[gi][gi].x, djj = G[gj][gj].x;
    const double a2 = acc[j].x * acc[j].x + acc[j].y * acc[j].y;
    if (dii > 0.0 && djj > 0.0 && a2 > tol * tol * dii * djj) rotate = 1;
  }
  __syncthreads();
  if (!rotate) return;
  if (tid == 0) atomicAdd(cnt + sweep % 3, 1);

  // ---- 3. one cyclic Jacobi sweep on the 32 x 32 Gram, accumulating Q
  for (int e = tid; e < JC * JC; e += JNT) {
    const int i = e / JC, j = e % JC;
    Q[i][j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  for (int step = 0; step < JC - 1; ++step) {
    if (tid < JC / 2) {
      auto idx = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + step) % (JC - 1); };
      int p = idx(tid), q = idx(JC - 1 - tid);
      if (p > q) { int tmp = p; p = q; q = tmp; }
      const double gpp = G[p][p].x, gqq = G[q][q].x;
      const double2 gpq = G[p][q];
      const double apq = sqrt(gpq.x * gpq.x + gpq.y * gpq.y);
      double c = 1.0, sn = 0.0;
      double2 e = make_double2(1.0, 0.0);
      if (apq > 0.0 && apq > 1e-300 && apq * apq > 1e-34 * gpp * gqq) {
        const double zeta = (gqq - gpp) / (2.0 * apq);
        const double tt = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        c = 1.0 / sqrt(1.0 + tt * tt);
        sn = tt * c;
        e = make_double2(gpq.x / apq, gpq.y / apq);
      }
      rc[tid] = c;
      rs[tid] = make_double2(sn * e.x, sn * e.y);   // s * e^{i alpha}
    }
    __syncthreads();
    // column update: G <- G J, Q <- Q J with J = [[c, s e], [-s conj e, c]]
    {
      const int pr = tid >> 4, row = tid & 15;
      auto idx = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + step) % (JC - 1); };
      int p = idx(pr), q = idx(JC - 1 - pr);
      if (p > q) { int tmp = p; p = q; q = tmp; }
      const double c = rc[pr];
      const cplx se = cmake(rs[pr].x, rs[pr].y);
      if (!(c == 1.0 && se.x == 0.0 && se.y == 0.0)) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = row + 16 * h;
          const cplx gp = cmake(G[r][p].x, G[r][p].y), gq = cmake(G[r][q].x, G[r][q].y);
          const cplx np_ = csub(cscale(gp, c), cmulc(gq, se));
          const cplx nq_ = cadd(cmul(gp, se), cscale(gq, c));
          G[r][p] = make_double2(np_.x, np_.y);
          G[r][q] = make_double2(nq_.x, nq_.y);
          const cplx qp = cmake(Q[r][p].x, Q[r][p].y), qq = cmake(Q[r][q].x, Q[r][q].y);
          const cplx mp = csub(cscale(qp, c), cmulc(qq, se));
          const cplx mq = cadd(cmul(qp, se), cscale(qq, c));
          Q[r][p] = make_double2(mp.x, mp.y);
          Q[r][q] = make_double2(mq.x, mq.y);
        }
      }
    }
    __syncthreads();
    // row update: G <- J^H G
    {
      const int pr = tid >> 4, col = tid & 15;
      auto idx = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + step) % (JC - 1); };
      int p = idx(pr), q = idx(JC - 1 - pr);
      if (p > q) { int tmp = p; p = q; q = tmp; }
      const double c = rc[pr];
      const cplx se = cmake(rs[pr].x, rs[pr].y);
      if (!(c == 1.0 && se.x == 0.0 && se.y == 0.0)) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int cc = col + 16 * h;
          const cplx gp = cmake(G[p][cc].x, G[p][cc].y), gq = cmake(G[q][cc].x, G[q][cc].y);
          // row p: c gp - s e gq ; row q: s conj(e) gp + c gq
          const cplx np_ = csub(cscale(gp, c), cmul(se, gq));
          const cplx nq_ = cadd(cmulc(gp, se), cscale(gq, c));
          G[p][cc] = make_double2(np_.x, np_.y);
          G[q][cc] = make_double2(nq_.x, nq_.y);
        }
      }
    }
    __syncthreads();
    if (tid < JC / 2) {
      auto idx = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + step) % (JC - 1); };
      int p = idx(tid), q = idx(JC - 1 - tid);
      if (!(rc[tid] == 1.0 && rs[tid].x == 0.0 && rs[tid].y == 0.0)) {
        G[p][q] = make_double2(0.0, 0.0);
        G[q][p] = make_double2(0.0, 0.0);
        G[p][p].y = 0.0;
        G[q][q].y = 0.0;
      }
    }
    __syncthreads();
  }

  // ---- 4. apply Q to the pair's columns over all stored rows
  const int rows_tot = s_rows_tot;
  const int ar = tid >> 4, aj0 = (tid & 15) * 2;
  for (int r0 = 0; r0 < rows_tot; r0 += JR) {
#pragma unroll
    for (int i = 0; i < (JR * JC) / JNT; ++i) {
      const int e = tid + JNT * i;
      const int r = e / JC, c = e % JC;
      double2 v = make_double2(0.0, 0.0);
      if (r0 + r < rows_tot && cols[c] >= 0)
        v = *reinterpret_cast<const double2*>(A + (int64_t)(r0 + r) * k + cols[c]);
      tile[r][c] = v;
    }
    __syncthreads();
    cplx out[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) out[j] = cmake(0.0, 0.0);
#pragma unroll 4
    for (int i = 0; i < JC; ++i) {
      const double2 a = tile[ar][i];
      const cplx ac = cmake(a.x, a.y);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const double2 q = Q[i][aj0 + j];
        cfma(out[j], ac, cmake(q.x, q.y));
      }
    }
    __syncthreads();
    if (r0 + ar < rows_tot) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int c = cols[aj0 + j];
        if (c >= 0) stc(A + (int64_t)(r0 + ar) * k + c, out[j]);
      }
    }
  }
}

// column norms + descending sort (ties by column index), one CTA per sector
constexpr int FNT = 512;

__global__ __launch_bounds__(FNT) void jacobi_finish_kernel(const SectorDesc* __restrict__ sd,
                                                            const cplx* __restrict__ abuf,
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
  for (int j = threadIdx.x; j < np2; j += FNT) {
    double s2 = -1.0;
    if (j < k) {
      s2 = 0.0;
      for (int r = 0; r < S.rows_g; ++r) s2 += cabs2(ldc(A + (int64_t)r * k + j));
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

}  // namespace

int jacobi_block_cols() { return JB; }

cudaError_t launch_jacobi_round(const SectorDesc* sd_dev, const JacobiWork* work_dev, int n_work,
                                int total_ctas, int t, void* abuf, int* rot_count, double tol,
                                int max_sweeps, cudaStream_t s) {
  if (total_ctas <= 0) return cudaSuccess;
  jacobi_round_kernel<<<total_ctas, JNT, 0, s>>>(sd_dev, work_dev, n_work, t,
                                                 reinterpret_cast<cplx*>(abuf), rot_count, tol,
                                                 max_sweeps);
  return cudaGetLastError();
}

cudaError_t launch_jacobi_finish(const SectorDesc* sd_dev, int n_sectors, int max_k,
                                 const void* abuf, double* sig, int* perm, cudaStream_t s) {
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
                                                    sig, perm);
  return cudaGetLastError();
}
