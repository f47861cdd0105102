// Blocked one-sided (Hestenes) Jacobi SVD of every sector, in FP64.
//
// Replaces the reference's per-sector cuSOLVER gesvd (src/beam_splitter_parallel/
// Rank.py:123) / LAPACK svd (src/MPO.py:258).  The Jacobi matrix of a sector is
// T = C diag(Lambda_R) when |L| >= |R| (its orthogonalised columns are sigma * V),
// or [T^H; I] when |L| < |R| (the identity rows accumulate V).  Columns are cut in
// blocks of 16; a round pairs the blocks by the circle method, and one CTA per block
// pair is split over 1-16 CTAs of a 16-CTA thread-block cluster by rows (all
// sectors of the update in one launch; small pairs share a cluster):
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

// D += A B on the FP64 tensor path, m8n8k4: a = A[lane>>2][lane&3],
// b = B[lane&3][lane>>2], d = (D[lane>>2][2(lane&3)], D[lane>>2][2(lane&3)+1])
__device__ __forceinline__ void dmma(double2& d, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d.x), "+d"(d.y)
               : "d"(a), "d"(b));
}

constexpr int JB = 16;        // columns per block
constexpr int JC = 2 * JB;    // columns per block pair
constexpr int JNT = 256;
constexpr int JCL = 16;       // CTAs per cluster (non-portable size, B200 supports 16)
constexpr int RMAX = 128;     // rows per CTA held in shared memory (2 CTAs per SM)

struct JacSmem {
  double2 tile[RMAX][JC + 1];   // this CTA's rows of the pair's 32 columns
  double2 G[JC][JC + 1];        // full pair Gram (identical in every CTA of the pair)
  double2 Q[JC][JC + 1];        // partial Gram, then the accumulated rotation
  double2 Gf[JC / 2][JC + 1];   // this CTA's slice of the reduced Gram (JC/cs rows, cs >= 2)
  double rc[JC / 2];            // rotations of the current inner step
  double2 rs[JC / 2];
  int cols[JC];
  JacobiWork W;
  int64_t aoff;
  int k, rows_g, rows_tot, rotate;
  double z2;
};

// Where a CTA of a round works: its sector, block pair, row part and columns.
struct JacTask {
  JacobiWork W;
  int pair, slot, part, cs, sweep, rr, valid, gslot;
};

__device__ __forceinline__ JacTask jac_task(const JacobiWork* __restrict__ work, int n_work, int t) {
  const int gc = blockIdx.x / JCL;
  int lo = 0, hi = n_work - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (work[mid].cta_start <= gc) lo = mid; else hi = mid - 1;
  }
  JacTask T;
  T.W = work[lo];
  const int cr = blockIdx.x % JCL;
  T.cs = T.W.cs;
  T.slot = cr / T.cs;
  T.part = cr % T.cs;
  T.pair = (gc - T.W.cta_start) * (JCL / T.cs) + T.slot;
  T.valid = T.pair < T.W.npairs;
  T.sweep = t / T.W.rounds;
  T.rr = t % T.W.rounds;
  T.gslot = gc * JCL + T.slot * T.cs;   // one slot per block pair of the launch
  return T;
}

// the pair's 32 columns (-1: padding) for round rr of the circle method
__device__ __forceinline__ int jac_col(const JacTask& T, int c, int k) {
  const int nbp = T.W.nblk + (T.W.nblk & 1);
  auto blk_at = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + T.rr) % (nbp - 1); };
  const int b = c < JB ? blk_at(T.pair) : blk_at(nbp - 1 - T.pair);
  const int col = b * JB + (c % JB);
  return (T.valid && b < T.W.nblk && col < k) ? col : -1;
}

__device__ __forceinline__ void jac_rows(const JacTask& T, int rows_tot, int rows_g, int& r0, int& nr,
                                         int& ng) {
  const int chunk = ((rows_tot + T.cs - 1) / T.cs + 15) / 16 * 16;
  r0 = T.part * chunk;
  nr = T.valid ? max(0, min(rows_tot, r0 + chunk) - r0) : 0;
  ng = T.valid ? max(0, min(rows_g, r0 + chunk) - r0) : 0;
}

// K1 of a round: pair Gram (rows split over cs CTAs of a cluster, reduced through
// distributed shared memory in a fixed order), convergence test, and -- on the pair's
// first CTA only -- one cyclic Jacobi sweep on the 32 x 32 Gram; Q and the rotate flag
// go to global memory for K2.  The other CTAs of the pair leave after the reduction.
__global__ __launch_bounds__(JNT) void jacobi_gram_kernel(const SectorDesc* __restrict__ sd,
                                                          const JacobiWork* __restrict__ work,
                                                          int n_work, int t,
                                                          const cplx* __restrict__ abuf,
                                                          int* __restrict__ rot_count,
                                                          const double* __restrict__ nf2,
                                                          double tol, int max_sweeps,
                                                          cplx* __restrict__ qbuf,
                                                          int* __restrict__ qflag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  JacSmem& S = *reinterpret_cast<JacSmem*>(smem_raw);
  cg::cluster_group cluster = cg::this_cluster();
  const int tid = threadIdx.x;
  const JacTask T = jac_task(work, n_work, t);
  if (tid == 0) {
    const SectorDesc& D = sd[T.W.sector];
    S.k = D.k;
    S.rows_g = D.rows_g;
    S.rows_tot = D.rows_tot;
    S.aoff = D.a_off;
    // numerical-rank floor: columns with |a|^2 <= z2 are exact zeros for the SVD
    const double zf = 16.0 * 2.220446049250313e-16 * sqrt((double)D.rows_g);
    S.z2 = zf * zf * nf2[T.W.sector];
    S.rotate = 0;
  }
  if (T.valid && T.part == 0 && tid == 0) qflag[T.gslot] = 0;
  __syncthreads();
  // every exit before the first cluster barrier depends on (sector, t) only, so the
  // whole cluster takes it together
  if (T.sweep >= max_sweeps) return;
  int* cnt = rot_count + 3 * T.W.sector;
  // the counter of sweep w+1 is cleared during sweep w (nobody else touches it then),
  // before the converged exit so that a converged sector keeps reading zeros
  if (T.rr == 0 && T.pair == 0 && T.part == 0 && tid == 0) cnt[(T.sweep + 1) % 3] = 0;
  if (T.sweep >= 1 && cnt[(T.sweep - 1) % 3] == 0) return;   // converged
  const int k = S.k;
  if (tid < JC) S.cols[tid] = jac_col(T, tid, k);
  int r0, nr, ng;
  jac_rows(T, S.rows_tot, S.rows_g, r0, nr, ng);
  const int rows_g = S.rows_g;
  const int cs = T.cs, part = T.part, sl = JC / cs, base = T.slot * cs;
  const cplx* A = abuf + S.aoff;
  __syncthreads();

  // ---- 1. this CTA's rows -> shared memory; partial Gram over its Gram rows
  for (int e = tid; e < ng * JC; e += JNT) {
    const int r = e / JC, c = e % JC;
    double2 v = make_double2(0.0, 0.0);
    if (S.cols[c] >= 0) v = *reinterpret_cast<const double2*>(A + (int64_t)(r0 + r) * k + S.cols[c]);
    S.tile[r][c] = v;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, li = lane >> 2, lk = lane & 3;
  {
    // G[i][j] = sum_r conj(X[r][i]) X[r][j] on the FP64 tensor path: warp w owns the
    // 8 x 8 tiles (I, J) = (w / 2, 2 (w % 2) + {0, 1}); rows in chunks of 4;
    // (ar - i ai)(br + i bi) = (ar br + ai bi) + i (ar bi - ai br)
    const int I = warp >> 1, J0 = 2 * (warp & 1);
    double2 gre[2] = {make_double2(0, 0), make_double2(0, 0)};
    double2 gim[2] = {make_double2(0, 0), make_double2(0, 0)};
    for (int k0 = 0; k0 < ng; k0 += 4) {
      const int r = k0 + lk;
      const double2 a = r < ng ? S.tile[r][8 * I + li] : make_double2(0.0, 0.0);
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {
        const double2 b = r < ng ? S.tile[r][8 * (J0 + jj) + li] : make_double2(0.0, 0.0);
        dmma(gre[jj], a.x, b.x);
        dmma(gre[jj], a.y, b.y);
        dmma(gim[jj], a.x, b.y);
        dmma(gim[jj], -a.y, b.x);
      }
    }
    // the partial Gram lives in Q's storage until the rotation is accumulated there
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) {
      const int row = 8 * I + li, col = 8 * (J0 + jj) + 2 * lk;
      S.Q[row][col] = make_double2(gre[jj].x, gim[jj].x);
      S.Q[row][col + 1] = make_double2(gre[jj].y, gim[jj].y);
    }
  }
  cluster.sync();
  // ---- 2. reduce: this CTA sums Gram rows [part*sl, part*sl + sl) over the pair's cs
  //         CTAs, in rank order
  if (T.valid && cs > 1) {
    for (int e = tid; e < sl * JC; e += JNT) {
      const int r = e / JC, c = e % JC;
      double sx = 0.0, sy = 0.0;
      for (int q = 0; q < cs; ++q) {
        const JacSmem* R = cluster.map_shared_rank(&S, base + q);
        const double2 v = R->Q[part * sl + r][c];
        sx += v.x;
        sy += v.y;
      }
      S.Gf[r][c] = make_double2(sx, sy);
    }
  }
  cluster.sync();
  // ---- 3. the pair's first CTA gathers the reduced Gram
  if (T.valid && part == 0) {
    for (int e = tid; e < JC * JC; e += JNT) {
      const int r = e / JC, c = e % JC;
      if (cs == 1) {
        S.G[r][c] = S.Q[r][c];
      } else {
        const JacSmem* R = cluster.map_shared_rank(&S, base + r / sl);
        S.G[r][c] = R->Gf[r % sl][c];
      }
    }
  }
  cluster.sync();   // after this no CTA touches another CTA's shared memory
  if (!(T.valid && part == 0)) return;

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
  if (tid == 0) atomicAdd(cnt + T.sweep % 3, 1);

  // ---- 5. one cyclic Jacobi sweep on the 32 x 32 Gram, accumulating Q.  A step rotates
  //         16 disjoint column pairs: threads 0-15 compute the rotations while the others
  //         fetch their operands; then G' = J^H G J, split into independent 2 x 2 blocks
  //         J_P1^H G[P1][P2] J_P2 (upper block triangle + Hermitian mirror), and Q' = Q J.
  for (int e = tid; e < JC * JC; e += JNT) S.Q[e / JC][e % JC] = make_double2((e / JC) == (e % JC) ? 1.0 : 0.0, 0.0);
  int P1 = -1, P2 = -1;
  if (tid < (JC / 2) * (JC / 2 + 1) / 2) {
    int rem = tid;
    P1 = 0;
    while (rem >= JC / 2 - P1) { rem -= JC / 2 - P1; ++P1; }
    P2 = P1 + rem;
  }
  const int qp = tid & 15, qr = tid >> 4;
  __syncthreads();
  for (int step = 0; step < JC - 1; ++step) {
    auto idx = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + step) % (JC - 1); };
    auto pq = [&](int P, int& p, int& q) {
      p = idx(P);
      q = idx(JC - 1 - P);
      if (p > q) { int tmp = p; p = q; q = tmp; }
    };
    // ---- phase A: rotations (zero-division form) and operand loads
    if (tid < JC / 2) {
      int p, q;
      pq(tid, p, q);
      const double a = S.G[p][p].x, d = S.G[q][q].x;
      const double2 g = S.G[p][q];
      const double g2 = g.x * g.x + g.y * g.y;
      double c = 1.0;
      double2 se = make_double2(0.0, 0.0);
      // cos 2t = |d - a| / r, r = sqrt((d - a)^2 + 4 |g|^2), c = sqrt((1 + cos 2t) / 2),
      // s e^{i alpha} = sign(d - a) g / (r c).  The off-diagonal threshold is tol / 4: a
      // pair the pair test flags must be rotated here even if this Gram's rounding
      // puts it slightly lower.
      if (g2 > 0.0 && a > z2 && d > z2 && a > t2 * d && d > t2 * a && g2 > 0.0625 * t2 * a * d) {
        const double dd = d - a;
        const double ir = rsqrt(fma(dd, dd, 4.0 * g2));
        const double c2 = fma(0.5 * fabs(dd), ir, 0.5);
        const double ic = rsqrt(c2);
        c = c2 * ic;
        const double f = copysign(ir * ic, dd);
        se = make_double2(f * g.x, f * g.y);
      }
      S.rc[tid] = c;
      S.rs[tid] = se;
    }
    int p1 = 0, q1 = 0, p2 = 0, q2 = 0, pa, qa;
    double2 b00 = make_double2(0, 0), b01 = b00, b10 = b00, b11 = b00;
    if (P1 >= 0) {
      pq(P1, p1, q1);
      pq(P2, p2, q2);
      b00 = S.G[p1][p2]; b01 = S.G[p1][q2]; b10 = S.G[q1][p2]; b11 = S.G[q1][q2];
    }
    pq(qp, pa, qa);
    const double2 qv0 = S.Q[qr][pa], qw0 = S.Q[qr][qa];
    const double2 qv1 = S.Q[qr + 16][pa], qw1 = S.Q[qr + 16][qa];
    __syncthreads();
    // ---- phase B: updates
    if (P1 >= 0) {
      const double c1 = S.rc[P1], c2v = S.rc[P2];
      const cplx s1 = cmake(S.rs[P1].x, S.rs[P1].y), s2 = cmake(S.rs[P2].x, S.rs[P2].y);
      const bool r1 = !(c1 == 1.0 && s1.x == 0.0 && s1.y == 0.0);
      const bool r2 = !(c2v == 1.0 && s2.x == 0.0 && s2.y == 0.0);
      if (r1 || r2) {
        const cplx B00 = cmake(b00.x, b00.y), B01 = cmake(b01.x, b01.y);
        const cplx B10 = cmake(b10.x, b10.y), B11 = cmake(b11.x, b11.y);
        // B J2: columns (p2, q2)
        const cplx x00 = csub(cscale(B00, c2v), cmulc(B01, s2)), x01 = cadd(cmul(B00, s2), cscale(B01, c2v));
        const cplx x10 = csub(cscale(B10, c2v), cmulc(B11, s2)), x11 = cadd(cmul(B10, s2), cscale(B11, c2v));
        // J1^H (B J2): rows (p1, q1)
        cplx y00 = csub(cscale(x00, c1), cmul(s1, x10)), y01 = csub(cscale(x01, c1), cmul(s1, x11));
        cplx y10 = cadd(cmulc(x00, s1), cscale(x10, c1)), y11 = cadd(cmulc(x01, s1), cscale(x11, c1));
        if (P1 == P2) {
          y01 = cmake(0.0, 0.0);
          y10 = cmake(0.0, 0.0);
          y00.y = 0.0;
          y11.y = 0.0;
          S.G[p1][p1] = make_double2(y00.x, y00.y);
          S.G[p1][q1] = make_double2(y01.x, y01.y);
          S.G[q1][p1] = make_double2(y10.x, y10.y);
          S.G[q1][q1] = make_double2(y11.x, y11.y);
        } else {
          S.G[p1][p2] = make_double2(y00.x, y00.y);
          S.G[p1][q2] = make_double2(y01.x, y01.y);
          S.G[q1][p2] = make_double2(y10.x, y10.y);
          S.G[q1][q2] = make_double2(y11.x, y11.y);
          // Hermitian mirror
          S.G[p2][p1] = make_double2(y00.x, -y00.y);
          S.G[q2][p1] = make_double2(y01.x, -y01.y);
          S.G[p2][q1] = make_double2(y10.x, -y10.y);
          S.G[q2][q1] = make_double2(y11.x, -y11.y);
        }
      }
    }
    {
      const double c = S.rc[qp];
      const cplx se = cmake(S.rs[qp].x, S.rs[qp].y);
      if (!(c == 1.0 && se.x == 0.0 && se.y == 0.0)) {
        const cplx v0 = cmake(qv0.x, qv0.y), w0 = cmake(qw0.x, qw0.y);
        const cplx v1 = cmake(qv1.x, qv1.y), w1 = cmake(qw1.x, qw1.y);
        const cplx n0 = csub(cscale(v0, c), cmulc(w0, se)), m0 = cadd(cmul(v0, se), cscale(w0, c));
        const cplx n1 = csub(cscale(v1, c), cmulc(w1, se)), m1 = cadd(cmul(v1, se), cscale(w1, c));
        S.Q[qr][pa] = make_double2(n0.x, n0.y);
        S.Q[qr][qa] = make_double2(m0.x, m0.y);
        S.Q[qr + 16][pa] = make_double2(n1.x, n1.y);
        S.Q[qr + 16][qa] = make_double2(m1.x, m1.y);
      }
    }
    __syncthreads();
  }
  // ---- 6. Q and the flag for K2
  cplx* qo = qbuf + (int64_t)T.gslot * JC * JC;
  for (int e = tid; e < JC * JC; e += JNT) {
    const double2 v = S.Q[e / JC][e % JC];
    qo[e] = cmake(v.x, v.y);
  }
  if (tid == 0) qflag[T.gslot] = 1;
}

// K2 of a round: every CTA of a rotated pair applies Q to its rows on the FP64 tensor
// path: warp w owns rows [16 w, 16 w + 16) (two 8-row tiles) x the four 8-column tiles;
// (tr + i ti)(qr + i qi) = (tr qr - ti qi) + i (tr qi + ti qr)
struct ApplySmem {
  double2 tile[RMAX][JC + 1];
  double2 Q[JC][JC + 1];
  int cols[JC];
};

__global__ __launch_bounds__(JNT) void jacobi_apply_kernel(const SectorDesc* __restrict__ sd,
                                                           const JacobiWork* __restrict__ work,
                                                           int n_work, int t, cplx* __restrict__ abuf,
                                                           int max_sweeps,
                                                           const cplx* __restrict__ qbuf,
                                                           const int* __restrict__ qflag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ApplySmem& S = *reinterpret_cast<ApplySmem*>(smem_raw);
  const int tid = threadIdx.x;
  const JacTask T = jac_task(work, n_work, t);
  if (!T.valid || T.sweep >= max_sweeps) return;
  if (!qflag[T.gslot]) return;   // converged sector, or a pair without rotation
  const SectorDesc& D = sd[T.W.sector];
  const int k = D.k;
  int r0, nr, ng;
  jac_rows(T, D.rows_tot, D.rows_g, r0, nr, ng);
  if (nr == 0) return;
  if (tid < JC) S.cols[tid] = jac_col(T, tid, k);
  const cplx* qi = qbuf + (int64_t)T.gslot * JC * JC;
  for (int e = tid; e < JC * JC; e += JNT) {
    const cplx v = ldc(qi + e);
    S.Q[e / JC][e % JC] = make_double2(v.x, v.y);
  }
  __syncthreads();
  cplx* A = abuf + D.a_off;
  for (int e = tid; e < nr * JC; e += JNT) {
    const int r = e / JC, c = e % JC;
    double2 v = make_double2(0.0, 0.0);
    if (S.cols[c] >= 0) v = *reinterpret_cast<const double2*>(A + (int64_t)(r0 + r) * k + S.cols[c]);
    S.tile[r][c] = v;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, li = lane >> 2, lk = lane & 3;
  if (16 * warp < nr) {
    double2 ore[2][4], oim[2][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) { ore[a][c] = make_double2(0, 0); oim[a][c] = make_double2(0, 0); }
#pragma unroll
    for (int k0 = 0; k0 < JC; k0 += 4) {
      double2 tv[2], q[4];
#pragma unroll
      for (int a = 0; a < 2; ++a) tv[a] = S.tile[16 * warp + 8 * a + li][k0 + lk];
#pragma unroll
      for (int c = 0; c < 4; ++c) q[c] = S.Q[k0 + lk][8 * c + li];
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          dmma(ore[a][c], tv[a].x, q[c].x);
          dmma(ore[a][c], -tv[a].y, q[c].y);
          dmma(oim[a][c], tv[a].x, q[c].y);
          dmma(oim[a][c], tv[a].y, q[c].x);
        }
    }
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const int row = 16 * warp + 8 * a + li;
      if (row >= nr) continue;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int c0 = S.cols[8 * c + 2 * lk], c1 = S.cols[8 * c + 2 * lk + 1];
        if (c0 >= 0) stc(A + (int64_t)(r0 + row) * k + c0, cmake(ore[a][c].x, oim[a][c].x));
        if (c1 >= 0) stc(A + (int64_t)(r0 + row) * k + c1, cmake(ore[a][c].y, oim[a][c].y));
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
                                const double* nf2, double tol, int max_sweeps, void* qbuf,
                                int* qflag, cudaStream_t s) {
  if (total_clusters <= 0) return cudaSuccess;
  static bool attr_done = false;
  const int smem1 = (int)sizeof(JacSmem), smem2 = (int)sizeof(ApplySmem);
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(jacobi_gram_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem1);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(jacobi_gram_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(jacobi_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem2);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(total_clusters * JCL, 1, 1);
  cfg.blockDim = dim3(JNT, 1, 1);
  cfg.dynamicSmemBytes = smem1;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = JCL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, jacobi_gram_kernel, sd_dev, work_dev, n_work, t,
                                     reinterpret_cast<const cplx*>(abuf), rot_count, nf2, tol,
                                     max_sweeps, reinterpret_cast<cplx*>(qbuf), qflag);
  if (e != cudaSuccess) return e;
  jacobi_apply_kernel<<<total_clusters * JCL, JNT, smem2, s>>>(
      sd_dev, work_dev, n_work, t, reinterpret_cast<cplx*>(abuf), max_sweeps,
      reinterpret_cast<const cplx*>(qbuf), qflag);
  return cudaGetLastError();
}

int jacobi_qslots(int total_clusters) { return total_clusters * JCL; }

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
