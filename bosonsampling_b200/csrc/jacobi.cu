// Blocked one-sided (Hestenes) Jacobi SVD of every sector, in FP64.
//
// Replaces the reference's per-sector cuSOLVER gesvd (src/beam_splitter_parallel/
// Rank.py:123) / LAPACK svd (src/MPO.py:258).  The Jacobi matrix of a sector is
// T = C diag(Lambda_R) when |L| >= |R| (its orthogonalised columns are sigma * V),
// or [T^H; I] when |L| < |R| (the identity rows accumulate V).  Columns are cut in
// blocks of 16; a round pairs the blocks by the circle method (all sectors of the
// update in one launch pair), and each block pair's rows are cut in parts of at most
// 128 rows:
//   1. (gram kernel) every part holding Gram rows forms its partial 32 x 32 Gram; the
//      last part to finish sums the partials in part order, tests the pair and, if a
//      column pair is not orthogonal to `tol` (relative), runs one cyclic two-sided
//      Jacobi sweep on the Gram (complex rotations, 16 disjoint pairs per step),
//      accumulating the 32 x 32 unitary Q;
//   2. (apply kernel) every part of a rotated pair applies Q to its rows.
// A sector is converged after a sweep without rotations; later rounds of it exit
// at once.  One-sided Jacobi keeps high relative accuracy for small singular values.
// Numerical rank: a column whose norm is <= 16 eps sqrt(rows) ||T||_F is rounding
// noise (the null space of a rank-deficient block); it takes part in no rotation and
// its singular value is reported as 0, as is a column below tol times its partner
// in a pair test.  Without this, noise columns never test orthogonal.
#include "common.cuh"
#include "kernels.h"

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
constexpr int RMAX = 128;     // rows of one part (Gram tile in shared memory)

// Where a CTA of a round works: its sector, block pair and row part.
struct JacTask {
  JacobiWork W;
  int pair, part, sweep, rr, slot;
};

// Gram launch: CTAs [gram_start, gram_start + npairs cs_g) of a work entry, pair-major;
// apply launch: [apply_start, apply_start + npairs cs).
__device__ __forceinline__ JacTask jac_task(const JacobiWork* __restrict__ work, int n_work, int t,
                                            bool apply) {
  const int b = blockIdx.x;
  int lo = 0, hi = n_work - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int st = apply ? work[mid].apply_start : work[mid].gram_start;
    if (st <= b) lo = mid; else hi = mid - 1;
  }
  JacTask T;
  T.W = work[lo];
  const int per = apply ? T.W.cs : T.W.cs_g;
  const int local = b - (apply ? T.W.apply_start : T.W.gram_start);
  T.pair = local / per;
  T.part = local % per;
  T.sweep = t / T.W.rounds;
  T.rr = t % T.W.rounds;
  T.slot = T.W.slot_start + T.pair;
  return T;
}

// circle method over n (even) positions: the item at position pos in step s; position 0
// is fixed, the others turn by one place per step, pairs are (P, n - 1 - P)
__device__ __forceinline__ int circle_at(int pos, int s, int n) {
  return pos == 0 ? 0 : 1 + (pos - 1 + s) % (n - 1);
}

// the pair's c-th column (c < 16: first block, else second; -1: padding)
__device__ __forceinline__ int jac_col(const JacTask& T, int c, int k) {
  const int nbp = T.W.nblk + (T.W.nblk & 1);
  const int b = c < JB ? circle_at(T.pair, T.rr, nbp) : circle_at(nbp - 1 - T.pair, T.rr, nbp);
  const int col = b * JB + (c % JB);
  return (b < T.W.nblk && col < k) ? col : -1;
}

struct GramSmem {
  union {
    double2 tile[RMAX][JC + 1];   // this part's Gram rows of the pair's 32 columns
    double2 G[JC][JC + 1];        // then the pair Gram (upper triangle, i <= j, is used)
  } u;
  double rc[JC / 2];              // rotations of the current inner step
  double2 rs[JC / 2];
  int cols[JC];
  int rotate, last;
  double z2;
};

// pair-Gram element (i, j) from the stored upper triangle
__device__ __forceinline__ cplx gget(const GramSmem& S, int i, int j) {
  if (i <= j) {
    const double2 v = S.u.G[i][j];
    return cmake(v.x, v.y);
  }
  const double2 v = S.u.G[j][i];
  return cmake(v.x, -v.y);
}

__device__ __forceinline__ void gput(GramSmem& S, int i, int j, cplx v) {
  if (i < j) S.u.G[i][j] = make_double2(v.x, v.y);
  else S.u.G[j][i] = make_double2(v.x, -v.y);
}

// the ordered column pair (p < q) of pair P in inner step s
__device__ __forceinline__ void inner_pq(int P, int s, int& p, int& q) {
  p = circle_at(P, s, JC);
  q = circle_at(JC - 1 - P, s, JC);
  if (p > q) { const int x = p; p = q; q = x; }
}

// Round kernel 1: the pair Gram and, in the pair's last CTA to finish, the test and one
// cyclic Jacobi sweep on it.
//   a. every part (up to RMAX Gram rows) loads its rows of the pair's 32 columns and
//      forms a partial Gram on the FP64 tensor path; with several parts the partials go
//      to global memory and the last part to arrive (an arrival counter per pair) sums
//      them in part order, so the Gram does not depend on arrival order;
//   b. no rotation if every column pair is orthogonal to `tol` (relative); else
//   c. a cyclic two-sided sweep (circle order, 16 disjoint rotations per step) on the
//      Gram, accumulating the 32 x 32 unitary Q, which goes to global memory with a
//      flag for the apply kernel.
// The step's rotations are computed once (16 threads) and read by all; the Gram keeps
// only its upper triangle; Q lives in registers in circle-position order -- thread
// (pair L, rows g, g + 16) holds the entries of the two positions of pair L and passes
// them to the neighbouring pairs by warp shuffles when the circle turns, so Q never
// touches shared memory.  After the 31 steps the circle is back at its start and every
// thread holds columns L and 31 - L.
__global__ __launch_bounds__(JNT) void jacobi_gram_kernel(const SectorDesc* __restrict__ sd,
                                                          const JacobiWork* __restrict__ work,
                                                          int n_work, int t,
                                                          const cplx* __restrict__ abuf,
                                                          int* __restrict__ rot_count,
                                                          const double* __restrict__ nf2,
                                                          double tol, int max_sweeps,
                                                          cplx* __restrict__ pbuf,
                                                          int* __restrict__ pcnt,
                                                          cplx* __restrict__ qbuf,
                                                          int* __restrict__ qflag,
                                                          unsigned long long* __restrict__ executed) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GramSmem& S = *reinterpret_cast<GramSmem*>(smem_raw);
  const int tid = threadIdx.x;
  const JacTask T = jac_task(work, n_work, t, false);
  if (T.part == 0 && tid == 0) qflag[T.slot] = 0;
  // every exit before the arrival counter depends on (sector, t) only
  if (T.sweep >= max_sweeps) return;
  int* cnt = rot_count + 3 * T.W.sector;
  // the counter of sweep w+1 is cleared during sweep w (nobody else touches it then),
  // before the converged exit so that a converged sector keeps reading zeros
  if (T.rr == 0 && T.pair == 0 && T.part == 0 && tid == 0) cnt[(T.sweep + 1) % 3] = 0;
  if (T.sweep >= 1 && cnt[(T.sweep - 1) % 3] == 0) return;   // converged
  const SectorDesc& D = sd[T.W.sector];
  const int k = D.k, rows_g = D.rows_g;
  const int r0 = T.part * T.W.chunk;
  const int ng = min(rows_g, r0 + T.W.chunk) - r0;   // >= 1: parts cover the Gram rows
  if (tid < JC) S.cols[tid] = jac_col(T, tid, k);
  if (tid == 0) {
    // numerical-rank floor: columns with |a|^2 <= z2 are exact zeros for the SVD
    const double zf = 16.0 * 2.220446049250313e-16 * sqrt((double)rows_g);
    S.z2 = zf * zf * nf2[T.W.sector];
    S.rotate = 0;
  }
  __syncthreads();

  // ---- a. rows -> shared memory (all loads of a thread in flight), partial Gram
  {
    const cplx* A = abuf + D.a_off;
    const int lane = tid & 31, wrow = tid >> 5;
    const int col = S.cols[lane];
    constexpr int PER = RMAX * JC / JNT;
    double2 v[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int r = wrow + i * (JNT / JC);
      v[i] = make_double2(0.0, 0.0);
      if (r < ng && col >= 0) v[i] = *reinterpret_cast<const double2*>(A + (int64_t)(r0 + r) * k + col);
    }
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int r = wrow + i * (JNT / JC);
      if (r < ng) S.u.tile[r][lane] = v[i];
    }
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, li = lane >> 2, lk = lane & 3;
  // G[i][j] = sum_r conj(X[r][i]) X[r][j] on 8 x 8 tiles, rows in chunks of 4;
  // (ar - i ai)(br + i bi) = (ar br + ai bi) + i (ar bi - ai br)
  // The Gram is Hermitian: only its 10 upper 8 x 8 tiles (I <= J) are formed, spread
  // over the warps so that no scheduler (warps w and w + 4) carries more than three.
  int I0, J0, I1 = 0, J1 = 0, nt = 1;
  switch (warp) {
    case 0: I0 = 0; J0 = 0; I1 = 0; J1 = 1; nt = 2; break;
    case 1: I0 = 0; J0 = 3; I1 = 1; J1 = 1; nt = 2; break;
    case 2: I0 = 1; J0 = 3; break;
    case 3: I0 = 2; J0 = 3; break;
    case 4: I0 = 0; J0 = 2; break;
    case 5: I0 = 1; J0 = 2; break;
    case 6: I0 = 2; J0 = 2; break;
    default: I0 = 3; J0 = 3; break;
  }
  double2 gre[2] = {make_double2(0, 0), make_double2(0, 0)};
  double2 gim[2] = {make_double2(0, 0), make_double2(0, 0)};
  for (int k0 = 0; k0 < ng; k0 += 4) {
    const int r = k0 + lk;
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) {
      if (jj >= nt) break;   // warp-uniform
      const int I = jj == 0 ? I0 : I1, J = jj == 0 ? J0 : J1;
      const double2 a = r < ng ? S.u.tile[r][8 * I + li] : make_double2(0.0, 0.0);
      const double2 b = r < ng ? S.u.tile[r][8 * J + li] : make_double2(0.0, 0.0);
      dmma(gre[jj], a.x, b.x);
      dmma(gre[jj], a.y, b.y);
      dmma(gim[jj], a.x, b.y);
      dmma(gim[jj], -a.y, b.x);
    }
  }
  __syncthreads();   // the tile is dead; G takes its place
  if (tid == 0) atomicAdd(executed, (unsigned long long)ng);   // executed: ng rows of 10 Gram tiles
  const int cs_g = T.W.cs_g;
  if (cs_g == 1) {
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) {
      if (jj >= nt) break;
      const int row = 8 * (jj == 0 ? I0 : I1) + li, c0 = 8 * (jj == 0 ? J0 : J1) + 2 * lk;
      S.u.G[row][c0] = make_double2(gre[jj].x, gim[jj].x);
      S.u.G[row][c0 + 1] = make_double2(gre[jj].y, gim[jj].y);
    }
  } else {
    cplx* pp = pbuf + (int64_t)blockIdx.x * JC * JC;
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) {
      if (jj >= nt) break;
      const int row = 8 * (jj == 0 ? I0 : I1) + li, c0 = 8 * (jj == 0 ? J0 : J1) + 2 * lk;
      __stcg(reinterpret_cast<double2*>(pp + row * JC + c0), make_double2(gre[jj].x, gim[jj].x));
      __stcg(reinterpret_cast<double2*>(pp + row * JC + c0 + 1), make_double2(gre[jj].y, gim[jj].y));
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      const int old = atomicAdd(pcnt + T.slot, 1);
      __threadfence();
      S.last = (old == cs_g - 1);
    }
    __syncthreads();
    if (!S.last) return;
    // the last part: fixed-order sum of the upper triangles of the pair's partials
    const cplx* p0 = pbuf + (int64_t)(blockIdx.x - T.part) * JC * JC;
    for (int e = tid; e < JC * JC; e += JNT) {
      const int i = e / JC, j = e % JC;
      if (j < i) continue;
      double sx = 0.0, sy = 0.0;
#pragma unroll 4
      for (int q = 0; q < cs_g; ++q) {
        const double2 v = __ldcg(reinterpret_cast<const double2*>(p0 + (int64_t)q * JC * JC + e));
        sx += v.x;
        sy += v.y;
      }
      S.u.G[i][j] = make_double2(sx, sy);
    }
    if (tid == 0) pcnt[T.slot] = 0;   // ready for the next round
  }
  __syncthreads();

  // ---- b. convergence test (relative tolerance on |a_i^H a_j|)
  if (tol <= 0.0) tol = fmax(8.0 * 2.220446049250313e-16, 4.0 * 2.220446049250313e-16 * sqrt((double)rows_g));
  const double t2 = tol * tol, z2 = S.z2;
  for (int e = tid; e < JC * JC; e += JNT) {
    const int i = e / JC, j = e % JC;
    if (j <= i) continue;
    const double dii = S.u.G[i][i].x, djj = S.u.G[j][j].x;
    const double2 g = S.u.G[i][j];
    const double a2 = g.x * g.x + g.y * g.y;
    // a column at the numerical-rank floor, or below tol times its partner, is rounding
    // noise along the partner and is never rotated against it
    if (dii > z2 && djj > z2 && dii > t2 * djj && djj > t2 * dii && a2 > t2 * dii * djj) S.rotate = 1;
  }
  __syncthreads();
  if (!S.rotate) return;
  if (tid == 0) atomicAdd(cnt + T.sweep % 3, 1);

  // ---- c. one cyclic Jacobi sweep on the Gram
  // block roles: thread < 136 updates the 2 x 2 block (P1, P2), P1 <= P2, of the pair
  // positions; lanes 0-15 of the last warp compute the step's rotations
  int P1 = -1, P2 = -1;
  if (tid < (JC / 2) * (JC / 2 + 1) / 2) {
    int rem = tid;
    P1 = 0;
    while (rem >= JC / 2 - P1) { rem -= JC / 2 - P1; ++P1; }
    P2 = P1 + rem;
  }
  const int rt = tid - (JNT - 32);
  const int L = tid & 15, grp = tid >> 4;
  // Q at step 0 is the identity: positions hold columns L (upper) and 31 - L (lower);
  // rows grp < 16 meet column L only on the diagonal, rows grp + 16 meet 31 - L
  cplx qu0 = cmake(grp == L ? 1.0 : 0.0, 0.0), qu1 = cmake(0.0, 0.0);
  cplx ql0 = cmake(0.0, 0.0), ql1 = cmake(grp + 16 == JC - 1 - L ? 1.0 : 0.0, 0.0);
  for (int step = 0; step < JC - 1; ++step) {
    // ---- phase A: rotations (zero-division form) and block operands
    if (rt >= 0 && rt < JC / 2) {
      int p, q;
      inner_pq(rt, step, p, q);
      const double a = S.u.G[p][p].x, d = S.u.G[q][q].x;
      const double2 g = S.u.G[p][q];
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
      S.rc[rt] = c;
      S.rs[rt] = se;
    }
    int p1 = 0, q1 = 0, p2 = 0, q2 = 0;
    cplx B00 = cmake(0.0, 0.0), B01 = B00, B10 = B00, B11 = B00;
    if (P1 >= 0) {
      inner_pq(P1, step, p1, q1);
      inner_pq(P2, step, p2, q2);
      B00 = gget(S, p1, p2);
      B01 = gget(S, p1, q2);
      B10 = gget(S, q1, p2);
      B11 = gget(S, q1, q2);
    }
    const int cu = circle_at(L, step, JC), cl = circle_at(JC - 1 - L, step, JC);
    __syncthreads();
    // ---- phase B: block updates G' = J^H G J, and Q' = Q J
    if (P1 >= 0) {
      const double c1 = S.rc[P1], c2v = S.rc[P2];
      const cplx s1 = cmake(S.rs[P1].x, S.rs[P1].y), s2 = cmake(S.rs[P2].x, S.rs[P2].y);
      const bool r1 = !(c1 == 1.0 && s1.x == 0.0 && s1.y == 0.0);
      const bool r2 = !(c2v == 1.0 && s2.x == 0.0 && s2.y == 0.0);
      if (r1 || r2) {
        // B J2: columns (p2, q2)
        const cplx x00 = csub(cscale(B00, c2v), cmulc(B01, s2)), x01 = cadd(cmul(B00, s2), cscale(B01, c2v));
        const cplx x10 = csub(cscale(B10, c2v), cmulc(B11, s2)), x11 = cadd(cmul(B10, s2), cscale(B11, c2v));
        // J1^H (B J2): rows (p1, q1)
        const cplx y00 = csub(cscale(x00, c1), cmul(s1, x10)), y01 = csub(cscale(x01, c1), cmul(s1, x11));
        const cplx y10 = cadd(cmulc(x00, s1), cscale(x10, c1)), y11 = cadd(cmulc(x01, s1), cscale(x11, c1));
        if (P1 == P2) {
          S.u.G[p1][p1] = make_double2(y00.x, 0.0);
          S.u.G[p1][q1] = make_double2(0.0, 0.0);
          S.u.G[q1][q1] = make_double2(y11.x, 0.0);
        } else {
          gput(S, p1, p2, y00);
          gput(S, p1, q2, y01);
          gput(S, q1, p2, y10);
          gput(S, q1, q2, y11);
        }
      }
    }
    {
      const double c = S.rc[L];
      const cplx se = cmake(S.rs[L].x, S.rs[L].y);
      if (!(c == 1.0 && se.x == 0.0 && se.y == 0.0)) {
        // columns (p, q) = (cu, cl) or (cl, cu): v = Q[:, p], w = Q[:, q]
        const bool up = cu < cl;
        const cplx v0 = up ? qu0 : ql0, w0 = up ? ql0 : qu0;
        const cplx v1 = up ? qu1 : ql1, w1 = up ? ql1 : qu1;
        const cplx n0 = csub(cscale(v0, c), cmulc(w0, se)), m0 = cadd(cmul(v0, se), cscale(w0, c));
        const cplx n1 = csub(cscale(v1, c), cmulc(w1, se)), m1 = cadd(cmul(v1, se), cscale(w1, c));
        qu0 = up ? n0 : m0;
        ql0 = up ? m0 : n0;
        qu1 = up ? n1 : m1;
        ql1 = up ? m1 : n1;
      }
      // turn the circle: position j takes the column of position j + 1 (31 -> 1), so
      // pair L's upper entry comes from pair L + 1's upper (pair 15: its own lower) and
      // its lower from pair L - 1's lower (pair 0: pair 1's upper); position 0 stays
      const cplx du0 = cmake(__shfl_down_sync(0xffffffffu, qu0.x, 1, 16), __shfl_down_sync(0xffffffffu, qu0.y, 1, 16));
      const cplx du1 = cmake(__shfl_down_sync(0xffffffffu, qu1.x, 1, 16), __shfl_down_sync(0xffffffffu, qu1.y, 1, 16));
      const cplx ul0 = cmake(__shfl_up_sync(0xffffffffu, ql0.x, 1, 16), __shfl_up_sync(0xffffffffu, ql0.y, 1, 16));
      const cplx ul1 = cmake(__shfl_up_sync(0xffffffffu, ql1.x, 1, 16), __shfl_up_sync(0xffffffffu, ql1.y, 1, 16));
      const cplx nu0 = L == 0 ? qu0 : (L == 15 ? ql0 : du0), nu1 = L == 0 ? qu1 : (L == 15 ? ql1 : du1);
      const cplx nl0 = L == 0 ? du0 : ul0, nl1 = L == 0 ? du1 : ul1;
      qu0 = nu0;
      qu1 = nu1;
      ql0 = nl0;
      ql1 = nl1;
    }
    __syncthreads();
  }
  // ---- Q (column order again) and the flag for the apply kernel
  cplx* qo = qbuf + (int64_t)T.slot * JC * JC;
  stc(qo + grp * JC + L, qu0);
  stc(qo + (grp + 16) * JC + L, qu1);
  stc(qo + grp * JC + (JC - 1 - L), ql0);
  stc(qo + (grp + 16) * JC + (JC - 1 - L), ql1);
  if (tid == 0) qflag[T.slot] = 1;
}

// Round kernel 2: every part of a rotated pair applies Q to its rows on the FP64 tensor
// path, straight from global memory into mma fragments: warp w owns rows
// [16 w, 16 w + 16), one 8-row tile at a time, x the four 8-column tiles.  The complex
// product takes three real products (Gauss):
// (tr + i ti)(qr + i qi) = (tr qr - ti qi) + i ((tr + ti)(qr + qi) - tr qr - ti qi).
__global__ __launch_bounds__(JNT) void jacobi_apply_kernel(const SectorDesc* __restrict__ sd,
                                                           const JacobiWork* __restrict__ work,
                                                           int n_work, int t, cplx* __restrict__ abuf,
                                                           int max_sweeps,
                                                           const cplx* __restrict__ qbuf,
                                                           const int* __restrict__ qflag,
                                                           unsigned long long* __restrict__ executed) {
  __shared__ double2 Qs[JC][JC + 1];
  __shared__ double Qsum[JC][JC + 1];   // Re Q + Im Q
  __shared__ int cols[JC];
  const int tid = threadIdx.x;
  const JacTask T = jac_task(work, n_work, t, true);
  if (T.sweep >= max_sweeps) return;
  if (!qflag[T.slot]) return;   // converged sector, or a pair without rotation
  const SectorDesc& D = sd[T.W.sector];
  const int k = D.k;
  const int r0 = T.part * T.W.chunk;
  const int nr = min(D.rows_tot, r0 + T.W.chunk) - r0;
  if (tid == 0) atomicAdd(executed + 1, (unsigned long long)nr);   // executed: nr rows rotated
  if (tid < JC) cols[tid] = jac_col(T, tid, k);
  const cplx* qi = qbuf + (int64_t)T.slot * JC * JC;
#pragma unroll
  for (int i = 0; i < JC * JC / JNT; ++i) {
    const int e = tid + i * JNT;
    const cplx v = ldc(qi + e);
    Qs[e / JC][e % JC] = make_double2(v.x, v.y);
    Qsum[e / JC][e % JC] = v.x + v.y;
  }
  __syncthreads();
  cplx* A = abuf + D.a_off;
  const int warp = tid >> 5, lane = tid & 31, li = lane >> 2, lk = lane & 3;
  if (16 * warp >= nr) return;
#pragma unroll 1
  for (int a = 0; a < 2; ++a) {
    const int row = 16 * warp + 8 * a + li;
    double2 tv[JC / 4];
#pragma unroll
    for (int kk = 0; kk < JC / 4; ++kk) {
      const int col = cols[4 * kk + lk];
      tv[kk] = make_double2(0.0, 0.0);
      if (row < nr && col >= 0) tv[kk] = *reinterpret_cast<const double2*>(A + (int64_t)(r0 + row) * k + col);
    }
    // t1 = Tr Qr, t2 = Ti Qi, t3 = (Tr + Ti)(Qr + Qi) on the four column tiles
    double2 t1[4], t2[4], t3[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      t1[c] = make_double2(0, 0);
      t2[c] = make_double2(0, 0);
      t3[c] = make_double2(0, 0);
    }
#pragma unroll
    for (int kk = 0; kk < JC / 4; ++kk) {
      const double ts = tv[kk].x + tv[kk].y;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const double2 q = Qs[4 * kk + lk][8 * c + li];
        const double qs = Qsum[4 * kk + lk][8 * c + li];
        dmma(t1[c], tv[kk].x, q.x);
        dmma(t2[c], tv[kk].y, q.y);
        dmma(t3[c], ts, qs);
      }
    }
    if (row < nr) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int c0 = cols[8 * c + 2 * lk], c1 = cols[8 * c + 2 * lk + 1];
        if (c0 >= 0)
          stc(A + (int64_t)(r0 + row) * k + c0, cmake(t1[c].x - t2[c].x, t3[c].x - t1[c].x - t2[c].x));
        if (c1 >= 0)
          stc(A + (int64_t)(r0 + row) * k + c1, cmake(t1[c].y - t2[c].y, t3[c].y - t1[c].y - t2[c].y));
      }
    }
  }
}

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
                                int gram_ctas, int apply_ctas, int t, void* abuf, int* rot_count,
                                const double* nf2, double tol, int max_sweeps, void* pbuf,
                                int* pcnt, void* qbuf, int* qflag, unsigned long long* executed,
                                cudaStream_t s) {
  if (gram_ctas <= 0) return cudaSuccess;
  const int smem1 = (int)sizeof(GramSmem);
  // once per process (thread-safe initialisation; several host threads launch rounds)
  static const cudaError_t attr = cudaFuncSetAttribute(
      jacobi_gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GramSmem));
  if (attr != cudaSuccess) return attr;
  jacobi_gram_kernel<<<gram_ctas, JNT, smem1, s>>>(
      sd_dev, work_dev, n_work, t, reinterpret_cast<const cplx*>(abuf), rot_count, nf2, tol,
      max_sweeps, reinterpret_cast<cplx*>(pbuf), pcnt, reinterpret_cast<cplx*>(qbuf), qflag, executed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  jacobi_apply_kernel<<<apply_ctas, JNT, 0, s>>>(sd_dev, work_dev, n_work, t,
                                                 reinterpret_cast<cplx*>(abuf), max_sweeps,
                                                 reinterpret_cast<const cplx*>(qbuf), qflag, executed);
  return cudaGetLastError();
}

int jacobi_rows_per_part() { return RMAX; }

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
