// Gram / Hermitian-eigen route of the per-sector SVD (the mixed-precision form).
//
// The reference takes a thin SVD of every sector (cuSOLVER gesvd,
// src/beam_splitter_parallel/Rank.py:122-125; LAPACK, src/MPO.py:258).  The truncation
// keeps only the largest chi singular triplets over all sectors (at chi = 1024 about a
// third of the candidates, cut near 3e-3 of the largest singular value), so this route
// forms the Gram matrix of each sector in FP64 and solves a Hermitian eigenproblem:
//   X = T (|L| >= |R|) or T^H (|L| < |R|), G = X^H X (k x k, k = min(|L|, |R|)),
//   1. Householder reduction of G to a real symmetric tridiagonal (d, e): G = Q T Q^H,
//      Q = H_0 ... H_{k-2}, H_j = I - tau_j v_j v_j^H (LAPACK's zhetd2 conventions,
//      lower storage), one thread-block cluster per sector, rows owned cyclically by
//      the cluster's CTAs, the rank-2 update of step j - 1 fused with the matrix-vector
//      product of step j (one read and one write of the trailing matrix per step), one
//      cluster barrier per step;
//   2. every eigenvalue by multisection of Sturm counts (one warp per eigenvalue, 32
//      points per pass), sigma = sqrt(lambda), zero below the numerical floor;
//   3. after the global top-chi selection: eigenvectors of the kept eigenvalues by
//      inverse iteration on T - lambda I (partial pivoting; members of tight clusters
//      of eigenvalues are orthogonalised against each other), then y = Q z.
// V = y directly when X = T^H (G = T T^H), else V = T Y diag(1/sigma) (a GEMM).
// Eigenvalue errors are about eps ||G||: singular values above ~1e-6 of the largest
// are accurate to ~1e-10 relative, far below the truncation cut.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include "common.cuh"
#include "kernels.h"
#include "pipeline.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr double EPS = 2.220446049250313e-16;
// Threads per CTA of the tridiagonalisation: two instantiations, 128 threads (6 CTAs per
// SM by registers) for the small size classes and 256 threads (2 per SM) for the classes
// from BSMPO_TD_WIDE on (0-4, default 4: none).  Measured at chi = 1024 with 16
// concurrent updates: 256 threads for every class 656-672 BS-updates/s against 733-744
// for none; for the classes with k > 320 only (BSMPO_TD_WIDE=2) 760-776 against 790-793
// in the same run -- the wider CTAs shorten the largest sector's chain but cost resident
// CTA slots the concurrent updates share.
constexpr int TD_NT = 128;
constexpr int TD_NT_WIDE = 256;
constexpr int TD_CLASSES = 4;   // cluster sizes 1, 2, 4, 8 CTAs per sector, by sector size
constexpr int TD_NW_MAX = TD_NT_WIDE / 32;
// bulk-copy ring of each warp: about BSMPO_TD_RING_KB per CTA, 1, 2 or TD_MAXSLOT row
// slots (pairs of rows share one pass over the vectors)
#ifndef BSMPO_TD_RING_KB
#define BSMPO_TD_RING_KB 64
#endif
constexpr int TD_MAXSLOT = 4;
#ifndef BSMPO_TD_PAIRS
#define BSMPO_TD_PAIRS 1   // rows two at a time (0: one at a time)
#endif
static_assert(TD_NW_MAX <= 8, "the per-warp scalars of the tridiagonalisation hold 8 warps");

// shared memory of the tridiagonalisation with `slots` ring slots per warp (kmax = the
// launch's largest k, cl = CTAs per sector): the row rings, v and w of two steps, the
// published and the copied row, p of the own rows (two steps), 64 scalars and the rings'
// mbarriers
__host__ __device__ inline size_t td_smem_for(int kmax, int cl, int slots, int nw) {
  const int own = kmax / cl + 1;
  return sizeof(cplx) * ((size_t)nw * slots * kmax + 6 * (size_t)kmax + 2 * (size_t)own) +
         64 * sizeof(double) + nw * TD_MAXSLOT * sizeof(uint64_t);
}

// ring slots per warp: a power of two, 2 to TD_MAXSLOT within about BSMPO_TD_RING_KB per
// CTA, fewer where a one-CTA sector of size kmax would not fit in 227 KB
__host__ __device__ inline int td_slots(int kmax, int nw) {
  const long long fit = (long long)BSMPO_TD_RING_KB * 1024 / ((long long)nw * kmax * (long long)sizeof(cplx));
  int s = fit >= TD_MAXSLOT ? TD_MAXSLOT : 2;
  while (s > 1 && td_smem_for(kmax, 1, s, nw) > 227 * 1024) s >>= 1;
  return s;
}

// dynamic shared memory of a tridiagonalisation launch with nw warps per CTA
__host__ __device__ inline size_t td_smem_bytes(int kmax, int cl, int nw) {
  return td_smem_for(kmax, cl, td_slots(kmax, nw), nw);
}

__device__ __forceinline__ cplx warp_sum(cplx v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// a - (x conj(y) + u conj(z)), eight fused multiply-adds (the rank-2 update of one entry)
__device__ __forceinline__ cplx crank2(cplx a, cplx x, cplx y, cplx u, cplx z) {
  a.x = fma(-x.x, y.x, a.x);
  a.x = fma(-x.y, y.y, a.x);
  a.x = fma(-u.x, z.x, a.x);
  a.x = fma(-u.y, z.y, a.x);
  a.y = fma(-x.y, y.x, a.y);
  a.y = fma(x.x, y.y, a.y);
  a.y = fma(-u.y, z.x, a.y);
  a.y = fma(u.x, z.y, a.y);
  return a;
}

// a / b for complex b != 0
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  const double den = b.x * b.x + b.y * b.y;
  return cmake((a.x * b.x + a.y * b.y) / den, (a.y * b.x - a.x * b.y) / den);
}

// ---------------------------------------------------------------------------------
// 1. Tridiagonalisation.  Cluster c handles sector list[c]; its cl CTAs (1, 2, 4 or 8,
//    by sector size: a small sector would spend its steps waiting at barriers of a big
//    cluster) own the rows i = rank (mod cl).  Every CTA holds the reflector vectors
//    and a copy of the row being reduced, so one cluster barrier per step suffices.
//    Step j (trailing size t = k - j - 1):
//    R   every CTA (warp 0): row j as the previous pass left it, minus the pending
//        rank-2 update of step j - 1, gives d_j and the reflector (zlarfg: beta real,
//        tau_j, v_j), computed redundantly and bit-identically in every CTA (the same
//        inputs, the same warp reduction);
//    P   every CTA, its rows i > j: A[i][l] -= v'_i conj(w'_l) + w'_i conj(v'_l) (v', w'
//        of step j - 1), write back, p_i = tau sum_l A[i][l] v_l, partial
//        c = sum conj(p_i) v_i; the owner of row j + 1 also publishes that row;
//    --  cluster barrier
//    G   every CTA: c = sum of the partials (fixed order), w_j = p - tau c / 2 v from the
//        owners' p, and a copy of the published row j + 1 (the next step's R); the owner
//        of row j stores v_j there for the back-transformation, d_j, e_j = beta, tau_j.
//    p and the partials are double-buffered by step parity; the published row is written
//    again only cl steps later: every next write follows the next barrier, which no CTA
//    passes before every CTA has finished its G.
//    Rows stream through shared memory.  Warp w of a CTA handles its own rows number
//    r = w (mod 4) in every step (row i = rank + r cl), through a private ring of row
//    slots: its lane 0 issues a bulk copy (cp.async.bulk, completion counted on the
//    slot's mbarrier) of the row's trailing segment as soon as the slot is free and the
//    warp has written that row back in the previous step, so the copies run ahead of
//    the pass -- across the barrier, G and the next R into the next step's first rows
//    -- instead of one L2 round trip per load.  A row is read and written by one warp
//    only; its write-back is ordered before the next bulk read of it by a proxy fence
//    of the writing lanes and the warp's synchronisation.
template <int TD_NT_, int MINB>
__global__ void __launch_bounds__(TD_NT_, MINB)
    tridiag_kernel(const SectorDesc* __restrict__ sd, const int* __restrict__ list, int kmax,
                   cplx* __restrict__ gbuf, double* __restrict__ dbuf, double* __restrict__ ebuf,
                   cplx* __restrict__ taubuf, int* __restrict__ err) {
  constexpr int TD_NT = TD_NT_;        // threads of this instantiation
  constexpr int TD_NW = TD_NT_ / 32;   // its warps, each streaming its own rows
  extern __shared__ __align__(128) unsigned char smem_raw[];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int TD_CL = (int)cluster.num_blocks();   // 1, 2, 4 or 8
  const int cls = __ffs(TD_CL) - 1;                // log2 of it
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int own_cap = kmax / TD_CL + 1;
  const int nslot = td_slots(kmax, TD_NW);         // 1, 2 or 4
  const int nss = __ffs(nslot) - 1;
  cplx* ring = reinterpret_cast<cplx*>(smem_raw);  // slot s of warp w: ring + (w nslot + s) kmax
  cplx* vb = ring + (size_t)TD_NW * nslot * kmax;  // v of two consecutive steps: vb + (j & 1) kmax
  cplx* wb = vb + 2 * kmax;                        // w likewise
  cplx* pub = wb + 2 * kmax;                       // row j + 1 as published by its owner
  cplx* nrow = pub + kmax;                         // this CTA's copy of the row being reduced
  cplx* pown = nrow + kmax;                        // p of the own rows: pown + (j & 1) own_cap
  // [0..3] partial c of the two parities, [4..5] tau of this step, [8..] warp partials
  double* scal = reinterpret_cast<double*>(pown + 2 * own_cap);
  uint64_t* bars = reinterpret_cast<uint64_t*>(scal + 64) + warp * TD_MAXSLOT;   // this warp's
  cplx* wring = ring + (size_t)warp * nslot * kmax;
  const SectorDesc& S = sd[list[blockIdx.x / TD_CL]];
  const int k = S.k;                   // the same for every CTA of the cluster
  cplx* A = gbuf + S.g_off;
  double* dd = dbuf + S.s_off;
  double* ee = ebuf + S.s_off;
  cplx* tt = taubuf + S.s_off;
  if (k <= 1) {
    if (k == 1 && rank == 0 && tid == 0) dd[0] = A[0].x;
    return;                            // uniform over the cluster
  }
  if (lane < TD_MAXSLOT) {
    mbar_init(bars + lane, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // ---- this warp's row sequence: (step s, own row r) with rows i = rank + r cl > s,
  // r = warp (mod 4), in step order, then row order; copies are issued in the same order
  // as the pass consumes them, element q into slot q mod nslot
  auto first_row = [&](int s) {
    const int r0 = s >= rank ? ((s - rank) >> cls) + 1 : 0;
    return r0 + ((warp - r0) & (TD_NW - 1));
  };
  int is = 0, ir = first_row(0);       // next element to copy
  int issued = 0, done = 0;            // elements copied / consumed
  int ls = -1, lr = 0;                 // the last consumed element
  auto issue = [&]() {
    // a free slot, and the row's write-back of the previous step done (consumption is in
    // sequence order, so the last consumed element tells)
    while (is < k - 1 && rank + (ir << cls) < k && issued < done + nslot &&
           (is == 0 || ls > is - 1 || (ls == is - 1 && lr >= ir))) {
      if (lane == 0) {
        const int slot = issued & (nslot - 1);
        const uint32_t bytes = (uint32_t)(k - is - 1) * (uint32_t)sizeof(cplx);
        mbar_expect_tx(bars + slot, bytes);
        bulk_load(wring + (size_t)slot * kmax, A + (int64_t)(rank + (ir << cls)) * k + is + 1, bytes,
                  bars + slot);
      }
      ++issued;
      ir += TD_NW;
      if (rank + (ir << cls) >= k) ir = first_row(++is);
    }
  };
  issue();

  double beta = 0.0;                   // this step's e_j (warp 0)
  for (int j = 0; j < k - 1; ++j) {
    const int par = j & 1;
    const bool owner = rank == (j & (TD_CL - 1));
    cplx* vcur = vb + par * kmax;
    const cplx* vprev = vb + (par ^ 1) * kmax;
    const cplx* wprev = wb + (par ^ 1) * kmax;
    // ---- R: the reflector of row j (warp 0 of every CTA; warp shuffles only)
    if (warp == 0) {
      const cplx* row = A + (int64_t)j * k;
      double part = 0.0;
      const cplx vj = j > 0 ? vprev[j] : cmake(0.0, 0.0), wj = j > 0 ? wprev[j] : cmake(0.0, 0.0);
      for (int l = j + lane; l < k; l += 32) {
        // row j as the previous pass left it (copied from its owner), the Gram at j = 0
        cplx a = j > 0 ? nrow[l] : ldc(row + l);
        if (j > 0) a = crank2(a, vj, ldc(wprev + l), wj, ldc(vprev + l));
        if (l == j) {
          if (owner) dd[j] = a.x;
        } else {
          const cplx x = cconj(a);
          vcur[l] = x;                  // x for now, scaled below
          if (l > j + 1) part += cabs2(x);
        }
      }
      const double xn2 = warp_sum(part);   // the same value in every lane
      __syncwarp();
      const cplx alpha = vcur[j + 1];
      cplx tau, sc;
      if (xn2 == 0.0 && alpha.y == 0.0) {
        tau = cmake(0.0, 0.0);
        beta = alpha.x;
        sc = cmake(0.0, 0.0);
      } else {
        beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2), alpha.x);
        tau = cmake((beta - alpha.x) / beta, -alpha.y / beta);
        sc = cdiv(cmake(1.0, 0.0), cmake(alpha.x - beta, alpha.y));
      }
      __syncwarp();                     // alpha read by every lane before vcur[j + 1] changes
      for (int l = j + 1 + lane; l < k; l += 32)
        vcur[l] = l == j + 1 ? cmake(1.0, 0.0) : cmul(sc, vcur[l]);
      if (lane == 0) {
        scal[4] = tau.x;
        scal[5] = tau.y;
      }
    }
    __syncthreads();
    const cplx tau = cmake(scal[4], scal[5]);
    // ---- P: fused update + matrix-vector product on this warp's rows
    {
      double cpx = 0.0, cpy = 0.0;
      cplx* pw = pown + par * own_cap;
      // rows two at a time where the ring holds two slots: one pass over the vectors for
      // both rows
      for (int r = first_row(j); rank + (r << cls) < k;) {
        const int r2 = r + TD_NW;
        const int i = rank + (r << cls), i2 = rank + (r2 << cls);
        const bool two = BSMPO_TD_PAIRS && nslot >= 2 && i2 < k;   // warp-uniform
        const int slot = done & (nslot - 1), slot2 = (done + 1) & (nslot - 1);
        // on expiry the error word is set and the pass goes on with what the slot holds
        mbar_wait_fast(bars + slot, (uint32_t)(done >> nss) & 1u, err);
        if (two) mbar_wait_fast(bars + slot2, (uint32_t)((done + 1) >> nss) & 1u, err);
        const cplx* srow = wring + (size_t)slot * kmax - (j + 1);     // srow[l], l > j
        const cplx* srow2 = wring + (size_t)slot2 * kmax - (j + 1);
        cplx* grow = A + (int64_t)i * k;
        cplx* grow2 = A + (int64_t)(two ? i2 : i) * k;
        const bool next = i == j + 1;  // the next reflector row (never the second): publish it
        const cplx vi = j > 0 ? vprev[i] : cmake(0.0, 0.0), wi = j > 0 ? wprev[i] : cmake(0.0, 0.0);
        const cplx vi2 = (j > 0 && two) ? vprev[i2] : cmake(0.0, 0.0);
        const cplx wi2 = (j > 0 && two) ? wprev[i2] : cmake(0.0, 0.0);
        cplx acc = cmake(0.0, 0.0), acc2 = cmake(0.0, 0.0);
        if (two && j > 0 && !next) {
          // the common case without per-entry tests
#pragma unroll 2
          for (int l = j + 1 + lane; l < k; l += 32) {
            const cplx vc = ldc(vcur + l), vp = ldc(vprev + l), wp = ldc(wprev + l);
            const cplx a = crank2(ldc(srow + l), vi, wp, wi, vp);
            const cplx a2 = crank2(ldc(srow2 + l), vi2, wp, wi2, vp);
            stc(grow + l, a);
            stc(grow2 + l, a2);
            cfma(acc, a, vc);
            cfma(acc2, a2, vc);
          }
        } else {
#pragma unroll 2
          for (int l = j + 1 + lane; l < k; l += 32) {
            cplx a = ldc(srow + l);
            cplx a2 = two ? ldc(srow2 + l) : cmake(0.0, 0.0);
            const cplx vc = ldc(vcur + l);
            if (j > 0) {
              const cplx vp = ldc(vprev + l), wp = ldc(wprev + l);
              a = crank2(a, vi, wp, wi, vp);
              stc(grow + l, a);
              if (two) {
                a2 = crank2(a2, vi2, wp, wi2, vp);
                stc(grow2 + l, a2);
              }
            }
            if (next) pub[l] = a;
            cfma(acc, a, vc);
            cfma(acc2, a2, vc);
          }
        }
        // the write-back before the next bulk read of these rows (async proxy)
        if (j > 0) asm volatile("fence.proxy.async.global;" ::: "memory");
        if (two) {
          // both rows in one butterfly: after the first exchange lanes 0-15 carry row i and
          // lanes 16-31 row i2; lane 0 ends with row i's sum and fetches row i2's from lane 16
          const bool hi = (lane & 16) != 0;
          const cplx send = hi ? acc : acc2;
          cplx keep = hi ? acc2 : acc;
          keep.x += __shfl_xor_sync(0xffffffffu, send.x, 16);
          keep.y += __shfl_xor_sync(0xffffffffu, send.y, 16);
#pragma unroll
          for (int o = 8; o > 0; o >>= 1) {
            keep.x += __shfl_xor_sync(0xffffffffu, keep.x, o);
            keep.y += __shfl_xor_sync(0xffffffffu, keep.y, o);
          }
          acc = keep;
          acc2 = cmake(__shfl_sync(0xffffffffu, keep.x, 16), __shfl_sync(0xffffffffu, keep.y, 16));
        } else {
          acc = warp_sum(acc);
        }
        if (lane == 0) {
          // p_i, and conj(p_i) v_i summed by lane 0 of each warp in row order
          const cplx p = cmul(tau, acc);
          pw[r] = p;
          const cplx cv = ccmul(p, vcur[i]);
          cpx += cv.x;
          cpy += cv.y;
          if (two) {
            const cplx p2 = cmul(tau, acc2);
            pw[r2] = p2;
            const cplx cv2 = ccmul(p2, vcur[i2]);
            cpx += cv2.x;
            cpy += cv2.y;
          }
        }
        __syncwarp();                  // every lane done with the slots and the rows
        done += two ? 2 : 1;
        ls = j;
        lr = two ? r2 : r;
        issue();
        r = two ? r2 + TD_NW : r2;
      }
      if (lane == 0) {
        scal[8 + 2 * warp] = cpx;
        scal[9 + 2 * warp] = cpy;
      }
      __syncthreads();
      if (tid == 0) {
        double sx = 0.0, sy = 0.0;
        for (int w = 0; w < TD_NW; ++w) { sx += scal[8 + 2 * w]; sy += scal[9 + 2 * w]; }
        scal[2 * par] = sx;
        scal[2 * par + 1] = sy;
      }
    }
    cluster.sync();
    // ---- G: w_j from every owner's p, the next row from its owner
    {
      double cx = 0.0, cy = 0.0;
      for (int q = 0; q < TD_CL; ++q) {   // fixed order: the same sum in every CTA
        const double* qs = cluster.map_shared_rank(scal, q);
        cx += qs[2 * par];
        cy += qs[2 * par + 1];
      }
      const cplx a2 = cscale(cmul(tau, cmake(cx, cy)), -0.5);
      cplx* wcur = wb + par * kmax;
      const cplx* rpub = cluster.map_shared_rank(pub, (j + 1) & (TD_CL - 1));
      for (int l = j + 1 + tid; l < k; l += TD_NT) {
        const cplx* rp = cluster.map_shared_rank(pown, l & (TD_CL - 1));
        wcur[l] = cadd(rp[par * own_cap + (l >> cls)], cmul(a2, vcur[l]));
        nrow[l] = rpub[l];
      }
      if (owner) {
        // v_j kept in row j for the back-transformation (row j has been read by every
        // CTA before the barrier, and no copy of it is issued after step j - 1)
        cplx* row = A + (int64_t)j * k;
        for (int l = j + 1 + tid; l < k; l += TD_NT) stc(row + l, vcur[l]);
        if (tid == 0) {
          ee[j] = beta;                 // thread 0 is lane 0 of warp 0, which formed it
          tt[j] = tau;
        }
      }
      __syncthreads();
    }
  }
  // last diagonal entry: row k - 1 (copied in the last G) minus the update of step k - 2
  if (rank == ((k - 1) & (TD_CL - 1)) && tid == 0) {
    const int j = k - 1;
    const cplx v = vb[((k - 2) & 1) * kmax + j], w = wb[((k - 2) & 1) * kmax + j];
    const cplx a = crank2(nrow[j], v, w, w, v);
    dd[j] = a.x;
  }
  cluster.sync();   // no CTA leaves while another may still read its shared memory
}

// ---------------------------------------------------------------------------------
// 2. Eigenvalues: warp i of sector s finds the i-th largest eigenvalue of (d, e) by
//    multisection: 32 Sturm counts per pass (one per lane), the interval shrinks 33x.
constexpr int BI_NT = 256;

__device__ __forceinline__ int sturm_count(const double* d, const double* e2, int k, double x,
                                           double pivmin) {
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int c = q < 0.0;
  for (int i = 1; i < k; ++i) {
    q = (d[i] - x) - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    c += q < 0.0;
  }
  return c;
}

__global__ __launch_bounds__(BI_NT) void bisect_kernel(const SectorDesc* __restrict__ sd,
                                                       const double* __restrict__ dbuf,
                                                       const double* __restrict__ ebuf,
                                                       double* __restrict__ lam) {
  extern __shared__ double bsm[];
  const SectorDesc& S = sd[blockIdx.y];
  const int k = S.k;
  const int first = blockIdx.x * (BI_NT / 32);
  if (first >= k) return;             // uniform over the CTA
  double* d = bsm;
  double* e2 = bsm + k;
  __shared__ double red[2][BI_NT / 32];
  __shared__ double bounds[3];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* dg = dbuf + S.s_off;
  const double* eg = ebuf + S.s_off;
  double lo = 1e300, hi = -1e300, emax = 0.0;
  for (int i = tid; i < k; i += BI_NT) {
    const double di = dg[i];
    const double ea = i > 0 ? fabs(eg[i - 1]) : 0.0, eb = i < k - 1 ? fabs(eg[i]) : 0.0;
    d[i] = di;
    if (i < k - 1) e2[i] = eg[i] * eg[i];
    lo = fmin(lo, di - ea - eb);
    hi = fmax(hi, di + ea + eb);
    emax = fmax(emax, eb * eb);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
  }
  if (lane == 0) { red[0][warp] = lo; red[1][warp] = hi; }
  __shared__ double red_e[BI_NT / 32];
  if (lane == 0) red_e[warp] = emax;
  __syncthreads();
  if (tid == 0) {
    double a = red[0][0], b = red[1][0], c = red_e[0];
    for (int w = 1; w < BI_NT / 32; ++w) { a = fmin(a, red[0][w]); b = fmax(b, red[1][w]); c = fmax(c, red_e[w]); }
    // widen by a few ulps of the bound so the extreme eigenvalues stay inside
    const double span = fmax(fabs(a), fabs(b));
    bounds[0] = a - 4.0 * EPS * span - 1e-300;
    bounds[1] = b + 4.0 * EPS * span + 1e-300;
    bounds[2] = 2.2250738585072014e-308 * fmax(1.0, c);   // pivmin
  }
  __syncthreads();
  const int i = first + warp;
  if (i >= k) return;
  const int target = k - 1 - i;        // eigenvalues below lambda_(i) (ascending index)
  const double pivmin = bounds[2];
  double a = bounds[0], b = bounds[1];
  const double tol_abs = 4.0 * EPS * fmax(fabs(a), fabs(b)) + 2.0 * pivmin;
  for (int it = 0; it < 16; ++it) {
    const double x = a + (double)(lane + 1) * ((b - a) / 33.0);
    const int c = sturm_count(d, e2, k, x, pivmin);
    const unsigned below = __ballot_sync(0xffffffffu, c <= target);
    const int L = __popc(below);       // counts rise with x: lanes 0..L-1 lie below
    const double xl = __shfl_sync(0xffffffffu, x, L > 0 ? L - 1 : 0);
    const double xh = __shfl_sync(0xffffffffu, x, L < 32 ? L : 31);
    const double na = L > 0 ? xl : a, nb = L < 32 ? xh : b;
    a = na;
    b = nb;
    // absolute accuracy of a few eps ||T|| (the tridiagonalisation's own error) is all
    // the selection and sigma = sqrt(lambda) need
    if (b - a <= tol_abs) break;   // warp-uniform
  }
  if (lane == 0) lam[S.s_off + i] = 0.5 * (a + b);
}

// Monotone order (bisection rounds independently), numerical floor, sigma and 1/sigma.
constexpr int FI_NT = 1024;
__global__ __launch_bounds__(FI_NT) void eig_finish_kernel(const SectorDesc* __restrict__ sd,
                                                           const double* __restrict__ lam,
                                                           double* __restrict__ sig,
                                                           double* __restrict__ invsig) {
  __shared__ double buf[2][FI_NT];
  const SectorDesc& S = sd[blockIdx.x];
  const int k = S.k;
  const int tid = threadIdx.x;
  // k <= FI_NT * 2 handled in two halves of the scan
  const double lmax = k > 0 ? lam[S.s_off] : 0.0;
  const double floor_l = 32.0 * EPS * (double)k * fabs(lmax);
  double carry = 1e300;
  for (int base = 0; base < k; base += FI_NT) {
    const int i = base + tid;
    double v = i < k ? lam[S.s_off + i] : 1e300;
    int cur = 0;
    buf[0][tid] = v;
    __syncthreads();
    for (int off = 1; off < FI_NT; off <<= 1) {   // inclusive prefix minimum
      const double x = buf[cur][tid];
      const double y = tid >= off ? buf[cur][tid - off] : 1e300;
      buf[cur ^ 1][tid] = fmin(x, y);
      cur ^= 1;
      __syncthreads();
    }
    v = fmin(buf[cur][tid], carry);
    if (i < k) {
      const double s = v > floor_l ? sqrt(v) : 0.0;
      sig[S.s_off + i] = s;
      invsig[S.s_off + i] = s > 0.0 ? 1.0 / s : 0.0;
    }
    carry = fmin(carry, buf[cur][FI_NT - 1]);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------
// 3a. Eigenvectors of the tridiagonal by inverse iteration, one thread per kept
//     eigenvalue.  T - lambda I = P L U with partial pivoting (U has two
//     superdiagonals), stored column-interleaved in the scratch (entry l of vector t
//     at l * kept + t, so a warp's accesses coalesce).  Start vector: a fixed
//     pseudo-random one; three solves, normalised.  Eigenvalues closer than `gaptol`
//     form a group handled by its first member, each vector orthogonalised against
//     the group's earlier ones after every solve.
constexpr int IV_NT = 128;

__device__ __forceinline__ double start_entry(int l, int t) {
  unsigned h = (unsigned)l * 2654435761u ^ ((unsigned)t * 40503u + 0x9e3779b9u);
  h ^= h >> 15;
  h *= 2246822519u;
  h ^= h >> 13;
  return ((double)(h & 0xffffu) + 0.5) / 32768.0 - 1.0;
}

__global__ __launch_bounds__(IV_NT) void invit_kernel(const SectorDesc* __restrict__ sd,
                                                      const double* __restrict__ dbuf,
                                                      const double* __restrict__ ebuf,
                                                      const double* __restrict__ lam,
                                                      double* __restrict__ scratch,
                                                      unsigned char* __restrict__ swp,
                                                      double* __restrict__ zbuf) {
  extern __shared__ double ism[];
  const SectorDesc& S = sd[blockIdx.y];
  const int k = S.k, kept = S.kept;
  const int t0 = blockIdx.x * IV_NT;
  if (t0 >= kept) return;
  double* d = ism;
  double* e = ism + k;
  for (int i = threadIdx.x; i < k; i += IV_NT) {
    d[i] = dbuf[S.s_off + i];
    e[i] = i < k - 1 ? ebuf[S.s_off + i] : 0.0;
  }
  __syncthreads();
  const int t = t0 + threadIdx.x;
  if (t >= kept) return;
  const double* lv = lam + S.s_off;
  const double norm = fmax(fabs(lv[0]), fabs(lv[k - 1]));
  const double gaptol = 1e-9 * norm;
  // group membership: not a leader if the previous kept eigenvalue is within gaptol
  if (t > 0 && lv[t - 1] - lv[t] <= gaptol) return;
  int g_end = t + 1;
  while (g_end < kept && lv[g_end - 1] - lv[g_end] <= gaptol) ++g_end;
  const double tiny = EPS * norm + 1e-300;
  // scratch layout of this sector: 4 arrays [k][kept] (u0, u1, u2, mult)
  double* U0 = scratch + 4 * S.y_off;   // 4 arrays of k x kept in the sector's 4 k^2 slots
  double* U1 = U0 + (int64_t)k * kept;
  double* U2 = U1 + (int64_t)k * kept;
  double* MU = U2 + (int64_t)k * kept;
  unsigned char* SW = swp + S.y_off;
  double* Z = zbuf + S.y_off;
  for (int m = t; m < g_end; ++m) {
    const double lambda = lv[m];
    // factor T - lambda I
    double p = d[0] - lambda, q = k > 1 ? e[0] : 0.0;
#pragma unroll 4
    for (int i = 0; i < k - 1; ++i) {
      const double ei = e[i], an = d[i + 1] - lambda, en = i + 1 < k - 1 ? e[i + 1] : 0.0;
      const int64_t o = (int64_t)i * kept + m;
      if (fabs(ei) > fabs(p)) {
        const double mu = p / ei;
        U0[o] = ei; U1[o] = an; U2[o] = en; MU[o] = mu; SW[o] = 1;
        const double np = q - mu * an, nq = -mu * en;
        p = np;
        q = nq;
      } else {
        if (p == 0.0) p = tiny;
        const double mu = ei / p;
        U0[o] = p; U1[o] = q; U2[o] = 0.0; MU[o] = mu; SW[o] = 0;
        p = an - mu * q;
        q = en;
      }
    }
    if (p == 0.0) p = tiny;
    {
      const int64_t o = (int64_t)(k - 1) * kept + m;
      U0[o] = p; U1[o] = 0.0; U2[o] = 0.0; MU[o] = 0.0; SW[o] = 0;
    }
    for (int it = 0; it < 3; ++it) {
      // right-hand side: start vector, or L^{-1} P z
      if (it == 0) {
        for (int i = 0; i < k; ++i) Z[(int64_t)i * kept + m] = start_entry(i, m);
      } else {
#pragma unroll 4
        for (int i = 0; i < k - 1; ++i) {
          const int64_t o = (int64_t)i * kept + m, o1 = o + kept;
          double bi = Z[o], bn = Z[o1];
          if (SW[o]) { const double x = bi; bi = bn; bn = x; }
          Z[o] = bi;
          Z[o1] = bn - MU[o] * bi;
        }
      }
      // back substitution U z = b, then normalise
      double z1 = 0.0, z2 = 0.0, nrm = 0.0;
#pragma unroll 4
      for (int i = k - 1; i >= 0; --i) {
        const int64_t o = (int64_t)i * kept + m;
        double u0 = U0[o];
        if (u0 == 0.0) u0 = tiny;
        const double z = (Z[o] - U1[o] * z1 - U2[o] * z2) / u0;
        Z[o] = z;
        z2 = z1;
        z1 = z;
        nrm += z * z;
      }
      // orthogonalise against the group's earlier vectors
      for (int g = t; g < m; ++g) {
        double dot = 0.0;
        for (int i = 0; i < k; ++i) dot += Z[(int64_t)i * kept + g] * Z[(int64_t)i * kept + m];
        nrm = 0.0;
        for (int i = 0; i < k; ++i) {
          const double z = Z[(int64_t)i * kept + m] - dot * Z[(int64_t)i * kept + g];
          Z[(int64_t)i * kept + m] = z;
          nrm += z * z;
        }
      }
      const double inv = nrm > 0.0 ? 1.0 / sqrt(nrm) : 0.0;
      for (int i = 0; i < k; ++i) Z[(int64_t)i * kept + m] *= inv;
    }
  }
}

// 3b. y = Q z = H_0 (H_1 (... H_{k-2} z)), one warp per kept vector; lane holds the
//     entries l = lane (mod 32).  Writes V = y ([k][kept], X = T^H) or Y for the GEMM.
constexpr int BT_NT = 128;

template <int NPL>
__global__ __launch_bounds__(BT_NT) void backtransform_kernel(const SectorDesc* __restrict__ sd,
                                                              const cplx* __restrict__ gbuf,
                                                              const cplx* __restrict__ taubuf,
                                                              const double* __restrict__ zbuf,
                                                              cplx* __restrict__ vbuf,
                                                              cplx* __restrict__ ybuf) {
  const SectorDesc& S = sd[blockIdx.y];
  const int k = S.k, kept = S.kept;
  const int lane = threadIdx.x & 31;
  const int t = blockIdx.x * (BT_NT / 32) + (threadIdx.x >> 5);
  if (t >= kept) return;
  const cplx* A = gbuf + S.g_off;
  const cplx* tau = taubuf + S.s_off;
  const double* Z = zbuf + S.y_off;
  cplx y[NPL];
#pragma unroll
  for (int c = 0; c < NPL; ++c) {
    const int l = lane + 32 * c;
    y[c] = l < k ? cmake(Z[(int64_t)l * kept + t], 0.0) : cmake(0.0, 0.0);
  }
  for (int j = k - 2; j >= 0; --j) {
    const cplx* v = A + (int64_t)j * k;     // v_j at columns j+1 .. k-1 (v[j+1] = 1)
    cplx dot = cmake(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < NPL; ++c) {
      const int l = lane + 32 * c;
      if (l > j && l < k) ccfma(dot, ldc(v + l), y[c]);
    }
    dot = warp_sum(dot);
    const cplx f = cmul(tau[j], dot);
#pragma unroll
    for (int c = 0; c < NPL; ++c) {
      const int l = lane + 32 * c;
      if (l > j && l < k) y[c] = csub(y[c], cmul(f, ldc(v + l)));
    }
  }
  cplx* out = S.left ? vbuf + S.v_off : ybuf + S.y_off;
#pragma unroll
  for (int c = 0; c < NPL; ++c) {
    const int l = lane + 32 * c;
    if (l < k) stc(out + (int64_t)l * kept + t, y[c]);
  }
}

}  // namespace

int eigen_max_k() {
  // every k up to the bound fits the tridiagonalisation's shared memory with one CTA per
  // sector (the row ring shrinks in steps as k grows, so the size is not monotone in k)
  static const int kmax = [] {
    int best = 0;
    for (int k = 1; k <= 32 * 32; ++k) {   // the back-transformation keeps 32 entries per lane
      if (td_smem_bytes(k, 1, TD_NT / 32) > 227 * 1024) break;
      best = k;
    }
    return best;
  }();
  return kmax;
}

// Size-class bounds (largest k of classes 0, 1, 2); BSMPO_TD_CLASSES="a,b,c" in the
// environment replaces them (read once).
int tridiag_class(int k) {
  static const int* bounds = [] {
    static int b[3] = {64, 320, 1024};   // the 8-CTA class stays unused up to k = 1024
    const char* e = std::getenv("BSMPO_TD_CLASSES");
    int x, y, z;
    if (e && std::sscanf(e, "%d,%d,%d", &x, &y, &z) == 3 && 0 < x && x < y && y < z) {
      b[0] = x; b[1] = y; b[2] = z;
    }
    return b;
  }();
  return k <= bounds[0] ? 0 : k <= bounds[1] ? 1 : k <= bounds[2] ? 2 : 3;
}

cudaError_t launch_tridiag(const SectorDesc* sd_dev, const int* list_dev, const int* class_count,
                           const int* class_kmax, void* gbuf, double* dbuf, double* ebuf,
                           void* taubuf, int* err, const cudaStream_t* streams) {
  // once per process: the largest dynamic shared memory any launch may ask for
  static const cudaError_t attr = [] {
    size_t most = 0, most_w = 0;
    for (int k = 1; k <= eigen_max_k(); ++k) {
      most = std::max(most, td_smem_bytes(k, 1, TD_NT / 32));
      const size_t w = td_smem_bytes(k, 1, TD_NT_WIDE / 32);
      if (w <= 227 * 1024) most_w = std::max(most_w, w);
    }
    cudaError_t e = cudaFuncSetAttribute(tridiag_kernel<TD_NT, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(tridiag_kernel<TD_NT_WIDE, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most_w);
    return e;
  }();
  if (attr != cudaSuccess) return attr;
  // the first size class on 256-thread CTAs (BSMPO_TD_WIDE, 0-4; 4: none), read once
  static const int wide = [] {
    const char* e = std::getenv("BSMPO_TD_WIDE");
    return (e && e[0] >= '0' && e[0] <= '4') ? e[0] - '0' : TD_CLASSES;
  }();
  int first = 0;
  for (int c = 0; c < TD_CLASSES; ++c) {
    const int count = class_count[c];
    if (count == 0) continue;
    const int cl = 1 << c;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(count * cl);
    // 256 threads where asked and where their larger rings fit the launch's shared memory
    const bool w = c >= wide && td_smem_bytes(class_kmax[c], 1, TD_NT_WIDE / 32) <= 227 * 1024;
    const int nt = w ? TD_NT_WIDE : TD_NT;
    cfg.blockDim = dim3(nt);
    cfg.dynamicSmemBytes = td_smem_bytes(class_kmax[c], cl, nt / 32);
    cfg.stream = streams[TD_CLASSES - 1 - c];   // the largest class on the caller's stream
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaError_t e = w ? cudaLaunchKernelEx(&cfg, tridiag_kernel<TD_NT_WIDE, 2>, sd_dev, list_dev + first,
                                           class_kmax[c], reinterpret_cast<cplx*>(gbuf), dbuf, ebuf,
                                           reinterpret_cast<cplx*>(taubuf), err)
                      : cudaLaunchKernelEx(&cfg, tridiag_kernel<TD_NT, 6>, sd_dev, list_dev + first,
                                           class_kmax[c], reinterpret_cast<cplx*>(gbuf), dbuf, ebuf,
                                           reinterpret_cast<cplx*>(taubuf), err);
    if (e != cudaSuccess) return e;
    first += count;
  }
  return cudaSuccess;
}

cudaError_t launch_bisect(const SectorDesc* sd_dev, int n_sectors, int kmax, const double* dbuf,
                          const double* ebuf, double* lam, double* sig, double* invsig,
                          cudaStream_t s) {
  if (n_sectors <= 0 || kmax <= 0) return cudaSuccess;
  const size_t smem = (size_t)2 * kmax * sizeof(double);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(bisect_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  dim3 grid(ceil_div(kmax, BI_NT / 32), n_sectors);
  bisect_kernel<<<grid, BI_NT, smem, s>>>(sd_dev, dbuf, ebuf, lam);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  eig_finish_kernel<<<n_sectors, FI_NT, 0, s>>>(sd_dev, lam, sig, invsig);
  return cudaGetLastError();
}

cudaError_t launch_eigvec(const SectorDesc* sd_dev, int n_sectors, int kmax, int kept_max,
                          const double* dbuf, const double* ebuf, const double* lam,
                          double* scratch, unsigned char* swp, double* zbuf, const void* gbuf,
                          const void* taubuf, void* vbuf, void* ybuf, cudaStream_t s) {
  if (n_sectors <= 0 || kept_max <= 0) return cudaSuccess;
  const size_t smem = (size_t)2 * kmax * sizeof(double);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(invit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  invit_kernel<<<dim3(ceil_div(kept_max, IV_NT), n_sectors), IV_NT, smem, s>>>(sd_dev, dbuf, ebuf, lam,
                                                                               scratch, swp, zbuf);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 grid(ceil_div(kept_max, BT_NT / 32), n_sectors);
  const cplx* G = reinterpret_cast<const cplx*>(gbuf);
  const cplx* T = reinterpret_cast<const cplx*>(taubuf);
  cplx* V = reinterpret_cast<cplx*>(vbuf);
  cplx* Y = reinterpret_cast<cplx*>(ybuf);
  const int npl = ceil_div(kmax, 32);
  if (npl <= 4) backtransform_kernel<4><<<grid, BT_NT, 0, s>>>(sd_dev, G, T, zbuf, V, Y);
  else if (npl <= 8) backtransform_kernel<8><<<grid, BT_NT, 0, s>>>(sd_dev, G, T, zbuf, V, Y);
  else if (npl <= 16) backtransform_kernel<16><<<grid, BT_NT, 0, s>>>(sd_dev, G, T, zbuf, V, Y);
  else if (npl <= 32) backtransform_kernel<32><<<grid, BT_NT, 0, s>>>(sd_dev, G, T, zbuf, V, Y);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}
