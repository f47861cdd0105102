// libbsmpo C ABI and host orchestration of the beam-splitter MPO update.
//
// The host keeps a mirror of the per-bond charge-block sizes (they change only when
// an update writes a new bond, and the update reports its kept counts), so every
// launch of an update is planned on the host without reading device data; the one
// device->host synchronisation per update reads the kept counts after selection.
//
// Per update (bond layout of src/MPO.py:158-303, GPU driver
// src/beam_splitter_parallel/Rank.py:32-206):
//   Theta grouped GEMM -> gate mix (C per sector and the Jacobi matrix) ->
//   blocked one-sided Jacobi rounds -> column norms + sort -> top-chi selection ->
//   [sync: kept counts] -> V extraction -> W = V^H C grouped GEMM -> scatter.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <queue>
#include <mutex>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bsmpo.h"
#include "common.cuh"
#include "kernels.h"

namespace {

thread_local std::string g_last_error;

constexpr int MAX_SWEEPS = 40;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct HostStage {
  void* p = nullptr;
  size_t bytes = 0;
};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

void set_global_error(const char* msg) { g_last_error = msg ? msg : ""; }

struct bsmpo_ctx {
  int n = 0, d = 0, chi = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  // workspaces come from this stream-ordered pool (shared with the workers): growing a
  // buffer never synchronises the device, so other workers' streams keep running
  cudaMemPool_t pool = nullptr;
  // workspace growth: counts, and pinned stages replaced by larger ones (freed at destroy:
  // releasing pinned memory synchronises the device, which would stall every worker)
  int64_t dev_grows = 0, host_grows = 0;
  std::vector<void*> retired_host;
  // host waits of an update sleep on this event (blocking synchronisation) instead of
  // spinning, so several workers' waits leave the host cores to the launching threads
  cudaEvent_t wait_ev = nullptr;
  cudaEvent_t poll_ev[2] = {nullptr, nullptr};   // Jacobi convergence polls (blocking sync)
  double cutoff = 0.0;
  // device state
  cplx* gamma = nullptr;     // [n][chi][chi]
  double* lam = nullptr;     // [n+1][chi]  (edges: 1 on occupied slots)
  int* charge = nullptr;     // [n+1][chi][2]
  bool loaded = false;
  // host mirror of block sizes: cnt[b * d*d + c0*d + c1]
  std::vector<int> cnt;
  // workspaces
  DevBuf theta, cbuf, abuf, wbuf, vbuf, sig, keys, perm, tab, tab2, rot, kept, u3, m4, env_l,
      env_r, part, outv, dims, nf2, qbuf, qflag, pbuf, pcnt;
  // Gram / eigen route of the sector SVD (precision != BSMPO_PRECISION_FP64)
  DevBuf gbuf, eigd, taub, invsig, escr, swp, zbuf, ybuf;
  // tensor-core contractions (BSMPO_PRECISION_TF32X3): groups and tensor maps of the
  // V / W GEMMs, and the pipeline's error word
  DevBuf tab3, tcerr;
  DevBuf jwork;   // executed Jacobi rows: pair-Gram rows, rotated rows (unsigned long long[2])
  HostStage stage3;
  int precision = BSMPO_PRECISION_FP64;
  // the tridiagonalisation's size classes run side by side: three more streams, forked
  // from and joined to `stream` with events
  cudaStream_t aux[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t fork_ev = nullptr, join_ev[3] = {nullptr, nullptr, nullptr};
  // tridiagonalisation phase timing (timing mode): events around the forked launches,
  // read at the update's kept-count synchronisation; streamed bytes and zhetrd flops
  cudaEvent_t td_ev0 = nullptr, td_ev1 = nullptr;
  double td_ms = 0.0, td_bytes = 0.0, td_flops = 0.0;
  int64_t td_phases = 0;
  // BSMPO_GRAM_POLICY (Gram route): 0 (default) exact Jacobi only where the candidates
  // cannot exceed chi; 1 also after a selection that keeps fewer than chi; 2 also where
  // the centre bond holds fewer than chi vectors
  int gram_policy = 0;
  // which contractions of BSMPO_PRECISION_TF32X3 go on the tensor cores (BSMPO_TC_MASK,
  // read at create): bit 0 the Theta block products, bit 1 W = V^H C; the others FP64.
  // Default: Theta only.  W = V^H C is formed at the scale of C (columns carry
  // 1 / Lambda_R) while its rows near the cut are ~sigma_cut / sigma_max smaller, so a
  // split-TF32 error relative to the dot product grows by that ratio there (measured:
  // 1.1e-4 / 1.3e-3 marginal error on the N=16 / N=32 circuits against 8.7e-6 / 1.0e-4
  // with Theta alone)
  int tc_mask = 1;
  // side streams (0-3, BSMPO_TD_FORK) for the tridiagonalisation's size-class launches:
  // the largest class present runs on the update's stream, the others on the side
  // streams, forked and joined with events.  With concurrent updates the streams of all
  // workers share the device's hardware queues (CUDA_DEVICE_MAX_CONNECTIONS, at most
  // 32); streams beyond that count are serialised with others
  int td_fork = 1;
  int n_aux = 0;   // side streams created
  HostStage stage, stage2, hres;
  // last update diagnostics (host)
  std::vector<int> last_cc, last_shape, last_kept, last_k;
  std::vector<int64_t> last_soff;
  double last_trunc = 0.0, last_gemm = 0.0, last_svd = 0.0, last_bytes = 0.0;
  int last_sweeps = 0;
  // opt-in stage timing (BSMPO_PROFILE=1): synchronises after every stage
  bool profile = false;
  double stage_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int64_t jacobi_rounds = 0, updates = 0;
  int jac_rows = 128;  // rows per part of a block pair in a Jacobi round (BSMPO_JACOBI_ROWS)
  // Jacobi-phase timing with CUDA events (no extra synchronisation): elapsed time is
  // read at the update's selection sync, when both events have completed
  bool timing = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double jac_ms = 0.0, jac_flops = 0.0;
  int64_t jac_launches = 0;
  int last_ns = 0;
  int64_t launches = 0;
  std::string err;
  // Concurrent updates of one brick-wall layer (bsmpo_run_mesh).  A worker context
  // shares its owner's state and host mirror (cnt_shared) and owns its workspaces and
  // stream; the owner keeps its workers and, after a mesh, points `diag` at the worker
  // that ran the mesh's last update.
  std::vector<int>* cnt_shared = nullptr;
  std::vector<bsmpo_ctx*> workers;
  int n_workers = 8;      // BSMPO_WORKERS / bsmpo_set_workers
  const bsmpo_ctx* diag = nullptr;
  int last_index = -1;    // worker: mesh index of the last update it ran
  std::vector<double> mesh_tw;   // truncation weight of every update of the last mesh
  int64_t route_count[2] = {0, 0};   // updates solved by Jacobi [0] and by the Gram route [1]
};

namespace {

int fail(bsmpo_ctx* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  g_last_error = msg;
  return code;
}

// the host mirror of the charge-block sizes (a worker's is its owner's)
std::vector<int>& mirror(bsmpo_ctx* h) { return h->cnt_shared ? *h->cnt_shared : h->cnt; }

// waits (sleeping) until the handle's stream has drained
// the forked streams of the tridiagonalisation's size classes and their events, created
// once (for a worker when it is made, so the order of stream creation, which decides
// the streams' hardware queues, is fixed)
int make_fork_streams(bsmpo_ctx* h) {
  if (h->fork_ev) return BSMPO_OK;
  if (cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    h->fork_ev = nullptr;
    return fail(h, BSMPO_ECUDA, "fork event creation failed");
  }
  for (int i = 0; i < std::min(h->td_fork, 3); ++i) {
    if (cudaStreamCreateWithFlags(&h->aux[i], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->join_ev[i], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return fail(h, BSMPO_ECUDA, "fork stream creation failed");
    }
    h->n_aux = i + 1;
  }
  return BSMPO_OK;
}

cudaError_t host_wait(bsmpo_ctx* h) {
  if (!h->wait_ev) {
    cudaError_t e = cudaEventCreateWithFlags(&h->wait_ev, cudaEventBlockingSync | cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaEventRecord(h->wait_ev, h->stream);
  if (e != cudaSuccess) return e;
  return cudaEventSynchronize(h->wait_ev);
}

#define CK(h, call)                                                                    \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail((h), BSMPO_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define CKL(h, call)            \
  do {                          \
    CK(h, call);                \
    (h)->launches++;            \
  } while (0)

int grow(bsmpo_ctx* h, DevBuf& b, size_t bytes) {
  if (bytes <= b.bytes) return BSMPO_OK;
  // stream-ordered: the old buffer is released after the stream's earlier work on it
  if (b.p) CK(h, cudaFreeAsync(b.p, h->stream));
  b.p = nullptr;
  b.bytes = 0;
  // the next power of two: a buffer grows at most a few times however its sectors grow
  // (a growth inside a timed layer costs a pool allocation on the worker's stream)
  size_t want = 4096;
  while (want < bytes + 256) want <<= 1;
  h->dev_grows++;
  if (cudaMallocFromPoolAsync(&b.p, want, h->pool, h->stream) != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return fail(h, BSMPO_ENOMEM, "device allocation of " + std::to_string(want) + " bytes failed");
  }
  b.bytes = want;
  return BSMPO_OK;
}

int grow_host(bsmpo_ctx* h, HostStage& b, size_t bytes) {
  if (bytes <= b.bytes) return BSMPO_OK;
  // the old stage may still be read by copies in flight: kept until destroy
  if (b.p) h->retired_host.push_back(b.p);
  b.p = nullptr;
  b.bytes = 0;
  // pinned host memory: rare, generous growth
  size_t want = std::max<size_t>(align_up(bytes + bytes / 2 + 256, 256), 1 << 20);
  h->host_grows++;
  CK(h, cudaMallocHost(&b.p, want));
  b.bytes = want;
  return BSMPO_OK;
}

// offsets of the lexicographic charge blocks of one bond (d*d + 1 entries)
void block_offsets(const int* cnt, int d, int* off) {
  off[0] = 0;
  for (int q = 0; q < d * d; ++q) off[q + 1] = off[q] + cnt[q];
}

struct Plan {
  UpdateTables tab;
  std::vector<int> tidx;
  std::vector<ThetaDesc> td;
  std::vector<SectorDesc> sd;
  std::vector<MixPair> pairs;
  std::vector<GemmGroup> gg;
  std::vector<GemmGroup> ggram;   // Gram G_s = X^H X of every sector (Gram route)
  std::vector<int> tdlist;        // sectors by tridiagonalisation size class (Gram route)
  std::vector<TcGroup> tcg;       // Theta groups on the tensor cores (TF32X3)
  std::vector<unsigned char> tcmaps;   // their two tensor maps (Gamma_L, Gamma_R)
  int tc_tiles = 0;
  int td_count[4] = {0, 0, 0, 0}, td_kmax[4] = {0, 0, 0, 0};
  std::vector<JacobiWork> jw;
  int mix_tiles = 0, gemm_tiles = 0, max_rounds = 0, max_k = 0, max_left_m2 = 0;
  int gram_ctas = 0, apply_ctas = 0, jac_slots = 0;   // every sector in one round
  int64_t theta_elems = 0, c_elems = 0, a_elems = 0, s_elems = 0, w_elems = 0, v_elems = 0;
  int64_t g_elems = 0, y_elems = 0;
  int gram_tiles = 0;
  double flops_theta = 0.0;
};

// Orders a round's work entries (most rounds per sweep first: those sectors set the
// length of the Jacobi phase, so their CTAs are dispatched first) and assigns their
// CTA ranges and block-pair slots.
void jacobi_launch_list(std::vector<JacobiWork>& w, int* gram_ctas, int* apply_ctas, int* slots) {
  std::stable_sort(w.begin(), w.end(), [](const JacobiWork& a, const JacobiWork& b) {
    return a.rounds * a.npairs * a.cs > b.rounds * b.npairs * b.cs;
  });
  int g = 0, a = 0, sl = 0;
  for (auto& x : w) {
    x.gram_start = g;
    x.apply_start = a;
    x.slot_start = sl;
    g += x.npairs * x.cs_g;
    a += x.npairs * x.cs;
    sl += x.npairs;
  }
  *gram_ctas = g;
  *apply_ctas = a;
  *slots = sl;
}

int make_plan(bsmpo_ctx* h, int mode, Plan& P) {
  const int d = h->d, dd = d * d;
  const std::vector<int>& cnt = mirror(h);
  const int* cL = &cnt[(size_t)mode * dd];
  const int* cC = &cnt[(size_t)(mode + 1) * dd];
  const int* cR = &cnt[(size_t)(mode + 2) * dd];
  UpdateTables& T = P.tab;
  std::memset(&T, 0, sizeof(T));
  T.d = d;
  T.chi = h->chi;
  T.mode = mode;
  block_offsets(cL, d, T.offL);
  block_offsets(cC, d, T.offC);
  block_offsets(cR, d, T.offR);
  for (int i = 0; i < BSMPO_MAX_Q; ++i) { T.sidx[i] = -1; T.pair_of[i] = -1; }
  // sector range: the reference loop (src/MPO.py:191-206) over occupied charges
  int hi0 = -1, hi1 = -1, lo0 = d, lo1 = d;
  for (int a0 = 0; a0 < d; ++a0)
    for (int a1 = 0; a1 < d; ++a1) {
      if (cL[a0 * d + a1] > 0) { hi0 = std::max(hi0, a0); hi1 = std::max(hi1, a1); }
      if (cR[a0 * d + a1] > 0) { lo0 = std::min(lo0, a0); lo1 = std::min(lo1, a1); }
    }
  auto rows_of = [&](int a0, int from1) { return T.offL[(a0 + 1) * d] - T.offL[a0 * d + from1]; };
  auto cols_of = [&](int b0, int to1) { return T.offR[b0 * d + to1 + 1] - T.offR[b0 * d]; };
  P.sd.clear();
  int64_t c_off = 0, a_off = 0, s_off = 0, w_off = 0, v_off = 0, g_off = 0, y_off = 0;
  for (int cc0 = lo0; cc0 <= hi0; ++cc0)
    for (int cc1 = lo1; cc1 <= hi1; ++cc1) {
      SectorDesc S;
      std::memset(&S, 0, sizeof(S));
      S.cc0 = cc0;
      S.cc1 = cc1;
      int m = 0, n = 0;
      for (int a0 = cc0; a0 < d; ++a0) { S.row_start[a0] = m; m += rows_of(a0, cc1); }
      for (int b0 = 0; b0 <= cc0; ++b0) { S.col_start[b0] = n; n += cols_of(b0, cc1); }
      if (m == 0 || n == 0) continue;
      S.m = m;
      S.n = n;
      S.left = m < n ? 1 : 0;
      S.k = S.left ? m : n;
      S.rows_g = S.left ? n : m;
      S.rows_tot = S.left ? n + m : m;
      S.c_off = c_off; c_off += (int64_t)m * n;
      S.a_off = a_off; a_off += (int64_t)S.rows_tot * S.k;
      S.s_off = s_off; s_off += S.k;
      S.w_off = w_off; w_off += (int64_t)S.k * n;
      S.v_off = v_off; v_off += (int64_t)m * S.k;
      S.g_off = g_off; g_off += (int64_t)S.k * S.k;
      S.y_off = y_off; y_off += (int64_t)S.k * S.k;
      T.sidx[cc0 * d + cc1] = (int)P.sd.size();
      P.sd.push_back(S);
    }
  const int ns = (int)P.sd.size();
  if (ns > BSMPO_MAX_Q) return fail(h, BSMPO_EINVAL, "too many sectors");
  for (int s = 0; s < ns; ++s) {
    const int p = T.sidx[P.sd[s].cc1 * d + P.sd[s].cc0];
    T.pair_of[s] = p;
  }
  T.n_sectors = ns;
  P.c_elems = c_off; P.a_elems = a_off; P.s_elems = s_off; P.w_elems = w_off; P.v_elems = v_off;
  P.g_elems = g_off; P.y_elems = y_off;
  // Theta groups (q, a0, b0)
  P.tidx.assign((size_t)dd * d * d, -1);
  P.td.clear();
  P.gg.clear();
  int64_t t_off = 0;
  int tiles = 0;
  const int TMt = zgemm_tile_m(), TNt = zgemm_tile_n();
  const int64_t chi2 = (int64_t)h->chi * h->chi;
  P.flops_theta = 0.0;
  for (int q0 = 0; q0 < d; ++q0)
    for (int q1 = 0; q1 < d; ++q1) {
      const int nk = cC[q0 * d + q1];
      if (nk == 0) continue;
      for (int a0 = q0; a0 < d; ++a0) {
        const int nrow = rows_of(a0, q1);
        if (nrow == 0) continue;
        for (int b0 = 0; b0 <= q0; ++b0) {
          const int ncol = cols_of(b0, q1);
          if (ncol == 0) continue;
          ThetaDesc D;
          D.q0 = q0; D.q1 = q1; D.a0 = a0; D.b0 = b0;
          D.row0 = T.offL[a0 * d + q1]; D.nrow = nrow;
          D.col0 = T.offR[b0 * d]; D.ncol = ncol;
          D.k0 = T.offC[q0 * d + q1]; D.nk = nk;
          D.off = t_off;
          t_off += (int64_t)nrow * ncol;
          P.tidx[((q0 * d + q1) * d + a0) * d + b0] = (int)P.td.size();
          P.td.push_back(D);
          GemmGroup g;
          std::memset(&g, 0, sizeof(g));
          g.M = nrow; g.N = ncol; g.K = nk;
          g.lda = h->chi; g.ldb = h->chi; g.ldc = ncol;
          g.opA = 0; g.opB = 0; g.beta = 0;
          g.tiles_n = ceil_div(ncol, TNt);
          g.tile_start = tiles;
          tiles += ceil_div(nrow, TMt) * g.tiles_n;
          g.a_off = (int64_t)mode * chi2 + (int64_t)D.row0 * h->chi + D.k0;
          g.b_off = (int64_t)(mode + 1) * chi2 + (int64_t)D.k0 * h->chi + D.col0;
          g.c_off = D.off;
          g.ks_off = g.rs_off = g.cs_off = -1;
          P.gg.push_back(g);
          P.flops_theta += 8.0 * nrow * (double)nk * ncol;
        }
      }
    }
  P.theta_elems = t_off;
  P.gemm_tiles = tiles;
  // Theta on the tensor cores: one tensor map per site tensor, groups address blocks
  P.tcg.clear();
  P.tcmaps.clear();
  P.tc_tiles = 0;
  if (h->precision == BSMPO_PRECISION_TF32X3 && (h->tc_mask & 1)) {
    const size_t mb = tc_map_bytes();
    P.tcmaps.assign(2 * mb, 0);
    const cplx* gl = h->gamma + (size_t)mode * chi2;
    const cplx* gr = h->gamma + (size_t)(mode + 1) * chi2;
    if (tc_encode_map(P.tcmaps.data(), gl, h->chi, h->chi, h->chi, 0) != cudaSuccess ||
        tc_encode_map(P.tcmaps.data() + mb, gr, h->chi, h->chi, h->chi, 2) != cudaSuccess)
      return fail(h, BSMPO_ECUDA, "tensor map encoding failed");
    const int tm = tc_tile_m(), tn = tc_tile_n();
    for (const ThetaDesc& D : P.td) {
      TcGroup g;
      std::memset(&g, 0, sizeof(g));
      g.M = D.nrow; g.N = D.ncol; g.K = D.nk;
      g.opA = 0; g.mapA = 0; g.mapB = 1;
      g.a_r0 = D.row0; g.a_c0 = D.k0; g.b_r0 = D.k0; g.b_c0 = D.col0;
      g.ldc = D.ncol;
      g.tiles_n = ceil_div(D.ncol, tn);
      g.tile_start = P.tc_tiles;
      P.tc_tiles += ceil_div(D.nrow, tm) * g.tiles_n;
      g.c_off = D.off;
      g.cs_off = -1;
      P.tcg.push_back(g);
    }
  }
  // Gram groups: G_s = X^H X, X = the first rows_g rows of the sector's Jacobi matrix
  // ([rows_g][k] row-major: T, or T^H when |L| < |R|)
  P.ggram.clear();
  int gtiles = 0;
  for (const SectorDesc& S : P.sd) {
    GemmGroup g;
    std::memset(&g, 0, sizeof(g));
    g.M = S.k; g.N = S.k; g.K = S.rows_g;
    g.lda = S.k; g.ldb = S.k; g.ldc = S.k;
    g.opA = 1; g.opB = 0; g.beta = 0;
    g.tiles_n = ceil_div(S.k, TNt);
    g.tile_start = gtiles;
    gtiles += ceil_div(S.k, TMt) * g.tiles_n;
    g.a_off = S.a_off; g.b_off = S.a_off; g.c_off = S.g_off;
    g.ks_off = g.rs_off = g.cs_off = -1;
    P.ggram.push_back(g);
  }
  P.gram_tiles = gtiles;
  P.tdlist.clear();
  for (int c = 0; c < 4; ++c) {
    P.td_count[c] = 0;
    P.td_kmax[c] = 0;
    for (int s = 0; s < (int)P.sd.size(); ++s)
      if (tridiag_class(P.sd[s].k) == c) {
        P.tdlist.push_back(s);
        P.td_count[c]++;
        P.td_kmax[c] = std::max(P.td_kmax[c], P.sd[s].k);
      }
  }
  T.n_theta = (int)P.td.size();
  // mix pairs (a >= b)
  P.pairs.clear();
  int mt = 0;
  for (int a0 = 0; a0 < d; ++a0)
    for (int a1 = 0; a1 < d; ++a1) {
      const int na = cL[a0 * d + a1];
      if (!na) continue;
      for (int b0 = 0; b0 <= a0; ++b0)
        for (int b1 = 0; b1 <= a1; ++b1) {
          const int nb = cR[b0 * d + b1];
          if (!nb) continue;
          MixPair M;
          M.a0 = a0; M.a1 = a1; M.b0 = b0; M.b1 = b1;
          M.row0 = T.offL[a0 * d + a1]; M.nrow = na;
          M.col0 = T.offR[b0 * d + b1]; M.ncol = nb;
          M.tile_start = mt;
          M.pad_ = 0;
          mt += ceil_div(na * nb, 256);
          P.pairs.push_back(M);
        }
    }
  P.mix_tiles = mt;
  T.n_pairs = (int)P.pairs.size();
  // Jacobi work
  P.jw.clear();
  P.max_rounds = 0;
  P.max_k = 0;
  P.max_left_m2 = 0;
  const int JBc = jacobi_block_cols();
  const int rmax = std::min(h->jac_rows, jacobi_rows_per_part());
  for (int s = 0; s < ns; ++s) {
    const SectorDesc& S = P.sd[s];
    P.max_k = std::max(P.max_k, S.k);
    if (S.left) P.max_left_m2 = std::max(P.max_left_m2, S.m * S.m);
    JacobiWork w;
    std::memset(&w, 0, sizeof(w));
    w.sector = s;
    w.nblk = ceil_div(S.k, JBc);
    const int nbp = w.nblk + (w.nblk & 1);
    w.npairs = nbp / 2;
    w.rounds = nbp - 1;
    // parts of at most rmax rows (multiples of 16), as even as that allows; every part
    // is non-empty, and the first cs_g hold the Gram rows
    const int cs0 = ceil_div(S.rows_tot, rmax);
    w.chunk = ceil_div(ceil_div(S.rows_tot, cs0), 16) * 16;
    w.cs = ceil_div(S.rows_tot, w.chunk);
    w.cs_g = ceil_div(S.rows_g, w.chunk);
    P.max_rounds = std::max(P.max_rounds, w.rounds);
    P.jw.push_back(w);
  }
  std::vector<JacobiWork> all(P.jw);
  jacobi_launch_list(all, &P.gram_ctas, &P.apply_ctas, &P.jac_slots);
  return BSMPO_OK;
}

// packs plan tables into the pinned stage and copies them to the device table buffer
struct TabLayout {
  size_t tab, tidx, td, sd, pairs, gg, ggram, tdlist, tcmaps, tcg, jw, total;
};

TabLayout layout_of(const Plan& P) {
  TabLayout L;
  size_t o = 0;
  L.tab = o; o = align_up(o + sizeof(UpdateTables), 256);
  L.tidx = o; o = align_up(o + P.tidx.size() * sizeof(int), 256);
  L.td = o; o = align_up(o + P.td.size() * sizeof(ThetaDesc) + 1, 256);
  L.sd = o; o = align_up(o + P.sd.size() * sizeof(SectorDesc) + 1, 256);
  L.pairs = o; o = align_up(o + P.pairs.size() * sizeof(MixPair) + 1, 256);
  L.gg = o; o = align_up(o + P.gg.size() * sizeof(GemmGroup) + 1, 256);
  L.ggram = o; o = align_up(o + P.ggram.size() * sizeof(GemmGroup) + 1, 256);
  L.tdlist = o; o = align_up(o + P.tdlist.size() * sizeof(int) + 1, 256);
  L.tcmaps = o; o = align_up(o + P.tcmaps.size() + 1, 256);
  L.tcg = o; o = align_up(o + P.tcg.size() * sizeof(TcGroup) + 1, 256);
  L.jw = o; o = align_up(o + P.jw.size() * sizeof(JacobiWork) + 1, 256);
  L.total = o;
  return L;
}

template <typename T>
void put(void* base, size_t off, const std::vector<T>& v) {
  if (!v.empty()) std::memcpy(static_cast<char*>(base) + off, v.data(), v.size() * sizeof(T));
}

int check_mode(bsmpo_ctx* h, int mode) {
  if (!h) return fail(nullptr, BSMPO_EINVAL, "null handle");
  if (!h->loaded) return fail(h, BSMPO_EINVAL, "no state loaded");
  if (mode < 0 || mode > h->n - 2) return fail(h, BSMPO_EINVAL, "mode out of range");
  return BSMPO_OK;
}

struct StageClock {
  bsmpo_ctx* h;
  std::chrono::steady_clock::time_point t0;
  explicit StageClock(bsmpo_ctx* hh) : h(hh), t0(std::chrono::steady_clock::now()) {}
  // stage i done: with profiling on, wait for the device and add the elapsed time
  int mark(int i) {
    if (!h->profile) return BSMPO_OK;
    CK(h, cudaStreamSynchronize(h->stream));
    auto t1 = std::chrono::steady_clock::now();
    h->stage_ms[i] += std::chrono::duration<double, std::milli>(t1 - t0).count();
    t0 = t1;
    return BSMPO_OK;
  }
};

int bs_update_impl(bsmpo_ctx* h, int mode, const cplx* u3_dev) {
  int rc = check_mode(h, mode);
  if (rc) return rc;
  StageClock clk(h);
  h->updates++;
  const int d = h->d, chi = h->chi, dd = d * d;
  cudaStream_t st = h->stream;
  Plan P;
  if ((rc = make_plan(h, mode, P))) return rc;
  const int ns = (int)P.sd.size();
  h->last_ns = ns;
  if (ns == 0) return fail(h, BSMPO_EINVAL, "update with an empty left or right bond");
  // workspaces
  if ((rc = grow(h, h->theta, std::max<int64_t>(P.theta_elems, 1) * sizeof(cplx)))) return rc;
  if ((rc = grow(h, h->cbuf, std::max<int64_t>(P.c_elems, 1) * sizeof(cplx)))) return rc;
  if ((rc = grow(h, h->abuf, std::max<int64_t>(P.a_elems, 1) * sizeof(cplx)))) return rc;
  if ((rc = grow(h, h->wbuf, std::max<int64_t>(P.w_elems, 1) * sizeof(cplx)))) return rc;
  if ((rc = grow(h, h->vbuf, std::max<int64_t>(P.v_elems, 1) * sizeof(cplx)))) return rc;
  if ((rc = grow(h, h->sig, std::max<int64_t>(P.s_elems, 1) * sizeof(double)))) return rc;
  if ((rc = grow(h, h->keys, std::max<int64_t>(P.s_elems, 1) * sizeof(double)))) return rc;
  if ((rc = grow(h, h->perm, std::max<int64_t>(P.s_elems, 1) * sizeof(int)))) return rc;
  if ((rc = grow(h, h->rot, (size_t)3 * ns * sizeof(int)))) return rc;
  if ((rc = grow(h, h->nf2, (size_t)ns * sizeof(double)))) return rc;
  const size_t pair_elems = (size_t)4 * jacobi_block_cols() * jacobi_block_cols();
  if ((rc = grow(h, h->qbuf, std::max(P.jac_slots, 1) * pair_elems * sizeof(cplx)))) return rc;
  if ((rc = grow(h, h->qflag, std::max(P.jac_slots, 1) * sizeof(int)))) return rc;
  if ((rc = grow(h, h->pcnt, std::max(P.jac_slots, 1) * sizeof(int)))) return rc;
  if ((rc = grow(h, h->pbuf, std::max(P.gram_ctas, 1) * pair_elems * sizeof(cplx)))) return rc;
  if ((rc = grow(h, h->kept, (size_t)(ns + 1) * sizeof(int) + 64))) return rc;
  const TabLayout L = layout_of(P);
  if ((rc = grow(h, h->tab, L.total))) return rc;
  if ((rc = grow_host(h, h->stage, L.total))) return rc;
  if ((rc = grow_host(h, h->hres, 4096 + (size_t)(ns + 2) * sizeof(int) + 6 * ns * sizeof(int)))) return rc;
  char* hs = static_cast<char*>(h->stage.p);
  std::memcpy(hs + L.tab, &P.tab, sizeof(UpdateTables));
  put(hs, L.tidx, P.tidx);
  put(hs, L.td, P.td);
  put(hs, L.sd, P.sd);
  put(hs, L.pairs, P.pairs);
  put(hs, L.gg, P.gg);
  put(hs, L.ggram, P.ggram);
  put(hs, L.tdlist, P.tdlist);
  put(hs, L.tcmaps, P.tcmaps);
  put(hs, L.tcg, P.tcg);
  std::vector<JacobiWork> active(P.jw);
  int gram_ctas = 0, apply_ctas = 0, slots = 0;
  jacobi_launch_list(active, &gram_ctas, &apply_ctas, &slots);
  put(hs, L.jw, active);
  char* dt = static_cast<char*>(h->tab.p);
  CK(h, cudaMemcpyAsync(dt, hs, L.total, cudaMemcpyHostToDevice, st));
  const UpdateTables* tab_d = reinterpret_cast<const UpdateTables*>(dt + L.tab);
  const int* tidx_d = reinterpret_cast<const int*>(dt + L.tidx);
  const ThetaDesc* td_d = reinterpret_cast<const ThetaDesc*>(dt + L.td);
  SectorDesc* sd_d = reinterpret_cast<SectorDesc*>(dt + L.sd);
  const MixPair* pairs_d = reinterpret_cast<const MixPair*>(dt + L.pairs);
  const GemmGroup* gg_d = reinterpret_cast<const GemmGroup*>(dt + L.gg);
  const GemmGroup* ggram_d = reinterpret_cast<const GemmGroup*>(dt + L.ggram);
  const int* tdlist_d = reinterpret_cast<const int*>(dt + L.tdlist);
  const bool tc = h->precision == BSMPO_PRECISION_TF32X3;
  const bool tc_theta = tc && (h->tc_mask & 1), tc_w = tc && (h->tc_mask & 2);
  // error word of the asynchronous pipelines (tensor-core GEMM, streamed
  // tridiagonalisation): set on the device when a bounded wait expires
  if (!h->tcerr.p) {
    if ((rc = grow(h, h->tcerr, sizeof(int)))) return rc;
    CK(h, cudaMemsetAsync(h->tcerr.p, 0, sizeof(int), st));
  }
  int* tcerr_d = reinterpret_cast<int*>(h->tcerr.p);
  // The Gram route drops singular values below ~2e-6 of a sector's largest.  Where the
  // update does not truncate to chi that is pure loss (W = V^H C carries them through
  // 1 / Lambda_R), so such updates take the exact Jacobi SVD: up front when the
  // candidates cannot exceed chi or the centre bond holds fewer than chi vectors, and
  // after the selection when fewer than chi survive.
  bool gram = h->precision != BSMPO_PRECISION_FP64;
  {
    // the centre bond's current dimension predicts the outcome: a bond below chi was not
    // truncated by the last update on it and is unlikely to be by this one
    int64_t sum_k = 0, centre = 0;
    for (const SectorDesc& S : P.sd) sum_k += S.k;
    const std::vector<int>& cm = mirror(h);
    for (int q = 0; q < dd; ++q) centre += cm[(size_t)(mode + 1) * dd + q];
    if (sum_k <= chi || (h->gram_policy >= 2 && centre < chi)) gram = false;
  }
  const JacobiWork* jw_d = reinterpret_cast<const JacobiWork*>(dt + L.jw);
  const int64_t chi2 = (int64_t)chi * chi;

  if ((rc = clk.mark(0))) return rc;
  // 1. Theta_q = Glc[a, q] Gcr[q, b] for every valid triple
  if (tc_theta)
    CKL(h, launch_tc_zgemm(reinterpret_cast<const TcGroup*>(dt + L.tcg), (int)P.tcg.size(), P.tc_tiles,
                           dt + L.tcmaps, h->theta.p, nullptr, tcerr_d, st));
  else
    CKL(h, launch_zgemm_grouped(h->gamma, h->gamma, h->theta.p, nullptr, gg_d, (int)P.gg.size(),
                                P.gemm_tiles, st));
  if ((rc = clk.mark(1))) return rc;
  // 2. identity rows of [T^H; I] and the gate mix
  if (!gram) CKL(h, launch_identity_rows(sd_d, ns, P.max_left_m2, h->abuf.p, st));
  CKL(h, launch_mix_d(d, tab_d, tidx_d, td_d, sd_d, pairs_d, (int)P.pairs.size(), P.mix_tiles,
                      u3_dev, h->theta.p, h->lam + (size_t)(mode + 2) * chi, h->cbuf.p, h->abuf.p,
                      st));
  if ((rc = clk.mark(2))) return rc;
  // 3. the sector SVD: Gram + Hermitian eigenproblem, or blocked one-sided Jacobi
  double* lam_d = nullptr;
  double* dbuf_d = nullptr;
  double* ebuf_d = nullptr;
  int* hk = reinterpret_cast<int*>(h->hres.p);
  double* htw = reinterpret_cast<double*>(static_cast<char*>(h->hres.p) + 512);
  int total_kept = 0;
  for (;;) {
  if (gram) {
    if (P.max_k > eigen_max_k())
      return fail(h, BSMPO_ECAPACITY, "a sector of dimension " + std::to_string(P.max_k) +
                                          " exceeds the Gram route's limit " + std::to_string(eigen_max_k()));
    if ((rc = grow(h, h->gbuf, std::max<int64_t>(P.g_elems, 1) * sizeof(cplx)))) return rc;
    if ((rc = grow(h, h->eigd, std::max<int64_t>(3 * P.s_elems, 1) * sizeof(double)))) return rc;
    if ((rc = grow(h, h->taub, std::max<int64_t>(P.s_elems, 1) * sizeof(cplx)))) return rc;
    if ((rc = grow(h, h->invsig, std::max<int64_t>(P.s_elems, 1) * sizeof(double)))) return rc;
    dbuf_d = reinterpret_cast<double*>(h->eigd.p);
    ebuf_d = dbuf_d + P.s_elems;
    lam_d = ebuf_d + P.s_elems;
    if (h->timing) CK(h, cudaEventRecord(h->ev0, st));
    CKL(h, launch_zgemm_grouped(h->abuf.p, h->abuf.p, h->gbuf.p, nullptr, ggram_d, (int)P.ggram.size(),
                                P.gram_tiles, st));
    {
      // the largest class present on the update's stream, the others spread over the
      // side streams (none: all one after another)
      if (h->td_fork > 0 && (rc = make_fork_streams(h))) return rc;
      const int naux = std::min(h->td_fork, h->n_aux);
      cudaStream_t ts[4] = {st, st, st, st};
      bool used[3] = {false, false, false};
      for (int c = 3, slot = -1; c >= 0; --c) {
        if (P.td_count[c] == 0) continue;
        if (slot >= 0 && naux > 0) {
          ts[3 - c] = h->aux[slot % naux];
          used[slot % naux] = true;
        }
        ++slot;
      }
      const bool fork = used[0] || used[1] || used[2];
      if (h->timing) {
        if (!h->td_ev0) {
          CK(h, cudaEventCreate(&h->td_ev0));
          CK(h, cudaEventCreate(&h->td_ev1));
        }
        CK(h, cudaEventRecord(h->td_ev0, st));
      }
      if (fork) {
        CK(h, cudaEventRecord(h->fork_ev, st));
        for (int i = 0; i < 3; ++i)
          if (used[i]) CK(h, cudaStreamWaitEvent(h->aux[i], h->fork_ev, 0));
      }
      CK(h, launch_tridiag(sd_d, tdlist_d, P.td_count, P.td_kmax, h->gbuf.p, dbuf_d, ebuf_d, h->taub.p,
                           tcerr_d, ts));
      for (int i = 0; i < 3; ++i)
        if (used[i]) {
          CK(h, cudaEventRecord(h->join_ev[i], h->aux[i]));
          CK(h, cudaStreamWaitEvent(st, h->join_ev[i], 0));
        }
      for (int c = 0; c < 4; ++c) h->launches += P.td_count[c] > 0;
      if (h->timing) CK(h, cudaEventRecord(h->td_ev1, st));
    }
    CK(h, launch_bisect(sd_d, ns, P.max_k, dbuf_d, ebuf_d, lam_d, reinterpret_cast<double*>(h->sig.p),
                        reinterpret_cast<double*>(h->invsig.p), st));
    h->launches += 2;
    if (h->timing) CK(h, cudaEventRecord(h->ev1, st));
    h->last_sweeps = 0;
    if ((rc = clk.mark(3))) return rc;
  } else {
    // 3. blocked one-sided Jacobi
    double* nf2 = reinterpret_cast<double*>(h->nf2.p);
    CKL(h, launch_sector_norms(sd_d, ns, h->abuf.p, nf2, st));
    CK(h, cudaMemsetAsync(h->rot.p, 0, (size_t)3 * ns * sizeof(int), st));
    CK(h, cudaMemsetAsync(h->pcnt.p, 0, std::max(P.jac_slots, 1) * sizeof(int), st));
    if ((rc = grow(h, h->jwork, 2 * sizeof(unsigned long long)))) return rc;
    CK(h, cudaMemsetAsync(h->jwork.p, 0, 2 * sizeof(unsigned long long), st));
    // Convergence polls run one chunk behind: after launching chunk c + 1 the host reads
    // the counters copied after chunk c, so the stream always has a chunk queued while the
    // host checks (a converged sector's rounds in the extra chunk exit at once).  Counters
    // and compacted launch tables alternate between two pinned slots.
    int* hrot_slot[2] = {reinterpret_cast<int*>(static_cast<char*>(h->hres.p) + 1024), nullptr};
    hrot_slot[1] = hrot_slot[0] + 3 * ns;
    const size_t jw_bytes = align_up(std::max<size_t>(P.jw.size(), 1) * sizeof(JacobiWork), 256);
    if ((rc = grow_host(h, h->stage2, 2 * jw_bytes))) return rc;
    char* jw_stage[2] = {static_cast<char*>(h->stage2.p), static_cast<char*>(h->stage2.p) + jw_bytes};
    for (cudaEvent_t& e : h->poll_ev)
      if (!e) CK(h, cudaEventCreateWithFlags(&e, cudaEventBlockingSync | cudaEventDisableTiming));
    int t = 0;
    const int t_max = MAX_SWEEPS * std::max(1, P.max_rounds);
    bool converged = false;
    int checks = 0;
    std::vector<int> conv_at(ns, -1);
    if (h->timing) CK(h, cudaEventRecord(h->ev0, st));
    const int chunk = std::max(1, P.max_rounds);   // one sweep of the largest sector
    int t_after[2] = {0, 0};
    auto launch_chunk = [&](int slot) -> int {
      for (int i = 0; i < chunk && t < t_max; ++i, ++t) {
        // tol <= 0: per-sector default 4 eps sqrt(rows of the Gram), at least 8 eps
        CK(h, launch_jacobi_round(sd_d, jw_d, (int)active.size(), gram_ctas, apply_ctas, t,
                                  h->abuf.p, reinterpret_cast<int*>(h->rot.p), nf2, 0.0, MAX_SWEEPS,
                                  h->pbuf.p, reinterpret_cast<int*>(h->pcnt.p), h->qbuf.p,
                                  reinterpret_cast<int*>(h->qflag.p),
                                  reinterpret_cast<unsigned long long*>(h->jwork.p), st));
        h->launches += 2;
      }
      CK(h, cudaMemcpyAsync(hrot_slot[slot], h->rot.p, (size_t)3 * ns * sizeof(int),
                            cudaMemcpyDeviceToHost, st));
      CK(h, cudaEventRecord(h->poll_ev[slot], st));
      t_after[slot] = t;
      return BSMPO_OK;
    };
    if ((rc = launch_chunk(0))) return rc;
    int cur = 0, compactions = 0;
    for (;;) {
      const bool more = t < t_max;
      if (more && (rc = launch_chunk(cur ^ 1))) return rc;
      CK(h, cudaEventSynchronize(h->poll_ev[cur]));
      ++checks;
      const int* hrot = hrot_slot[cur];
      bool all = true;
      for (int s = 0; s < ns; ++s) {
        // a converged sector leaves the launches, and its counters are stale from then on
        if (conv_at[s] >= 0) continue;
        const int R = P.jw[s].rounds;
        const int done = t_after[cur] / R;
        if (done < 1 || hrot[3 * s + (done - 1) % 3] != 0) { all = false; continue; }
        conv_at[s] = done;
      }
      if (all) { converged = true; break; }
      if (!more) break;
      // drop converged sectors (and those out of sweeps) from the launches after the queued
      // chunk: the table copy is stream-ordered after it
      std::vector<JacobiWork> next;
      for (const auto& w : P.jw)
        if (conv_at[w.sector] < 0 && t / w.rounds < MAX_SWEEPS) next.push_back(w);
      if (next.size() < active.size() && !next.empty()) {
        active.swap(next);
        jacobi_launch_list(active, &gram_ctas, &apply_ctas, &slots);
        char* stg = jw_stage[compactions++ & 1];
        put(stg, 0, active);
        CK(h, cudaMemcpyAsync(dt + L.jw, stg, active.size() * sizeof(JacobiWork),
                              cudaMemcpyHostToDevice, st));
      }
      cur ^= 1;
    }
    if (h->timing) {
      CK(h, cudaMemcpyAsync(static_cast<char*>(h->hres.p) + 2048, h->jwork.p, 2 * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, st));
      CK(h, cudaEventRecord(h->ev1, st));
    }
    // sweeps the slowest sector needed (its last one without rotations included); t also
    // counts the chunk queued after convergence, whose rounds exit at once
    {
      int sw = 0;
      for (int s = 0; s < ns; ++s) sw = std::max(sw, conv_at[s] >= 0 ? conv_at[s] : t / P.jw[s].rounds);
      h->last_sweeps = sw;
    }
    h->jacobi_rounds += t;   // launched rounds, including the drained chunk
    if (h->timing) {
      float ms = 0.f;
      CK(h, cudaEventSynchronize(h->ev1));
      CK(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
      h->jac_ms += ms;
      h->jac_launches += t;
      // flops of the executed work, counted on the device: every row that formed a
      // partial pair Gram contributes its 10 upper 8 x 8 tiles (640 complex MACs), every
      // rotated row 32 x 32 complex MACs; 8 flops per complex MAC.  Pairs that did not
      // rotate and sectors that had converged do no apply work and are not counted.
      const unsigned long long* hw =
          reinterpret_cast<const unsigned long long*>(static_cast<char*>(h->hres.p) + 2048);
      h->jac_flops += 8.0 * 640.0 * (double)hw[0] + 8.0 * 1024.0 * (double)hw[1];
    }
    if ((rc = clk.mark(3))) return rc;
    if (!converged) {
      std::string msg = "Jacobi SVD did not converge (mode " + std::to_string(mode) + ")";
      for (int s = 0; s < ns; ++s) {
        const int R = P.jw[s].rounds, done = t_after[cur] / R;
        if (conv_at[s] >= 0) continue;
        const SectorDesc& S = P.sd[s];
        msg += "; sector (" + std::to_string(S.cc0) + "," + std::to_string(S.cc1) + ") m=" +
               std::to_string(S.m) + " n=" + std::to_string(S.n) + " sweeps=" + std::to_string(done) +
               " rotations=" + std::to_string(hrot_slot[cur][3 * s + (done - 1 + 3) % 3]);
        break;
      }
      return fail(h, BSMPO_ECONVERGE, msg);
    }
    CKL(h, launch_jacobi_finish(sd_d, ns, P.max_k, h->abuf.p, nf2,
                                reinterpret_cast<double*>(h->sig.p),
                                reinterpret_cast<int*>(h->perm.p), st));
  }
  // 4. selection -> kept counts (the one host sync of the update)
  int* kept_d = reinterpret_cast<int*>(h->kept.p);
  double* trunc_d = reinterpret_cast<double*>(static_cast<char*>(h->kept.p) +
                                              align_up((size_t)(ns + 1) * sizeof(int), 16));
  CKL(h, launch_select(tab_d, sd_d, ns, reinterpret_cast<double*>(h->sig.p),
                       reinterpret_cast<double*>(h->keys.p), h->cutoff, chi, kept_d, trunc_d, st));
  CK(h, cudaMemcpyAsync(hk, kept_d, (size_t)(ns + 1) * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(h, cudaMemcpyAsync(htw, trunc_d, sizeof(double), cudaMemcpyDeviceToHost, st));
  int* htc = reinterpret_cast<int*>(static_cast<char*>(h->hres.p) + 1000);
  CK(h, cudaMemcpyAsync(htc, tcerr_d, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(h, host_wait(h));
  if (*htc != 0)
    return fail(h, BSMPO_ECUDA, "tensor-core GEMM or tridiagonalisation: a pipeline wait expired (error word set)");
  total_kept = hk[ns];
  if (gram && total_kept < chi && h->cutoff == 0.0 && h->gram_policy >= 1) {
    // not truncated to chi: redo the SVD exactly (the Gram matrix and the eigen buffers
    // are not needed any more; the Jacobi matrix is intact)
    gram = false;
    CKL(h, launch_identity_rows(sd_d, ns, P.max_left_m2, h->abuf.p, st));
    continue;
  }
  break;
  }
  h->route_count[gram ? 1 : 0]++;
  if (gram && h->timing) {
    // eigen phase of the Gram route (Gram GEMM, tridiagonalisation, bisection): both
    // events completed before the kept counts arrived
    float ms = 0.f;
    CK(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->jac_ms += ms;
    h->jac_launches += 4;
    // algorithmic flops: the Gram (8 k^2 rows, complex MACs) and the Householder
    // reduction of a k x k Hermitian matrix (16/3 k^3, LAPACK's zhetrd count)
    for (const SectorDesc& S : P.sd)
      h->jac_flops += 8.0 * (double)S.k * S.k * S.rows_g + 16.0 / 3.0 * (double)S.k * S.k * S.k;
    float tms = 0.f;
    CK(h, cudaEventElapsedTime(&tms, h->td_ev0, h->td_ev1));
    h->td_ms += tms;
    h->td_phases++;
    for (const SectorDesc& S : P.sd) {
      // step j reads and writes the (k - j - 1)^2 trailing matrix once: 32 B per entry
      const double k = S.k;
      h->td_bytes += 32.0 * (k - 1.0) * k * (2.0 * k - 1.0) / 6.0;
      h->td_flops += 16.0 / 3.0 * k * k * k;
    }
  }
  if ((rc = clk.mark(4))) return rc;
  // 5. V (Jacobi: extracted from the converged columns; Gram route: eigenvectors, and
  // V = T Y diag(1/sigma) where X = T) and W = V^H C
  std::vector<GemmGroup> wg, vg;
  int wtiles = 0, vtiles = 0, max_vm = 0, kept_max = 0;
  double flops_w = 0.0;
  const int TMt = zgemm_tile_m(), TNt = zgemm_tile_n();
  for (int s = 0; s < ns; ++s) {
    const SectorDesc& S = P.sd[s];
    const int kp = hk[s];
    max_vm = std::max(max_vm, kp * S.m);
    kept_max = std::max(kept_max, kp);
    if (kp == 0) continue;
    GemmGroup g;
    std::memset(&g, 0, sizeof(g));
    g.M = kp; g.N = S.n; g.K = S.m;
    g.lda = kp; g.ldb = S.n; g.ldc = S.n;
    g.opA = 1; g.opB = 0; g.beta = 0;
    g.tiles_n = ceil_div(S.n, TNt);
    g.tile_start = wtiles;
    wtiles += ceil_div(kp, TMt) * g.tiles_n;
    g.a_off = S.v_off; g.b_off = S.c_off; g.c_off = S.w_off;
    g.ks_off = g.rs_off = g.cs_off = -1;
    wg.push_back(g);
    flops_w += 8.0 * kp * (double)S.m * S.n;
    if (gram && !S.left) {
      // V [m][kp] = T [m][k] Y [k][kp] diag(1 / sigma)
      GemmGroup v;
      std::memset(&v, 0, sizeof(v));
      v.M = S.m; v.N = kp; v.K = S.k;
      v.lda = S.k; v.ldb = kp; v.ldc = kp;
      v.opA = 0; v.opB = 0; v.beta = 0;
      v.tiles_n = ceil_div(kp, TNt);
      v.tile_start = vtiles;
      vtiles += ceil_div(S.m, TMt) * v.tiles_n;
      v.a_off = S.a_off; v.b_off = S.y_off; v.c_off = S.v_off;
      v.ks_off = v.rs_off = -1;
      v.cs_off = S.s_off;
      vg.push_back(v);
      flops_w += 8.0 * kp * (double)S.m * S.k;
    }
  }
  const size_t wbytes = align_up(wg.size() * sizeof(GemmGroup) + 1, 256);
  const size_t vbytes = align_up(vg.size() * sizeof(GemmGroup) + 1, 256);
  if ((rc = grow(h, h->tab2, wbytes + vbytes))) return rc;
  if ((rc = grow_host(h, h->stage2, wbytes + vbytes))) return rc;
  put(h->stage2.p, 0, wg);
  put(h->stage2.p, wbytes, vg);
  CK(h, cudaMemcpyAsync(h->tab2.p, h->stage2.p, wbytes + vbytes, cudaMemcpyHostToDevice, st));
  const GemmGroup* wg_d = reinterpret_cast<const GemmGroup*>(h->tab2.p);
  const GemmGroup* vg_d = reinterpret_cast<const GemmGroup*>(static_cast<char*>(h->tab2.p) + wbytes);
  if (gram) {
    const size_t ye = (size_t)std::max<int64_t>(P.y_elems, 1);
    if ((rc = grow(h, h->escr, 4 * ye * sizeof(double)))) return rc;
    if ((rc = grow(h, h->swp, ye))) return rc;
    if ((rc = grow(h, h->zbuf, ye * sizeof(double)))) return rc;
    if ((rc = grow(h, h->ybuf, ye * sizeof(cplx)))) return rc;
    CK(h, launch_eigvec(sd_d, ns, P.max_k, kept_max, dbuf_d, ebuf_d, lam_d,
                        reinterpret_cast<double*>(h->escr.p), reinterpret_cast<unsigned char*>(h->swp.p),
                        reinterpret_cast<double*>(h->zbuf.p), h->gbuf.p, h->taub.p, h->vbuf.p, h->ybuf.p,
                        st));
    h->launches += 2;
    // V = T Y diag(1/sigma) stays FP64: it divides by sigma (down to ~3e-3 of the largest
    // at the cut), which would magnify a TF32 error into V's orthogonality, and a
    // non-orthonormal V leaks into W = V^H C at the scale of C
    if (!vg.empty())
      CKL(h, launch_zgemm_grouped(h->abuf.p, h->ybuf.p, h->vbuf.p, reinterpret_cast<double*>(h->invsig.p),
                                  vg_d, (int)vg.size(), vtiles, st));
  } else {
    CKL(h, launch_extract_v(sd_d, ns, max_vm, h->abuf.p, reinterpret_cast<double*>(h->sig.p),
                            reinterpret_cast<int*>(h->perm.p), h->vbuf.p, st));
  }
  if (tc_w) {
    // W = V^H C on the tensor cores: two tensor maps per group
    const size_t mb = tc_map_bytes();
    std::vector<unsigned char> maps;
    std::vector<TcGroup> tw;
    int tw_tiles = 0;
    const int tm = tc_tile_m(), tn = tc_tile_n();
    bool enc_ok = true;
    auto add_map = [&](const void* base, int rows, int cols, int ld, int kind) -> int {
      const int idx = (int)(maps.size() / mb);
      maps.resize(maps.size() + mb);
      if (tc_encode_map(maps.data() + (size_t)idx * mb, base, rows, cols, ld, kind) != cudaSuccess) enc_ok = false;
      return idx;
    };
    const cplx* V0 = reinterpret_cast<const cplx*>(h->vbuf.p);
    const cplx* C0 = reinterpret_cast<const cplx*>(h->cbuf.p);
    for (int s = 0; s < ns; ++s) {
      const SectorDesc& S = P.sd[s];
      const int kp = hk[s];
      if (kp == 0) continue;
      TcGroup g;
      std::memset(&g, 0, sizeof(g));
      g.M = kp; g.N = S.n; g.K = S.m; g.opA = 1;
      g.mapA = add_map(V0 + S.v_off, S.m, kp, kp, 1);
      g.mapB = add_map(C0 + S.c_off, S.m, S.n, S.n, 2);
      g.ldc = S.n;
      g.tiles_n = ceil_div(S.n, tn);
      g.tile_start = tw_tiles;
      tw_tiles += ceil_div(kp, tm) * g.tiles_n;
      g.c_off = S.w_off;
      g.cs_off = -1;
      tw.push_back(g);
    }
    if (!enc_ok) return fail(h, BSMPO_ECUDA, "tensor map encoding failed");
    const size_t o_tw = align_up(maps.size(), 256);
    const size_t total = align_up(o_tw + tw.size() * sizeof(TcGroup) + 1, 256);
    if ((rc = grow(h, h->tab3, total))) return rc;
    if ((rc = grow_host(h, h->stage3, total))) return rc;
    std::memcpy(h->stage3.p, maps.data(), maps.size());
    put(h->stage3.p, o_tw, tw);
    CK(h, cudaMemcpyAsync(h->tab3.p, h->stage3.p, total, cudaMemcpyHostToDevice, st));
    const char* t3 = static_cast<const char*>(h->tab3.p);
    CKL(h, launch_tc_zgemm(reinterpret_cast<const TcGroup*>(t3 + o_tw), (int)tw.size(), tw_tiles, t3,
                           h->wbuf.p, nullptr, tcerr_d, st));
  } else {
    CKL(h, launch_zgemm_grouped(h->vbuf.p, h->cbuf.p, h->wbuf.p, nullptr, wg_d, (int)wg.size(), wtiles, st));
  }
  if ((rc = clk.mark(5))) return rc;
  // 6. scatter into Gamma[mode], Gamma[mode+1], Lambda / charge of bond mode+1
  CKL(h, launch_scatter(tab_d, sd_d, ns, total_kept, chi, h->charge + (size_t)mode * chi * 2,
                        h->charge + (size_t)(mode + 2) * chi * 2, h->vbuf.p, h->wbuf.p,
                        reinterpret_cast<double*>(h->sig.p), h->gamma + (size_t)mode * chi2,
                        h->gamma + (size_t)(mode + 1) * chi2, h->lam + (size_t)(mode + 1) * chi,
                        h->charge + (size_t)(mode + 1) * chi * 2, st));
  if ((rc = clk.mark(6))) return rc;
  // algorithmic minimum bytes: read Glc, Gcr, write Gamma_L, Gamma_R (complex128)
  {
    double nl = 0, nc = 0, nr = 0;
    const std::vector<int>& cnt = mirror(h);
    for (int q = 0; q < dd; ++q) {
      nl += cnt[(size_t)mode * dd + q];
      nc += cnt[(size_t)(mode + 1) * dd + q];
      nr += cnt[(size_t)(mode + 2) * dd + q];
    }
    h->last_bytes = 16.0 * (nl * nc + nc * nr + ((double)nl + nr) * total_kept);
  }
  // host mirror and diagnostics
  int* cM = &mirror(h)[(size_t)(mode + 1) * dd];
  std::fill(cM, cM + dd, 0);
  h->last_cc.assign(2 * ns, 0);
  h->last_shape.assign(2 * ns, 0);
  h->last_kept.assign(ns, 0);
  h->last_k.assign(ns, 0);
  h->last_soff.assign(ns, 0);
  double svd_flops = 0.0;
  for (int s = 0; s < ns; ++s) {
    const SectorDesc& S = P.sd[s];
    cM[S.cc0 * d + S.cc1] = hk[s];
    h->last_cc[2 * s] = S.cc0;
    h->last_cc[2 * s + 1] = S.cc1;
    h->last_shape[2 * s] = S.m;
    h->last_shape[2 * s + 1] = S.n;
    h->last_kept[s] = hk[s];
    h->last_k[s] = S.k;
    h->last_soff[s] = S.s_off;
    // one sweep: every column pair's Gram (rows_g) and rotation (rows_tot), 8 flops / complex MAC
    svd_flops += 4.0 * (double)S.k * S.k * (S.rows_g + S.rows_tot);
  }
  h->last_trunc = *htw;
  h->last_gemm = P.flops_theta + flops_w;
  h->last_svd = svd_flops * h->last_sweeps;
  return BSMPO_OK;
}

M8 transpose_to_m8(const double* S) {
  // S = [[s00, s01], [s10, s11]] acting on the state -> tensor of M = S^T
  M8 m;
  m.v[0] = S[0]; m.v[1] = S[1];   // M00 = S00
  m.v[2] = S[4]; m.v[3] = S[5];   // M01 = S10
  m.v[4] = S[2]; m.v[5] = S[3];   // M10 = S01
  m.v[6] = S[6]; m.v[7] = S[7];   // M11 = S11
  return m;
}

void free_workspaces(bsmpo_ctx* h) {
  DevBuf* bufs[] = {&h->theta, &h->cbuf, &h->abuf, &h->wbuf, &h->vbuf, &h->sig, &h->keys,
                    &h->perm, &h->tab, &h->tab2, &h->rot, &h->kept, &h->u3, &h->m4,
                    &h->env_l, &h->env_r, &h->part, &h->outv, &h->dims, &h->nf2, &h->qbuf,
                    &h->qflag, &h->pbuf, &h->pcnt, &h->gbuf, &h->eigd, &h->taub, &h->invsig,
                    &h->escr, &h->swp, &h->zbuf, &h->ybuf, &h->tab3, &h->tcerr, &h->jwork};
  for (DevBuf* b : bufs)
    if (b->p) cudaFreeAsync(b->p, h->stream);
  cudaStreamSynchronize(h->stream);
  HostStage* hs[] = {&h->stage, &h->stage2, &h->stage3, &h->hres};
  for (HostStage* b : hs)
    if (b->p) cudaFreeHost(b->p);
  for (void* p : h->retired_host) cudaFreeHost(p);
  h->retired_host.clear();
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->wait_ev) cudaEventDestroy(h->wait_ev);
  for (cudaEvent_t& e : h->poll_ev)
    if (e) cudaEventDestroy(e);
  if (h->fork_ev) cudaEventDestroy(h->fork_ev);
  if (h->td_ev0) cudaEventDestroy(h->td_ev0);
  if (h->td_ev1) cudaEventDestroy(h->td_ev1);
  for (int i = 0; i < 3; ++i) {
    if (h->aux[i]) { cudaStreamSynchronize(h->aux[i]); cudaStreamDestroy(h->aux[i]); }
    if (h->join_ev[i]) cudaEventDestroy(h->join_ev[i]);
  }
}

void destroy_worker(bsmpo_ctx* w);

// A worker context for concurrent updates: the owner's state, its own stream.
int make_worker(bsmpo_ctx* h, bsmpo_ctx** out) {
  bsmpo_ctx* w = new bsmpo_ctx();
  w->n = h->n; w->d = h->d; w->chi = h->chi; w->device = h->device;
  w->gamma = h->gamma; w->lam = h->lam; w->charge = h->charge;
  w->pool = h->pool;
  w->loaded = true;
  w->cnt_shared = &h->cnt;
  w->profile = h->profile;
  w->td_fork = h->td_fork;
  if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete w;
    return fail(h, BSMPO_ECUDA, "worker stream creation failed");
  }
  if (w->td_fork && make_fork_streams(w) != BSMPO_OK) {
    const std::string msg = w->err;
    destroy_worker(w);
    return fail(h, BSMPO_ECUDA, msg);
  }
  *out = w;
  return BSMPO_OK;
}

void destroy_worker(bsmpo_ctx* w) {
  cudaStreamSynchronize(w->stream);
  free_workspaces(w);
  cudaStreamDestroy(w->stream);
  delete w;   // the state belongs to the owner
}

// Runs the updates of a mesh on the owner's workers.  Two beam splitters conflict when
// their modes differ by 0 or 1 (shared site); update k depends on the latest earlier
// update at modes m_k - 1, m_k and m_k + 1 -- nothing else it touches is written by
// another update (modes 2 apart share only a bond both read).  Workers take the
// lowest-numbered update whose dependencies have finished (host side: after their
// host mirror entries are written; device side: the worker's stream waits for the
// events recorded at their ends), so consecutive brick-wall layers overlap.  Every
// update computes exactly what it computes alone.
// The host side of a mesh over a host-resident state: the first update touching site s,
// first[s], copies the site in on its own stream before it starts, and the last, last[s],
// copies it out after it ends.  Every later update touching the site depends on the
// first one (they share a site), and the last one on every earlier one, so the copies
// need no events of their own; they run in the workers' streams, where they overlap the
// other workers' updates without extra streams (which would share the device's hardware
// queues with the workers' streams).
struct HostStream {
  std::vector<int> first, last;
  const char* gamma_in = nullptr;
  char* gamma_out = nullptr;
  size_t site_bytes = 0;
};

int run_mesh_concurrent(bsmpo_ctx* h, int n_bs, const int* modes, const cplx* u3, int nw,
                        HostStream* hs = nullptr) {
  const int d3 = h->d * h->d * h->d;
  int rc;
  while ((int)h->workers.size() < nw) {
    bsmpo_ctx* w = nullptr;
    if ((rc = make_worker(h, &w))) return rc;
    h->workers.push_back(w);
  }
  for (int k = 0; k < nw; ++k) {
    bsmpo_ctx* w = h->workers[k];
    w->cutoff = h->cutoff;
    w->precision = h->precision;
    w->gram_policy = h->gram_policy;
    w->tc_mask = h->tc_mask;
    w->td_fork = h->td_fork;
    w->jac_rows = h->jac_rows;
    w->timing = h->timing;
    if (w->timing && !w->ev0) {
      CK(h, cudaEventCreate(&w->ev0));
      CK(h, cudaEventCreate(&w->ev1));
    }
    w->last_index = -1;
  }
  // dependencies
  std::vector<int> pred((size_t)3 * n_bs, -1), remaining(n_bs, 0);
  std::vector<std::vector<int>> succ(n_bs);
  {
    std::vector<int> last(h->n, -1);
    for (int k = 0; k < n_bs; ++k) {
      const int m = modes[k];
      int c = 0;
      for (int dm = -1; dm <= 1; ++dm) {
        const int mm = m + dm;
        if (mm < 0 || mm > h->n - 2 || last[mm] < 0) continue;
        pred[(size_t)3 * k + c++] = last[mm];
        succ[last[mm]].push_back(k);
      }
      remaining[k] = c;
      last[m] = k;
    }
  }
  std::vector<cudaEvent_t> done_ev(n_bs, nullptr);
  for (int k = 0; k < n_bs; ++k)
    if (cudaEventCreateWithFlags(&done_ev[k], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      for (cudaEvent_t e : done_ev) if (e) cudaEventDestroy(e);
      return fail(h, BSMPO_ECUDA, "event creation failed");
    }
  std::mutex mu;
  std::condition_variable cv;
  std::priority_queue<int, std::vector<int>, std::greater<int>> ready;
  for (int k = 0; k < n_bs; ++k)
    if (remaining[k] == 0) ready.push(k);
  int finished = 0;
  int err_code = BSMPO_OK;
  std::string err_msg;
  std::vector<std::thread> pool;
  for (int wk = 0; wk < nw; ++wk)
    pool.emplace_back([&, wk]() {
      bsmpo_ctx* w = h->workers[wk];
      cudaSetDevice(h->device);
      for (;;) {
        int k;
        {
          std::unique_lock<std::mutex> lock(mu);
          cv.wait(lock, [&] { return err_code || finished == n_bs || !ready.empty(); });
          if (err_code || ready.empty()) break;
          k = ready.top();
          ready.pop();
        }
        int r = BSMPO_OK;
        for (int c = 0; c < 3 && !r; ++c) {
          const int j = pred[(size_t)3 * k + c];
          if (j >= 0 && cudaStreamWaitEvent(w->stream, done_ev[j], 0) != cudaSuccess)
            r = fail(w, BSMPO_ECUDA, "cudaStreamWaitEvent failed");
        }
        for (int site = modes[k]; hs && site <= modes[k] + 1 && !r; ++site)
          if (hs->first[site] == k &&
              cudaMemcpyAsync(reinterpret_cast<char*>(h->gamma) + (size_t)site * hs->site_bytes,
                              hs->gamma_in + (size_t)site * hs->site_bytes, hs->site_bytes,
                              cudaMemcpyHostToDevice, w->stream) != cudaSuccess)
            r = fail(w, BSMPO_ECUDA, "site copy-in failed");
        if (!r) r = bs_update_impl(w, modes[k], u3 + (size_t)k * d3);
        if (!r) h->mesh_tw[k] = w->last_trunc;   // each k is written by one worker only
        if (!r && cudaEventRecord(done_ev[k], w->stream) != cudaSuccess)
          r = fail(w, BSMPO_ECUDA, "cudaEventRecord failed");
        for (int site = modes[k]; hs && site <= modes[k] + 1 && !r; ++site)
          // the site's final value of this mesh: copied out behind the update
          if (hs->last[site] == k &&
              cudaMemcpyAsync(hs->gamma_out + (size_t)site * hs->site_bytes,
                              reinterpret_cast<const char*>(h->gamma) + (size_t)site * hs->site_bytes,
                              hs->site_bytes, cudaMemcpyDeviceToHost, w->stream) != cudaSuccess)
            r = fail(w, BSMPO_ECUDA, "site copy-out failed");
        std::lock_guard<std::mutex> lock(mu);
        if (r) {
          if (!err_code) { err_code = r; err_msg = w->err; }
        } else {
          w->last_index = std::max(w->last_index, k);
          ++finished;
          for (int s2 : succ[k])
            if (--remaining[s2] == 0) ready.push(s2);
        }
        cv.notify_all();
      }
    });
  for (auto& t : pool) t.join();
  for (int wk = 0; wk < nw; ++wk) {
    const cudaError_t e = host_wait(h->workers[wk]);
    if (e != cudaSuccess && !err_code) { err_code = BSMPO_ECUDA; err_msg = cudaGetErrorString(e); }
  }
  for (cudaEvent_t e : done_ev) cudaEventDestroy(e);
  if (err_code) return fail(h, err_code, err_msg);
  // counters and the last update's diagnostics
  int best = -1;
  for (int k = 0; k < nw; ++k) {
    bsmpo_ctx* w = h->workers[k];
    h->launches += w->launches;
    h->updates += w->updates;
    h->jacobi_rounds += w->jacobi_rounds;
    for (int q = 0; q < 2; ++q) { h->route_count[q] += w->route_count[q]; w->route_count[q] = 0; }
    h->jac_ms += w->jac_ms;
    h->jac_flops += w->jac_flops;
    h->jac_launches += w->jac_launches;
    h->td_ms += w->td_ms; h->td_bytes += w->td_bytes; h->td_flops += w->td_flops; h->td_phases += w->td_phases;
    h->dev_grows += w->dev_grows; h->host_grows += w->host_grows;
    w->dev_grows = w->host_grows = 0;
    w->td_ms = w->td_bytes = w->td_flops = 0.0;
    w->td_phases = 0;
    for (int q = 0; q < 8; ++q) h->stage_ms[q] += w->stage_ms[q];
    w->launches = w->updates = w->jacobi_rounds = w->jac_launches = 0;
    w->jac_ms = w->jac_flops = 0.0;
    for (int q = 0; q < 8; ++q) w->stage_ms[q] = 0.0;
    if (w->last_index > best) { best = w->last_index; h->diag = w; }
  }
  return BSMPO_OK;
}

int env_all(bsmpo_ctx* h) {
  const int n = h->n, d = h->d, chi = h->chi, dd = d * d;
  cudaStream_t st = h->stream;
  int rc;
  if ((rc = grow(h, h->env_l, (size_t)(n + 1) * chi * sizeof(cplx)))) return rc;
  if ((rc = grow(h, h->env_r, (size_t)(n + 1) * chi * sizeof(cplx)))) return rc;
  std::vector<int> dims(n + 1);
  for (int b = 0; b <= n; ++b) {
    int s = 0;
    for (int q = 0; q < dd; ++q) s += h->cnt[(size_t)b * dd + q];
    dims[b] = s;
  }
  if ((rc = grow(h, h->dims, (size_t)(n + 1) * sizeof(int)))) return rc;
  if ((rc = grow_host(h, h->stage2, std::max<size_t>(h->stage2.bytes, (n + 1) * sizeof(int))))) return rc;
  std::memcpy(h->stage2.p, dims.data(), (n + 1) * sizeof(int));
  CK(h, cudaMemcpyAsync(h->dims.p, h->stage2.p, (n + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
  cplx* R = reinterpret_cast<cplx*>(h->env_r.p);
  cplx* Lv = reinterpret_cast<cplx*>(h->env_l.p);
  const int64_t chi2 = (int64_t)chi * chi;
  CKL(h, launch_env_init(d, chi, h->charge + (size_t)n * chi * 2, h->lam + (size_t)n * chi,
                         R + (size_t)n * chi, st));
  for (int b = n - 1; b >= 0; --b)
    CKL(h, launch_env_right_step(d, chi, h->gamma + (size_t)b * chi2, h->charge + (size_t)b * chi * 2,
                                 h->lam + (size_t)b * chi, R + (size_t)(b + 1) * chi,
                                 R + (size_t)b * chi, dims[b], dims[b + 1], st));
  CKL(h, launch_env_init(d, chi, h->charge, h->lam, Lv, st));
  for (int b = 0; b < n; ++b)
    CKL(h, launch_env_left_step(d, chi, h->gamma + (size_t)b * chi2,
                                h->charge + (size_t)(b + 1) * chi * 2, h->lam + (size_t)(b + 1) * chi,
                                Lv + (size_t)b * chi, Lv + (size_t)(b + 1) * chi, dims[b], dims[b + 1],
                                st));
  return BSMPO_OK;
}

}  // namespace

extern "C" {

const char* bsmpo_version(void) { return "bsmpo 0.1 (sm_100a, FP64 plain path)"; }

const char* bsmpo_last_error(const bsmpo_ctx* h) {
  if (h) return h->err.c_str();
  return g_last_error.c_str();
}

int bsmpo_bs_angle_grad(int d, int n_gates, const double* theta, const double* phi, const void* ubar,
                        double* grad, void* stream) {
  if (d < 1 || d > BSMPO_MAX_D || n_gates < 0 || (n_gates > 0 && (!theta || !phi || !ubar || !grad)))
    return fail(nullptr, BSMPO_EINVAL, "bad argument");
  if (n_gates == 0) return BSMPO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  // per gate: M = T^T and dM/dtheta, dM/dphi of T(theta, phi) = [[e^{i phi} c, -s], [e^{i phi} s, c]]
  std::vector<double> m4((size_t)n_gates * 8), dm4((size_t)n_gates * 16);
  for (int g = 0; g < n_gates; ++g) {
    const double c = std::cos(theta[g]), s = std::sin(theta[g]);
    const double er = std::cos(phi[g]), ei = std::sin(phi[g]);
    const double T[8] = {er * c, ei * c, -s, 0.0, er * s, ei * s, c, 0.0};
    const double Tt[8] = {-er * s, -ei * s, -c, 0.0, er * c, ei * c, -s, 0.0};        // dT/dtheta
    const double Tp[8] = {-ei * c, er * c, 0.0, 0.0, -ei * s, er * s, 0.0, 0.0};      // dT/dphi
    const M8 a = transpose_to_m8(T), b = transpose_to_m8(Tt), e = transpose_to_m8(Tp);
    for (int j = 0; j < 8; ++j) {
      m4[(size_t)g * 8 + j] = a.v[j];
      dm4[(size_t)g * 16 + j] = b.v[j];
      dm4[(size_t)g * 16 + 8 + j] = e.v[j];
    }
  }
  void* dev = nullptr;
  const size_t bytes = (m4.size() + dm4.size()) * sizeof(double);
  cudaError_t e = cudaMallocAsync(&dev, bytes, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dev, m4.data(), m4.size() * sizeof(double), cudaMemcpyHostToDevice, st);
  double* dm4_dev = static_cast<double*>(dev) + m4.size();
  if (e == cudaSuccess) e = cudaMemcpyAsync(dm4_dev, dm4.data(), dm4.size() * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_fock_angle_grad(d, n_gates, static_cast<double*>(dev), dm4_dev, ubar, grad, st);
  if (dev) cudaFreeAsync(dev, st);
  const cudaError_t e2 = cudaStreamSynchronize(st);   // the host arrays above are read by the copies
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) return fail(nullptr, BSMPO_ECUDA, cudaGetErrorString(e));
  return BSMPO_OK;
}

int bsmpo_unitary(int d, const double* M, void* u_out, void* stream) {
  if (d < 1 || d > BSMPO_MAX_D || !M || !u_out) return fail(nullptr, BSMPO_EINVAL, "bad argument");
  M8 m;
  for (int i = 0; i < 8; ++i) m.v[i] = M[i];
  cudaError_t e = launch_fock_tensor_single(d, m, u_out, nullptr, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(nullptr, BSMPO_ECUDA, cudaGetErrorString(e));
  return BSMPO_OK;
}

int bsmpo_unitary_tr(int d, double t_re, double t_im, double r_re, double r_im, double* u_re,
                     double* u_im, void* stream) {
  if (d < 1 || d > BSMPO_MAX_D || !u_re || !u_im) return fail(nullptr, BSMPO_EINVAL, "bad argument");
  // M = [[t, -conj r], [r, conj t]]
  M8 m;
  m.v[0] = t_re; m.v[1] = t_im;
  m.v[2] = -r_re; m.v[3] = r_im;
  m.v[4] = r_re; m.v[5] = r_im;
  m.v[6] = t_re; m.v[7] = -t_im;
  cudaError_t e = launch_fock_tensor_single(d, m, u_re, u_im, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(nullptr, BSMPO_ECUDA, cudaGetErrorString(e));
  return BSMPO_OK;
}

int bsmpo_contract_sector(int d, int cc0, int cc1, const void* u, const void* glc, const void* gcr,
                          const int* cl, const int* cc, const int* cr, int len_l, int len_c,
                          int len_r, void* c, void* stream) {
  if (d < 1 || d > BSMPO_MAX_D || len_l < 0 || len_c < 0 || len_r < 0 || !u || !c)
    return fail(nullptr, BSMPO_EINVAL, "bad argument");
  if (cc0 < 0 || cc1 < 0 || cc0 >= d || cc1 >= d) return fail(nullptr, BSMPO_EINVAL, "bad centre charge");
  cudaError_t e = launch_contract_sector(d, cc0, cc1, u, glc, gcr, cl, cc, cr, len_l, len_c, len_r, c,
                                         (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(nullptr, BSMPO_ECUDA, cudaGetErrorString(e));
  return BSMPO_OK;
}

int bsmpo_contract_mps(int d, int tau, const void* u, const void* glc, const void* gcr, const double* ll,
                       const double* lc, const double* lr, const int* cl, const int* cc, const int* cr,
                       int len_l, int len_c, int len_r, void* t, void* stream) {
  if (d < 1 || d > BSMPO_MAX_D || len_l < 0 || len_c < 0 || len_r < 0 || !u || !t)
    return fail(nullptr, BSMPO_EINVAL, "bad argument");
  if (tau < 0 || tau >= d) return fail(nullptr, BSMPO_EINVAL, "bad centre charge");
  if ((len_l > 0 && (!glc || !ll || !cl)) || (len_r > 0 && (!gcr || !lr || !cr)) || (len_c > 0 && (!lc || !cc)))
    return fail(nullptr, BSMPO_EINVAL, "null input");
  cudaError_t e = launch_contract_mps(d, tau, u, glc, gcr, ll, lc, lr, cl, cc, cr, len_l, len_c, len_r, t,
                                      (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(nullptr, BSMPO_ECUDA, cudaGetErrorString(e));
  return BSMPO_OK;
}

int bsmpo_zgemm_tf32x3(int M, int N, int K, const void* a, int lda, int opA, const void* b, int ldb,
                       void* c, int ldc, void* stream) {
  if (M < 0 || N < 0 || K < 1 || !a || !b || !c || (opA != 0 && opA != 1) || ldb < N || ldc < N ||
      lda < (opA ? M : K))
    return fail(nullptr, BSMPO_EINVAL, "bsmpo_zgemm_tf32x3: bad argument");
  if (M == 0 || N == 0) return BSMPO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t mb = tc_map_bytes();
  const size_t o_g = align_up(2 * mb, 256), o_err = o_g + 256, total = o_err + 256;
  std::vector<unsigned char> host(total, 0);
  if (tc_encode_map(host.data(), a, opA ? K : M, opA ? M : K, lda, opA ? 1 : 0) != cudaSuccess ||
      tc_encode_map(host.data() + mb, b, K, N, ldb, 2) != cudaSuccess)
    return fail(nullptr, BSMPO_ECUDA, "bsmpo_zgemm_tf32x3: tensor map encoding failed");
  TcGroup g;
  std::memset(&g, 0, sizeof(g));
  g.M = M; g.N = N; g.K = K; g.opA = opA; g.mapA = 0; g.mapB = 1;
  g.ldc = ldc;
  g.tiles_n = ceil_div(N, tc_tile_n());
  g.tile_start = 0;
  g.cs_off = -1;
  std::memcpy(host.data() + o_g, &g, sizeof(g));
  void* dev = nullptr;
  cudaError_t e = cudaMallocAsync(&dev, total, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dev, host.data(), total, cudaMemcpyHostToDevice, st);
  int herr = 0;
  char* dc = static_cast<char*>(dev);
  if (e == cudaSuccess)
    e = launch_tc_zgemm(reinterpret_cast<const TcGroup*>(dc + o_g), 1, ceil_div(M, tc_tile_m()) * g.tiles_n, dc, c,
                        nullptr, reinterpret_cast<int*>(dc + o_err), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, dc + o_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (dev) cudaFreeAsync(dev, st);
  if (e != cudaSuccess) return fail(nullptr, BSMPO_ECUDA, std::string("bsmpo_zgemm_tf32x3: ") + cudaGetErrorString(e));
  if (herr) return fail(nullptr, BSMPO_ECUDA, "bsmpo_zgemm_tf32x3: a pipeline wait expired");
  return BSMPO_OK;
}

int bsmpo_create(int n, int d, int chi, int flags, bsmpo_ctx** out) {
  if (!out) return fail(nullptr, BSMPO_EINVAL, "null output handle");
  *out = nullptr;
  if (n < 2 || d < 1 || d > BSMPO_MAX_D || chi < 1 || chi > 8192 || flags != 0)
    return fail(nullptr, BSMPO_EINVAL, "bad create arguments");
  bsmpo_ctx* h = new bsmpo_ctx();
  h->n = n; h->d = d; h->chi = chi;
  cudaGetDevice(&h->device);
  const size_t gbytes = (size_t)n * chi * chi * sizeof(cplx);
  if (cudaMalloc(&h->gamma, gbytes) != cudaSuccess ||
      cudaMalloc(&h->lam, (size_t)(n + 1) * chi * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->charge, (size_t)(n + 1) * chi * 2 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(h->gamma); cudaFree(h->lam); cudaFree(h->charge);
    delete h;
    return fail(nullptr, BSMPO_ENOMEM, "state allocation failed");
  }
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = h->device;
  if (cudaMemPoolCreate(&h->pool, &props) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(h->gamma); cudaFree(h->lam); cudaFree(h->charge);
    delete h;
    return fail(nullptr, BSMPO_ECUDA, "memory pool creation failed");
  }
  // keep released workspace memory in the pool (no release at synchronisation points)
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(h->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  // a block freed on one worker's stream is not handed to another worker's allocation
  // with a hidden dependency on the first stream's pending work (which would serialise
  // concurrent updates whenever a workspace grows); such blocks are reused once their
  // free is known to be complete
  int no = 0;
  cudaMemPoolSetAttribute(h->pool, cudaMemPoolReuseAllowInternalDependencies, &no);
  cudaMemPoolSetAttribute(h->pool, cudaMemPoolReuseAllowOpportunistic, &no);
  h->cnt.assign((size_t)(n + 1) * d * d, 0);
  const char* prof = std::getenv("BSMPO_PROFILE");
  h->profile = prof && prof[0] == '1';
  const char* jr = std::getenv("BSMPO_JACOBI_ROWS");
  if (jr && std::atoi(jr) >= 16) h->jac_rows = std::atoi(jr);
  const char* tm = std::getenv("BSMPO_TC_MASK");
  if (tm && tm[0] >= '0' && tm[0] <= '3') h->tc_mask = tm[0] - '0';
  const char* gp = std::getenv("BSMPO_GRAM_POLICY");
  if (gp && gp[0] >= '0' && gp[0] <= '2') h->gram_policy = gp[0] - '0';
  const char* tf = std::getenv("BSMPO_TD_FORK");
  if (tf && tf[0] >= '0' && tf[0] <= '3') h->td_fork = tf[0] - '0';
  const char* nwk = std::getenv("BSMPO_WORKERS");
  if (nwk && std::atoi(nwk) >= 1 && std::atoi(nwk) <= 64) h->n_workers = std::atoi(nwk);
  *out = h;
  return BSMPO_OK;
}

int bsmpo_destroy(bsmpo_ctx* h) {
  if (!h) return BSMPO_OK;
  for (bsmpo_ctx* w : h->workers) destroy_worker(w);
  h->workers.clear();
  cudaStreamSynchronize(h->stream);
  free_workspaces(h);
  if (h->pool) cudaMemPoolDestroy(h->pool);
  cudaFree(h->gamma); cudaFree(h->lam); cudaFree(h->charge);
  delete h;
  return BSMPO_OK;
}

int bsmpo_set_workers(bsmpo_ctx* h, int n_workers) {
  if (!h) return fail(nullptr, BSMPO_EINVAL, "null handle");
  if (n_workers < 1 || n_workers > 64) return fail(h, BSMPO_EINVAL, "workers must be 1..64");
  h->n_workers = n_workers;
  return BSMPO_OK;
}

int bsmpo_set_stream(bsmpo_ctx* h, void* stream) {
  if (!h) return fail(nullptr, BSMPO_EINVAL, "null handle");
  h->stream = (cudaStream_t)stream;
  return BSMPO_OK;
}

int bsmpo_set_precision(bsmpo_ctx* h, int precision) {
  if (!h) return fail(nullptr, BSMPO_EINVAL, "null handle");
  if (precision != BSMPO_PRECISION_FP64 && precision != BSMPO_PRECISION_FP64_GRAM &&
      precision != BSMPO_PRECISION_TF32X3)
    return fail(h, BSMPO_EINVAL, "unknown precision mode " + std::to_string(precision));
  h->precision = precision;
  return BSMPO_OK;
}

int bsmpo_set_cutoff(bsmpo_ctx* h, double cutoff) {
  if (!h) return fail(nullptr, BSMPO_EINVAL, "null handle");
  if (!(cutoff >= 0.0) || cutoff >= 1.0) return fail(h, BSMPO_EINVAL, "cutoff must be in [0, 1)");
  h->cutoff = cutoff;
  return BSMPO_OK;
}

}  // extern "C"

// Validates the charges and Lambda of a state (host copies: hc [(n+1) chi][2], hl
// [(n+1) chi] with the inner bonds filled) and rebuilds the host mirror of the block
// sizes; fills the edge Lambda of hl (1 on the occupied slots of bonds 0 and n).
// Checks one bond (host copies: hc [chi][2], hl [chi]; hl is not read on the edge bonds 0
// and n) and writes its block sizes to row [d*d]: sorted, occupied slots first, charges in
// range, Lambda > 0 on the occupied slots and 0 on the empty ones.
int validate_bond(bsmpo_ctx* h, int b, const int* hc, const double* hl, int* row) {
  const int n = h->n, d = h->d, chi = h->chi;
  std::fill(row, row + d * d, 0);
  bool empty_seen = false;
  int p0 = -1, p1 = -1;
  for (int i = 0; i < chi; ++i) {
    const int c0 = hc[(size_t)i * 2], c1 = hc[(size_t)i * 2 + 1];
    const bool occ = c0 < d;
    if (!occ) {
      if (c0 != d || c1 != d)
        return fail(h, BSMPO_EINVAL, "bond " + std::to_string(b) + ": empty slots must carry (d, d)");
      empty_seen = true;
      if (b > 0 && b < n && hl[i] != 0.0)
        return fail(h, BSMPO_EINVAL, "bond " + std::to_string(b) + ": Lambda on an empty slot");
      continue;
    }
    if (empty_seen) return fail(h, BSMPO_EINVAL, "bond " + std::to_string(b) + ": occupied slot after an empty one");
    if (c0 < 0 || c1 < 0 || c1 >= d) return fail(h, BSMPO_EINVAL, "bond " + std::to_string(b) + ": charge out of range");
    if (c0 < p0 || (c0 == p0 && c1 < p1))
      return fail(h, BSMPO_EINVAL, "bond " + std::to_string(b) + ": charges not sorted");
    if (b > 0 && b < n && !(hl[i] > 0.0))
      return fail(h, BSMPO_EINVAL, "bond " + std::to_string(b) + ": occupied slot with Lambda <= 0");
    p0 = c0; p1 = c1;
    row[c0 * d + c1]++;
  }
  return BSMPO_OK;
}

int validate_state(bsmpo_ctx* h, const int* hc, double* hl) {
  const int n = h->n, d = h->d, chi = h->chi;
  for (int b = 0; b <= n; ++b) {
    const int rc = validate_bond(h, b, hc + (size_t)b * chi * 2, hl + (size_t)b * chi, &h->cnt[(size_t)b * d * d]);
    if (rc) return rc;
  }
  for (int b : {0, n})
    for (int i = 0; i < chi; ++i) hl[(size_t)b * chi + i] = hc[((size_t)b * chi + i) * 2] < d ? 1.0 : 0.0;
  return BSMPO_OK;
}

extern "C" {

int bsmpo_load_state(bsmpo_ctx* h, const void* gamma, const double* lambda, const int* charge) {
  if (!h || !gamma || !lambda || !charge) return fail(h, BSMPO_EINVAL, "null argument");
  const int n = h->n, chi = h->chi;
  cudaStream_t st = h->stream;
  h->loaded = false;
  CK(h, cudaMemcpyAsync(h->gamma, gamma, (size_t)n * chi * chi * sizeof(cplx),
                        cudaMemcpyDeviceToDevice, st));
  CK(h, cudaMemcpyAsync(h->lam + chi, lambda, (size_t)(n - 1) * chi * sizeof(double),
                        cudaMemcpyDeviceToDevice, st));
  CK(h, cudaMemcpyAsync(h->charge, charge, (size_t)(n + 1) * chi * 2 * sizeof(int),
                        cudaMemcpyDeviceToDevice, st));
  std::vector<int> hc((size_t)(n + 1) * chi * 2);
  std::vector<double> hl((size_t)(n + 1) * chi, 0.0);
  CK(h, cudaMemcpyAsync(hc.data(), charge, hc.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(h, cudaMemcpyAsync(hl.data() + chi, lambda, (size_t)(n - 1) * chi * sizeof(double),
                        cudaMemcpyDeviceToHost, st));
  CK(h, cudaStreamSynchronize(st));
  int rc = validate_state(h, hc.data(), hl.data());
  if (rc) return rc;
  CK(h, cudaMemcpyAsync(h->lam, hl.data(), chi * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(h, cudaMemcpyAsync(h->lam + (size_t)n * chi, hl.data() + (size_t)n * chi, chi * sizeof(double),
                        cudaMemcpyHostToDevice, st));
  CK(h, cudaStreamSynchronize(st));
  h->loaded = true;
  return BSMPO_OK;
}

int bsmpo_init_product(bsmpo_ctx* h, const double* rho, int total_photons) {
  if (!h || !rho) return fail(h, BSMPO_EINVAL, "null argument");
  const int n = h->n, d = h->d, chi = h->chi, dd = d * d;
  if (total_photons >= d) return fail(h, BSMPO_EINVAL, "total_photons must be < d (or negative: none)");
  // bond charges, right to left: (ket, bra) photons right of the bond, at most d - 1
  std::vector<std::vector<int>> bonds(n + 1);   // flat charge index c0 * d + c1, sorted
  bonds[n] = {0};
  std::vector<char> mark(dd);
  for (int b = n - 1; b >= 0; --b) {
    std::fill(mark.begin(), mark.end(), 0);
    if (b == 0) {
      // every diagonal total, reachable or not (or only the post-selected one)
      for (int c = 0; c < d; ++c)
        if (total_photons < 0 || c == total_photons) mark[c * d + c] = 1;
    } else {
      const double* r = rho + (size_t)b * dd * 2;
      for (int q : bonds[b + 1]) {
        const int c0 = q / d, c1 = q % d;
        for (int o0 = 0; o0 + c0 < d; ++o0)
          for (int o1 = 0; o1 + c1 < d; ++o1)
            if (r[(o0 * d + o1) * 2] != 0.0 || r[(o0 * d + o1) * 2 + 1] != 0.0)
              mark[(c0 + o0) * d + c1 + o1] = 1;
      }
    }
    for (int q = 0; q < dd; ++q)
      if (mark[q]) bonds[b].push_back(q);
    if ((int)bonds[b].size() > chi)
      return fail(h, BSMPO_ECAPACITY, "chi = " + std::to_string(chi) + " is smaller than the product-state "
                                      "bond dimension " + std::to_string(bonds[b].size()));
  }
  std::vector<int> hc((size_t)(n + 1) * chi * 2, d);
  std::vector<double> hl((size_t)(n + 1) * chi, 0.0);
  std::fill(h->cnt.begin(), h->cnt.end(), 0);
  for (int b = 0; b <= n; ++b)
    for (size_t i = 0; i < bonds[b].size(); ++i) {
      const int q = bonds[b][i];
      hc[((size_t)b * chi + i) * 2] = q / d;
      hc[((size_t)b * chi + i) * 2 + 1] = q % d;
      hl[(size_t)b * chi + i] = 1.0;
      h->cnt[(size_t)b * dd + q]++;
    }
  int rc;
  if ((rc = grow(h, h->m4, (size_t)n * dd * sizeof(cplx)))) return rc;
  cudaStream_t st = h->stream;
  CK(h, cudaMemcpyAsync(h->charge, hc.data(), hc.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  CK(h, cudaMemcpyAsync(h->lam, hl.data(), hl.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(h, cudaMemcpyAsync(h->m4.p, rho, (size_t)n * dd * sizeof(cplx), cudaMemcpyHostToDevice, st));
  CKL(h, launch_product_fill(n, d, chi, h->charge, h->m4.p, h->gamma, st));
  CK(h, cudaStreamSynchronize(st));
  h->loaded = true;
  h->diag = nullptr;
  return BSMPO_OK;
}

int bsmpo_canonicalize(bsmpo_ctx* h) {
  int rc = check_mode(h, 0);
  if (rc) return rc;
  // right-to-left sweep of identity-gate updates (the reference's Canonicalize,
  // src/MPO.py:137-155, whose phase-only gate acts as the identity on product inputs)
  const double I[8] = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0};
  for (int mode = h->n - 2; mode >= 0; --mode)
    if ((rc = bsmpo_bs_update(h, mode, I))) return rc;
  return BSMPO_OK;
}

int bsmpo_store_state(bsmpo_ctx* h, void* gamma, double* lambda, int* charge) {
  if (!h || !h->loaded) return fail(h, BSMPO_EINVAL, "no state loaded");
  const int n = h->n, chi = h->chi;
  cudaStream_t st = h->stream;
  if (gamma) CK(h, cudaMemcpyAsync(gamma, h->gamma, (size_t)n * chi * chi * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
  if (lambda) CK(h, cudaMemcpyAsync(lambda, h->lam + chi, (size_t)(n - 1) * chi * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (charge) CK(h, cudaMemcpyAsync(charge, h->charge, (size_t)(n + 1) * chi * 2 * sizeof(int), cudaMemcpyDeviceToDevice, st));
  CK(h, cudaStreamSynchronize(st));
  return BSMPO_OK;
}

int bsmpo_get_site(bsmpo_ctx* h, int site, void* gamma) {
  if (!h || !h->loaded) return fail(h, BSMPO_EINVAL, "no state loaded");
  if (!gamma || site < 0 || site >= h->n) return fail(h, BSMPO_EINVAL, "bad argument");
  const size_t elems = (size_t)h->chi * h->chi;
  CK(h, cudaMemcpyAsync(gamma, h->gamma + (size_t)site * elems, elems * sizeof(cplx), cudaMemcpyDeviceToDevice,
                        h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return BSMPO_OK;
}

int bsmpo_put_site(bsmpo_ctx* h, int site, const void* gamma) {
  if (!h || !h->loaded) return fail(h, BSMPO_EINVAL, "no state loaded");
  if (!gamma || site < 0 || site >= h->n) return fail(h, BSMPO_EINVAL, "bad argument");
  const size_t elems = (size_t)h->chi * h->chi;
  CK(h, cudaMemcpyAsync(h->gamma + (size_t)site * elems, gamma, elems * sizeof(cplx), cudaMemcpyDeviceToDevice,
                        h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return BSMPO_OK;
}

int bsmpo_get_bond(bsmpo_ctx* h, int bond, double* lambda, int* charge) {
  if (!h || !h->loaded) return fail(h, BSMPO_EINVAL, "no state loaded");
  if (!lambda || !charge || bond < 1 || bond >= h->n) return fail(h, BSMPO_EINVAL, "bad argument");
  const int chi = h->chi;
  CK(h, cudaMemcpyAsync(lambda, h->lam + (size_t)bond * chi, chi * sizeof(double), cudaMemcpyDeviceToDevice,
                        h->stream));
  CK(h, cudaMemcpyAsync(charge, h->charge + (size_t)bond * chi * 2, chi * 2 * sizeof(int),
                        cudaMemcpyDeviceToDevice, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return BSMPO_OK;
}

int bsmpo_put_bond(bsmpo_ctx* h, int bond, const double* lambda, const int* charge) {
  if (!h || !h->loaded) return fail(h, BSMPO_EINVAL, "no state loaded");
  if (!lambda || !charge || bond < 1 || bond >= h->n) return fail(h, BSMPO_EINVAL, "bad argument");
  const int chi = h->chi, dd = h->d * h->d;
  // checked before it is written: a rejected bond leaves the state as it was
  std::vector<double> hl(chi);
  std::vector<int> hc((size_t)chi * 2), row(dd);
  CK(h, cudaMemcpyAsync(hl.data(), lambda, chi * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaMemcpyAsync(hc.data(), charge, chi * 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  const int rc = validate_bond(h, bond, hc.data(), hl.data(), row.data());
  if (rc) return rc;
  CK(h, cudaMemcpyAsync(h->lam + (size_t)bond * chi, lambda, chi * sizeof(double), cudaMemcpyDeviceToDevice,
                        h->stream));
  CK(h, cudaMemcpyAsync(h->charge + (size_t)bond * chi * 2, charge, chi * 2 * sizeof(int),
                        cudaMemcpyDeviceToDevice, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  std::copy(row.begin(), row.end(), h->cnt.begin() + (size_t)bond * dd);
  return BSMPO_OK;
}

int bsmpo_bs_update_tensor(bsmpo_ctx* h, int mode, const void* u) {
  if (!u) return fail(h, BSMPO_EINVAL, "null tensor");
  if (h) h->diag = nullptr;
  return bs_update_impl(h, mode, reinterpret_cast<const cplx*>(u));
}

int bsmpo_bs_update(bsmpo_ctx* h, int mode, const double* S) {
  int rc = check_mode(h, mode);
  if (rc) return rc;
  if (!S) return fail(h, BSMPO_EINVAL, "null matrix");
  const int d = h->d;
  if ((rc = grow(h, h->u3, (size_t)d * d * d * sizeof(cplx)))) return rc;
  CKL(h, launch_fock_tensor_single(d, transpose_to_m8(S), h->u3.p, nullptr, h->stream));
  h->diag = nullptr;
  return bs_update_impl(h, mode, reinterpret_cast<const cplx*>(h->u3.p));
}

}  // extern "C"

// A mesh of beam splitters (T(theta, phi) each) on the loaded state; with hs, over the
// host-resident state whose sites are arriving (see HostStream).
int run_mesh_impl(bsmpo_ctx* h, int n_bs, const int* modes, const double* theta, const double* phi,
                  HostStream* hs) {
  h->mesh_tw.assign(n_bs, 0.0);
  if (n_bs == 0) return BSMPO_OK;
  const int d = h->d, d3 = d * d * d;
  int rc;
  if ((rc = grow(h, h->u3, (size_t)n_bs * d3 * sizeof(cplx)))) return rc;
  if ((rc = grow(h, h->m4, (size_t)n_bs * 8 * sizeof(double)))) return rc;
  std::vector<double> m4((size_t)n_bs * 8);
  for (int i = 0; i < n_bs; ++i) {
    // T(theta, phi) = [[e^{i phi} c, -s], [e^{i phi} s, c]]; tensor of M = T^T
    const double c = std::cos(theta[i]), s = std::sin(theta[i]);
    const double er = std::cos(phi[i]), ei = std::sin(phi[i]);
    double S[8] = {er * c, ei * c, -s, 0.0, er * s, ei * s, c, 0.0};
    M8 m = transpose_to_m8(S);
    for (int j = 0; j < 8; ++j) m4[(size_t)i * 8 + j] = m.v[j];
  }
  if ((rc = grow_host(h, h->stage2, std::max(h->stage2.bytes, m4.size() * sizeof(double))))) return rc;
  std::memcpy(h->stage2.p, m4.data(), m4.size() * sizeof(double));
  CK(h, cudaMemcpyAsync(h->m4.p, h->stage2.p, m4.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CKL(h, launch_fock_tensor(d, n_bs, reinterpret_cast<const double*>(h->m4.p), h->u3.p, h->stream));
  // the stage is reused by the updates, and worker streams read u3: drain the stream
  CK(h, cudaStreamSynchronize(h->stream));
  const int nw = std::min(h->n_workers, n_bs);
  if (nw > 1 || hs)
    return run_mesh_concurrent(h, n_bs, modes, reinterpret_cast<const cplx*>(h->u3.p), std::max(nw, 1), hs);
  h->diag = nullptr;
  for (int i = 0; i < n_bs; ++i) {
    rc = bs_update_impl(h, modes[i], reinterpret_cast<const cplx*>(h->u3.p) + (size_t)i * d3);
    if (rc) return rc;
    h->mesh_tw[i] = h->last_trunc;
  }
  return BSMPO_OK;
}

int check_mesh_args(bsmpo_ctx* h, int n_bs, const int* modes, const double* theta, const double* phi) {
  if (!h || n_bs < 0 || (n_bs > 0 && (!modes || !theta || !phi))) return fail(h, BSMPO_EINVAL, "bad argument");
  for (int i = 0; i < n_bs; ++i)
    if (modes[i] < 0 || modes[i] > h->n - 2) return fail(h, BSMPO_EINVAL, "mode out of range");
  return BSMPO_OK;
}

extern "C" {

int bsmpo_run_mesh(bsmpo_ctx* h, int n_bs, const int* modes, const double* theta, const double* phi) {
  int rc = check_mesh_args(h, n_bs, modes, theta, phi);
  if (rc) return rc;
  if (!h->loaded) return fail(h, BSMPO_EINVAL, "no state loaded");
  return run_mesh_impl(h, n_bs, modes, theta, phi, nullptr);
}

int bsmpo_run_mesh_host(bsmpo_ctx* h, int n_bs, const int* modes, const double* theta, const double* phi,
                        const void* gamma_in, const double* lambda_in, const int* charge_in, void* gamma_out,
                        double* lambda_out, int* charge_out) {
  int rc = check_mesh_args(h, n_bs, modes, theta, phi);
  if (rc) return rc;
  if (!gamma_in || !lambda_in || !charge_in || !gamma_out || !lambda_out || !charge_out)
    return fail(h, BSMPO_EINVAL, "null argument");
  const int n = h->n, chi = h->chi;
  const size_t site_bytes = (size_t)chi * chi * sizeof(cplx);
  cudaStream_t st = h->stream;
  h->loaded = false;
  // the bonds: validated on the host, copied in before any site
  std::vector<double> hl((size_t)(n + 1) * chi, 0.0);
  std::memcpy(hl.data() + chi, lambda_in, (size_t)(n - 1) * chi * sizeof(double));
  if ((rc = validate_state(h, charge_in, hl.data()))) return rc;
  CK(h, cudaMemcpyAsync(h->lam, hl.data(), hl.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(h, cudaMemcpyAsync(h->charge, charge_in, (size_t)(n + 1) * chi * 2 * sizeof(int), cudaMemcpyHostToDevice, st));
  CK(h, cudaStreamSynchronize(st));
  h->loaded = true;
  HostStream hs;
  hs.first.assign(n, -1);
  hs.last.assign(n, -1);
  hs.gamma_in = static_cast<const char*>(gamma_in);
  hs.gamma_out = static_cast<char*>(gamma_out);
  hs.site_bytes = site_bytes;
  for (int k = n_bs - 1; k >= 0; --k) hs.first[modes[k]] = hs.first[modes[k] + 1] = k;
  for (int k = 0; k < n_bs; ++k) hs.last[modes[k]] = hs.last[modes[k] + 1] = k;
  // the sites no update touches: in and straight out on the handle's stream
  for (int s = 0; s < n; ++s)
    if (hs.first[s] < 0) {
      CK(h, cudaMemcpyAsync(reinterpret_cast<char*>(h->gamma) + (size_t)s * site_bytes,
                            hs.gamma_in + (size_t)s * site_bytes, site_bytes, cudaMemcpyHostToDevice, st));
      CK(h, cudaMemcpyAsync(hs.gamma_out + (size_t)s * site_bytes,
                            reinterpret_cast<const char*>(h->gamma) + (size_t)s * site_bytes, site_bytes,
                            cudaMemcpyDeviceToHost, st));
    }
  rc = run_mesh_impl(h, n_bs, modes, theta, phi, &hs);
  if (rc) {
    cudaStreamSynchronize(st);
    h->loaded = false;   // the device state is incomplete
    return rc;
  }
  // the bonds, once every update has finished (the workers are drained)
  CK(h, cudaMemcpyAsync(lambda_out, h->lam + chi, (size_t)(n - 1) * chi * sizeof(double), cudaMemcpyDeviceToHost,
                        st));
  CK(h, cudaMemcpyAsync(charge_out, h->charge, (size_t)(n + 1) * chi * 2 * sizeof(int), cudaMemcpyDeviceToHost,
                        st));
  CK(h, cudaStreamSynchronize(st));
  return BSMPO_OK;
}

int bsmpo_mesh_truncation(const bsmpo_ctx* h, double* weights, int cap) {
  if (!h || (!weights && cap > 0)) return fail(nullptr, BSMPO_EINVAL, "bad argument");
  const int nb = (int)h->mesh_tw.size();
  if (!weights) return nb;   // size query
  if (cap < nb) return fail(const_cast<bsmpo_ctx*>(h), BSMPO_ECAPACITY, "weights buffer too small");
  std::copy(h->mesh_tw.begin(), h->mesh_tw.end(), weights);
  return nb;
}

int bsmpo_apply_phases(bsmpo_ctx* h, const double* phases) {
  if (!h || !phases) return fail(h, BSMPO_EINVAL, "bad argument");
  if (!h->loaded) return fail(h, BSMPO_EINVAL, "no state loaded");
  const int chi = h->chi;
  for (int m = 0; m < h->n; ++m)
    CKL(h, launch_phase(h->d, chi, phases[m], h->charge + (size_t)m * chi * 2,
                        h->charge + (size_t)(m + 1) * chi * 2, h->gamma + (size_t)m * chi * chi,
                        h->stream));
  return BSMPO_OK;
}

int bsmpo_observables(bsmpo_ctx* h, double* trace, double* marginals) {
  if (!h || !trace) return fail(h, BSMPO_EINVAL, "bad argument");
  if (!h->loaded) return fail(h, BSMPO_EINVAL, "no state loaded");
  const int n = h->n, d = h->d, chi = h->chi;
  int rc;
  if ((rc = env_all(h))) return rc;
  const int chunk_rows = 32;
  const int nchunk = ceil_div(chi, chunk_rows);
  if ((rc = grow(h, h->part, (size_t)n * nchunk * d * sizeof(cplx)))) return rc;
  if ((rc = grow(h, h->outv, ((size_t)n * d + 1) * sizeof(cplx)))) return rc;
  cplx* out = reinterpret_cast<cplx*>(h->outv.p);
  CKL(h, launch_sum_vector(h->env_r.p, chi, out + (size_t)n * d, h->stream));
  if (marginals)
    CKL(h, launch_marginals(n, d, chi, h->gamma, h->charge, h->env_l.p, h->env_r.p,
                            reinterpret_cast<const int*>(h->dims.p), h->part.p, chunk_rows, out,
                            h->stream));
  if ((rc = grow_host(h, h->hres, std::max(h->hres.bytes, ((size_t)n * d + 1) * sizeof(cplx) + 8192)))) return rc;
  cplx* ho = reinterpret_cast<cplx*>(static_cast<char*>(h->hres.p) + 4096);
  CK(h, cudaMemcpyAsync(ho, out, ((size_t)n * d + 1) * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  trace[0] = ho[(size_t)n * d].x;
  trace[1] = ho[(size_t)n * d].y;
  if (marginals)
    for (int i = 0; i < n * d; ++i) { marginals[2 * i] = ho[i].x; marginals[2 * i + 1] = ho[i].y; }
  return BSMPO_OK;
}

int bsmpo_last_update_info(const bsmpo_ctx* hc, int* n_sectors, int* sector_cc, int* shape,
                           int* sigma_len, double* sigma, int sigma_cap, int* kept,
                           double* trunc_weight) {
  if (!hc) return fail(nullptr, BSMPO_EINVAL, "null handle");
  // after a concurrent mesh the last update's data live in the worker that ran it
  bsmpo_ctx* h = const_cast<bsmpo_ctx*>(hc->diag ? hc->diag : hc);
  const int ns = h->last_ns;
  if (n_sectors) *n_sectors = ns;
  if (sector_cc) std::copy(h->last_cc.begin(), h->last_cc.end(), sector_cc);
  if (shape) std::copy(h->last_shape.begin(), h->last_shape.end(), shape);
  if (sigma_len) std::copy(h->last_k.begin(), h->last_k.end(), sigma_len);
  if (kept) std::copy(h->last_kept.begin(), h->last_kept.end(), kept);
  if (trunc_weight) *trunc_weight = h->last_trunc;
  if (sigma) {
    int64_t tot = 0;
    for (int k : h->last_k) tot += k;
    if (tot > sigma_cap) return fail(const_cast<bsmpo_ctx*>(hc), BSMPO_ECAPACITY, "sigma buffer too small");
    CK(h, cudaMemcpyAsync(sigma, h->sig.p, tot * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
  }
  return BSMPO_OK;
}

int bsmpo_last_update_work(const bsmpo_ctx* hc, double* gemm_flops, double* svd_flops,
                           double* min_bytes) {
  if (!hc) return fail(nullptr, BSMPO_EINVAL, "null handle");
  const bsmpo_ctx* h = hc->diag ? hc->diag : hc;
  if (gemm_flops) *gemm_flops = h->last_gemm;
  if (svd_flops) *svd_flops = h->last_svd;
  if (min_bytes) *min_bytes = h->last_bytes;
  return BSMPO_OK;
}

int bsmpo_bond_dims(const bsmpo_ctx* h, int* dims) {
  if (!h || !dims) return fail(nullptr, BSMPO_EINVAL, "bad argument");
  const int dd = h->d * h->d;
  for (int b = 0; b <= h->n; ++b) {
    int s = 0;
    for (int q = 0; q < dd; ++q) s += h->cnt[(size_t)b * dd + q];
    dims[b] = s;
  }
  return BSMPO_OK;
}

int64_t bsmpo_kernel_launches(const bsmpo_ctx* h) { return h ? h->launches : 0; }

int bsmpo_workspace_stats(const bsmpo_ctx* h, int64_t* out) {
  if (!h || !out) return fail(const_cast<bsmpo_ctx*>(h), BSMPO_EINVAL, "null argument");
  out[0] = h->dev_grows;
  out[1] = h->host_grows;
  // bytes held by the handle and its workers
  int64_t dev = 0, host = 0;
  auto add = [&](const bsmpo_ctx* c) {
    const DevBuf* bufs[] = {&c->theta, &c->cbuf, &c->abuf, &c->wbuf, &c->vbuf, &c->sig, &c->keys,
                            &c->perm, &c->tab, &c->tab2, &c->rot, &c->kept, &c->u3, &c->m4,
                            &c->env_l, &c->env_r, &c->part, &c->outv, &c->dims, &c->nf2, &c->qbuf,
                            &c->qflag, &c->pbuf, &c->pcnt, &c->gbuf, &c->eigd, &c->taub, &c->invsig,
                            &c->escr, &c->swp, &c->zbuf, &c->ybuf, &c->tab3, &c->tcerr, &c->jwork};
    for (const DevBuf* b : bufs) dev += (int64_t)b->bytes;
    const HostStage* hs[] = {&c->stage, &c->stage2, &c->stage3, &c->hres};
    for (const HostStage* b : hs) host += (int64_t)b->bytes;
  };
  add(h);
  for (const bsmpo_ctx* w : h->workers) add(w);
  out[2] = dev;
  out[3] = host;
  return BSMPO_OK;
}

int bsmpo_svd_routes(const bsmpo_ctx* h, int64_t* counts) {
  if (!h || !counts) return fail(nullptr, BSMPO_EINVAL, "bad argument");
  counts[0] = h->route_count[0];
  counts[1] = h->route_count[1];
  return BSMPO_OK;
}

int bsmpo_set_timing(bsmpo_ctx* h, int on) {
  if (!h) return fail(nullptr, BSMPO_EINVAL, "null handle");
  if (on && !h->ev0) {
    CK(h, cudaEventCreate(&h->ev0));
    CK(h, cudaEventCreate(&h->ev1));
  }
  h->timing = on != 0;
  h->jac_ms = h->jac_flops = 0.0;
  h->jac_launches = 0;
  h->td_ms = h->td_bytes = h->td_flops = 0.0;
  h->td_phases = 0;
  return BSMPO_OK;
}

int bsmpo_tridiag_timing(const bsmpo_ctx* h, double* ms, double* bytes, double* flops, int64_t* phases) {
  if (!h) return fail(nullptr, BSMPO_EINVAL, "null handle");
  if (ms) *ms = h->td_ms;
  if (bytes) *bytes = h->td_bytes;
  if (flops) *flops = h->td_flops;
  if (phases) *phases = h->td_phases;
  return BSMPO_OK;
}

int bsmpo_jacobi_timing(const bsmpo_ctx* h, double* ms, double* flops, int64_t* launches) {
  if (!h) return fail(nullptr, BSMPO_EINVAL, "null handle");
  if (ms) *ms = h->jac_ms;
  if (flops) *flops = h->jac_flops;
  if (launches) *launches = h->jac_launches;
  return BSMPO_OK;
}

int bsmpo_stage_times(const bsmpo_ctx* h, double* ms, int n) {
  if (!h || !ms || n < 10) return fail(nullptr, BSMPO_EINVAL, "bad argument");
  for (int i = 0; i < 8; ++i) ms[i] = h->stage_ms[i];
  ms[8] = (double)h->jacobi_rounds;
  ms[9] = (double)h->updates;
  return BSMPO_OK;
}

}  // extern "C"
