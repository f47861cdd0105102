/*
 * bsmpo.h -- C ABI of libbsmpo.so, the B200 (sm_100a) beam-splitter MPO update.
 *
 * One BS update of a U(1)-symmetric density-matrix MPO = Fock beam-splitter tensor
 * -> per-charge-block two-site contraction -> per-sector SVD -> top-chi truncation
 * -> scatter into the two site tensors.  Everything runs on the device; the library
 * owns the MPO state and its workspaces.
 *
 * Conventions
 *   - Every function returns 0 on success and a negative BSMPO_E* code on failure;
 *     bsmpo_last_error() gives a message.  No C++ exception crosses the ABI.
 *   - Pointers documented "device" are CUDA device pointers; "host" pointers are
 *     plain host memory.  `stream` arguments are cudaStream_t (NULL = legacy default).
 *   - complex128 is interleaved (re, im) doubles.
 *   - State layout (the reference's, src/MPO.py:114-132 and
 *     src/beam_splitter_parallel/Full.py:56-63, in double precision):
 *       gamma  [n][chi][chi] complex128   Gamma[site][left bond][right bond]
 *       lambda [n-1][chi]    double       Lambda on bond i+1 (between sites i, i+1)
 *       charge [n+1][chi][2] int32        (ket, bra) photons right of the bond,
 *                                         sorted lexicographically, empty = (d, d)
 *   - One handle is used from one host thread at a time.
 */
#ifndef BSMPO_H
#define BSMPO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BSMPO_OK 0
#define BSMPO_EINVAL -1      /* bad argument / inconsistent state */
#define BSMPO_ECUDA -2       /* CUDA runtime error */
#define BSMPO_ENOMEM -3      /* device allocation failed */
#define BSMPO_ECAPACITY -4   /* a workspace bound was exceeded */
#define BSMPO_ECONVERGE -5   /* the per-sector SVD did not converge */

typedef struct bsmpo_ctx bsmpo_ctx;

/* Library version string. */
const char* bsmpo_version(void);

/* Message of the last error on `h` (or of the last handle-less call when h == NULL). */
const char* bsmpo_last_error(const bsmpo_ctx* h);

/* Gradient with respect to the angles of n_gates mesh beam splitters T(theta, phi) =
 * [[e^{i phi} cos, -sin], [e^{i phi} sin, cos]] (host theta[], phi[]), given ubar
 * (device complex128 [n_gates][d][d][d]), the gradient of a real loss with respect to each
 * gate's tensor U[new_a][new_b][old_a] (as bsmpo_run_mesh builds it; pairing
 * Re sum conj(ubar) dU).  Writes grad (device double [n_gates][2]: dL/dtheta, dL/dphi).
 * The reference has no gradient (it runs forward only); the differentiation form's
 * adjoint (bosonsampling_b200.adjoint) uses this for the gates.  Synchronises stream. */
int bsmpo_bs_angle_grad(int d, int n_gates, const double* theta, const double* phi,
                        const void* ubar, double* grad, void* stream);

/* Two-mode Fock beam-splitter tensor.  Replaces cuda_kernels.Rand_U / u_kernel
 * (src/cuda_kernels.py:18-50, src/u_kernel.cu:37-71) and the CPU Rand_BS_MPS
 * (src/MPO.py:6-18).  M is the 2x2 single-particle matrix of the reference's
 * convention, a+ -> M00 a+ + M10 b+, b+ -> M01 a+ + M11 b+ (for the reference's
 * (t, r): M = [[t, -conj r], [r, conj t]]), given as 8 host doubles
 * (re, im of M00, M01, M10, M11).  Writes U[n][m][l] = <l, n+m-l| M |n, m> for
 * 0 <= n, m, l < d (zero where n+m-l is outside [0, d)) as complex128 to the device
 * buffer u_out (d^3 entries).  Integer powers in FP64: exact at r = 0 and t = 0. */
int bsmpo_unitary(int d, const double* M, void* u_out, void* stream);

/* Same, for the reference's (t, r) pair, writing split real / imaginary parts
 * (the layout of cuda_kernels.Rand_U): u_re, u_im are device double[d^3]. */
int bsmpo_unitary_tr(int d, double t_re, double t_im, double r_re, double r_im,
                     double* u_re, double* u_im, void* stream);

/* One centre-charge sector of the two-site contraction.  Replaces
 * cuda_kernels.update_MPO / update_MPO_kernel.cu:kernel (src/cuda_kernels.py:101-127,
 * src/update_MPO_kernel.cu:193-733), without the reference's x8 alignment padding:
 *   C[l][r] = sum_c Glc[l][c] Gcr[c][r] U(cl0-cc0, cc0-cr0, cl0-q0(c))
 *                                       conj U(cl1-cc1, cc1-cr1, cl1-q1(c))
 * over c with cl >= q(c) >= cr componentwise (else the term is 0).
 *   u    device complex128 [d][d][d] (bsmpo_unitary output, U[new_a][new_b][old_a])
 *   glc  device complex128 [len_l][len_c] row-major; gcr [len_c][len_r]
 *   cl   device int32 [len_l][2]; cc [len_c][2] (sorted); cr [len_r][2]
 *   c    device complex128 [len_l][len_r] output (overwritten). */
int bsmpo_contract_sector(int d, int cc0, int cc1, const void* u,
                          const void* glc, const void* gcr,
                          const int* cl, const int* cc, const int* cr,
                          int len_l, int len_c, int len_r, void* c, void* stream);

/* The pure-state (MPS) variant of the contraction.  Replaces cuda_kernels.update_MPS /
 * update_kernel.cu:kernel (src/cuda_kernels.py:72-90, src/update_kernel.cu:193-769),
 * one charge (photon number) per bond index:
 *   T[l][r] = LL[l] LR[r] sum_c LC[c] Glc[l][c] Gcr[c][r] U(cl - tau, tau - cr, cl - q(c))
 * over c with cl >= q(c) >= cr (else the term is 0; T is 0 where cl - tau or tau - cr
 * falls outside [0, d)).
 *   u    device complex128 [d][d][d]; glc [len_l][len_c]; gcr [len_c][len_r]
 *   ll, lc, lr device double Lambda of the rows / centre entries / columns
 *   cl, cc, cr device int32 charges; t device complex128 [len_l][len_r] (overwritten). */
int bsmpo_contract_mps(int d, int tau, const void* u, const void* glc, const void* gcr, const double* ll,
                       const double* lc, const double* lr, const int* cl, const int* cc, const int* cr,
                       int len_l, int len_c, int len_r, void* t, void* stream);

/* Complex GEMM on the tensor cores with three TF32 split products (hi*hi + hi*lo +
 * lo*hi, FP32 accumulation): C[m][n] = sum_k op(A)[m][k] B[k][n], the contraction
 * primitive of BSMPO_PRECISION_TF32X3 (the reference's update_MPO_kernel.cu GEMM,
 * src/update_MPO_kernel.cu:193-733, computes in FP32 SIMT).  Device complex128
 * row-major matrices: op(A) = A [M][K] (opA 0, lda >= K) or A^H with A stored [K][M]
 * (opA 1, lda >= M); B [K][N]; C [M][N] is overwritten.  Synchronises `stream`; error
 * about 2^-21 relative per product. */
int bsmpo_zgemm_tf32x3(int M, int N, int K, const void* a, int lda, int opA, const void* b, int ldb,
                       void* c, int ldc, void* stream);

/* Create a handle for an n-mode chain with local cutoff d and bond dimension chi.
 * Allocates the device state (n chi^2 complex128) and workspaces on the current
 * device.  flags: reserved, pass 0. */
int bsmpo_create(int n, int d, int chi, int flags, bsmpo_ctx** out);
int bsmpo_destroy(bsmpo_ctx* h);

/* Stream used by all following calls on h (default: the legacy default stream). */
int bsmpo_set_stream(bsmpo_ctx* h, void* stream);

/* How the sector SVD and the contractions are computed (bsmpo_set_precision):
 *   BSMPO_PRECISION_FP64       one-sided Jacobi SVD in FP64, FP64 contractions: the
 *                              plain path, equal to the reference CPU algorithm
 *                              (src/MPO.py:254-279) to ~1e-12 (the default);
 *   BSMPO_PRECISION_FP64_GRAM  FP64 contractions, per-sector Gram matrix and Hermitian
 *                              eigenproblem in FP64 (Householder tridiagonalisation,
 *                              bisection, inverse iteration): singular values below
 *                              about 2e-6 of the largest are dropped as zero.  An
 *                              update whose candidates cannot exceed chi (the growing
 *                              bonds of the first layers) is solved by the exact Jacobi
 *                              SVD instead: nothing is truncated there, and dropping
 *                              small values there is pure loss (W = V^H C carries them
 *                              through 1 / Lambda_R).  The environment variable
 *                              BSMPO_GRAM_POLICY, read at create, widens that rule:
 *                              1 adds updates that keep fewer than chi after the
 *                              selection (the SVD is redone), 2 also those whose centre
 *                              bond holds fewer than chi vectors. */
#define BSMPO_PRECISION_FP64 0
#define BSMPO_PRECISION_FP64_GRAM 1
/*   BSMPO_PRECISION_TF32X3     the Gram route with the two-site contraction (the Theta
 *                              block products) on the tensor cores (tcgen05): 3 x TF32
 *                              split products, FP32 accumulation; the Gram, the
 *                              eigenproblem, V = T Y / sigma, W = V^H C, Lambda and the
 *                              observables stay FP64 (BSMPO_TC_MASK=3 in the environment
 *                              at create also puts W on the tensor cores).  Measured
 *                              marginal error against FP64: ~1e-5 (N=16, chi=64) to
 *                              ~1e-4 (N=32, chi=256) of the trace -- the FP32
 *                              accumulation of the split products bounds it, so this
 *                              mode does not reach 1e-6 on these circuits. */
#define BSMPO_PRECISION_TF32X3 2
int bsmpo_set_precision(bsmpo_ctx* h, int precision);

/* Relative singular-value cutoff: a singular value s is kept only if
 * s > cutoff * (largest singular value of that update).  0 (the default) keeps every
 * s > 0, the reference's rule (src/MPO.py:272-279 with the Lambda > 0 masks). */
int bsmpo_set_cutoff(bsmpo_ctx* h, double cutoff);

/* Copy a state into / out of the handle.  Device pointers in the layout above.
 * load validates it (sorted charges, sentinel d for empty slots, Lambda > 0 on
 * occupied internal slots). */
int bsmpo_load_state(bsmpo_ctx* h, const void* gamma, const double* lambda, const int* charge);
int bsmpo_store_state(bsmpo_ctx* h, void* gamma, double* lambda, int* charge);

/* One site or one bond of the loaded state, copied between the handle and device
 * buffers of the caller: the units of the halo exchange of a circuit partitioned over
 * several handles (ranks), replacing the per-site Gamma / Lambda / charge messages of
 * src/fully_parallel/Full.py:70-103 and the per-request state shipping of
 * src/beam_splitter_parallel/Full.py:149-166.  Site 0..n-1: Gamma[site], complex128
 * chi x chi.  Bond 1..n-1 (between sites bond-1 and bond): Lambda double[chi] and
 * charges int32[chi][2].  put_bond validates the bond as load_state does and leaves the
 * state unchanged when it is rejected.  All return with the copy complete. */
int bsmpo_get_site(bsmpo_ctx* h, int site, void* gamma);
int bsmpo_put_site(bsmpo_ctx* h, int site, const void* gamma);
int bsmpo_get_bond(bsmpo_ctx* h, int bond, double* lambda, int* charge);
int bsmpo_put_bond(bsmpo_ctx* h, int bond, const double* lambda, const int* charge);

/* Product-state MPO built on the device: the filling of the reference's Initialize
 * (src/MPO.py:56-109) for an arbitrary density matrix per mode.  rho: host
 * complex128 [n][d][d] (rho[site][ket occupation][bra occupation]).  Bond charges are
 * the (ket, bra) photons right of the bond, at most d - 1 each; bond 0 lists every
 * diagonal total (c, c), c < d, or only (total_photons, total_photons) when
 * total_photons >= 0 (the reference's post-selected photon number).  Lambda = 1 on
 * occupied slots.  BSMPO_ECAPACITY if a bond needs more than chi slots. */
int bsmpo_init_product(bsmpo_ctx* h, const double* rho, int total_photons);

/* Right-to-left sweep of identity-gate updates over every bond: the canonicalising
 * sweep of the reference's Initialize (src/MPO.py:137-155). */
int bsmpo_canonicalize(bsmpo_ctx* h);

/* Apply a beam splitter to modes (mode, mode+1): the per-BS unit of work of
 * RankWorker.RankProcess (src/beam_splitter_parallel/Rank.py:32-206) and
 * InitializationMPO.Update (src/MPO.py:158-303), fully on the device.
 * S: host double[8], the 2x2 single-particle unitary acting on the state
 * (a photon entering mode j leaves mode i with amplitude S[i][j]). */
int bsmpo_bs_update(bsmpo_ctx* h, int mode, const double* S);

/* Same with an explicit device tensor U[new_a][new_b][old_a] (complex128 d^3), e.g.
 * the reference's Rand_BS_MPS tensor or bsmpo_unitary output. */
int bsmpo_bs_update_tensor(bsmpo_ctx* h, int mode, const void* u);

/* Run a whole mesh (the walk of src/beam_splitter_parallel/Full.py:149-202):
 * n_bs beam splitters T(theta, phi) = [[e^{i phi} cos, -sin], [e^{i phi} sin, cos]]
 * on (modes[i], modes[i]+1), in the given order.  Host arrays.  Consecutive entries
 * whose modes differ pairwise by 2 or more (a brick-wall layer) touch disjoint sites
 * and run concurrently on the handle's workers (bsmpo_set_workers); the result is the
 * same as applying them one by one.  Returns with all work complete. */
int bsmpo_run_mesh(bsmpo_ctx* h, int n_bs, const int* modes, const double* theta,
                   const double* phi);

/* The same mesh over a host-resident state (the reference keeps the state in host
 * memory and moves each update's blocks to the device and back:
 * src/beam_splitter_parallel/Rank.py:63-68 and 198-199).  The input state
 * (gamma_in [n][chi][chi] complex128, lambda_in [n-1][chi], charge_in [n+1][chi][2], the
 * bsmpo_load_state layout, host memory) is validated, its bonds are copied in, and
 * each site of Gamma is copied in by the first update touching it, on that update's
 * stream, and copied to gamma_out by the last one, so one update's transfers overlap
 * the other updates' compute (both directions need page-locked host memory to run
 * asynchronously).  lambda_out and charge_out are written at the end.  The outputs may
 * alias the inputs.  On return the device holds the same state (as after
 * bsmpo_load_state + bsmpo_run_mesh) and all copies are complete.  On error the
 * device state is not loaded. */
int bsmpo_run_mesh_host(bsmpo_ctx* h, int n_bs, const int* modes, const double* theta,
                        const double* phi, const void* gamma_in, const double* lambda_in,
                        const int* charge_in, void* gamma_out, double* lambda_out,
                        int* charge_out);

/* Truncation weight (sum of discarded sigma^2) of every update of the last
 * bsmpo_run_mesh call, in mesh order, into host weights[cap].  Returns the number of
 * updates (>= 0; weights == NULL only queries it) or a negative code
 * (BSMPO_ECAPACITY if cap is too small).  The
 * reference computes no truncation weight (src/MPO.py:272-279 discards silently). */
int bsmpo_mesh_truncation(const bsmpo_ctx* h, double* weights, int cap);

/* Number of updates bsmpo_run_mesh runs at once (1..64, default 8 or the environment
 * variable BSMPO_WORKERS at create).  Each worker owns a stream and its own workspaces
 * (grown on demand, freed by bsmpo_destroy).  Replaces the reference's dispatch of one
 * layer's beam splitters to separate MPI ranks (src/beam_splitter_parallel/
 * Full.py:149-166, Rank.py:32-206) within one GPU. */
int bsmpo_set_workers(bsmpo_ctx* h, int n_workers);

/* Output phase screen exp(i phase_m n_m) on every mode (host double[n]). */
int bsmpo_apply_phases(bsmpo_ctx* h, const double* phases);

/* Trace (summary.Probability, src/summary.py:11-26) and single-mode photon-number
 * marginals P[i][k] = Prob(k photons in mode i), un-normalised, in FP64.
 * Host outputs: trace[2] (re, im), marginals[n][d][2] (re, im); marginals may be NULL. */
int bsmpo_observables(bsmpo_ctx* h, double* trace, double* marginals);

/* Diagnostics of the last update (host buffers, capacities in entries):
 *   n_sectors; per sector (in loop order) its centre charge sector_cc[s][2],
 *   |L_s|, |R_s| in shape[s][2], the number of singular values sigma_len[s]
 *   (descending, packed in sigma), the kept count kept[s]; and the truncation
 *   weight (sum of discarded sigma^2).  Any output pointer may be NULL. */
int bsmpo_last_update_info(const bsmpo_ctx* h, int* n_sectors, int* sector_cc, int* shape,
                           int* sigma_len, double* sigma, int sigma_cap, int* kept,
                           double* trunc_weight);

/* Work counters of the last update (host): algorithmic flops of the contraction
 * GEMMs and of the SVD step, and the bytes the update had to move at minimum. */
int bsmpo_last_update_work(const bsmpo_ctx* h, double* gemm_flops, double* svd_flops,
                           double* min_bytes);

/* Bond dimensions (occupied slots) of every bond, host int[n+1]. */
int bsmpo_bond_dims(const bsmpo_ctx* h, int* dims);

/* Updates solved by the Jacobi SVD (counts[0]) and by the Gram route (counts[1]) since
 * creation (host int64[2]). */
int bsmpo_svd_routes(const bsmpo_ctx* h, int64_t* counts);

/* Workspace growth since creation (host int64[4]): [0] device workspace allocations
 * (stream-ordered, from the handle's pool), [1] pinned host stage allocations, [2]
 * device bytes and [3] pinned bytes held now by the handle and its workers.  Workspaces
 * grow on demand to the largest update seen and are kept until bsmpo_destroy; a
 * replaced pinned stage is also kept until then (releasing pinned memory would
 * synchronise the device). */
int bsmpo_workspace_stats(const bsmpo_ctx* h, int64_t* out);

/* Number of kernels this handle has launched since creation. */
int64_t bsmpo_kernel_launches(const bsmpo_ctx* h);

/* Time the SVD phase of every update with CUDA events on the handle's stream: the
 * Jacobi rounds (BSMPO_PRECISION_FP64) or the Gram + tridiagonalisation + bisection
 * kernels (Gram route).  on != 0 enables and resets the counters. */
int bsmpo_set_timing(bsmpo_ctx* h, int on);

/* Accumulated SVD-phase device time (ms), its algorithmic flops and its launches since
 * bsmpo_set_timing(h, 1).  Jacobi: the executed work counted on the device (rows that
 * formed a partial pair Gram, 640 complex MACs each, and rotated rows, 1024 each);
 * Gram route: 8 k^2 rows (the Gram) + 16/3 k^3 (Householder reduction) per sector;
 * 8 flops per complex MAC. */
int bsmpo_jacobi_timing(const bsmpo_ctx* h, double* ms, double* flops, int64_t* launches);

/* Device time (ms) of the Householder tridiagonalisation phase of the Gram route (its
 * forked size-class launches, CUDA events on the update's stream) since
 * bsmpo_set_timing(h, 1), with the bytes its fused passes stream (every step reads and
 * writes the trailing matrix once: 32 B per complex entry) and its flops (16/3 k^3 per
 * sector, LAPACK's zhetrd count), and the number of phases. */
int bsmpo_tridiag_timing(const bsmpo_ctx* h, double* ms, double* bytes, double* flops, int64_t* phases);

/* Stage timing, filled only when the handle was created with BSMPO_PROFILE=1 in the
 * environment (each stage then ends with a stream synchronisation).  ms[0..7]:
 * plan+upload, Theta GEMM, mix, Jacobi rounds, finish+select+sync, V/W, scatter,
 * (unused); ms[8] = Jacobi round launches, ms[9] = updates.  n >= 10. */
int bsmpo_stage_times(const bsmpo_ctx* h, double* ms, int n);

/* Largest bond dimension bsmpo_trace_noalloc accepts. */
#define BSMPO_NOALLOC_MAX_CHI 4096

/* MPO trace without any device allocation.  No counterpart in the reference: it is
 * for callers that cannot call cudaMalloc -- code running under a framework that owns
 * all device memory (a caching allocator that must see every allocation), or a hook
 * between beam-splitter updates that must not incur an allocation's implicit device
 * synchronisation.  Computes the same trace as bsmpo_observables from caller-owned
 * device buffers in the state layout above (gamma [n][chi][chi] complex128, lambda
 * [n-1][chi], charge [n+1][chi][2]); writes (re, im) to the device buffer trace_out
 * (2 doubles), on `stream`.  Its scratch is a fixed array inside the library,
 * 2 * BSMPO_NOALLOC_MAX_CHI + 256 complex128 entries (about 135 KB) that every GPU
 * loading the library keeps until the process exits; chi > BSMPO_NOALLOC_MAX_CHI is
 * rejected with BSMPO_EINVAL.  The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress, with the device current) and caches it.  That
 * first call also makes CUDA load the library's code and the array onto the device
 * (lazy module loading), which does take device memory once: make the first call on
 * each device early, before a framework reserves the whole device and before any
 * stream capture.  The cached address does not survive cudaDeviceReset: do not call
 * this function again in a process after resetting the device.  `stream` must belong
 * to the current device on every call (checked: BSMPO_EINVAL otherwise).  A CUDA error
 * already pending from earlier work makes the call fail with BSMPO_ECUDA before it
 * launches anything.  All calls share the array, and every call rewrites all of the
 * scratch it reads: calls that overlap on the GPU (other streams, other host threads)
 * race; serialise them.  Errors: see bsmpo_last_error(NULL). */
int bsmpo_trace_noalloc(int n, int d, int chi, const void* gamma, const double* lambda,
                        const int* charge, double* trace_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BSMPO_H */
