// Internal launch interface of libbsmpo's kernels (host side, C++).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/bsmpo.h"

// Message returned by bsmpo_last_error(NULL) (capi.cu).
void set_global_error(const char* msg);

// Largest local cutoff d supported (charge tables are d x d).
#define BSMPO_MAX_D 8
#define BSMPO_MAX_Q (BSMPO_MAX_D * BSMPO_MAX_D)

// ---------------------------------------------------------------- fock.cu
cudaError_t launch_fock_tensor(int d, int n_gates, const double* m4_dev, void* u_dev,
                               cudaStream_t s);
// One gate with M passed by value; writes interleaved complex (u_im == nullptr) or
// split real / imaginary double arrays.
struct M8 { double v[8]; };
// dL/dtheta, dL/dphi of every gate T(theta, phi) from the gradient of its tensor: m4 and
// dm4 (device) hold per gate M (8 doubles) and dM/dtheta, dM/dphi (16 doubles); grad gets
// 2 doubles per gate.
cudaError_t launch_fock_angle_grad(int d, int n_gates, const double* m4_dev, const double* dm4_dev,
                                   const void* ubar_dev, double* grad_dev, cudaStream_t s);
cudaError_t launch_fock_tensor_single(int d, M8 m, void* u_re_or_cplx, double* u_im,
                                      cudaStream_t s);

// ---------------------------------------------------------------- zgemm.cu
// One group of a grouped complex128 GEMM:  C = rs[m] cs[n] sum_k op(A)(m,k) ks[k] op(B)(k,n)
// op 0: as stored (row-major A[m][k], B[k][n]); op 1: conjugate transpose (A stored
// [k][m], B stored [n][k]).  Offsets are in complex elements (scales in doubles) from
// the launch's base pointers; a negative scale offset means "none".
struct GemmGroup {
  int M, N, K;
  int lda, ldb, ldc;
  int opA, opB;
  int beta;          // 0: C = result, 1: C += result
  int tiles_n;       // ceil(N / tile N)
  int tile_start;    // first flat tile index of this group
  int pad_;
  int64_t a_off, b_off, c_off;
  int64_t ks_off, rs_off, cs_off;
};

cudaError_t launch_zgemm_grouped(const void* a, const void* b, void* c, const double* scale,
                                 const GemmGroup* groups_dev, int n_groups, int total_tiles,
                                 cudaStream_t s);
int zgemm_tile_m();
int zgemm_tile_n();

// ---------------------------------------------------------------- plan descriptors
// Theta group (q, a0, b0): Theta_q[rows of left group a0 with a1 >= q1]
//                                 [cols of right group b0 with b1 <= q1]
//                         = Glc[rows][centre block q] @ Gcr[centre block q][cols]
struct ThetaDesc {
  int q0, q1, a0, b0;
  int row0, nrow, col0, ncol, k0, nk;
  int64_t off;            // storage [nrow][ncol] in the Theta workspace
};

struct SectorDesc {
  int cc0, cc1;
  int m, n;            // |L_s|, |R_s|
  int k;               // columns of the Jacobi matrix: n when !left, m when left
  int left;            // 1: Jacobi on [T^H; I_m] (m < n), 0: on T (m >= n)
  int rows_g;          // rows entering the pair Gram (m or n)
  int rows_tot;        // stored rows of the Jacobi matrix (m or n + m)
  int kept;            // filled after selection
  int slot0;           // first slot of this sector on the new bond
  int64_t c_off;       // C[m][n] row-major (complex)
  int64_t a_off;       // Jacobi matrix, row-major [rows_tot][k] (complex)
  int64_t s_off;       // singular values / keys / permutation (k entries)
  int64_t w_off;       // W = V^H C, [kept][n] row-major (complex)
  int64_t v_off;       // V, [m][kept] row-major (complex)
  int64_t g_off;       // Gram / Householder vectors, [k][k] (complex; Gram route only)
  int64_t y_off;       // k x k slots (Gram route): eigenvectors [k][kept], scratch
  int row_start[BSMPO_MAX_D];   // row of L_s where left group a0 (a1 >= cc1 part) starts
  int col_start[BSMPO_MAX_D];   // column of R_s where right group b0 (b1 <= cc1 part) starts
};

// One (left block a, right block b), a >= b, of the gate mix, cut in tiles of 256 elements.
struct MixPair {
  int a0, a1, b0, b1;
  int row0, nrow;      // left-bond rows of block a
  int col0, ncol;      // right-bond columns of block b
  int tile_start;      // first flat CTA index of this pair
  int pad_;
};

// Per-update tables shared by several kernels (device copy, one per update).
struct UpdateTables {
  int d, chi, mode;
  int n_sectors, n_theta, n_pairs;
  int offL[BSMPO_MAX_Q + 1], offC[BSMPO_MAX_Q + 1], offR[BSMPO_MAX_Q + 1];
  int sidx[BSMPO_MAX_Q];                          // sector index of centre charge, or -1
  int pair_of[BSMPO_MAX_Q];                       // sector index of the (cc1, cc0) sector, or -1
};

// ---------------------------------------------------------------- sector.cu
// Theta -> C (every sector, row-major) and the Jacobi matrix (T or [T^H; I]).
cudaError_t launch_mix_d(int d, const UpdateTables* tab_dev, const int* tidx_dev,
                         const ThetaDesc* td_dev, const SectorDesc* sd_dev,
                         const MixPair* pairs_dev, int n_pairs, int total_tiles, const void* u3,
                         const void* theta, const double* lam_r, void* cbuf, void* abuf,
                         cudaStream_t s);
// Identity rows of [T^H; I_m] for the `left` sectors.
cudaError_t launch_identity_rows(const SectorDesc* sd_dev, int n_sectors, int max_elems,
                                 void* abuf, cudaStream_t s);
// Deterministic top-chi with ket/bra pair symmetrisation; writes kept counts into
// sd_dev[s].kept and kept_out[s], slot starts, and the truncation weight.
cudaError_t launch_select(const UpdateTables* tab_dev, SectorDesc* sd_dev, int n_sectors,
                          const double* sig, double* keys, double cutoff, int chi,
                          int* kept_out, double* trunc_out, cudaStream_t s);
// conj(V) rows for the kept vectors of every sector.
cudaError_t launch_extract_v(const SectorDesc* sd_dev, int n_sectors, int max_elems,
                             const void* abuf, const double* sig, const int* perm, void* vbuf,
                             cudaStream_t s);
// New Gamma_L (= Gamma[mode]), Gamma_R (= Gamma[mode+1]), Lambda and charges of bond mode+1.
cudaError_t launch_scatter(const UpdateTables* tab_dev, const SectorDesc* sd_dev, int n_sectors,
                           int total_kept, int chi, const int* charge_l, const int* charge_r,
                           const void* vbuf, const void* wbuf, const double* sig,
                           void* gamma_l, void* gamma_r, double* lam_c, int* charge_c,
                           cudaStream_t s);
// exp(i phi (n_ket - n_bra)) on every element of one site tensor.
cudaError_t launch_phase(int d, int chi, double phi, const int* charge_l, const int* charge_r,
                         void* gamma, cudaStream_t s);

// ---------------------------------------------------------------- jacobi.cu
// One round of the blocked one-sided Jacobi SVD for every active sector.
struct JacobiWork {
  int sector;       // index into the SectorDesc array
  int nblk;         // column blocks
  int npairs;       // block pairs per round
  int rounds;       // rounds per sweep
  int cs;           // row parts per block pair (rows_tot in parts of `chunk` rows)
  int cs_g;         // parts holding Gram rows (the first rows_g rows)
  int chunk;        // rows per part (multiple of 16, at most jacobi_rows_per_part())
  int gram_start;   // first CTA of this sector in the gram launch (npairs * cs_g CTAs)
  int apply_start;  // first CTA in the apply launch (npairs * cs CTAs)
  int slot_start;   // first block-pair slot (Q, flag and arrival counter)
  int pad_[2];
};
// rows of one part of a block pair
int jacobi_rows_per_part();
int jacobi_block_cols();
// One round of every listed sector: the gram kernel (partial Grams -> pbuf, 32 x 32
// complex per gram CTA; the last part of a pair reduces, tests and solves, writing Q
// and the flag of its slot), then the apply kernel.  pcnt (one int per slot) must be
// zero before the first round; the kernels leave it zero.  executed[0] / executed[1]
// count the rows that formed a partial pair Gram / were rotated (the executed work).
cudaError_t launch_jacobi_round(const SectorDesc* sd_dev, const JacobiWork* work_dev, int n_work,
                                int gram_ctas, int apply_ctas, int t, void* abuf, int* rot_count,
                                const double* nf2, double tol, int max_sweeps, void* pbuf,
                                int* pcnt, void* qbuf, int* qflag, unsigned long long* executed,
                                cudaStream_t s);
// Largest number of Jacobi-matrix rows (|L| + |R| or |L|) a sector may have.
// ||T_s||_F^2 of each sector's Jacobi matrix (Gram rows), fixed-order reduction.
cudaError_t launch_sector_norms(const SectorDesc* sd_dev, int n_sectors, const void* abuf,
                                double* nf2, cudaStream_t s);
// Column norms (0 below the numerical-rank floor), descending sort (ties by column
// index): sig[s_off..], perm[s_off..].
cudaError_t launch_jacobi_finish(const SectorDesc* sd_dev, int n_sectors, int max_k,
                                 const void* abuf, const double* nf2, double* sig, int* perm,
                                 cudaStream_t s);

// ---------------------------------------------------------------- eigen.cu
// Gram / Hermitian-eigen route of the sector SVD (see eigen.cu).  gbuf holds every
// sector's Gram G = X^H X (k x k at g_off), overwritten by the Householder vectors.
int eigen_max_k();
// Sectors go in four launches by size class (tridiag_class: 1, 2, 4 or 8 CTAs per
// sector): list_dev holds the sector indices grouped by class, class_count / class_kmax
// (host, 4 entries) the number of sectors and their largest k per class.  Class c goes
// on streams[3 - c] (the caller forks and joins them; streams[0] is its own).  err: a
// device word set to 1 when a bulk-copy wait expired (zeroed by the caller).
int tridiag_class(int k);
cudaError_t launch_tridiag(const SectorDesc* sd_dev, const int* list_dev, const int* class_count,
                           const int* class_kmax, void* gbuf, double* dbuf, double* ebuf,
                           void* taubuf, int* err, const cudaStream_t* streams);
// eigenvalues (lam, descending), singular values sig = sqrt(lam) (0 below the floor), 1/sig
cudaError_t launch_bisect(const SectorDesc* sd_dev, int n_sectors, int kmax, const double* dbuf,
                          const double* ebuf, double* lam, double* sig, double* invsig,
                          cudaStream_t s);
// eigenvectors of the kept eigenvalues (sd[s].kept): V ([k][kept] at v_off) of the
// sectors with X = T^H, Y ([k][kept] at y_off) of the others
cudaError_t launch_eigvec(const SectorDesc* sd_dev, int n_sectors, int kmax, int kept_max,
                          const double* dbuf, const double* ebuf, const double* lam,
                          double* scratch, unsigned char* swp, double* zbuf, const void* gbuf,
                          const void* taubuf, void* vbuf, void* ybuf, cudaStream_t s);

// ---------------------------------------------------------------- tcgemm.cu
// One group of the tensor-core (tcgen05, 3 x TF32) grouped complex GEMM:
//   C[c_off + m ldc + n] = sum_k op(A)[m][k] B[k][n] (x scale[cs_off + n])
// A and B are read through TMA tensor maps (index mapA / mapB into the launch's map
// array, FP64 views of complex matrices): op(A) = A ([m][k] at row a_r0 + m, column
// a_c0 + k; opA 0) or A^H (A stored [k][m] at row a_r0 + k, column a_c0 + m; opA 1);
// B [k][n] at row b_r0 + k, column b_c0 + n.  Offsets in complex elements.
struct TcGroup {
  int M, N, K;
  int opA;
  int tiles_n, tile_start;
  int mapA, mapB;
  int a_r0, a_c0, b_r0, b_c0;
  int ldc, pad_;
  int64_t c_off, cs_off;
};
int tc_tile_m();
int tc_tile_n();
size_t tc_map_bytes();
// Encodes a tensor map (tc_map_bytes() bytes at map_out) of the complex matrix at base
// (rows x cols, leading dimension ld, complex elements) with the box of operand `kind`:
// 0 = A [m][k], 1 = A stored [k][m], 2 = B [k][n].
cudaError_t tc_encode_map(void* map_out, const void* base, int rows, int cols, int ld, int kind);
// err: device int, set to nonzero if a pipeline wait of the kernel expired.
cudaError_t launch_tc_zgemm(const TcGroup* groups_dev, int n_groups, int total_tiles, const void* maps_dev,
                            void* c, const double* scale, int* err, cudaStream_t s);

// ---------------------------------------------------------------- contract.cu
// Standalone sector contraction with per-element charges (the update_MPO drop-in).
cudaError_t launch_contract_sector(int d, int cc0, int cc1, const void* u, const void* glc,
                                   const void* gcr, const int* cl, const int* cc, const int* cr,
                                   int len_l, int len_c, int len_r, void* c, cudaStream_t s);

// ---------------------------------------------------------------- state.cu
// Product-state Gamma from the bond charges (sorted, sentinel d) and the per-site
// density matrices rho[site][o_ket][o_bra] (complex, n d^2 entries).
cudaError_t launch_product_fill(int n, int d, int chi, const int* charge, const void* rho,
                                void* gamma, cudaStream_t s);

// Pure-state (MPS) variant of the contraction, one int32 charge per index.
cudaError_t launch_contract_mps(int d, int tau, const void* u, const void* glc, const void* gcr,
                                const double* ll, const double* lc, const double* lr, const int* cl,
                                const int* cc, const int* cr, int len_l, int len_c, int len_r, void* t,
                                cudaStream_t s);

// ---------------------------------------------------------------- observables.cu
// env_r[b] (b = n..0) and env_l[b] (b = 0..n), complex, masked to ket == bra charges.
cudaError_t launch_env_right_step(int d, int chi, const void* gamma_b, const int* charge_b,
                                  const double* lam_b, const void* r_next, void* r_out,
                                  int rows, int cols, cudaStream_t s);
cudaError_t launch_env_left_step(int d, int chi, const void* gamma_b, const int* charge_next,
                                 const double* lam_next, const void* l_cur, void* l_out,
                                 int rows, int cols, cudaStream_t s);
cudaError_t launch_env_init(int d, int chi, const int* charge_b, const double* lam_b, void* v,
                            cudaStream_t s);
// partial marginal bins: part[site][chunk][d] complex, then reduced into out[site][d].
cudaError_t launch_marginals(int n, int d, int chi, const void* gamma, const int* charge,
                             const void* env_l, const void* env_r, const int* dims,
                             void* part, int chunk_rows, void* out, cudaStream_t s);
cudaError_t launch_sum_vector(const void* v, int len, void* out, cudaStream_t s);
