// Grouped complex GEMM on the 5th-generation tensor cores (tcgen05), 3 x TF32 split
// products with FP32 accumulation: the contractions of the mixed-precision form.
//
//   C[m][n] = sum_k op(A)[m][k] B[k][n] (x cs[n]),  op(A) = A or A^H,
//
// with FP64 complex inputs and outputs.  The complex product is one real GEMM:
// A_int (M x 2K, the interleaved storage of A read as reals) times B_emb (2K x 2N,
// every complex b as the 2 x 2 block [[Re b, Im b], [-Im b, Re b]]) gives C_int, the
// interleaved storage of C.  Every real operand x is split into TF32 hi = tf32(x) and
// lo = tf32(x - hi); the accumulator takes hi*hi + hi*lo + lo*hi (about 2^-21 relative
// per product instead of TF32's 2^-11).
//
// One CTA per 128 x 64 complex tile (MMA M = 128, N = 128 reals), 192 threads:
//   warp 0     TMA producer: cp.async.bulk.tensor of the raw FP64 tiles of A and B
//              (8 complex of K per k-block) into a 4-stage ring;
//   warp 1     allocates 128 TMEM columns; one lane issues tcgen05.mma kind::tf32
//              (6 per k-block: 3 products x 2 MMA K-steps) and tcgen05.commit;
//   warps 2-5  split each raw k-block into TF32 hi / lo in the canonical K-major
//              core-matrix layout (no swizzle), zeroing K beyond the group (the TMA box
//              may run into a neighbouring charge block), then read the accumulator with
//              tcgen05.ld and write C.
// Every mbarrier wait is bounded (about one second of clock): on expiry the kernel sets
// the error word and every role leaves its loop, so a fault in the pipeline ends the
// launch instead of hanging the GPU.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>

#include "common.cuh"
#include "kernels.h"
#include "pipeline.cuh"

namespace {

constexpr int TC_BM = 128;                      // complex rows of C per tile (MMA M)
constexpr int TC_BN = 64;                       // complex columns of C per tile (MMA N / 2)
constexpr int TC_BK = 8;                        // complex K per k-block (16 reals)
constexpr int TC_RAW = 4;                       // raw FP64 stages
constexpr int TC_CV = 2;                        // converted TF32 stages
constexpr int TC_NT = 192;
constexpr int RAW_A_BYTES = TC_BM * TC_BK * 16;   // 16 KB (box 16 x 128 or 256 x 8 doubles)
constexpr int RAW_B_BYTES = TC_BK * TC_BN * 16;   // 8 KB (box 128 x 8 doubles)
constexpr int RAW_STAGE = RAW_A_BYTES + RAW_B_BYTES;
constexpr int OP_BYTES = 128 * 2 * TC_BK * 4;     // 128 rows x 16 TF32 = 8 KB
constexpr int CV_STAGE = 4 * OP_BYTES;            // A hi, A lo, B hi, B lo
constexpr int TC_SMEM = TC_RAW * RAW_STAGE + TC_CV * CV_STAGE + 1024 + 1024;

// instruction descriptor, kind::tf32: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9 and
// 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(128 >> 3) << 17) |
                              ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// shared-memory matrix descriptor, K-major, no swizzle: core matrices of 8 rows x 16 B;
// the two 16-byte K chunks of one MMA are LBO = 128 B apart, 8-row groups SBO = 512 B
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)(128 >> 4) << 16;
  d |= (uint64_t)(512 >> 4) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version of this architecture
  return d;                 // base offset 0, layout type 0 (no swizzle)
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(TC_IDESC), "r"(accum));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void split_tf32(double x, float& hi, float& lo) {
  uint32_t h, l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"((float)x));
  hi = __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"((float)(x - (double)hi)));
  lo = __uint_as_float(l);
}

// byte offset of the 16-byte chunk c (4 TF32 of K) of row r in an operand tile
__device__ __forceinline__ int op_off(int r, int c) { return (r >> 3) * 512 + c * 128 + (r & 7) * 16; }

__device__ __forceinline__ void st_shared_f4(unsigned char* p, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}

__global__ void __launch_bounds__(TC_NT, 1)
    tc_zgemm_kernel(const TcGroup* __restrict__ groups, int n_groups, const CUtensorMap* __restrict__ maps,
                    cplx* __restrict__ C, const double* __restrict__ scale, int* __restrict__ err) {
  extern __shared__ unsigned char smem_dyn[];
  // 1024-byte aligned regions
  unsigned char* base = smem_dyn + ((1024 - (smem_u32(smem_dyn) & 1023)) & 1023);
  unsigned char* raw = base;
  unsigned char* cv = raw + TC_RAW * RAW_STAGE;
  uint64_t* bars = reinterpret_cast<uint64_t*>(cv + TC_CV * CV_STAGE);
  uint64_t* raw_full = bars;
  uint64_t* raw_empty = bars + TC_RAW;
  uint64_t* cv_full = bars + 2 * TC_RAW;
  uint64_t* cv_empty = cv_full + TC_CV;
  uint64_t* acc_full = cv_empty + TC_CV;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_full + 1);
  TcGroup* gsh = reinterpret_cast<TcGroup*>(bars + 32);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    int lo = 0, hi = n_groups - 1;
    const int t = blockIdx.x;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (groups[mid].tile_start <= t) lo = mid; else hi = mid - 1;
    }
    *gsh = groups[lo];
    for (int s = 0; s < TC_RAW; ++s) {
      mbar_init(raw_full + s, 1);
      mbar_init(raw_empty + s, 4);   // one arrival per converter warp
    }
    for (int s = 0; s < TC_CV; ++s) {
      mbar_init(cv_full + s, 4);
      mbar_init(cv_empty + s, 1);    // tcgen05.commit
    }
    mbar_init(acc_full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const TcGroup g = *gsh;
  const uint32_t tmem = *tmem_slot;
  const int local = blockIdx.x - g.tile_start;
  const int m0 = (local / g.tiles_n) * TC_BM, n0 = (local % g.tiles_n) * TC_BN;
  const int nkb = (g.K + TC_BK - 1) / TC_BK;
  bool ok = true;

  if (warp == 0) {
    // ---- TMA producer
    if (lane == 0) {
      const CUtensorMap* ma = maps + g.mapA;
      const CUtensorMap* mb = maps + g.mapB;
      for (int kb = 0; kb < nkb && ok; ++kb) {
        const int s = kb % TC_RAW;
        if (kb >= TC_RAW) ok = mbar_wait(raw_empty + s, ((kb / TC_RAW) - 1) & 1, err);
        if (!ok) break;
        unsigned char* dst = raw + s * RAW_STAGE;
        mbar_expect_tx(raw_full + s, RAW_STAGE);
        const int k0 = kb * TC_BK;
        if (g.opA == 0)   // A[m][k]: box 8 complex of K x 128 rows
          tma_load_2d(dst, ma, 2 * (g.a_c0 + k0), g.a_r0 + m0, raw_full + s);
        else              // A stored [k][m]: box 128 complex of M x 8 rows
          tma_load_2d(dst, ma, 2 * (g.a_c0 + m0), g.a_r0 + k0, raw_full + s);
        tma_load_2d(dst + RAW_A_BYTES, mb, 2 * (g.b_c0 + n0), g.b_r0 + k0, raw_full + s);
      }
    }
  } else if (warp == 1) {
    // ---- MMA issue (one lane)
    if (lane == 0) {
      for (int kb = 0; kb < nkb && ok; ++kb) {
        const int s = kb % TC_CV;
        ok = mbar_wait(cv_full + s, (kb / TC_CV) & 1, err);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t st = smem_u32(cv + s * CV_STAGE);
        const uint32_t ahi = st, alo = st + OP_BYTES, bhi = st + 2 * OP_BYTES, blo = st + 3 * OP_BYTES;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
          const uint32_t o = kk * 256;   // two 16-byte K chunks per MMA (K = 8 TF32)
          mma_tf32(tmem, umma_desc(alo + o), umma_desc(bhi + o), (kb | kk) ? 1u : 0u);
          mma_tf32(tmem, umma_desc(ahi + o), umma_desc(blo + o), 1u);
          mma_tf32(tmem, umma_desc(ahi + o), umma_desc(bhi + o), 1u);
        }
        mma_commit(cv_empty + s);       // frees the stage once these MMAs have read it
      }
      if (ok) mma_commit(acc_full);
    }
  } else {
    // ---- converters (warps 2-5, 128 threads), then the epilogue
    const int ct = tid - 64;
    for (int kb = 0; kb < nkb && ok; ++kb) {
      const int rs = kb % TC_RAW, cs = kb % TC_CV;
      ok = mbar_wait(raw_full + rs, (kb / TC_RAW) & 1, err);
      if (ok && kb >= TC_CV) ok = mbar_wait(cv_empty + cs, ((kb / TC_CV) - 1) & 1, err);
      if (!ok) break;
      const double2* ra = reinterpret_cast<const double2*>(raw + rs * RAW_STAGE);
      const double2* rb = reinterpret_cast<const double2*>(raw + rs * RAW_STAGE + RAW_A_BYTES);
      unsigned char* ov = cv + cs * CV_STAGE;
      const int kvalid = g.K - kb * TC_BK;   // complex K entries of this block inside the group
      // A row ct: A_int[ct][2k] = Re, [2k + 1] = Im (conjugated for A^H)
      {
        float h[16], l[16];
#pragma unroll
        for (int k = 0; k < TC_BK; ++k) {
          double2 v = make_double2(0.0, 0.0);
          if (k < kvalid) {
            v = g.opA == 0 ? ra[ct * TC_BK + k] : ra[k * TC_BM + ct];
            if (g.opA) v.y = -v.y;
          }
          split_tf32(v.x, h[2 * k], l[2 * k]);
          split_tf32(v.y, h[2 * k + 1], l[2 * k + 1]);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          st_shared_f4(ov + op_off(ct, c), h[4 * c], h[4 * c + 1], h[4 * c + 2], h[4 * c + 3]);
          st_shared_f4(ov + OP_BYTES + op_off(ct, c), l[4 * c], l[4 * c + 1], l[4 * c + 2], l[4 * c + 3]);
        }
      }
      // B_emb^T row ct = 2n + c: (Re b, -Im b) for c = 0, (Im b, Re b) for c = 1
      {
        const int n = ct >> 1, c1 = ct & 1;
        float h[16], l[16];
#pragma unroll
        for (int k = 0; k < TC_BK; ++k) {
          double2 v = make_double2(0.0, 0.0);
          if (k < kvalid) v = rb[k * TC_BN + n];
          const double x0 = c1 ? v.y : v.x, x1 = c1 ? v.x : -v.y;
          split_tf32(x0, h[2 * k], l[2 * k]);
          split_tf32(x1, h[2 * k + 1], l[2 * k + 1]);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          st_shared_f4(ov + 2 * OP_BYTES + op_off(ct, c), h[4 * c], h[4 * c + 1], h[4 * c + 2], h[4 * c + 3]);
          st_shared_f4(ov + 3 * OP_BYTES + op_off(ct, c), l[4 * c], l[4 * c + 1], l[4 * c + 2], l[4 * c + 3]);
        }
      }
      // generic-proxy writes -> visible to the tensor cores (async proxy)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(raw_empty + rs);
        mbar_arrive(cv_full + cs);
      }
    }
    // ---- epilogue: TMEM lanes 32 q .. 32 q + 31 (q = warp mod 4) are rows m0 + 32 q + lane
    if (ok) ok = mbar_wait(acc_full, 0, err);
    if (ok) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int q = warp & 3;
      const int row = m0 + 32 * q + lane;
      const double* csp = g.cs_off >= 0 ? scale + g.cs_off : nullptr;
#pragma unroll 1
      for (int chunk = 0; chunk < 4; ++chunk) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * chunk);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
            "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
            "[%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
              "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
              "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
              "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < g.M) {
          cplx* crow = C + g.c_off + (int64_t)row * g.ldc;
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int n = n0 + 16 * chunk + i;
            if (n < g.N) {
              const double s = csp ? csp[n] : 1.0;
              stc(crow + n, cmake((double)__uint_as_float(r[2 * i]) * s, (double)__uint_as_float(r[2 * i + 1]) * s));
            }
          }
        }
      }
    }
  }
  // ---- teardown: every role is done with TMEM before it is released
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
  }
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

}  // namespace

int tc_tile_m() { return TC_BM; }
int tc_tile_n() { return TC_BN; }

cudaError_t tc_encode_map(void* map_out, const void* base, int rows, int cols, int ld, int opA_box) {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  if (!g_encode) return cudaErrorNotSupported;
  // FP64 view: inner dimension 2 cols doubles, `rows` rows of 16 ld bytes
  const cuuint64_t dims[2] = {(cuuint64_t)2 * (cols > 0 ? cols : 1), (cuuint64_t)(rows > 0 ? rows : 1)};
  const cuuint64_t strides[1] = {(cuuint64_t)16 * (ld > 0 ? ld : 1)};
  cuuint32_t box[2];
  if (opA_box == 0) { box[0] = 2 * TC_BK; box[1] = TC_BM; }        // A [m][k]
  else if (opA_box == 1) { box[0] = 2 * TC_BM; box[1] = TC_BK; }   // A stored [k][m]
  else { box[0] = 2 * TC_BN; box[1] = TC_BK; }                     // B [k][n]
  const cuuint32_t estr[2] = {1, 1};
  CUtensorMap* m = reinterpret_cast<CUtensorMap*>(map_out);
  const CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

size_t tc_map_bytes() { return sizeof(CUtensorMap); }

cudaError_t launch_tc_zgemm(const TcGroup* groups_dev, int n_groups, int total_tiles, const void* maps_dev,
                            void* c, const double* scale, int* err, cudaStream_t s) {
  if (total_tiles <= 0 || n_groups <= 0) return cudaSuccess;
  static const cudaError_t attr =
      cudaFuncSetAttribute(tc_zgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
  if (attr != cudaSuccess) return attr;
  tc_zgemm_kernel<<<total_tiles, TC_NT, TC_SMEM, s>>>(groups_dev, n_groups,
                                                      reinterpret_cast<const CUtensorMap*>(maps_dev),
                                                      reinterpret_cast<cplx*>(c), scale, err);
  return cudaGetLastError();
}
