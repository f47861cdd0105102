// MPO trace for callers that must not allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code that runs under a
// framework owning every byte of device memory (a caching allocator that has to see
// each allocation and may have reserved the whole device), or a monitoring hook
// between beam-splitter updates that must not trigger the implicit device
// synchronisation an allocation can cause.  bsmpo_trace_noalloc gives them the MPO
// trace (the same quantity as bsmpo_observables) from caller-owned input and output
// buffers only.  Its scratch -- two environment vectors of at most
// BSMPO_NOALLOC_MAX_CHI complex128 entries and the partial sums of the final
// reduction -- lives in the file-scope array below, which every GPU that loads the
// library holds until the process exits.
#include <mutex>
#include <string>

#include "../../include/bsmpo.h"
#include "common.cuh"
#include "kernels.h"

namespace {

constexpr int NA_NT = 256;
// scratch: [0, chi) and [chi, 2 chi) environment vectors (ping-pong), then NA_NT partials
constexpr size_t NA_SCRATCH_ENTRIES = 2 * (size_t)BSMPO_NOALLOC_MAX_CHI + NA_NT;

static __device__ __align__(256) cplx g_noalloc_scratch[NA_SCRATCH_ENTRIES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_setup_mutex;
cplx* g_scratch_dev[NA_MAX_DEVICES] = {nullptr};

__device__ __forceinline__ bool na_diag(int2 c, int d) { return c.x < d && c.x == c.y; }

// R[i] = 1 on the occupied ket == bra slots of the last bond
__global__ void na_init_kernel(int d, int chi, const int2* __restrict__ cb, cplx* __restrict__ r) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < chi; i += gridDim.x * blockDim.x)
    r[i] = na_diag(cb[i], d) ? cmake(1.0, 0.0) : cmake(0.0, 0.0);
}

// r_out[a] = mask_b(a) sum_j gamma_b[a][j] r_in[j], one warp per row; lam == nullptr on
// the edge bond 0 (its Lambda is 1 on every occupied slot)
__global__ void na_step_kernel(int d, int chi, const cplx* __restrict__ g, const int2* __restrict__ cb,
                               const double* __restrict__ lam, const cplx* __restrict__ rin,
                               cplx* __restrict__ rout) {
  const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (a >= chi) return;
  cplx acc = cmake(0.0, 0.0);
  const bool ok = na_diag(cb[a], d) && (lam == nullptr || lam[a] > 0.0);
  if (ok)
    for (int j = lane; j < chi; j += 32) cfma(acc, ldc(g + (int64_t)a * chi + j), ldc(rin + j));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  if (lane == 0) rout[a] = acc;
}

// trace = sum_a r[a], one CTA, fixed-order tree (partials kept in the scratch array)
__global__ void na_sum_kernel(int chi, const cplx* __restrict__ r, cplx* __restrict__ part,
                              double* __restrict__ out) {
  cplx acc = cmake(0.0, 0.0);
  for (int i = threadIdx.x; i < chi; i += NA_NT) acc = cadd(acc, r[i]);
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int s = NA_NT / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) part[threadIdx.x] = cadd(part[threadIdx.x], part[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = part[0].x;
    out[1] = part[0].y;
  }
}

int na_fail(int code, const std::string& msg) {
  set_global_error(msg.c_str());
  return code;
}

// device address of the scratch array on the current device, looked up once per device
int na_scratch(cplx** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return na_fail(BSMPO_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= NA_MAX_DEVICES) return na_fail(BSMPO_EINVAL, "device index out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return na_fail(BSMPO_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_dev[dev] = static_cast<cplx*>(p);
  }
  *out = g_scratch_dev[dev];
  return BSMPO_OK;
}

}  // namespace

extern "C" int bsmpo_trace_noalloc(int n, int d, int chi, const void* gamma, const double* lambda,
                                   const int* charge, double* trace_out, void* stream) {
  if (n < 2 || d < 1 || d > BSMPO_MAX_D || chi < 1)
    return na_fail(BSMPO_EINVAL, "bsmpo_trace_noalloc: bad n, d or chi");
  if (chi > BSMPO_NOALLOC_MAX_CHI)
    return na_fail(BSMPO_EINVAL, "bsmpo_trace_noalloc: chi = " + std::to_string(chi) +
                                     " exceeds the allocation-free limit " +
                                     std::to_string(BSMPO_NOALLOC_MAX_CHI));
  if (!gamma || !lambda || !charge || !trace_out)
    return na_fail(BSMPO_EINVAL, "bsmpo_trace_noalloc: null pointer");
  // an error left by earlier, unrelated work is reported as such, not as ours
  cudaError_t pe = cudaPeekAtLastError();
  if (pe != cudaSuccess)
    return na_fail(BSMPO_ECUDA, std::string("bsmpo_trace_noalloc: pending CUDA error from earlier work: ") +
                                    cudaGetErrorString(pe));
  cudaStream_t st = (cudaStream_t)stream;
  // the scratch address is per device: the stream must belong to the current device
  int cur = -1, sdev = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e == cudaSuccess) e = cudaStreamGetDevice(st, &sdev);
  if (e != cudaSuccess)
    return na_fail(BSMPO_ECUDA, std::string("bsmpo_trace_noalloc: ") + cudaGetErrorString(e));
  if (sdev != cur)
    return na_fail(BSMPO_EINVAL, "bsmpo_trace_noalloc: the stream belongs to device " +
                                     std::to_string(sdev) + ", the current device is " +
                                     std::to_string(cur));
  cplx* scratch = nullptr;
  int rc = na_scratch(&scratch);
  if (rc) return rc;
  const cplx* G = reinterpret_cast<const cplx*>(gamma);
  const int2* C = reinterpret_cast<const int2*>(charge);
  const int64_t chi2 = (int64_t)chi * chi;
  cplx* r[2] = {scratch, scratch + chi};
  cplx* part = scratch + 2 * (size_t)BSMPO_NOALLOC_MAX_CHI;
  auto launched = [](const char* what) -> int {
    const cudaError_t le = cudaGetLastError();
    if (le == cudaSuccess) return BSMPO_OK;
    return na_fail(BSMPO_ECUDA, std::string("bsmpo_trace_noalloc: ") + what + ": " + cudaGetErrorString(le));
  };
  na_init_kernel<<<ceil_div(chi, 256), 256, 0, st>>>(d, chi, C + (int64_t)n * chi, r[n & 1]);
  if ((rc = launched("init"))) return rc;
  for (int b = n - 1; b >= 0; --b) {
    // R_b from R_{b+1}; bond b's Lambda is lambda[b-1] for interior bonds
    na_step_kernel<<<ceil_div(chi * 32, 256), 256, 0, st>>>(
        d, chi, G + (int64_t)b * chi2, C + (int64_t)b * chi, b > 0 ? lambda + (int64_t)(b - 1) * chi : nullptr,
        r[(b + 1) & 1], r[b & 1]);
    if ((rc = launched("environment step"))) return rc;
  }
  na_sum_kernel<<<1, NA_NT, 0, st>>>(chi, r[0], part, trace_out);
  return launched("sum");
}
