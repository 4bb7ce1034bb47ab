// Allocation-free pair scoring: swe_score_pairs_noalloc.
//
// Some callers cannot call cudaMalloc: real-time or embedded hosts that must
// not touch the device allocator once they have started, and programs whose
// device memory is all owned by their own pooling allocator, which this
// library cannot see or grow.  They already hold their inputs and outputs on
// the device; this entry point scores pairs from those buffers and allocates
// nothing.
//
// The 32-bit wavefront needs one scratch column per warp for sequences longer
// than one 512-column chunk.  Here that scratch is a file-scope device array of
// NOALLOC_SCRATCH_INTS ints (4 MiB, held by every GPU that loads the library
// until the process exits).  Each warp gets max_len + 1 ints of it, so a call
// runs min(1024, 2^20 / (max_len + 1)) warps; the longest sequence a call may
// reference is SWE_NOALLOC_MAX_LEN symbols.  A second static word counts the
// pairs that reference a sequence longer than the caller's max_len; every
// call clears it before its kernel runs.
//
// Host code cannot pass the arrays' names to a kernel (on the host they are
// only stand-ins for the device symbols), so the device addresses are looked
// up with cudaGetSymbolAddress, with the device current, on the first call
// made on it, and kept together with the CUDA context that was current then:
// a call from another context of the same device (one a driver-API caller
// made current) looks them up again.  A cudaDeviceReset invalidates them, and
// the context made after it may carry the old handle, so the call is not
// meant to be used after a reset.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "swgpu.h"
#include "sw_kernels.cuh"
#include "sw_wavefront32.cuh"

namespace swgpu {

constexpr int NOALLOC_SCRATCH_INTS = 1 << 20;
static __device__ __align__(256) int g_noalloc_scratch[NOALLOC_SCRATCH_INTS];
// pairs of the current call whose sequence is longer than max_len
static __device__ __align__(256) unsigned g_noalloc_rejected;

struct NoAllocParams {
  const char* seqs;      // sequence bytes; sequence i starts at seqs + off[i]
  const int64_t* off;
  const int* len;
  const int* pairs;      // 2 * npairs indices (a, b)
  long long npairs;
  unsigned* out;         // npairs distances
  int max_len;
  int* scratch;          // device address of g_noalloc_scratch
  unsigned* rejected;    // device address of g_noalloc_rejected
  long long stride;      // ints per warp = max_len + 1
  int nwarps;
};

// One warp per pair, like the explicit-pair mode of generic_kernel, but the
// sequences are caller-owned C strings (the effective symbols are s[1..len])
// and the boundary columns live in the static scratch array.
__global__ void __launch_bounds__(256) noalloc_pairs_kernel(NoAllocParams p) {
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  if (gw >= p.nwarps) return;
  int* scratch = p.scratch + (long long)gw * p.stride;
  for (long long w = gw; w < p.npairs; w += p.nwarps) {
    const int ia = p.pairs[2 * w], ib = p.pairs[2 * w + 1];
    const int la = p.len[ia], lb = p.len[ib];
    if (la > p.max_len || lb > p.max_len || la < 0 || lb < 0) {
      // longer than the caller declared: the scratch slice would overflow
      if (lane == 0) {
        p.out[w] = 0xFFFFFFFFu;
        atomicAdd(p.rejected, 1u);
      }
      continue;
    }
    const uint8_t* A = reinterpret_cast<const uint8_t*>(p.seqs + p.off[ia]) + 1;
    const uint8_t* B = reinterpret_cast<const uint8_t*>(p.seqs + p.off[ib]) + 1;
    const uint8_t* R = A;
    const uint8_t* Cc = B;
    int lr = la, lc = lb;
    if (lc > lr) {
      R = B;
      Cc = A;
      lr = lb;
      lc = la;
    }
    const int best = sw32_warp(R, lr, Cc, lc, scratch, lane);
    if (lane == 0) p.out[w] = 4u * (unsigned)max(la, lb) - (unsigned)best;
  }
}

namespace {
std::mutex g_setup_mu;
struct DeviceSymbols {
  void* ctx = nullptr;  // the context current when the addresses were taken
  int* scratch = nullptr;
  unsigned* rejected = nullptr;
};
DeviceSymbols g_symbols[64];

// The calling thread's current CUDA context (driver API, reached through the
// runtime's entry-point query so the library needs no link to libcuda), or
// nullptr when there is none or the query is unavailable.
void* current_context() {
  typedef int (*CtxGetCurrentFn)(void**);
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (CtxGetCurrentFn) nullptr;
    }
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}
}  // namespace

}  // namespace swgpu

extern "C" swe_status swe_score_pairs_noalloc(const char* seqs, const int64_t* off, const int* len,
                                              const int* pairs, int64_t npairs, unsigned* out, int max_len,
                                              void* stream) {
  using namespace swgpu;
  if (npairs < 0 || max_len < 0 || max_len > SWE_NOALLOC_MAX_LEN) return SWE_ERR_INVALID;
  if (npairs == 0) return SWE_OK;
  if (!seqs || !off || !len || !pairs || !out) return SWE_ERR_INVALID;
  // an error left by the caller's own earlier work is theirs: report it, keep it
  if (cudaPeekAtLastError() != cudaSuccess) return SWE_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return SWE_ERR_NO_DEVICE;
  }
  DeviceSymbols sym;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    void* ctx = current_context();
    if (!g_symbols[dev].scratch || !ctx || ctx != g_symbols[dev].ctx) {
      void* a = nullptr;
      void* r = nullptr;
      if (cudaGetSymbolAddress(&a, g_noalloc_scratch) != cudaSuccess || !a ||
          cudaGetSymbolAddress(&r, g_noalloc_rejected) != cudaSuccess || !r) {
        cudaGetLastError();
        return SWE_ERR_CUDA;
      }
      g_symbols[dev].scratch = static_cast<int*>(a);
      g_symbols[dev].rejected = static_cast<unsigned*>(r);
      // the lookup sets up the device's primary context when none was current yet
      g_symbols[dev].ctx = ctx ? ctx : current_context();
    }
    sym = g_symbols[dev];
  }
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  NoAllocParams p;
  p.seqs = seqs;
  p.off = off;
  p.len = len;
  p.pairs = pairs;
  p.npairs = npairs;
  p.out = out;
  p.max_len = max_len;
  p.scratch = sym.scratch;
  p.rejected = sym.rejected;
  p.stride = (long long)max_len + 1;
  long long warps = NOALLOC_SCRATCH_INTS / p.stride;
  if (warps > 1024) warps = 1024;
  if (warps > npairs) warps = npairs;
  p.nwarps = (int)warps;
  const int blocks = (p.nwarps + 7) / 8;
  // the counter keeps the previous call's value: clear it first
  if (cudaMemsetAsync(sym.rejected, 0, sizeof(unsigned), st) != cudaSuccess) {
    cudaGetLastError();
    return SWE_ERR_CUDA;
  }
  noalloc_pairs_kernel<<<blocks, 256, 0, st>>>(p);
  if (cudaGetLastError() != cudaSuccess) return SWE_ERR_CUDA;
  unsigned rejected = 0;
  if (cudaMemcpyAsync(&rejected, sym.rejected, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return SWE_ERR_CUDA;
  }
  return rejected ? SWE_ERR_INVALID : SWE_OK;
}
