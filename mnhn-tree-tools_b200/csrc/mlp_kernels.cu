// Kernels of the learned prefilter (sm_100a).
//
//   kmer_kernel            k-mer counts per sequence (kmers.c semantics), L1-normalised
//   gemm_bf16_tn_kernel    C = A * B^T on the 5th-generation tensor cores: operand
//                          tiles arrive by TMA (128-byte swizzle) into a 4-stage
//                          shared-memory ring, one thread issues tcgen05.mma into a
//                          128 x 128 fp32 accumulator in tensor memory, and four
//                          warps read it back with tcgen05.ld for a fused epilogue
//                          (bias, GELU or GELU', bf16 / transposed bf16 / fp32
//                          outputs, column sums for bias gradients)
//   gather_rows_kernel     batch rows of the feature matrix as bf16 (+ transpose)
//   pair_loss_kernel       MSE between embedding distance and target, with dE
//   adam_kernel, publish_kernel
//   candidates_kernel      all pairs of a set: exact length bound + embedding margin
#include <cstdio>

#include "mlp_kernels.cuh"
#include "sw_device.cuh"

namespace swgpu {

// ---------------------------------------------------------------------------
// k-mer features
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) kmer_kernel(const uint8_t* __restrict__ codes,
                                                   const int64_t* __restrict__ code_off,
                                                   const int* __restrict__ len, const uint8_t* __restrict__ first_code,
                                                   int n, int k, float* __restrict__ out) {
  extern __shared__ int km_hist[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nb = 1 << (2 * k);
  int* hist = km_hist + warp * nb;
  for (int b = lane; b < nb; b += 32) hist[b] = 0;
  __syncwarp();
  const int gw = blockIdx.x * (blockDim.x >> 5) + warp, nw = gridDim.x * (blockDim.x >> 5);
  for (int i = gw; i < n; i += nw) {
    const int L = len[i];
    const uint8_t* c = codes + code_off[i];
    const uint8_t c0 = first_code[i];
    const int nwin = L > k ? L - k : 0;  // windows 0 .. L-k-1
    int valid = 0;
    for (int w = lane; w < nwin; w += 32) {
      int idx = 0;
      bool ok = true;
      for (int t = 0; t < k; ++t) {
        const int p = w + t;
        const uint8_t s = p == 0 ? c0 : c[p - 1];
        ok = ok && s < 4;
        idx |= (s & 3) << (2 * t);
      }
      if (ok) {
        atomicAdd(&hist[idx], 1);
        ++valid;
      }
    }
    for (int o = 16; o > 0; o >>= 1) valid += __shfl_xor_sync(0xFFFFFFFFu, valid, o);
    __syncwarp();
    const float inv = valid > 0 ? 1.0f / (float)valid : 0.0f;
    float* row = out + (long long)i * nb;
    for (int b = lane; b < nb; b += 32) {
      row[b] = (float)hist[b] * inv;
      hist[b] = 0;
    }
    __syncwarp();
  }
}

cudaError_t launch_kmer_features(const uint8_t* codes, const int64_t* code_off, const int* len,
                                 const uint8_t* first_code, int n, int k, float* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (k < 1 || k > 6) return cudaErrorInvalidValue;
  const size_t smem = (size_t)4 * (1u << (2 * k)) * sizeof(int);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kmer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int grid = (n + 3) / 4 < 148 * 8 ? (n + 3) / 4 : 148 * 8;
  kmer_kernel<<<grid, 128, smem, st>>>(codes, code_off, len, first_code, n, k, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// GELU (exact erf form)
// ---------------------------------------------------------------------------
__host__ __device__ float gelu_ref(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// ---------------------------------------------------------------------------
// tcgen05 / TMA building blocks (inline PTX)
// ---------------------------------------------------------------------------
constexpr int G_BM = 128, G_BK = 64, G_STAGES = 4;
constexpr int G_TILE_BYTES = G_BM * G_BK * 2;  // 16 KB: the A tile (128 x 64)
// Per tile width BN (128, or 64 when 128-wide tiles would leave SMs idle):
// the B tile (BN x 64), the stage, the tensor-memory columns of the
// accumulator and the instruction descriptor.
template <int BN>
struct GemmShape {
  static constexpr int B_BYTES = BN * G_BK * 2;
  static constexpr int STAGE_BYTES = G_TILE_BYTES + B_BYTES;
  static constexpr int TMEM_COLS = BN;  // a power of two >= 32
};
// Warp w drains accumulator rows 32*(w%4) .. +31 (the tensor-memory lanes its
// quarter may read) and 32 columns from 32*(w/4): 16 warps for 128-wide tiles
// (one CTA per SM), 8 for 64-wide ones (two CTAs per SM).  The epilogue runs
// after the tile's last MMA, so spreading it over more warps shortens the CTA.
template <int BN>
constexpr int gemm_threads() {
  return BN == 128 ? 512 : 256;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// D[tmem] (+)= A[smem desc] * B[smem desc]^T, kind::f16 (bf16 inputs, fp32 accumulator)
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major operand tile written by TMA
// with 128-byte swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart
// (stride byte offset), leading byte offset unused (1), descriptor version 1,
// layout type 2 = 128-byte swizzle.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor: fp32 accumulator, bf16 A and B, both K-major,
// N = BN (bits 17-22 hold N/8), M = 128 (bits 24-28 hold M/16).
template <int BN>
__host__ __device__ constexpr uint32_t gemm_idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(G_BM >> 4) << 24);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// One CTA per 128 x BN tile of C.  Warp 0 lane 0 feeds the stage ring with
// TMA, warp 1 lane 0 issues the MMAs (4 per 64-wide K step) and commits each
// stage back to the producer; then every warp drains its part of the accumulator.
template <int BN>
__global__ void __launch_bounds__(gemm_threads<BN>(), BN == 64 ? 2 : 1)
    gemm_bf16_tn_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, int M, int N,
                        int K, GemmEpi ep) {
  using S = GemmShape<BN>;
  extern __shared__ uint8_t g_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(g_smem_raw) + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full_bar[G_STAGES], empty_bar[G_STAGES], done_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int s_issued, s_consumed;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * G_BM, n0 = blockIdx.x * BN;
  const int nk = K / G_BK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < G_STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    s_issued = 0;
    s_consumed = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(S::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == 0 && lane == 0) {  // producer
    int kt = 0;
    for (; kt < nk; ++kt) {
      const int s = kt % G_STAGES, use = kt / G_STAGES;
      if (use > 0 && !mbar_wait_bounded(&empty_bar[s], (unsigned)((use - 1) & 1), ep.wait_limit)) {
        atomicOr(ep.status, KST_TIMEOUT);
        break;
      }
      uint8_t* a_tile = smem + s * S::STAGE_BYTES;
      uint8_t* b_tile = a_tile + G_TILE_BYTES;
      mbar_arrive_expect_tx(&full_bar[s], S::STAGE_BYTES);
      tma_load_2d(a_tile, &ta, kt * G_BK, m0, &full_bar[s]);
      tma_load_2d(b_tile, &tb, kt * G_BK, n0, &full_bar[s]);
    }
    s_issued = kt;
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    int kt = 0;
    for (; kt < nk; ++kt) {
      const int s = kt % G_STAGES, use = kt / G_STAGES;
      if (!mbar_wait_bounded(&full_bar[s], (unsigned)(use & 1), ep.wait_limit)) {
        atomicOr(ep.status, KST_TIMEOUT);
        break;
      }
      tc_fence_after();
      const uint64_t adesc = sw128_desc(smem_u32(smem + s * S::STAGE_BYTES));
      const uint64_t bdesc = sw128_desc(smem_u32(smem + s * S::STAGE_BYTES + G_TILE_BYTES));
#pragma unroll
      for (int k = 0; k < G_BK / 16; ++k)  // 16 bf16 = 32 bytes per MMA step along K
        tc_mma(tmem, adesc + 2 * k, bdesc + 2 * k, gemm_idesc<BN>(), (kt | k) != 0 ? 1u : 0u);
      tc_commit(&empty_bar[s]);  // the stage is free once these MMAs have read it
    }
    s_consumed = kt;
    tc_commit(&done_bar);  // accumulator complete
  }
  __syncwarp();

  // epilogue: warp w drains rows 32*(w%4) .. +31 (its tensor-memory lane
  // quarter) and columns 32*(w/4) .. +31
  int ok = 0;
  if (lane == 0) ok = mbar_wait_bounded(&done_bar, 0, ep.wait_limit) ? 1 : 0;
  ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
  if (!ok && lane == 0) atomicOr(ep.status, KST_TIMEOUT);
  tc_fence_after();
  const int quarter = warp & 3, slice = warp >> 2;
  const int m = m0 + quarter * 32 + lane;
  if (ok) {
    for (int c = slice * 32; c < slice * 32 + 32; c += 16) {
      uint32_t r[16];
      tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c, r);
      const long long rowoff = (long long)m * N + n0 + c;
      float v[16];
      if (ep.gelu_in) {
        const float4* gi = reinterpret_cast<const float4*>(ep.gelu_in + rowoff);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 z = gi[q];
          v[4 * q] = z.x, v[4 * q + 1] = z.y, v[4 * q + 2] = z.z, v[4 * q + 3] = z.w;
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]) * gelu_grad(v[j]);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
      }
      if (ep.bias) {
        const float4* bb = reinterpret_cast<const float4*>(ep.bias + n0 + c);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 b = bb[q];
          v[4 * q] += b.x, v[4 * q + 1] += b.y, v[4 * q + 2] += b.z, v[4 * q + 3] += b.w;
        }
      }
      if (ep.out_pre) {
        float4* o = reinterpret_cast<float4*>(ep.out_pre + rowoff);
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      }
      if (ep.act) {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = gelu_ref(v[j]);
      }
      if (ep.out_f32) {
        float4* o = reinterpret_cast<float4*>(ep.out_f32 + rowoff);
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      }
      if (ep.out_bf16) {  // 16 values = two 16-byte stores
        uint32_t w[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
          w[q] = *reinterpret_cast<const uint32_t*>(&h2);
        }
        uint4* o = reinterpret_cast<uint4*>(ep.out_bf16 + rowoff);
        o[0] = make_uint4(w[0], w[1], w[2], w[3]);
        o[1] = make_uint4(w[4], w[5], w[6], w[7]);
      }
      if (ep.out_bf16_t) {  // lanes hold consecutive rows: each store is one 64-byte run
#pragma unroll
        for (int j = 0; j < 16; ++j) ep.out_bf16_t[(long long)(n0 + c + j) * M + m] = __float2bfloat16_rn(v[j]);
      }
      if (ep.colsum_part) {  // this warp's 32 rows: one partial row of the column sums
        float* part = ep.colsum_part + (long long)(m0 / 32 + quarter) * N + n0 + c;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          float t = v[j];
          for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
          if (lane == 0) part[j] = t;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    // copies issued but never consumed (after a timeout) land before the CTA leaves
    for (int kt = s_consumed; kt < s_issued; ++kt)
      mbar_wait_bounded(&full_bar[kt % G_STAGES], (unsigned)((kt / G_STAGES) & 1), ep.wait_limit);
  }
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TMEM_COLS)
                 : "memory");
  }
}

__global__ void colsum_reduce_kernel(const float* __restrict__ part, int rows, int N, float* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += part[(long long)r * N + n];
  out[n] = s;
}

cudaError_t launch_colsum_reduce(const float* part, int rows, int N, float* out, cudaStream_t st) {
  if (N <= 0) return cudaSuccess;
  colsum_reduce_kernel<<<(N + 127) / 128, 128, 0, st>>>(part, rows, N, out);
  return cudaGetLastError();
}

size_t gemm_smem_bytes(int bn) {
  return (size_t)G_STAGES * (bn == 64 ? GemmShape<64>::STAGE_BYTES : GemmShape<128>::STAGE_BYTES) + 1024;
}

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// Tensor map of a row-major bf16 [rows x cols] matrix, box 64 (cols) x box_rows, 128-byte swizzle.
cudaError_t make_map(CUtensorMap* map, const __nv_bfloat16* base, int rows, int cols, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  const cuuint32_t box[2] = {(cuuint32_t)G_BK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace

int gemm_force_bn = 0;

static cudaError_t launch_gemm_bn(int bn, const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K,
                                  const GemmEpi& ep, cudaStream_t st) {
  CUtensorMap ma, mb;
  cudaError_t e = make_map(&ma, A, M, K, G_BM);
  if (e == cudaSuccess) e = make_map(&mb, B, N, K, bn);
  if (e != cudaSuccess) return e;
  static bool attr64 = false, attr128 = false;
  bool& attr = bn == 64 ? attr64 : attr128;
  auto kern = bn == 64 ? gemm_bf16_tn_kernel<64> : gemm_bf16_tn_kernel<128>;
  if (!attr) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem_bytes(bn));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  dim3 grid(N / bn, M / G_BM);
  kern<<<grid, bn == 64 ? gemm_threads<64>() : gemm_threads<128>(), gemm_smem_bytes(bn), st>>>(ma, mb, M, N, K, ep);
  return cudaGetLastError();
}

cudaError_t launch_gemm_bf16_tn(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K,
                                const GemmEpi& ep, cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0 || M % G_BM || N % 64 || K % G_BK) return cudaErrorInvalidValue;
  // operands and every epilogue array are read and written in 16-byte units
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(ep.bias) |
       reinterpret_cast<uintptr_t>(ep.gelu_in) | reinterpret_cast<uintptr_t>(ep.out_pre) |
       reinterpret_cast<uintptr_t>(ep.out_f32) | reinterpret_cast<uintptr_t>(ep.out_bf16)) & 15)
    return cudaErrorInvalidValue;
  // 128-wide tiles unless fewer than half the SMs would get one (or N is not
  // a multiple of 128): then 64-wide tiles, two CTAs per SM.  Measured on
  // B200 with M = 4,096: N = 256 and 128 (64 and 32 tiles) 13.5 -> 11.4 and
  // 9.8 -> 8.4 us; N = 512 (128 tiles) 16.5 -> 17.7 us, so it keeps 128.
  int dev = 0, sms = 148;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int bn = (N % 128 != 0 || 2LL * (M / G_BM) * (N / 128) < sms) ? 64 : 128;
  if (gemm_force_bn == 64 || gemm_force_bn == 128) {
    if (gemm_force_bn == 128 && N % 128) return cudaErrorInvalidValue;
    return launch_gemm_bn(gemm_force_bn, A, B, M, N, K, ep, st);
  }
  return launch_gemm_bn(bn, A, B, M, N, K, ep, st);
}

// ---------------------------------------------------------------------------
// training-step helpers
// ---------------------------------------------------------------------------
__global__ void gather_rows_kernel(const float* __restrict__ X, int D, const int* __restrict__ idx, int rows, int M,
                                   float scale, __nv_bfloat16* __restrict__ out, __nv_bfloat16* __restrict__ out_t) {
  __shared__ float tile[32][33];
  const int r0 = blockIdx.y * 32, d0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  for (int rr = ty; rr < 32; rr += 8) {
    const int r = r0 + rr, d = d0 + tx;
    float v = 0.f;
    if (r < rows && d < D) v = scale * X[(long long)idx[r] * D + d];
    tile[rr][tx] = v;
    if (r < M && d < D) out[(long long)r * D + d] = __float2bfloat16_rn(v);
  }
  __syncthreads();
  if (out_t)
    for (int dd = ty; dd < 32; dd += 8) {
      const int d = d0 + dd, r = r0 + tx;
      if (d < D && r < M) out_t[(long long)d * M + r] = __float2bfloat16_rn(tile[tx][dd]);
    }
}

cudaError_t launch_gather_rows(const float* X, int D, const int* idx, int rows, int M, float scale,
                               __nv_bfloat16* out, __nv_bfloat16* out_t, cudaStream_t st) {
  dim3 grid((D + 31) / 32, (M + 31) / 32);
  gather_rows_kernel<<<grid, 256, 0, st>>>(X, D, idx, rows, M, scale, out, out_t);
  return cudaGetLastError();
}

__global__ void pair_loss_kernel(const float* __restrict__ E, int D, const float* __restrict__ target, int P, int M,
                                 float* loss, __nv_bfloat16* __restrict__ dE, __nv_bfloat16* __restrict__ dE_t,
                                 const float* __restrict__ w_over) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int p = gw; p < P; p += nw) {
    const float* ea = E + (long long)(2 * p) * D;
    const float* eb = ea + D;
    float s = 0.f;
    for (int d = lane; d < D; d += 32) {
      const float x = ea[d] - eb[d];
      s += x * x;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    const float dist = sqrtf(s);
    const float r = dist - target[p];
    const float w = (w_over && r > 0.f) ? w_over[p] : 1.0f;  // an over-estimate may weigh more
    if (lane == 0) atomicAdd(loss, w * r * r / (float)P);
    const float c = dist > 1e-20f ? 2.0f * w * r / ((float)P * dist) : 0.0f;
    for (int d = lane; d < D; d += 32) {
      const float g = c * (ea[d] - eb[d]);
      const __nv_bfloat16 gp = __float2bfloat16_rn(g), gn = __float2bfloat16_rn(-g);
      dE[(long long)(2 * p) * D + d] = gp;
      dE[(long long)(2 * p + 1) * D + d] = gn;
      dE_t[(long long)d * M + 2 * p] = gp;
      dE_t[(long long)d * M + 2 * p + 1] = gn;
    }
  }
}

cudaError_t launch_pair_loss(const float* E, int D, const float* target, int P, int M, float* loss,
                             __nv_bfloat16* dE, __nv_bfloat16* dE_t, const float* w_over, cudaStream_t st) {
  // the loss depends on embedding differences only: the last layer's bias gradient is zero
  if (P <= 0) return cudaSuccess;
  const int grid = (P + 7) / 8 < 148 * 4 ? (P + 7) / 8 : 148 * 4;
  pair_loss_kernel<<<grid, 256, 0, st>>>(E, D, target, P, M, loss, dE, dE_t, w_over);
  return cudaGetLastError();
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float bc1,
                            float bc2, float wd) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * ((mi / bc1) / (sqrtf(vi / bc2) + eps) + wd * w[i]);
  }
}

cudaError_t launch_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                        float eps, float bc1, float bc2, float wd, cudaStream_t st) {
  adam_kernel<<<148 * 4, 256, 0, st>>>(w, g, m, v, n, lr, b1, b2, eps, bc1, bc2, wd);
  return cudaGetLastError();
}

__global__ void publish_kernel(const float* __restrict__ W, int R, int C, __nv_bfloat16* __restrict__ Wb,
                               __nv_bfloat16* __restrict__ Wt) {
  __shared__ float tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int rr = ty; rr < 32; rr += 8) {
    const int r = r0 + rr, c = c0 + tx;
    const float v = (r < R && c < C) ? W[(long long)r * C + c] : 0.f;
    tile[rr][tx] = v;
    if (r < R && c < C) Wb[(long long)r * C + c] = __float2bfloat16_rn(v);
  }
  __syncthreads();
  for (int cc = ty; cc < 32; cc += 8) {
    const int c = c0 + cc, r = r0 + tx;
    if (c < C && r < R) Wt[(long long)c * R + r] = __float2bfloat16_rn(tile[tx][cc]);
  }
}

cudaError_t launch_publish(const float* W, int R, int C, __nv_bfloat16* Wb, __nv_bfloat16* Wt, cudaStream_t st) {
  dim3 grid((C + 31) / 32, (R + 31) / 32);
  publish_kernel<<<grid, 256, 0, st>>>(W, R, C, Wb, Wt);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// candidates: 64 x 64 position tiles of one set, upper triangle
// ---------------------------------------------------------------------------
constexpr int C_T = 64;

template <int D>
__global__ void __launch_bounds__(256) candidates_kernel(const float* __restrict__ emb, const int* __restrict__ orig,
                                                         const int* __restrict__ len, int first, int n, long long T,
                                                         MarginTable margins, int use_emb, int2* __restrict__ pairs,
                                                         unsigned long long cap, unsigned long long* count,
                                                         uint32_t* __restrict__ keys, uint8_t* __restrict__ has) {
  extern __shared__ float c_smem[];
  float (*ei)[D + 1] = reinterpret_cast<float (*)[D + 1]>(c_smem);
  float (*ej)[D + 1] = reinterpret_cast<float (*)[D + 1]>(c_smem + C_T * (D + 1));
  __shared__ int li[C_T], lj[C_T], oi[C_T], oj[C_T];
  const int nt = (n + C_T - 1) / C_T;
  const long long ntiles = (long long)nt * (nt + 1) / 2;
  const int lane = threadIdx.x & 31;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    // tile t -> (bi, bj) with bi <= bj, row-major over the upper triangle
    int bi = 0;
    long long rem = t;
    while (rem >= nt - bi) {
      rem -= nt - bi;
      ++bi;
    }
    const int bj = bi + (int)rem;
    const int i0 = bi * C_T, j0 = bj * C_T;
    __syncthreads();
    for (int x = threadIdx.x; x < C_T; x += blockDim.x) {
      const int pi = i0 + x, pj = j0 + x;
      oi[x] = pi < n ? orig[first + pi] : -1;
      oj[x] = pj < n ? orig[first + pj] : -1;
      li[x] = pi < n ? len[oi[x]] : 0;
      lj[x] = pj < n ? len[oj[x]] : 0;
    }
    __syncthreads();
    if (use_emb) {
      for (int x = threadIdx.x; x < C_T * D; x += blockDim.x) {
        const int r = x / D, d = x % D;
        ei[r][d] = oi[r] >= 0 ? emb[(long long)oi[r] * D + d] : 0.f;
        ej[r][d] = oj[r] >= 0 ? emb[(long long)oj[r] * D + d] : 0.f;
      }
      __syncthreads();
    }
    // each thread: a 4 x 4 block of pairs (rows ty*4.., cols tx*4..) of the 64 x 64 tile
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4] = {};
    if (use_emb) {
      for (int d = 0; d < D; ++d) {
        float a[4], b[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          a[q] = ei[ty * 4 + q][d];
          b[q] = ej[tx * 4 + q][d];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const float df = a[q] - b[r];
            acc[q][r] = fmaf(df, df, acc[q][r]);
          }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int xi = ty * 4 + q, xj = tx * 4 + r;
        const int pi = i0 + xi, pj = j0 + xj;
        bool cand = pi < n && pj < n && pi < pj;
        uint32_t key = 0;
        if (cand) {
          const int la = li[xi], lb = lj[xj];
          const int mx = la > lb ? la : lb, mn = la > lb ? lb : la;
          cand = 4LL * (mx - mn) <= T;
          if (cand && use_emb) {
            float m = margins.m[margins.n - 1];
            for (int b = 0; b < margins.n - 1; ++b)
              if (mx < margins.upper[b]) {
                m = margins.m[b];
                break;
              }
            const float thr0 = (float)T / (4.0f * (float)(mx > 0 ? mx : 1));
            const float thr = thr0 + m;
            cand = thr >= 0.f && acc[q][r] <= thr * thr;
            // squared embedding distance over the squared threshold: the
            // grouping's edge order (a non-negative float's bits order like it)
            key = __float_as_uint(thr0 > 0.f ? acc[q][r] / (thr0 * thr0) : acc[q][r]);
          }
        }
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, cand);
        if (bal) {
          unsigned long long base = 0;
          if (lane == 0) base = atomicAdd(count, (unsigned long long)__popc(bal));
          base = __shfl_sync(0xFFFFFFFFu, base, 0);
          if (cand) {
            const unsigned long long at = base + __popc(bal & ((1u << lane) - 1u));
            if (at < cap) {
              pairs[at] = make_int2(oi[xi], oj[xj]);
              if (keys) keys[at] = key;
            }
            if (has) {
              has[oi[xi]] = 1;
              has[oj[xj]] = 1;
            }
          }
        }
      }
  }
}

cudaError_t launch_candidates(const float* emb, int D, const int* orig, const int* len, int first, int n,
                              long long T, const MarginTable& margins, int use_emb, int2* pairs,
                              uint32_t* keys, unsigned long long cap, unsigned long long* count, uint8_t* has,
                              cudaStream_t st) {
  if (margins.n < 1 || margins.n > MARGIN_BUCKETS) return cudaErrorInvalidValue;
  if (n <= 1) return cudaSuccess;
  if (D != 128) return cudaErrorInvalidValue;
  const long long nt = (n + C_T - 1) / C_T;
  const long long ntiles = nt * (nt + 1) / 2;
  const int grid = (int)(ntiles < 148 * 4 ? ntiles : 148 * 4);
  const size_t smem = use_emb ? (size_t)2 * C_T * (128 + 1) * sizeof(float) : 0;
  if (smem) {
    cudaError_t e = cudaFuncSetAttribute(candidates_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  candidates_kernel<128><<<grid, 256, smem, st>>>(emb, orig, len, first, n, T, margins, use_emb, pairs, cap,
                                                  count, keys, has);
  return cudaGetLastError();
}

__global__ void pair_dist_kernel(const float* __restrict__ emb, int D, const int* __restrict__ a,
                                 const int* __restrict__ b, long long np, float* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long p = gw; p < np; p += nw) {
    const float* x = emb + (long long)a[p] * D;
    const float* y = emb + (long long)b[p] * D;
    float s = 0.f;
    for (int d = lane; d < D; d += 32) {
      const float t = x[d] - y[d];
      s = fmaf(t, t, s);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if (lane == 0) out[p] = sqrtf(s);
  }
}

cudaError_t launch_pair_dist(const float* emb, int D, const int* a, const int* b, long long np, float* out,
                             cudaStream_t st) {
  if (np <= 0) return cudaSuccess;
  const long long g = (np + 7) / 8;
  pair_dist_kernel<<<(int)(g < 148 * 8 ? g : 148 * 8), 256, 0, st>>>(emb, D, a, b, np, out);
  return cudaGetLastError();
}

}  // namespace swgpu
