// Point datasets (k-mer frequency vectors, PCA projections) with the L1 / L2
// distances of dbscan_L1 / dbscan_L2 (dbscan.c:563-779): every pair's
// distance in one launch into the engine's 32-bit distance matrix, after which
// the threshold kernel, the DBSCAN replay and the adaptive sweep run unchanged.
//
// Exactness.  The reference's AVX path accumulates, per pair, over the
// dimensions in order: L2 dist = fma(a-b, a-b, dist) (dbscan.c:661-665, an
// FMA build), L1 dist = dist + |a-b| (dbscan.c:672-675), starting from +0.
// point_dist_kernel does the same operations in the same order with
// explicitly rounded intrinsics, so every distance has the reference's bits.
// Since fl(a-b) = -fl(b-a), the matrix is exactly symmetric and each upper
// triangle tile writes both halves.  Distances are never -0, so their bit
// patterns order like the floats; NaN patterns sort above +inf and never pass
// a threshold, as NaN <= eps is false.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "staging.cuh"

namespace swgpu {
namespace {

constexpr int PT_TILE = 128;   // points per tile side
constexpr int PT_KC = 16;      // dimensions per shared-memory stage
constexpr int PT_THREADS = 256;

// Two float32 values in one 64-bit register (x in the low half) and back.
__device__ __forceinline__ uint64_t pack2(float x, float y) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ void unpack2(uint64_t v, float& x, float& y) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(v));
}
// Element-wise float32 pairs, each element rounded as its scalar operation.
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// One CTA per upper-triangle tile (bi <= bj) of 128 x 128 pairs; each thread
// holds 8 x 8 pairs: rows i0 + {ty*4 .. ty*4+3, 64+ty*4 .. 64+ty*4+3}, the
// same pattern of columns from tx.  Operands stream through shared memory in
// stages of 16 dimensions, the next stage loaded into registers while the
// current one is used.  L2 works on float32 pairs (sub.f32x2 / fma.f32x2:
// two columns per instruction, each element rounded exactly as the scalar
// operation), with the A operand stored twice in shared memory so that a pair
// (a, a) is one 8-byte load; L1 stays scalar (its |a-b| has no pair form).
template <int METRIC, bool VEC>
__global__ void __launch_bounds__(PT_THREADS, 2)
    point_dist_kernel(const float* __restrict__ V, int64_t n_pad, int n, int dims, const int2* __restrict__ tiles,
                      int ntiles, uint32_t* __restrict__ D, unsigned* __restrict__ max_bits) {
  constexpr bool PAIRS = METRIC == SWE_METRIC_L2;
  constexpr int AW = PAIRS ? 2 * PT_TILE : PT_TILE;  // floats per A row of a stage
  __shared__ __align__(16) float sA[2][PT_KC][AW];
  __shared__ __align__(16) float sB[2][PT_KC][PT_TILE];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  unsigned local_max = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int i0 = tiles[t].x * PT_TILE, j0 = tiles[t].y * PT_TILE;
    float acc[8][8];
    uint64_t acc2[8][4];  // the L2 accumulators as pairs of columns (2cp, 2cp+1)
#pragma unroll
    for (int r = 0; r < 8; ++r) {
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[r][c] = 0.0f;
#pragma unroll
      for (int cp = 0; cp < 4; ++cp) acc2[r][cp] = 0ull;  // +0.0f in both halves
    }
    // stage loads: 2 x 512 float4 per stage, 2 + 2 per thread
    float4 ra[2], rb[2];
    auto fetch = [&](int k0) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int q = threadIdx.x + h * PT_THREADS;  // 0..511
        const int kk = q >> 5, c4 = (q & 31) * 4;
        if (k0 + kk < dims) {
          ra[h] = *reinterpret_cast<const float4*>(V + (int64_t)(k0 + kk) * n_pad + i0 + c4);
          rb[h] = *reinterpret_cast<const float4*>(V + (int64_t)(k0 + kk) * n_pad + j0 + c4);
        } else {
          ra[h] = make_float4(0.f, 0.f, 0.f, 0.f);
          rb[h] = ra[h];
        }
      }
    };
    auto stash = [&](int buf) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int q = threadIdx.x + h * PT_THREADS;
        const int kk = q >> 5, c4 = (q & 31) * 4;
        if (PAIRS) {  // each A value twice: (a0, a0, a1, a1), (a2, a2, a3, a3)
          *reinterpret_cast<float4*>(&sA[buf][kk][2 * c4]) = make_float4(ra[h].x, ra[h].x, ra[h].y, ra[h].y);
          *reinterpret_cast<float4*>(&sA[buf][kk][2 * c4 + 4]) = make_float4(ra[h].z, ra[h].z, ra[h].w, ra[h].w);
        } else {
          *reinterpret_cast<float4*>(&sA[buf][kk][c4]) = ra[h];
        }
        *reinterpret_cast<float4*>(&sB[buf][kk][c4]) = rb[h];
      }
    };
    fetch(0);
    __syncthreads();  // the previous tile's last stage is no longer read
    stash(0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < dims; k0 += PT_KC) {
      const bool more = k0 + PT_KC < dims;
      if (more) fetch(k0 + PT_KC);
      const int kc = min(PT_KC, dims - k0);
      if (PAIRS) {
        for (int kk = 0; kk < kc; ++kk) {
          const float4 p0 = *reinterpret_cast<const float4*>(&sA[buf][kk][2 * (ty * 4)]);
          const float4 p1 = *reinterpret_cast<const float4*>(&sA[buf][kk][2 * (ty * 4) + 4]);
          const float4 p2 = *reinterpret_cast<const float4*>(&sA[buf][kk][2 * (64 + ty * 4)]);
          const float4 p3 = *reinterpret_cast<const float4*>(&sA[buf][kk][2 * (64 + ty * 4) + 4]);
          const float4 b0 = *reinterpret_cast<const float4*>(&sB[buf][kk][tx * 4]);
          const float4 b1 = *reinterpret_cast<const float4*>(&sB[buf][kk][64 + tx * 4]);
          const uint64_t ap[8] = {pack2(p0.x, p0.y), pack2(p0.z, p0.w), pack2(p1.x, p1.y), pack2(p1.z, p1.w),
                                  pack2(p2.x, p2.y), pack2(p2.z, p2.w), pack2(p3.x, p3.y), pack2(p3.z, p3.w)};
          const uint64_t bp[4] = {pack2(b0.x, b0.y), pack2(b0.z, b0.w), pack2(b1.x, b1.y), pack2(b1.z, b1.w)};
#pragma unroll
          for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int cp = 0; cp < 4; ++cp) {
              const uint64_t d = sub2(ap[r], bp[cp]);
              acc2[r][cp] = fma2(d, d, acc2[r][cp]);
            }
        }
      } else
      for (int kk = 0; kk < kc; ++kk) {
        const float4 a0 = *reinterpret_cast<const float4*>(&sA[buf][kk][ty * 4]);
        const float4 a1 = *reinterpret_cast<const float4*>(&sA[buf][kk][64 + ty * 4]);
        const float4 b0 = *reinterpret_cast<const float4*>(&sB[buf][kk][tx * 4]);
        const float4 b1 = *reinterpret_cast<const float4*>(&sB[buf][kk][64 + tx * 4]);
        const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
        const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            const float d = __fsub_rn(a[r], b[c]);
            acc[r][c] = METRIC == SWE_METRIC_L2 ? __fmaf_rn(d, d, acc[r][c]) : __fadd_rn(acc[r][c], fabsf(d));
          }
      }
      if (more) {
        stash(buf ^ 1);
        __syncthreads();
        buf ^= 1;
      }
    }
    if (PAIRS) {
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int cp = 0; cp < 4; ++cp) unpack2(acc2[r][cp], acc[r][2 * cp], acc[r][2 * cp + 1]);
    }
    // both halves of the matrix
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = i0 + (r < 4 ? ty * 4 + r : 64 + ty * 4 + r - 4);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j = j0 + h * 64 + tx * 4;
        if (i < n)
          for (int c = 0; c < 4; ++c)
            if (j + c < n) local_max = max(local_max, __float_as_uint(acc[r][h * 4 + c]));
        if (VEC) {
          if (i < n && j < n)
            *reinterpret_cast<uint4*>(D + (int64_t)i * n + j) =
                make_uint4(__float_as_uint(acc[r][h * 4]), __float_as_uint(acc[r][h * 4 + 1]),
                           __float_as_uint(acc[r][h * 4 + 2]), __float_as_uint(acc[r][h * 4 + 3]));
        } else if (i < n) {
          for (int c = 0; c < 4; ++c)
            if (j + c < n) D[(int64_t)i * n + j + c] = __float_as_uint(acc[r][h * 4 + c]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int j = j0 + (c < 4 ? tx * 4 + c : 64 + tx * 4 + c - 4);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = i0 + h * 64 + ty * 4;
        if (VEC) {
          if (j < n && i < n)
            *reinterpret_cast<uint4*>(D + (int64_t)j * n + i) =
                make_uint4(__float_as_uint(acc[h * 4][c]), __float_as_uint(acc[h * 4 + 1][c]),
                           __float_as_uint(acc[h * 4 + 2][c]), __float_as_uint(acc[h * 4 + 3][c]));
        } else if (j < n) {
          for (int r = 0; r < 4; ++r)
            if (i + r < n) D[(int64_t)j * n + i + r] = __float_as_uint(acc[h * 4 + r][c]);
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) local_max = max(local_max, __shfl_xor_sync(0xFFFFFFFFu, local_max, o));
  if ((threadIdx.x & 31) == 0) atomicMax(max_bits, local_max);
}

uint32_t float_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, sizeof u);
  return u;
}

}  // namespace

swe_status need_sequences(swe_ctx* ctx) {
  if (ctx->metric != 0) return fail(ctx, SWE_ERR_STATE, "the upload holds points, not sequences");
  return SWE_OK;
}

long long ctx_threshold(const swe_ctx* ctx, float eps) {
  if (ctx->metric == SWE_METRIC_L2) {
    const float e2 = eps * eps;  // epsilon_square, dbscan.c:578
    if (e2 != e2) return -1;
    return (long long)float_bits(e2);  // >= +0: a square is never -0
  }
  if (ctx->metric == SWE_METRIC_L1) {
    if (!(eps >= 0.0f)) return -1;       // no distance is below a negative eps
    return eps == 0.0f ? 0 : (long long)float_bits(eps);  // -0 admits the distance +0
  }
  return eps_threshold(eps);
}

long long ctx_fixed_point(const swe_ctx* ctx) {
  if (ctx->metric == 0) return 4LL * ctx->max_len;  // every Smith-Waterman distance is <= 4*max_len
  return ctx->point_max_bits <= 0x7F800000u ? (long long)ctx->point_max_bits : -1;  // NaN: none
}

long long ctx_sweep_key(const swe_ctx* ctx, float eps) {
  if (ctx->metric == SWE_METRIC_L2 && !(eps >= 0.0f)) return -1;
  return ctx_threshold(ctx, eps);
}

long long engine_fixed_point(const swe_ctx* ctx) { return ctx_fixed_point(ctx); }
long long engine_sweep_key(const swe_ctx* ctx, float eps) { return ctx_sweep_key(ctx, eps); }

}  // namespace swgpu

using namespace swgpu;

extern "C" {

swe_status swe_upload_points(swe_ctx* ctx, const float* const* values, int dims, int n, int metric) {
  if (!ctx) return SWE_ERR_INVALID;
  if (metric != SWE_METRIC_L1 && metric != SWE_METRIC_L2) return fail(ctx, SWE_ERR_INVALID, "unknown metric");
  if (n < 0 || dims < 0 || (n > 0 && dims > 0 && !values)) return fail(ctx, SWE_ERR_INVALID, "bad point arrays");
  for (int d = 0; n > 0 && d < dims; ++d)
    if (!values[d]) return fail(ctx, SWE_ERR_INVALID, "bad point arrays");
  if (swe_status s = select_device(ctx)) return s;
  if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
  ctx->graph = nullptr;
  ctx->scored = false;
  ctx->masked = false;
  ctx->bits_T = LLONG_MIN;
  ctx->bits_set = -1;
  ctx->upload_gen += 1;
  ctx->metric = metric;
  ctx->dims = dims;
  ctx->n = n;
  ctx->max_len = 0;
  ctx->len.assign(n, 0);
  ctx->tiles.clear();
  ctx->n_sets = 1;
  ctx->set_first = {0, n};
  ctx->set_nfast = {n};
  ctx->set_base = {0, (long long)n * n};
  ctx->order.resize(n);
  ctx->pos.resize(n);
  for (int i = 0; i < n; ++i) ctx->order[i] = ctx->pos[i] = i;
  ctx->set_of.assign(n, 0);
  ctx->stats = swe_stats{};
  ctx->stats.n_sequences = n;
  ctx->stats.unique_pairs = (int64_t)n * (n - 1) / 2;
  ctx->stats.cells = (double)n * (n - 1) / 2.0 * dims;  // pair-dimensions
  ctx->dist_bytes = 4;
  ctx->stats.dist_bytes = 4;
  ctx->point_max_bits = 0;
  if (n == 0) {
    ctx->scored = true;
    return SWE_OK;
  }
  cudaStream_t st = ctx->st;
  CK(ctx->d_pos.alloc(n));
  CK(ctx->d_order.alloc(n));
  CK(cpy(ctx, ctx->d_pos.p, ctx->pos.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  CK(cpy(ctx, ctx->d_order.p, ctx->order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  const int64_t nn = (int64_t)n * n;
  ctx->d_D16.release();
  if (ctx->d_D32.n < (size_t)nn + 4 || ctx->d_D32.n > 2 * ((size_t)nn + 4)) ctx->d_D32.release();
  CK(ctx->d_D32.alloc((size_t)nn + 4));  // 16 bytes of slack: the threshold pass copies aligned windows

  // points, dimension-major, padded with zeros to whole tiles
  const int nt = (n + PT_TILE - 1) / PT_TILE;
  const int64_t n_pad = (int64_t)nt * PT_TILE;
  CK(ctx->d_points.alloc((size_t)std::max<int64_t>((int64_t)dims * n_pad, 4)));
  if (dims > 0) {
    // dimension-major rows of n_pad floats (zeros after point n-1), assembled
    // chunk by chunk in the pinned staging buffers
    const size_t chunk = stage_chunk(ctx);
    Staging* sg = nullptr;
    if (swe_status s = staging_ready(ctx, chunk, &sg)) return s;
    const size_t row_bytes = sizeof(float) * (size_t)n_pad, used = sizeof(float) * (size_t)n;
    swe_status s = staged_h2d(ctx, sg, chunk, ctx->d_points.p, row_bytes * dims, [&](char* dst, size_t a, size_t b) {
      split_copy(a, b, [&](size_t x, size_t y) {
        for (size_t p = x; p < y;) {
          const size_t d = p / row_bytes, in = p - d * row_bytes, e = std::min(y, (d + 1) * row_bytes);
          const size_t real = in < used ? std::min(e - p, used - in) : 0;
          if (real) memcpy(dst + (p - a), reinterpret_cast<const char*>(values[d]) + in, real);
          if (e - p > real) memset(dst + (p - a) + real, 0, e - p - real);
          p = e;
        }
      });
    });
    if (s) return s;
  }
  std::vector<int2> tiles;
  tiles.reserve((size_t)nt * (nt + 1) / 2);
  for (int bi = 0; bi < nt; ++bi)
    for (int bj = bi; bj < nt; ++bj) tiles.push_back(make_int2(bi, bj));
  DevBuf<int2> d_tiles;
  CK(d_tiles.alloc(tiles.size()));
  CK(cpy(ctx, d_tiles.p, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(ctx->d_ctr.p, 0, sizeof(unsigned), st));
  const int grid = (int)std::min<size_t>(tiles.size(), (size_t)ctx->num_sms * 2);
  const bool vec = (n & 3) == 0;
  CK(cudaEventRecord(ctx->ev[2], st));
  ctx->stats.kernel_launches += 1;
  if (metric == SWE_METRIC_L2) {
    if (vec)
      point_dist_kernel<SWE_METRIC_L2, true><<<grid, PT_THREADS, 0, st>>>(ctx->d_points.p, n_pad, n, dims, d_tiles.p,
                                                                          (int)tiles.size(), ctx->d_D32.p,
                                                                          ctx->d_ctr.p);
    else
      point_dist_kernel<SWE_METRIC_L2, false><<<grid, PT_THREADS, 0, st>>>(
          ctx->d_points.p, n_pad, n, dims, d_tiles.p, (int)tiles.size(), ctx->d_D32.p, ctx->d_ctr.p);
  } else {
    if (vec)
      point_dist_kernel<SWE_METRIC_L1, true><<<grid, PT_THREADS, 0, st>>>(ctx->d_points.p, n_pad, n, dims, d_tiles.p,
                                                                          (int)tiles.size(), ctx->d_D32.p,
                                                                          ctx->d_ctr.p);
    else
      point_dist_kernel<SWE_METRIC_L1, false><<<grid, PT_THREADS, 0, st>>>(
          ctx->d_points.p, n_pad, n, dims, d_tiles.p, (int)tiles.size(), ctx->d_D32.p, ctx->d_ctr.p);
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev[3], st));
  unsigned mx = 0;
  CK(cpy(ctx, &mx, ctx->d_ctr.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
  ctx->stats.ms_score_pass = ms;
  ctx->stats.ms_fast_kernel = ms;
  ctx->point_max_bits = mx;
  ctx->scored = true;
  return SWE_OK;
}

}  // extern "C"
