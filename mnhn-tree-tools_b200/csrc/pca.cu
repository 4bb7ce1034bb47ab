// kmer2pca on the GPU (kmer2pca.c:286-597): the sample table resident in HBM,
// the feature sums and the covariance matrix from one tiled pass over it, and
// the projections of every sample onto the leading eigenvectors, and between
// them the Householder reduction and the bisection of the eigen-decomposition
// (the inverse iteration for the few wanted vectors is host code,
// pca_eigen.cpp).
//
// What the reference computes (kmer2pca.c):
//   means       m_i = (sum of x_ki over all n samples) / n              (466-481)
//   covariance  C_ij = (sum over k < n4 of (x_kj - m_j)(x_ki - m_i)) / n (337-463)
//               in 4-lane AVX Kahan sums.  Its scalar tail is guarded by
//               `!n_samples%4`, which is 0 for every n_samples > 0, so the last
//               n % 4 samples never enter the sums: n4 = n - n % 4.
//   projection  p_ji = sum over k of x_jk v_ik in the order of k, raw
//               (uncentred) samples, v_i the eigenvector of the i-th largest
//               eigenvalue, a multiply-add per term on an FMA build (141-211)
//
// Integer tables (every fasta2kmer table holds shorts) are kept as int16 and
// take an exact route: the GPU forms P_ij = sum over k < n4 of x_ki x_kj and the
// column sums T_i over the same samples in float64, where every product and
// partial sum is an integer below 2^53 (n4 max|x|^2 < 2^53), so no addition
// rounds and the order of the additions does not matter.  The host adds the
// last n % 4 rows to T for the sums S over all samples and evaluates
//   C_ij = (n^2 P_ij - n (S_i T_j + S_j T_i) + n4 S_i S_j) / n^3
// with an exact 128-bit numerator, converted to double once and divided by n
// three times: the exact value of the reference's sum up to four roundings
// (the reference rounds every centred value and partial sum).
// Other tables (fractions, or integers outside the int16 range) are kept as
// float64: the GPU centres each value as the reference does (x - m_i, m from
// the column sums) and sums the products with FMAs over sample slices that are
// added in a fixed order, which is the reference's sum up to rounding.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "staging.cuh"

namespace swgpu {

struct PcaState {
  DevBuf<int16_t> d_x16;
  DevBuf<double> d_x64, d_part, d_gram, d_colpart, d_shift, d_vec, d_proj;
  DevBuf<double> d_eig, d_tri;  // eigen-decomposition: the matrix, then per-column vectors
  int64_t n = 0, nf = 0;
  bool resident = false;  // a table is on the device
  bool int16 = false;     // held as int16 (integral values in the int16 range)
  bool exact = false;     // covariance by the exact integer route
  std::vector<double> tail;  // per feature: sum of the last n % 4 samples
  // the Householder reduction's 3 (n - 2) launches, captured once per size and
  // buffers and replayed (kernel-to-kernel gaps instead of host launches)
  cudaGraphExec_t red_graph = nullptr;
  int64_t red_n = 0;
  const double* red_A = nullptr;
  const double* red_tri = nullptr;
  ~PcaState() {
    if (red_graph) cudaGraphExecDestroy(red_graph);
  }
};

void pca_state_destroy(PcaState* ps) { delete ps; }

namespace {

constexpr int PG_TILE = 64;     // features per Gram tile side
constexpr int PG_K = 16;        // samples per shared-memory stage
constexpr int PG_THREADS = 256;

__device__ __forceinline__ double val(int16_t x) { return (double)x; }
__device__ __forceinline__ double val(double x) { return x; }

// Column sums of rows [0, rows): CTA column blockIdx.y sums rows
// [y * chunk_rows, (y+1) * chunk_rows) of 256 features, one feature per thread
// (consecutive threads read consecutive features of a row).
template <typename T>
__global__ void __launch_bounds__(256) pca_colsum_kernel(const T* __restrict__ X, int64_t nf, int64_t rows,
                                                         int64_t chunk_rows, double* __restrict__ colpart) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const int64_t r0 = (int64_t)blockIdx.y * chunk_rows, r1 = min(rows, r0 + chunk_rows);
  double s = 0.0;
  for (int64_t r = r0; r < r1; ++r) s += val(X[r * nf + f]);
  colpart[(int64_t)blockIdx.y * nf + f] = s;
}

// Gram tiles: CTA (t, s) forms the 64 x 64 feature tile t of the lower
// triangle (block row bi >= block column bj, t = bi (bi + 1) / 2 + bj) over
// the samples of slice s, sum over k of (x_ki - c_i)(x_kj - c_j) with c the
// shift (CENTER) or 0, into part[s][i][j].  Samples stream through shared
// memory 16 at a time; thread (ty, tx) holds features i = i0 + ty + 16 a and
// j = j0 + tx + 16 b (a, b < 4), so that a warp's operand reads are one
// broadcast and one contiguous 128-byte row.  Rows past the slice and
// features past nf load as 0 (after centring).
template <typename T, bool CENTER>
__global__ void __launch_bounds__(PG_THREADS) pca_gram_kernel(const T* __restrict__ X, int64_t nf, int64_t rows,
                                                              int64_t slice_rows, const double* __restrict__ shift,
                                                              double* __restrict__ part) {
  __shared__ double sA[PG_K][PG_TILE];
  __shared__ double sB[PG_K][PG_TILE];
  const int64_t t = blockIdx.x;
  int64_t bi = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while (bi > 0 && bi * (bi + 1) / 2 > t) --bi;
  const int64_t bj = t - bi * (bi + 1) / 2;
  const int64_t i0 = bi * PG_TILE, j0 = bj * PG_TILE;
  const int64_t r0 = (int64_t)blockIdx.y * slice_rows, r1 = min(rows, r0 + slice_rows);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int lc = threadIdx.x & 63, lr = threadIdx.x >> 6;  // load column; load rows lr + 4 q
  const bool a_in = i0 + lc < nf, b_in = j0 + lc < nf;
  const double ca = CENTER && a_in ? shift[i0 + lc] : 0.0, cb = CENTER && b_in ? shift[j0 + lc] : 0.0;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int64_t k0 = r0; k0 < r1; k0 += PG_K) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int rr = lr + 4 * q;
      const int64_t k = k0 + rr;
      double va = 0.0, vb = 0.0;
      if (k < r1) {
        const T* row = X + k * nf;
        if (a_in) va = CENTER ? __dsub_rn(val(row[i0 + lc]), ca) : val(row[i0 + lc]);
        if (b_in) vb = CENTER ? __dsub_rn(val(row[j0 + lc]), cb) : val(row[j0 + lc]);
      }
      sA[rr][lc] = va;
      sB[rr][lc] = vb;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < PG_K; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int x = 0; x < 4; ++x) a[x] = sA[kk][ty + 16 * x];
#pragma unroll
      for (int y = 0; y < 4; ++y) b[y] = sB[kk][tx + 16 * y];
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = __fma_rn(a[x], b[y], acc[x][y]);
    }
    __syncthreads();
  }
  double* out = part + (int64_t)blockIdx.y * nf * nf;
#pragma unroll
  for (int x = 0; x < 4; ++x) {
    const int64_t i = i0 + ty + 16 * x;
    if (i >= nf) continue;
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int64_t j = j0 + tx + 16 * y;
      if (j < nf) out[i * nf + j] = acc[x][y];
    }
  }
}

// G[i][j] (i >= j) = sum over slices, in slice order, of part[s][i][j].
__global__ void __launch_bounds__(256) pca_fold_kernel(const double* __restrict__ part, int nslices, int64_t nf,
                                                       double* __restrict__ G) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nf * nf) return;
  const int64_t i = idx / nf, j = idx - i * nf;
  if (j > i) return;
  double s = 0.0;
  for (int q = 0; q < nslices; ++q) s += part[(int64_t)q * nf * nf + idx];
  G[idx] = s;
}

// p[j][i] = sum over k of x_jk v_ik, one multiply-add per k in order.
template <typename T>
__global__ void __launch_bounds__(256) pca_project_kernel(const T* __restrict__ X, int64_t n, int64_t nf,
                                                          const double* __restrict__ V, int64_t dims,
                                                          double* __restrict__ P) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * dims) return;
  const int64_t j = idx / dims, i = idx - j * dims;
  const T* x = X + j * nf;
  const double* v = V + i * nf;
  double acc = 0.0;
  for (int64_t k = 0; k < nf; ++k) acc = __fma_rn(val(x[k]), v[k], acc);
  P[idx] = acc;
}

// ---- eigen-decomposition of the covariance matrix ------------------------
// The Householder reduction of the host solver (pca_eigen.cpp) with the matrix
// in device memory (n_features^2 doubles, L2-resident for 5-mers), three
// launches per column k: the reflector from row k (one CTA), p = tau A22 u
// (a warp per row of the trailing block), and the rank-2 update
// A22 -= u w^T + w u^T, w = p - (tau/2)(p.u) u, of the whole trailing block
// (every CTA forms p.u itself).  Then every eigenvalue of the tridiagonal by
// bisection on Sturm counts, a thread per eigenvalue.  The few wanted
// eigenvectors come from inverse iteration and the stored reflectors on the
// host.

// Sum of v over the CTA (blockDim.x a multiple of 32), returned to every thread.
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();  // sh may still be read by a previous call
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
  return t;
}

// Reflector of step k from x = A[k][k+1 .. n-1] (the column below the
// diagonal): u (u[0] = 1) to `u` and into row k, tau[k], d[k] = A[k][k] and
// e[k] = beta.  One CTA.
__global__ void __launch_bounds__(1024) tri_reflector_kernel(double* __restrict__ A, int64_t n, int64_t k,
                                                             double* __restrict__ u, double* __restrict__ tau,
                                                             double* __restrict__ dd, double* __restrict__ ee) {
  __shared__ double sh[32];
  const int64_t m = n - k - 1;
  double* x = A + k * n + k + 1;
  const double alpha = x[0];
  double s = 0.0;
  for (int64_t i = 1 + threadIdx.x; i < m; i += blockDim.x) s = __fma_rn(x[i], x[i], s);
  const double sigma = block_sum(s, sh);  // every read of x above happens before the writes below
  double t = 0.0, beta = alpha, scale = 0.0;
  if (sigma != 0.0) {
    const double norm = sqrt(alpha * alpha + sigma);
    beta = alpha <= 0.0 ? norm : -norm;
    scale = 1.0 / (alpha - beta);
    t = (beta - alpha) / beta;
  }
  for (int64_t i = threadIdx.x; i < m; i += blockDim.x) {
    const double ui = i == 0 ? 1.0 : x[i] * scale;
    u[i] = ui;
    x[i] = ui;
  }
  if (threadIdx.x == 0) {
    tau[k] = t;
    dd[k] = A[k * n + k];
    ee[k] = beta;
  }
}

// p[i] = tau[k] * sum over j of A[k+1+i][k+1+j] u[j], a warp per row.
__global__ void __launch_bounds__(256) tri_symv_kernel(const double* __restrict__ A, int64_t n, int64_t k,
                                                       const double* __restrict__ u, const double* __restrict__ tau,
                                                       double* __restrict__ p) {
  const double t = tau[k];
  if (t == 0.0) return;
  const int64_t m = n - k - 1;
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < m; i += warps) {
    const double* row = A + (k + 1 + i) * n + k + 1;
    double s = 0.0;
    for (int64_t j = lane; j < m; j += 32) s = __fma_rn(row[j], u[j], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) p[i] = t * s;
  }
}

// A22 -= u w^T + w u^T over the whole trailing block, rows spread over CTAs.
__global__ void __launch_bounds__(256) tri_update_kernel(double* __restrict__ A, int64_t n, int64_t k,
                                                         const double* __restrict__ u, const double* __restrict__ tau,
                                                         const double* __restrict__ p) {
  __shared__ double sh[32];
  const double t = tau[k];
  if (t == 0.0) return;
  const int64_t m = n - k - 1;
  double s = 0.0;
  for (int64_t j = threadIdx.x; j < m; j += blockDim.x) s = __fma_rn(p[j], u[j], s);
  const double K = 0.5 * t * block_sum(s, sh);
  for (int64_t i = blockIdx.x; i < m; i += gridDim.x) {
    const double ui = u[i], wi = p[i] - K * ui;
    double* row = A + (k + 1 + i) * n + k + 1;
    for (int64_t j = threadIdx.x; j < m; j += blockDim.x) {
      const double uj = u[j], wj = p[j] - K * uj;
      row[j] -= ui * wj + wi * uj;
    }
  }
}

// Eigenvalue j of the tridiagonal (d, e2 = e^2): the point where the Sturm
// count passes from j to j + 1, bisected from [lo, hi] to a few ulps.
__global__ void __launch_bounds__(128) tri_bisect_kernel(const double* __restrict__ d, const double* __restrict__ e2,
                                                         int64_t n, double lo, double hi, double pivmin, double tnorm,
                                                         double* __restrict__ lam) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double l = lo, u = hi;
  for (int it = 0; it < 200; ++it) {
    const double tol = 2 * DBL_EPSILON * fmax(fabs(l), fabs(u)) + DBL_EPSILON * tnorm + pivmin;
    const double mid = l + 0.5 * (u - l);
    if (u - l <= tol || mid <= l || mid >= u) break;
    int64_t c = 0;
    double q = d[0] - mid;
    if (fabs(q) < pivmin) q = -pivmin;
    c += q <= 0.0;
    for (int64_t i = 1; i < n; ++i) {
      q = d[i] - mid - e2[i - 1] / q;
      if (fabs(q) < pivmin) q = -pivmin;
      c += q <= 0.0;
    }
    if (c > j) u = mid;
    else l = mid;
  }
  lam[j] = l + 0.5 * (u - l);
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

swe_status pca_state(swe_ctx* ctx, PcaState** out) {
  if (!ctx->pca) {
    ctx->pca = new (std::nothrow) PcaState();
    if (!ctx->pca) return fail(ctx, SWE_ERR_OOM, "pca state");
  }
  *out = ctx->pca;
  return SWE_OK;
}

// Device buffers above 1 GB are given back after a call.
void trim_pca_state(PcaState* ps) {
  constexpr size_t KEEP = size_t(1) << 30;
  if (ps->d_part.n * sizeof(double) > KEEP) ps->d_part.release();
  if (ps->d_gram.n * sizeof(double) > KEEP) ps->d_gram.release();
  if (ps->d_proj.n * sizeof(double) > KEEP) ps->d_proj.release();
}

// Checks the table, picks its device form and copies it to the device.
swe_status pca_upload(swe_ctx* ctx, const double* data, int64_t n, int64_t nf, PcaState** out, swe_pca_info* info) {
  if (n < 1 || nf < 1 || !data) return fail(ctx, SWE_ERR_INVALID, "pca: empty or missing table");
  if (nf > 65536 || n > ((int64_t)1 << 40) / nf) return fail(ctx, SWE_ERR_INVALID, "pca: table too large");
  if (swe_status s = select_device(ctx)) return s;
  PcaState* ps = nullptr;
  if (swe_status s = pca_state(ctx, &ps)) return s;
  const auto t0 = std::chrono::steady_clock::now();
  ps->resident = false;
  const int64_t total = n * nf;
  // integral values in the int16 range, and their largest magnitude
  const int T = copy_threads((size_t)total * sizeof(double));
  std::vector<int> ok(T, 1);
  std::vector<double> big(T, 0.0);
  host_parallel(T, T, [&](int64_t w) {
    const int64_t a = total * w / T, b = total * (w + 1) / T;
    int good = 1;
    double m = 0.0;
    for (int64_t e = a; e < b; ++e) {
      const double x = data[e];
      good &= (x >= -32768.0) & (x <= 32767.0) & (x == std::floor(x));
      m = std::max(m, std::fabs(x));
    }
    ok[w] = good;
    big[w] = m;
  });
  bool is16 = true;
  double maxabs = 0.0;
  for (int w = 0; w < T; ++w) {
    is16 = is16 && ok[w];
    maxabs = std::max(maxabs, big[w]);
  }
  const int64_t n4 = n - n % 4;
  ps->n = n;
  ps->nf = nf;
  ps->int16 = is16;
  ps->exact = is16 && (double)n4 * maxabs * maxabs < 9007199254740992.0;  // 2^53
  ps->tail.assign((size_t)nf, 0.0);
  for (int64_t k = n4; k < n; ++k)
    for (int64_t f = 0; f < nf; ++f) ps->tail[f] += data[k * nf + f];

  const size_t chunk = stage_chunk(ctx);
  Staging* sg = nullptr;
  if (swe_status s = staging_ready(ctx, chunk, &sg)) return s;
  size_t bytes;
  if (is16) {
    ps->d_x64.release();
    CK(ps->d_x16.alloc((size_t)total));
    bytes = (size_t)total * sizeof(int16_t);
    if (swe_status s = staged_h2d(ctx, sg, chunk, ps->d_x16.p, bytes, [&](char* dst, size_t a, size_t b) {
          split_copy(a / 2, b / 2, [&](size_t x, size_t y) {
            int16_t* o = reinterpret_cast<int16_t*>(dst) + (x - a / 2);
            for (size_t e = x; e < y; ++e) o[e - x] = (int16_t)data[e];
          });
        }))
      return s;
  } else {
    ps->d_x16.release();
    CK(ps->d_x64.alloc((size_t)total));
    bytes = (size_t)total * sizeof(double);
    if (swe_status s = staged_h2d(ctx, sg, chunk, ps->d_x64.p, bytes, [&](char* dst, size_t a, size_t b) {
          split_copy(a, b, [&](size_t x, size_t y) {
            memcpy(dst + (x - a), reinterpret_cast<const char*>(data) + x, y - x);
          });
        }))
      return s;
  }
  CK(cudaStreamSynchronize(ctx->st));
  ps->resident = true;
  if (info) {
    info->exact = ps->exact ? 1 : 0;
    info->h2d_bytes = (int64_t)bytes;
    info->ms_upload = ms_since(t0);
  }
  *out = ps;
  return SWE_OK;
}

template <typename T>
swe_status launch_colsum(swe_ctx* ctx, PcaState* ps, const T* X, int64_t rows, int64_t* nchunks) {
  const int64_t nf = ps->nf;
  const int64_t fblocks = (nf + 255) / 256;
  int64_t nch = std::max<int64_t>(1, (4 * (int64_t)ctx->num_sms + fblocks - 1) / fblocks);
  nch = std::min<int64_t>(nch, std::max<int64_t>(1, rows / 64));
  nch = std::min<int64_t>(nch, 65535);
  const int64_t chunk_rows = (rows + nch - 1) / nch;
  nch = (rows + chunk_rows - 1) / chunk_rows;
  CK(ps->d_colpart.alloc((size_t)(nch * nf)));
  pca_colsum_kernel<T><<<dim3((unsigned)fblocks, (unsigned)nch), 256, 0, ctx->st>>>(X, nf, rows, chunk_rows,
                                                                                      ps->d_colpart.p);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches += 1;
  *nchunks = nch;
  return SWE_OK;
}

template <typename T>
swe_status launch_gram(swe_ctx* ctx, PcaState* ps, const T* X, int64_t rows, bool center, int* nslices) {
  const int64_t nf = ps->nf;
  const int64_t nt = (nf + PG_TILE - 1) / PG_TILE;
  const int64_t tiles = nt * (nt + 1) / 2;
  const int64_t want = 6 * (int64_t)ctx->num_sms;  // about two waves of three CTAs per SM
  int64_t s = std::max<int64_t>(1, (want + tiles - 1) / tiles);
  s = std::min<int64_t>(s, std::max<int64_t>(1, rows / 256));
  s = std::min<int64_t>(s, std::max<int64_t>(1, (int64_t)(((size_t)1 << 27) / ((size_t)nf * nf))));  // <= 1 GB
  s = std::min<int64_t>(s, 65535);
  int64_t slice_rows = (rows + s - 1) / s;
  slice_rows = (slice_rows + PG_K - 1) / PG_K * PG_K;
  s = (rows + slice_rows - 1) / slice_rows;
  CK(ps->d_part.alloc((size_t)(s * nf * nf)));
  const dim3 grid((unsigned)tiles, (unsigned)s);
  if (center)
    pca_gram_kernel<T, true><<<grid, PG_THREADS, 0, ctx->st>>>(X, nf, rows, slice_rows, ps->d_shift.p, ps->d_part.p);
  else
    pca_gram_kernel<T, false><<<grid, PG_THREADS, 0, ctx->st>>>(X, nf, rows, slice_rows, nullptr, ps->d_part.p);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches += 1;
  *nslices = (int)s;
  return SWE_OK;
}

// Covariance of the resident table into cov (n_features^2, row-major).
swe_status pca_covariance(swe_ctx* ctx, PcaState* ps, double* cov, swe_pca_info* info) {
  const int64_t n = ps->n, nf = ps->nf, n4 = n - n % 4;
  cudaStream_t st = ctx->st;
  std::vector<double> S(ps->tail), Tsum((size_t)nf, 0.0);
  float ms_cov = 0.0f, ms_gram = 0.0f;
  if (n4 > 0) {
    CK(cudaEventRecord(ctx->ev[0], st));
    int64_t nch = 0;
    if (ps->int16) {
      if (swe_status s = launch_colsum<int16_t>(ctx, ps, ps->d_x16.p, n4, &nch)) return s;
    } else if (swe_status s = launch_colsum<double>(ctx, ps, ps->d_x64.p, n4, &nch)) {
      return s;
    }
    std::vector<double> colpart((size_t)(nch * nf));
    CK(cpy(ctx, colpart.data(), ps->d_colpart.p, sizeof(double) * colpart.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int64_t c = 0; c < nch; ++c)
      for (int64_t f = 0; f < nf; ++f) Tsum[f] += colpart[c * nf + f];
  }
  for (int64_t f = 0; f < nf; ++f) S[f] = Tsum[f] + ps->tail[f];
  if (n4 == 0) {  // no sample enters the reference's sums
    std::fill(cov, cov + nf * nf, 0.0);
    if (info) info->ms_covariance = info->ms_gram = 0.0;
    return SWE_OK;
  }
  const bool center = !ps->exact;
  if (center) {  // the means, subtracted from every value inside the Gram kernel
    std::vector<double> m((size_t)nf);
    for (int64_t f = 0; f < nf; ++f) m[f] = S[f] / (double)n;
    CK(ps->d_shift.alloc((size_t)nf));
    CK(cpy(ctx, ps->d_shift.p, m.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, st));
  }
  CK(cudaEventRecord(ctx->ev[1], st));
  int ns = 0;
  if (ps->int16) {
    if (swe_status s = launch_gram<int16_t>(ctx, ps, ps->d_x16.p, n4, center, &ns)) return s;
  } else if (swe_status s = launch_gram<double>(ctx, ps, ps->d_x64.p, n4, center, &ns)) {
    return s;
  }
  CK(cudaEventRecord(ctx->ev[2], st));
  CK(ps->d_gram.alloc((size_t)(nf * nf)));
  const int64_t cells = nf * nf;
  pca_fold_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(ps->d_part.p, ns, nf, ps->d_gram.p);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches += 1;
  CK(cudaEventRecord(ctx->ev[3], st));
  CK(cpy(ctx, cov, ps->d_gram.p, sizeof(double) * (size_t)cells, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  CK(cudaEventElapsedTime(&ms_gram, ctx->ev[1], ctx->ev[2]));
  CK(cudaEventElapsedTime(&ms_cov, ctx->ev[0], ctx->ev[3]));
  if (info) {
    info->ms_gram = ms_gram;
    info->ms_covariance = ms_cov;
  }
  // the lower triangle holds the sums; finish on the host threads
  const double dn = (double)n;
  host_parallel(nf, copy_threads((size_t)cells * sizeof(double)) * 2, [&](int64_t i) {
    if (center) {
      for (int64_t j = 0; j <= i; ++j) cov[i * nf + j] = cov[i * nf + j] / dn;
      return;
    }
    const __int128 N = n, N4 = n4, Si = (__int128)(int64_t)S[i], Ti = (__int128)(int64_t)Tsum[i];
    for (int64_t j = 0; j <= i; ++j) {
      const __int128 P = (__int128)(int64_t)cov[i * nf + j];
      const __int128 Sj = (__int128)(int64_t)S[j], Tj = (__int128)(int64_t)Tsum[j];
      const __int128 Q = N * N * P - N * (Si * Tj + Sj * Ti) + N4 * Si * Sj;
      cov[i * nf + j] = (double)Q / dn / dn / dn;
    }
  });
  for (int64_t i = 0; i < nf; ++i)
    for (int64_t j = 0; j < i; ++j) cov[j * nf + i] = cov[i * nf + j];
  return SWE_OK;
}

swe_status pca_project(swe_ctx* ctx, PcaState* ps, const double* vectors, int64_t dims, double* proj,
                       swe_pca_info* info) {
  const int64_t n = ps->n, nf = ps->nf;
  cudaStream_t st = ctx->st;
  CK(ps->d_vec.alloc((size_t)(dims * nf)));
  CK(ps->d_proj.alloc((size_t)(n * dims)));
  CK(cpy(ctx, ps->d_vec.p, vectors, sizeof(double) * (size_t)(dims * nf), cudaMemcpyHostToDevice, st));
  const int64_t items = n * dims;
  if ((items + 255) / 256 > INT_MAX) return fail(ctx, SWE_ERR_INVALID, "pca: too many projections for one launch");
  CK(cudaEventRecord(ctx->ev[0], st));
  const unsigned blocks = (unsigned)((items + 255) / 256);
  if (ps->int16)
    pca_project_kernel<int16_t><<<blocks, 256, 0, st>>>(ps->d_x16.p, n, nf, ps->d_vec.p, dims, ps->d_proj.p);
  else
    pca_project_kernel<double><<<blocks, 256, 0, st>>>(ps->d_x64.p, n, nf, ps->d_vec.p, dims, ps->d_proj.p);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches += 1;
  CK(cudaEventRecord(ctx->ev[1], st));
  CK(cpy(ctx, proj, ps->d_proj.p, sizeof(double) * (size_t)items, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
  if (info) info->ms_project = ms;
  return SWE_OK;
}

// Eigenvalues (ascending) and the eigenvectors of the n_vectors largest ones
// of the symmetric host matrix cov, reduced and bisected on the GPU.  Diagonal
// and small matrices go to the host solver.
swe_status pca_eigen_device(swe_ctx* ctx, const double* cov, int64_t n, int64_t n_vectors, double* eigenvalues,
                            double* vectors, double* ms_out) {
  const auto t0 = std::chrono::steady_clock::now();
  for (int64_t i = 0; i < n * n; ++i)
    if (!std::isfinite(cov[i])) return fail(ctx, SWE_ERR_INVALID, "pca: matrix entry not finite");
  if (n < 64 || pca_eigen_diagonal(cov, n, n_vectors, eigenvalues, vectors)) {
    swe_status s = n < 64 ? swe_pca_eigen(cov, n, n_vectors, eigenvalues, vectors) : SWE_OK;
    if (ms_out) *ms_out = ms_since(t0);
    return s ? fail(ctx, s, "pca: eigen-decomposition failed") : SWE_OK;
  }
  if (swe_status s = select_device(ctx)) return s;
  PcaState* ps = nullptr;
  if (swe_status s = pca_state(ctx, &ps)) return s;
  cudaStream_t st = ctx->st;
  CK(ps->d_eig.alloc((size_t)(n * n)));
  CK(ps->d_tri.alloc((size_t)(6 * n)));  // u, p, tau, d, e, then d, e^2 / eigenvalues
  double* A = ps->d_eig.p;
  double *u = ps->d_tri.p, *p = u + n, *tau = p + n, *dd = tau + n, *ee = dd + n, *lam = ee + n;
  CK(cpy(ctx, A, cov, sizeof(double) * (size_t)(n * n), cudaMemcpyHostToDevice, st));
  const int sms = ctx->num_sms;
  if (!ps->red_graph || ps->red_n != n || ps->red_A != A || ps->red_tri != u) {
    if (ps->red_graph) cudaGraphExecDestroy(ps->red_graph);
    ps->red_graph = nullptr;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int64_t k = 0; k + 2 < n; ++k) {
      const int64_t m = n - k - 1;
      tri_reflector_kernel<<<1, 1024, 0, st>>>(A, n, k, u, tau, dd, ee);
      tri_symv_kernel<<<(unsigned)std::min<int64_t>((m + 7) / 8, 8 * (int64_t)sms), 256, 0, st>>>(A, n, k, u, tau,
                                                                                                 p);
      tri_update_kernel<<<(unsigned)std::min<int64_t>(m, 4 * (int64_t)sms), 256, 0, st>>>(A, n, k, u, tau, p);
    }
    const cudaError_t le = cudaGetLastError();
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (le != cudaSuccess || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return cuda_fail(ctx, le != cudaSuccess ? le : ce, "pca: capturing the reduction");
    }
    const cudaError_t ie = cudaGraphInstantiate(&ps->red_graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      ps->red_graph = nullptr;
      return cuda_fail(ctx, ie, "pca: instantiating the reduction");
    }
    ps->red_n = n;
    ps->red_A = A;
    ps->red_tri = u;
  }
  CK(cudaGraphLaunch(ps->red_graph, st));
  ctx->stats.kernel_launches += 3 * (n - 2);
  std::vector<double> Ah((size_t)(n * n)), tau_h(n), d(n), e(n), e2(n);
  CK(cpy(ctx, tau_h.data(), tau, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CK(cpy(ctx, d.data(), dd, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CK(cpy(ctx, e.data(), ee, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CK(cpy(ctx, Ah.data(), A, sizeof(double) * (size_t)(n * n), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  d[n - 2] = Ah[(n - 2) * n + n - 2];
  d[n - 1] = Ah[(n - 1) * n + n - 1];
  e[n - 2] = Ah[(n - 2) * n + n - 1];
  // Gershgorin bounds and the pivot floor, as the host bisection takes them
  double lo = d[0], hi = d[0], emax2 = 0.0, tnorm = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double r = (i > 0 ? std::fabs(e[i - 1]) : 0) + (i + 1 < n ? std::fabs(e[i]) : 0);
    lo = std::min(lo, d[i] - r);
    hi = std::max(hi, d[i] + r);
    if (i + 1 < n) {
      e2[i] = e[i] * e[i];
      emax2 = std::max(emax2, e2[i]);
    }
  }
  tnorm = std::max(std::fabs(lo), std::fabs(hi));
  const double pivmin = DBL_MIN * std::max(1.0, emax2);
  const double pad = 2 * DBL_EPSILON * tnorm + 2 * pivmin;
  // d and e^2 into the device scratch (over u and p), eigenvalues into lam
  CK(cpy(ctx, u, d.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
  CK(cpy(ctx, p, e2.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
  tri_bisect_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(u, p, n, lo - pad, hi + pad, pivmin, tnorm, lam);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches += 1;
  CK(cpy(ctx, eigenvalues, lam, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  pca_vectors_from_tridiagonal(Ah.data(), tau_h.data(), d.data(), e.data(), n, eigenvalues, n_vectors, vectors);
  if (n * n * sizeof(double) > (size_t(1) << 30)) ps->d_eig.release();
  if (ms_out) *ms_out = ms_since(t0);
  return SWE_OK;
}

}  // namespace
}  // namespace swgpu

using namespace swgpu;

namespace {

// Runs a call's body with host allocation failures turned into SWE_ERR_OOM
// (nothing is thrown across the C ABI) and the call's info cleared first.
template <class F>
swe_status pca_call(swe_ctx* ctx, swe_pca_info* info, F&& body) {
  if (!ctx) return SWE_ERR_INVALID;
  if (info) *info = swe_pca_info{};
  try {
    return body();
  } catch (const std::bad_alloc&) {
    return fail(ctx, SWE_ERR_OOM, "pca: host allocation failed");
  }
}

}  // namespace

extern "C" {

swe_status swe_pca_covariance(swe_ctx* ctx, const double* data, int64_t n_samples, int64_t n_features, double* cov,
                              swe_pca_info* info) {
  return pca_call(ctx, info, [&]() -> swe_status {
    if (!cov) return fail(ctx, SWE_ERR_INVALID, "pca: no covariance buffer");
    PcaState* ps = nullptr;
    if (swe_status s = pca_upload(ctx, data, n_samples, n_features, &ps, info)) return s;
    swe_status s = pca_covariance(ctx, ps, cov, info);
    trim_pca_state(ps);
    return s;
  });
}

swe_status swe_pca_project(swe_ctx* ctx, const double* data, int64_t n_samples, int64_t n_features,
                           const double* vectors, int64_t dimensions, double* projections, swe_pca_info* info) {
  return pca_call(ctx, info, [&]() -> swe_status {
    if (dimensions < 1 || dimensions > n_features || !vectors || !projections)
      return fail(ctx, SWE_ERR_INVALID, "pca: bad projection arguments");
    PcaState* ps = nullptr;
    if (data) {
      if (swe_status s = pca_upload(ctx, data, n_samples, n_features, &ps, info)) return s;
    } else {
      ps = ctx->pca;
      if (!ps || !ps->resident || ps->n != n_samples || ps->nf != n_features)
        return fail(ctx, SWE_ERR_STATE, "pca: no resident table of this shape");
      if (swe_status s = select_device(ctx)) return s;
    }
    swe_status s = pca_project(ctx, ps, vectors, dimensions, projections, info);
    trim_pca_state(ps);
    return s;
  });
}

swe_status swe_pca_eigen_gpu(swe_ctx* ctx, const double* cov, int64_t n_features, int64_t n_vectors,
                             double* eigenvalues, double* vectors) {
  return pca_call(ctx, nullptr, [&]() -> swe_status {
    const int64_t n = n_features;
    if (n < 0 || n_vectors < 0 || n_vectors > n || (n > 0 && (!cov || !eigenvalues)) ||
        (n_vectors > 0 && !vectors) || n > 65536)
      return fail(ctx, SWE_ERR_INVALID, "pca: bad eigen-decomposition arguments");
    if (n == 0) return SWE_OK;
    return pca_eigen_device(ctx, cov, n, n_vectors, eigenvalues, vectors, nullptr);
  });
}

swe_status swe_pca(swe_ctx* ctx, const double* data, int64_t n_samples, int64_t n_features, int64_t dimensions,
                   double* eigenvalues, double* projections, swe_pca_info* info) {
  return pca_call(ctx, info, [&]() -> swe_status {
    if (dimensions < 1 || dimensions > n_features || !eigenvalues || !projections)
      return fail(ctx, SWE_ERR_INVALID, "pca: bad arguments");
    PcaState* ps = nullptr;
    if (swe_status s = pca_upload(ctx, data, n_samples, n_features, &ps, info)) return s;
    std::vector<double> cov((size_t)(n_features * n_features)), vec((size_t)(dimensions * n_features));
    if (swe_status s = pca_covariance(ctx, ps, cov.data(), info)) return s;
    double ms_eigen = 0.0;
    if (swe_status s = pca_eigen_device(ctx, cov.data(), n_features, dimensions, eigenvalues, vec.data(), &ms_eigen))
      return s;
    if (info) info->ms_eigen = ms_eigen;
    swe_status s = pca_project(ctx, ps, vec.data(), dimensions, projections, info);
    trim_pca_state(ps);
    return s;
  });
}

}  // extern "C"
