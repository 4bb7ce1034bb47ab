// Kernels of the learned prefilter: k-mer features, the tcgen05 BF16 GEMM
// that carries every dense layer (forward and backward), GELU, the pair
// loss, Adam, and the embedding-distance candidate pass.  No counterpart in
// the reference except the k-mer definition (kmers.c:157-241).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace swgpu {

// ---------------------------------------------------------------------------
// k-mer features
// ---------------------------------------------------------------------------
// Counts of the 4^k k-mers of every sequence, windows starting at 0 .. len-k-1
// (the last window is not counted, kmers.c:167-229), index bits 2i..2i+1 =
// base i with A0 C1 G2 T3 (kmers.c:26-63); a window holding any other symbol
// counts nothing.  Sequence i is s[0] = first_code[i] followed by
// codes[code_off[i] .. + len-1) (the engine's effective codes s[1..len]).
// out[i * 4^k + b] = count_b / sum of counts (0 for a sequence without any).
cudaError_t launch_kmer_features(const uint8_t* codes, const int64_t* code_off, const int* len,
                                 const uint8_t* first_code, int n, int k, float* out, cudaStream_t st);

// ---------------------------------------------------------------------------
// tcgen05 GEMM: C[M x N] = A[M x K] * B[N x K]^T, A and B bf16 row-major
// (K contiguous), fp32 accumulation in tensor memory.  M and N multiples of
// 128, K a multiple of 64.  The epilogue applies, in this order:
//   v = acc;  v *= gelu'(gelu_in[m][n]) if gelu_in;  v += bias[n] if bias;
//   out_pre[m][n] = v;  v = gelu(v) if act;  then out_f32 / out_bf16 /
//   out_bf16_t[n][m] = v, and colsum_part[m / 32][n] = the sum of v over the
//   32 rows m / 32 * 32 .. +31 (plain stores; launch_colsum_reduce adds the
//   M / 32 partial rows in a fixed order, so column sums are deterministic).
// ---------------------------------------------------------------------------
struct GemmEpi {
  const float* bias;
  int act;                   // 1 = exact GELU
  const float* gelu_in;      // [M x N] pre-activation of a GELU (backward)
  float* out_pre;            // [M x N]
  float* out_f32;            // [M x N]
  __nv_bfloat16* out_bf16;   // [M x N]
  __nv_bfloat16* out_bf16_t; // [N x M]
  float* colsum_part;        // [M / 32 x N]
  unsigned* status;          // KST_TIMEOUT when a bounded wait gave up
  unsigned wait_limit;
};
cudaError_t launch_gemm_bf16_tn(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K,
                                const GemmEpi& ep, cudaStream_t st);
size_t gemm_smem_bytes(int bn);
// out[n] = sum over r = 0 .. rows-1, in order, of part[r][n].
cudaError_t launch_colsum_reduce(const float* part, int rows, int N, float* out, cudaStream_t st);
// Test hook: 64 or 128 forces that tile width (0: chosen by shape).
extern int gemm_force_bn;

// Exact GELU, x * Phi(x), and its derivative.
__host__ __device__ float gelu_ref(float x);

// ---------------------------------------------------------------------------
// helpers of the training step
// ---------------------------------------------------------------------------
// Rows of the batch: out[r] = scale * X[idx[r]] as bf16 (M rows of width D;
// rows r >= rows get zeros), out_t the transpose [D x M].
cudaError_t launch_gather_rows(const float* X, int D, const int* idx, int rows, int M, float scale,
                               __nv_bfloat16* out, __nv_bfloat16* out_t, cudaStream_t st);
// Pair loss over rows (2p, 2p+1): r = ||E[2p] - E[2p+1]|| - target[p],
// loss += w r^2 / P with w = w_over[p] when r > 0 (w_over may be NULL: w = 1);
// dE = d loss / dE written as bf16 [M x D] and transposed bf16 [D x M].
// Rows >= 2P get zero gradient.
cudaError_t launch_pair_loss(const float* E, int D, const float* target, int P, int M, float* loss,
                             __nv_bfloat16* dE, __nv_bfloat16* dE_t, const float* w_over, cudaStream_t st);
// Adam on a flat fp32 parameter vector, with decoupled weight decay wd
// (w -= lr * (m_hat / (sqrt(v_hat) + eps) + wd * w)).
cudaError_t launch_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                        float eps, float bc1, float bc2, float wd, cudaStream_t st);
// bf16 copy and bf16 transpose of an fp32 [R x C] matrix.
cudaError_t launch_publish(const float* W, int R, int C, __nv_bfloat16* Wb, __nv_bfloat16* Wt, cudaStream_t st);

// ---------------------------------------------------------------------------
// candidates
// ---------------------------------------------------------------------------
// Margins by the pair's longer length: bucket b (b < n-1) holds max lengths
// below upper[b], the last bucket everything else.
constexpr int MARGIN_BUCKETS = 8;
struct MarginTable {
  int n;
  int upper[MARGIN_BUCKETS];
  float m[MARGIN_BUCKETS];
};

// Candidate pairs of one set (sorted positions first .. first+n-1 of
// `orig`): a pair i < j is a candidate when 4*|len_i - len_j| <= T (a bound
// every exact distance obeys: d >= 4*(max - min)) and, with use_emb, when
// emb_dist(i, j) <= T / (4*max(len_i, len_j)) + margin(max).  Candidates go to
// pairs[] (original indices, up to cap; the count, also beyond cap, in
// *count); keys[] (may be NULL) gets at the same index the bits of the pair's
// squared embedding distance over its squared threshold (0 without
// embeddings), the order in which the grouping joins pairs; has[i] = 1 (may
// be NULL) for every sequence in a candidate.  Embeddings are per original
// index, D floats each.
cudaError_t launch_candidates(const float* emb, int D, const int* orig, const int* len, int first, int n,
                              long long T, const MarginTable& margins, int use_emb, int2* pairs,
                              uint32_t* keys, unsigned long long cap, unsigned long long* count, uint8_t* has,
                              cudaStream_t st);
// Embedding distances of explicit pairs (original indices).
cudaError_t launch_pair_dist(const float* emb, int D, const int* a, const int* b, long long np, float* out,
                             cudaStream_t st);

}  // namespace swgpu
