// Learned prefilter: k-mer features -> MLP embedding (1024 -> 512 -> 256 ->
// 128, GELU, bf16 weights, fp32 accumulation) trained so that the L2
// distance of two embeddings predicts the normalised Smith-Waterman distance
// d / (4 * max(len_a, len_b)) of the pair.  Every dense layer, forward and
// backward, runs on the tcgen05 GEMM of mlp_kernels.cu; Adam keeps fp32
// master weights and republishes bf16 copies (and their transposes, which
// the backward GEMMs read) after every step.
//
// No counterpart in the reference; the features follow kmers.c:157-241.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "engine_ctx.cuh"
#include "mlp_kernels.cuh"

namespace swgpu {

struct PrefilterState {
  static constexpr int D0 = 1024, D1 = 512, D2 = 256, D3 = 128;
  static constexpr long long OFF_W1 = 0, OFF_B1 = OFF_W1 + (long long)D1 * D0;
  static constexpr long long OFF_W2 = OFF_B1 + D1, OFF_B2 = OFF_W2 + (long long)D2 * D1;
  static constexpr long long OFF_W3 = OFF_B2 + D2, OFF_B3 = OFF_W3 + (long long)D3 * D2;
  static constexpr long long NPARAM = OFF_B3 + D3;
  // features are L1-normalised counts (sum 1 over 1024 bins); the network
  // sees them scaled by this constant so typical inputs are O(0.1)
  static constexpr float IN_SCALE = 32.0f;

  DevBuf<float> w, g, m, v;
  DevBuf<__nv_bfloat16> W1b, W1t, W2b, W2t, W3b, W3t;
  long long adam_t = 0;
  bool init = false;

  // features and embeddings of the current upload
  DevBuf<float> X, emb;
  int feat_gen = -1, emb_gen = -1;
  bool emb_external = false;  // embeddings given by the caller (swe_prefilter_set_embeddings)

  // candidate pairs of the last prefiltered pass with their grouping keys,
  // the pairs sorted by key (ties by pair), per-sequence "in a candidate" flags
  DevBuf<int2> cand, cand_tmp;
  DevBuf<uint32_t> key, key_tmp;
  DevBuf<uint8_t> sort_tmp;
  DevBuf<unsigned long long> cand_count;
  DevBuf<uint8_t> has;
  HostPinned<int2> h_cand;

  // batch buffers (M rows)
  int M = 0;
  DevBuf<int> idx;
  DevBuf<float> target, wover;
  DevBuf<__nv_bfloat16> Xg, Xgt, A1, A1t, A2, A2t, dE, dEt, dZ2, dZ2t, dZ1t;
  DevBuf<float> Z1, Z2, E, loss;
  DevBuf<float> cpart;  // partial column sums of the bias gradients [M / 32 x D1]
  DevBuf<unsigned> status;
};

void prefilter_destroy(PrefilterState* pf) { delete pf; }

namespace {

using PS = PrefilterState;

swe_status pf_need(swe_ctx* ctx, bool need_init) {
  if (swe_status s = need_sequences(ctx)) return s;
  if (!ctx->pf) ctx->pf = new PrefilterState();
  if (need_init && !ctx->pf->init) return fail(ctx, SWE_ERR_STATE, "prefilter not initialised");
  return SWE_OK;
}

swe_status ensure_batch(swe_ctx* ctx, int M) {
  PS* pf = ctx->pf;
  if (pf->M >= M) return SWE_OK;
  CK(pf->idx.alloc(M));
  CK(pf->target.alloc(M));
  CK(pf->wover.alloc(M));
  CK(pf->Xg.alloc((size_t)M * PS::D0));
  CK(pf->Xgt.alloc((size_t)M * PS::D0));
  CK(pf->A1.alloc((size_t)M * PS::D1));
  CK(pf->A1t.alloc((size_t)M * PS::D1));
  CK(pf->A2.alloc((size_t)M * PS::D2));
  CK(pf->A2t.alloc((size_t)M * PS::D2));
  CK(pf->dE.alloc((size_t)M * PS::D3));
  CK(pf->dEt.alloc((size_t)M * PS::D3));
  CK(pf->dZ2.alloc((size_t)M * PS::D2));
  CK(pf->dZ2t.alloc((size_t)M * PS::D2));
  CK(pf->dZ1t.alloc((size_t)M * PS::D1));
  CK(pf->Z1.alloc((size_t)M * PS::D1));
  CK(pf->Z2.alloc((size_t)M * PS::D2));
  CK(pf->E.alloc((size_t)M * PS::D3));
  CK(pf->cpart.alloc((size_t)(M / 32) * PS::D1));
  CK(pf->loss.alloc(1));
  CK(pf->status.alloc(1));
  pf->M = M;
  return SWE_OK;
}

swe_status publish(swe_ctx* ctx) {
  PS* pf = ctx->pf;
  cudaStream_t st = ctx->st;
  ctx->stats.kernel_launches += 3;
  CK(launch_publish(pf->w.p + PS::OFF_W1, PS::D1, PS::D0, pf->W1b.p, pf->W1t.p, st));
  CK(launch_publish(pf->w.p + PS::OFF_W2, PS::D2, PS::D1, pf->W2b.p, pf->W2t.p, st));
  CK(launch_publish(pf->w.p + PS::OFF_W3, PS::D3, PS::D2, pf->W3b.p, pf->W3t.p, st));
  return SWE_OK;
}

GemmEpi epi(swe_ctx* ctx) {
  GemmEpi e{};
  e.status = ctx->pf->status.p;
  e.wait_limit = 1u << 22;
  return e;
}

swe_status gemm(swe_ctx* ctx, const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K, const GemmEpi& e) {
  ctx->stats.kernel_launches += 1;
  CK(launch_gemm_bf16_tn(A, B, M, N, K, e, ctx->st));
  return SWE_OK;
}

swe_status ensure_features(swe_ctx* ctx) {
  PS* pf = ctx->pf;
  if (pf->feat_gen == ctx->upload_gen) return SWE_OK;
  CK(pf->X.alloc((size_t)std::max(ctx->n, 1) * PS::D0));
  ctx->stats.kernel_launches += 1;
  CK(launch_kmer_features(ctx->d_codes.p, ctx->d_off.p, ctx->d_len.p, ctx->d_first.p, ctx->n, 5, pf->X.p, ctx->st));
  pf->feat_gen = ctx->upload_gen;
  return SWE_OK;
}

// Forward pass of `rows` gathered rows (pf->idx) padded to M.
swe_status forward(swe_ctx* ctx, int rows, int M) {
  PS* pf = ctx->pf;
  cudaStream_t st = ctx->st;
  ctx->stats.kernel_launches += 1;
  CK(launch_gather_rows(pf->X.p, PS::D0, pf->idx.p, rows, M, PS::IN_SCALE, pf->Xg.p, pf->Xgt.p, st));
  GemmEpi e1 = epi(ctx);
  e1.bias = pf->w.p + PS::OFF_B1;
  e1.out_pre = pf->Z1.p;
  e1.act = 1;
  e1.out_bf16 = pf->A1.p;
  e1.out_bf16_t = pf->A1t.p;
  if (swe_status s = gemm(ctx, pf->Xg.p, pf->W1b.p, M, PS::D1, PS::D0, e1)) return s;
  GemmEpi e2 = epi(ctx);
  e2.bias = pf->w.p + PS::OFF_B2;
  e2.out_pre = pf->Z2.p;
  e2.act = 1;
  e2.out_bf16 = pf->A2.p;
  e2.out_bf16_t = pf->A2t.p;
  if (swe_status s = gemm(ctx, pf->A1.p, pf->W2b.p, M, PS::D2, PS::D1, e2)) return s;
  GemmEpi e3 = epi(ctx);
  e3.bias = pf->w.p + PS::OFF_B3;
  e3.out_f32 = pf->E.p;
  if (swe_status s = gemm(ctx, pf->A2.p, pf->W3b.p, M, PS::D3, PS::D2, e3)) return s;
  return SWE_OK;
}

// Loss and gradients (into pf->g) of P pairs on rows (2p, 2p+1); weighted
// over-estimates when over_weighted (weights staged by stage_pairs).
swe_status loss_grad(swe_ctx* ctx, int P, int M, bool over_weighted = false) {
  PS* pf = ctx->pf;
  cudaStream_t st = ctx->st;
  if (swe_status s = forward(ctx, 2 * P, M)) return s;
  CK(cudaMemsetAsync(pf->g.p, 0, sizeof(float) * PS::NPARAM, st));
  CK(cudaMemsetAsync(pf->dE.p, 0, sizeof(__nv_bfloat16) * (size_t)M * PS::D3, st));
  CK(cudaMemsetAsync(pf->dEt.p, 0, sizeof(__nv_bfloat16) * (size_t)M * PS::D3, st));
  ctx->stats.kernel_launches += 1;
  CK(launch_pair_loss(pf->E.p, PS::D3, pf->target.p, P, M, pf->loss.p, pf->dE.p, pf->dEt.p,
                      over_weighted ? pf->wover.p : nullptr, st));
  GemmEpi e5 = epi(ctx);  // dW3 = dE^T A2
  e5.out_f32 = pf->g.p + PS::OFF_W3;
  if (swe_status s = gemm(ctx, pf->dEt.p, pf->A2t.p, PS::D3, PS::D2, M, e5)) return s;
  GemmEpi e6 = epi(ctx);  // dZ2 = (dE W3) * gelu'(Z2); db2
  e6.gelu_in = pf->Z2.p;
  e6.out_bf16 = pf->dZ2.p;
  e6.out_bf16_t = pf->dZ2t.p;
  e6.colsum_part = pf->cpart.p;
  if (swe_status s = gemm(ctx, pf->dE.p, pf->W3t.p, M, PS::D2, PS::D3, e6)) return s;
  ctx->stats.kernel_launches += 1;
  CK(launch_colsum_reduce(pf->cpart.p, M / 32, PS::D2, pf->g.p + PS::OFF_B2, st));
  GemmEpi e7 = epi(ctx);  // dW2 = dZ2^T A1
  e7.out_f32 = pf->g.p + PS::OFF_W2;
  if (swe_status s = gemm(ctx, pf->dZ2t.p, pf->A1t.p, PS::D2, PS::D1, M, e7)) return s;
  GemmEpi e8 = epi(ctx);  // dZ1 = (dZ2 W2) * gelu'(Z1); db1
  e8.gelu_in = pf->Z1.p;
  e8.out_bf16_t = pf->dZ1t.p;
  e8.colsum_part = pf->cpart.p;
  if (swe_status s = gemm(ctx, pf->dZ2.p, pf->W2t.p, M, PS::D1, PS::D2, e8)) return s;
  ctx->stats.kernel_launches += 1;
  CK(launch_colsum_reduce(pf->cpart.p, M / 32, PS::D1, pf->g.p + PS::OFF_B1, st));
  GemmEpi e9 = epi(ctx);  // dW1 = dZ1^T (scaled X)
  e9.out_f32 = pf->g.p + PS::OFF_W1;
  if (swe_status s = gemm(ctx, pf->dZ1t.p, pf->Xgt.p, PS::D1, PS::D0, M, e9)) return s;
  return SWE_OK;
}

swe_status check_status(swe_ctx* ctx) {
  unsigned s = 0;
  CK(cpy(ctx, &s, ctx->pf->status.p, sizeof(s), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return check_kernel_status(ctx, s);
}

// Pair rows and normalised targets d / (4 * max(len_a, len_b)) for pairs
// [k0, k0+P); with over_weight != 1, the weight of an over-estimate of each
// pair (over_weight for pairs with d <= over_T, 1 for the others).
swe_status stage_pairs(swe_ctx* ctx, const int* a, const int* b, const unsigned* d, long long k0, int P, int M,
                       std::vector<int>& hidx, std::vector<float>& ht, long long over_T = -1,
                       float over_weight = 1.0f) {
  hidx.assign(M, 0);
  ht.assign(std::max(P, 1), 0.f);
  std::vector<float> hw;
  if (over_weight != 1.0f) hw.assign(std::max(P, 1), 1.0f);
  for (int p = 0; p < P; ++p) {
    const int x = a[k0 + p], y = b[k0 + p];
    hidx[2 * p] = x;
    hidx[2 * p + 1] = y;
    const int mx = std::max(ctx->len[x], ctx->len[y]);
    ht[p] = mx > 0 ? (float)d[k0 + p] / (4.0f * (float)mx) : 0.f;
    if (!hw.empty() && (long long)d[k0 + p] <= over_T) hw[p] = over_weight;
  }
  PS* pf = ctx->pf;
  CK(cpy(ctx, pf->idx.p, hidx.data(), sizeof(int) * M, cudaMemcpyHostToDevice, ctx->st));
  CK(cpy(ctx, pf->target.p, ht.data(), sizeof(float) * std::max(P, 1), cudaMemcpyHostToDevice, ctx->st));
  if (!hw.empty()) CK(cpy(ctx, pf->wover.p, hw.data(), sizeof(float) * hw.size(), cudaMemcpyHostToDevice, ctx->st));
  return SWE_OK;
}

swe_status check_pairs(swe_ctx* ctx, const int* a, const int* b, long long np) {
  for (long long k = 0; k < np; ++k)
    if (a[k] < 0 || a[k] >= ctx->n || b[k] < 0 || b[k] >= ctx->n)
      return fail(ctx, SWE_ERR_INVALID, "pair index out of range");
  return SWE_OK;
}

}  // namespace

}  // namespace swgpu

using namespace swgpu;

extern "C" {

swe_status swe_kmer_features(swe_ctx* ctx, int k, float* out) {
  if (!ctx || k < 1 || k > 6) return SWE_ERR_INVALID;
  if (swe_status s = need_sequences(ctx)) return s;
  if (swe_status s = select_device(ctx)) return s;
  if (ctx->n == 0) return SWE_OK;
  const size_t nb = (size_t)1 << (2 * k);
  DevBuf<float> tmp;
  CK(tmp.alloc((size_t)ctx->n * nb));
  ctx->stats.kernel_launches += 1;
  CK(launch_kmer_features(ctx->d_codes.p, ctx->d_off.p, ctx->d_len.p, ctx->d_first.p, ctx->n, k, tmp.p, ctx->st));
  if (out) CK(cpy(ctx, out, tmp.p, sizeof(float) * ctx->n * nb, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return SWE_OK;
}

swe_status swe_prefilter_init(swe_ctx* ctx, uint64_t seed) {
  if (!ctx) return SWE_ERR_INVALID;
  if (swe_status s = select_device(ctx)) return s;
  if (swe_status s = pf_need(ctx, false)) return s;
  PS* pf = ctx->pf;
  std::vector<float> h(PS::NPARAM);
  std::mt19937_64 rng(seed);
  auto fill = [&](long long off, long long count, int fan_in) {
    const float a = 1.0f / std::sqrt((float)fan_in);
    std::uniform_real_distribution<float> U(-a, a);
    for (long long i = 0; i < count; ++i) h[off + i] = U(rng);
  };
  fill(PS::OFF_W1, (long long)PS::D1 * PS::D0, PS::D0);
  fill(PS::OFF_B1, PS::D1, PS::D0);
  fill(PS::OFF_W2, (long long)PS::D2 * PS::D1, PS::D1);
  fill(PS::OFF_B2, PS::D2, PS::D1);
  fill(PS::OFF_W3, (long long)PS::D3 * PS::D2, PS::D2);
  fill(PS::OFF_B3, PS::D3, PS::D2);
  CK(pf->w.alloc(PS::NPARAM));
  CK(pf->g.alloc(PS::NPARAM));
  CK(pf->m.alloc(PS::NPARAM));
  CK(pf->v.alloc(PS::NPARAM));
  CK(pf->W1b.alloc((size_t)PS::D1 * PS::D0));
  CK(pf->W1t.alloc((size_t)PS::D1 * PS::D0));
  CK(pf->W2b.alloc((size_t)PS::D2 * PS::D1));
  CK(pf->W2t.alloc((size_t)PS::D2 * PS::D1));
  CK(pf->W3b.alloc((size_t)PS::D3 * PS::D2));
  CK(pf->W3t.alloc((size_t)PS::D3 * PS::D2));
  CK(cpy(ctx, pf->w.p, h.data(), sizeof(float) * PS::NPARAM, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemsetAsync(pf->m.p, 0, sizeof(float) * PS::NPARAM, ctx->st));
  CK(cudaMemsetAsync(pf->v.p, 0, sizeof(float) * PS::NPARAM, ctx->st));
  if (swe_status s = publish(ctx)) return s;
  CK(cudaStreamSynchronize(ctx->st));
  pf->adam_t = 0;
  pf->init = true;
  pf->emb_gen = -1;
  return SWE_OK;
}

int64_t swe_prefilter_param_count(void) { return PS::NPARAM; }

swe_status swe_prefilter_params(swe_ctx* ctx, float* get, const float* set) {
  if (!ctx) return SWE_ERR_INVALID;
  if (swe_status s = select_device(ctx)) return s;
  if (swe_status s = pf_need(ctx, true)) return s;
  PS* pf = ctx->pf;
  if (get) CK(cpy(ctx, get, pf->w.p, sizeof(float) * PS::NPARAM, cudaMemcpyDeviceToHost, ctx->st));
  if (set) {
    CK(cpy(ctx, pf->w.p, set, sizeof(float) * PS::NPARAM, cudaMemcpyHostToDevice, ctx->st));
    if (swe_status s = publish(ctx)) return s;
    pf->emb_gen = -1;
  }
  CK(cudaStreamSynchronize(ctx->st));
  return SWE_OK;
}

swe_status swe_prefilter_loss_grad(swe_ctx* ctx, const int* a, const int* b, const unsigned* dist, int npairs,
                                   float* loss, float* grad) {
  if (!ctx || npairs <= 0 || !a || !b || !dist) return SWE_ERR_INVALID;
  if (swe_status s = select_device(ctx)) return s;
  if (swe_status s = pf_need(ctx, true)) return s;
  if (swe_status s = check_pairs(ctx, a, b, npairs)) return s;
  const int M = (2 * npairs + 127) / 128 * 128;
  if (swe_status s = ensure_batch(ctx, M)) return s;
  if (swe_status s = ensure_features(ctx)) return s;
  PS* pf = ctx->pf;
  std::vector<int> hidx;
  std::vector<float> ht;
  if (swe_status s = stage_pairs(ctx, a, b, dist, 0, npairs, M, hidx, ht)) return s;
  CK(cudaMemsetAsync(pf->loss.p, 0, sizeof(float), ctx->st));
  CK(cudaMemsetAsync(pf->status.p, 0, sizeof(unsigned), ctx->st));
  if (swe_status s = loss_grad(ctx, npairs, M)) return s;
  if (loss) CK(cpy(ctx, loss, pf->loss.p, sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
  if (grad) CK(cpy(ctx, grad, pf->g.p, sizeof(float) * PS::NPARAM, cudaMemcpyDeviceToHost, ctx->st));
  return check_status(ctx);
}

swe_status swe_prefilter_train(swe_ctx* ctx, const int* a, const int* b, const unsigned* dist, int64_t npairs,
                               int epochs, int batch_pairs, float lr, float weight_decay, uint64_t seed,
                               float over_eps, float over_weight, float* epoch_loss) {
  if (!ctx || npairs <= 0 || !a || !b || !dist || epochs < 0 || batch_pairs <= 0 || !(lr > 0) ||
      !(weight_decay >= 0) || !(over_weight > 0))
    return SWE_ERR_INVALID;
  const long long over_T = over_weight != 1.0f ? eps_threshold(over_eps) : -1;
  if (swe_status s = select_device(ctx)) return s;
  if (swe_status s = pf_need(ctx, true)) return s;
  if (swe_status s = check_pairs(ctx, a, b, npairs)) return s;
  PS* pf = ctx->pf;
  const int P = (int)std::min<int64_t>(batch_pairs, npairs);
  const int M = (2 * P + 127) / 128 * 128;
  if (swe_status s = ensure_batch(ctx, M)) return s;
  if (swe_status s = ensure_features(ctx)) return s;
  std::vector<long long> order(npairs);
  std::iota(order.begin(), order.end(), 0LL);
  std::vector<int> sa(npairs), sb(npairs);
  std::vector<unsigned> sd(npairs);
  std::mt19937_64 rng(seed);
  std::vector<int> hidx;
  std::vector<float> ht;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(order.begin(), order.end(), rng);
    for (long long k = 0; k < npairs; ++k) {
      sa[k] = a[order[k]];
      sb[k] = b[order[k]];
      sd[k] = dist[order[k]];
    }
    CK(cudaMemsetAsync(pf->loss.p, 0, sizeof(float), ctx->st));
    CK(cudaMemsetAsync(pf->status.p, 0, sizeof(unsigned), ctx->st));
    long long steps = 0;
    for (long long k0 = 0; k0 + P <= npairs; k0 += P, ++steps) {  // full batches only
      if (swe_status s = stage_pairs(ctx, sa.data(), sb.data(), sd.data(), k0, P, M, hidx, ht, over_T, over_weight))
        return s;
      if (swe_status s = loss_grad(ctx, P, M, over_weight != 1.0f)) return s;
      pf->adam_t++;
      const float bc1 = 1.0f - std::pow(b1, (float)pf->adam_t), bc2 = 1.0f - std::pow(b2, (float)pf->adam_t);
      ctx->stats.kernel_launches += 1;
      CK(launch_adam(pf->w.p, pf->g.p, pf->m.p, pf->v.p, PS::NPARAM, lr, b1, b2, eps, bc1, bc2, weight_decay,
                     ctx->st));
      if (swe_status s = publish(ctx)) return s;
    }
    float sum = 0;
    CK(cpy(ctx, &sum, pf->loss.p, sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    if (swe_status s = check_status(ctx)) return s;
    if (epoch_loss) epoch_loss[ep] = steps ? sum / (float)steps : 0.f;
  }
  pf->emb_gen = -1;
  return SWE_OK;
}

swe_status swe_prefilter_embed(swe_ctx* ctx, float* out) {
  if (!ctx) return SWE_ERR_INVALID;
  if (swe_status s = select_device(ctx)) return s;
  if (swe_status s = pf_need(ctx, true)) return s;
  PS* pf = ctx->pf;
  const int n = ctx->n;
  if ((pf->emb_gen != ctx->upload_gen || pf->emb_external) && n > 0) {
    if (swe_status s = ensure_features(ctx)) return s;
    const int chunk = std::min(16384, (n + 127) / 128 * 128);
    if (swe_status s = ensure_batch(ctx, chunk)) return s;
    CK(pf->emb.alloc((size_t)n * PS::D3));
    CK(cudaMemsetAsync(pf->status.p, 0, sizeof(unsigned), ctx->st));
    std::vector<int> hidx(chunk);
    for (int r0 = 0; r0 < n; r0 += chunk) {
      const int rows = std::min(chunk, n - r0);
      const int M = (rows + 127) / 128 * 128;
      for (int r = 0; r < M; ++r) hidx[r] = r0 + std::min(r, rows - 1);
      CK(cpy(ctx, pf->idx.p, hidx.data(), sizeof(int) * M, cudaMemcpyHostToDevice, ctx->st));
      if (swe_status s = forward(ctx, rows, M)) return s;
      CK(cudaMemcpyAsync(pf->emb.p + (size_t)r0 * PS::D3, pf->E.p, sizeof(float) * (size_t)rows * PS::D3,
                         cudaMemcpyDeviceToDevice, ctx->st));
      CK(cudaStreamSynchronize(ctx->st));  // hidx is reused
    }
    if (swe_status s = check_status(ctx)) return s;
    pf->emb_gen = ctx->upload_gen;
    pf->emb_external = false;
  }
  if (out && n > 0) CK(cpy(ctx, out, pf->emb.p, sizeof(float) * (size_t)n * PS::D3, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return SWE_OK;
}

swe_status swe_prefilter_pair_dist(swe_ctx* ctx, const int* a, const int* b, int64_t np, float* out) {
  if (!ctx || np < 0 || (np > 0 && (!a || !b || !out))) return SWE_ERR_INVALID;
  if (np == 0) return SWE_OK;
  if (swe_status s = check_pairs(ctx, a, b, np)) return s;
  if (swe_status s = swe_prefilter_embed(ctx, nullptr)) return s;
  DevBuf<int> da, db;
  DevBuf<float> dout;
  CK(da.alloc(np));
  CK(db.alloc(np));
  CK(dout.alloc(np));
  CK(cpy(ctx, da.p, a, sizeof(int) * np, cudaMemcpyHostToDevice, ctx->st));
  CK(cpy(ctx, db.p, b, sizeof(int) * np, cudaMemcpyHostToDevice, ctx->st));
  ctx->stats.kernel_launches += 1;
  CK(launch_pair_dist(ctx->pf->emb.p, PS::D3, da.p, db.p, np, dout.p, ctx->st));
  CK(cpy(ctx, out, dout.p, sizeof(float) * np, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return SWE_OK;
}

swe_status swe_prefilter_set_embeddings(swe_ctx* ctx, const float* emb) {
  if (!ctx || (!emb && ctx->n > 0)) return SWE_ERR_INVALID;
  if (swe_status s = select_device(ctx)) return s;
  if (swe_status s = pf_need(ctx, false)) return s;
  PS* pf = ctx->pf;
  CK(pf->emb.alloc((size_t)std::max(ctx->n, 1) * PS::D3));
  if (ctx->n > 0)
    CK(cpy(ctx, pf->emb.p, emb, sizeof(float) * (size_t)ctx->n * PS::D3, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  pf->emb_gen = ctx->upload_gen;
  pf->emb_external = true;
  return SWE_OK;
}

swe_status swe_score_prefiltered(swe_ctx* ctx, float eps, const swe_margins* margins, int use_emb,
                                 swe_prefilter_stats* out) {
  if (!ctx || (use_emb && !margins)) return SWE_ERR_INVALID;
  MarginTable mt{};
  mt.n = 1;
  if (margins) {
    if (margins->n < 1 || margins->n > SWE_MARGIN_BUCKETS) return fail(ctx, SWE_ERR_INVALID, "1..8 margin buckets");
    mt.n = margins->n;
    for (int b = 0; b < mt.n; ++b) {
      mt.upper[b] = margins->upper[b];
      mt.m[b] = margins->margin[b];
      if (b > 0 && b < mt.n - 1 && mt.upper[b] <= mt.upper[b - 1])
        return fail(ctx, SWE_ERR_INVALID, "margin bucket bounds must increase");
    }
  }
  if (swe_status s = select_device(ctx)) return s;
  if (swe_status s = pf_need(ctx, false)) return s;
  PS* pf = ctx->pf;
  swe_prefilter_stats st{};
  using clk = std::chrono::steady_clock;
  auto ms_since = [](clk::time_point t) { return std::chrono::duration<double, std::milli>(clk::now() - t).count(); };
  const auto t0 = clk::now();
  if (use_emb && !(pf->emb_external && pf->emb_gen == ctx->upload_gen)) {
    if (!pf->init) return fail(ctx, SWE_ERR_STATE, "prefilter not initialised");
    if (swe_status s = swe_prefilter_embed(ctx, nullptr)) return s;
  }
  st.ms_embed = ms_since(t0);
  const long long T = eps_threshold(eps);
  // candidate pairs of every set with their grouping keys, and the flags
  const auto t1 = clk::now();
  const unsigned long long cap = 1ull << 25;
  CK(pf->cand.alloc(cap));
  CK(pf->key.alloc(cap));
  CK(pf->cand_count.alloc(1));
  CK(pf->has.alloc(std::max(ctx->n, 1)));
  CK(cudaMemsetAsync(pf->cand_count.p, 0, sizeof(unsigned long long), ctx->st));
  CK(cudaMemsetAsync(pf->has.p, 0, std::max(ctx->n, 1), ctx->st));
  if (T >= 0 && ctx->n > 1) {
    for (int k = 0; k < ctx->n_sets; ++k) {
      const int f = ctx->set_first[k], nk = ctx->set_first[k + 1] - f;
      if (nk < 2) continue;
      ctx->stats.kernel_launches += 1;
      CK(launch_candidates(use_emb ? pf->emb.p : nullptr, PS::D3, ctx->d_order.p, ctx->d_len.p, f, nk, T, mt,
                           use_emb, pf->cand.p, pf->key.p, cap, pf->cand_count.p, pf->has.p, ctx->st));
    }
  }
  unsigned long long count = 0;
  CK(cpy(ctx, &count, pf->cand_count.p, sizeof(count), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  st.candidates = (int64_t)count;
  const int n = ctx->n;
  std::vector<uint8_t> has;
  const bool group = use_emb && count > 0 && count <= cap;
  if (count <= cap) {
    if (group) {
      // pairs in key order, ties by pair (a deterministic order whatever order
      // the candidate kernel appended them in): sort by pair, then stably by key
      uint64_t* pv = reinterpret_cast<uint64_t*>(pf->cand.p);
      CK(pf->cand_tmp.alloc(count));
      CK(pf->key_tmp.alloc(count));
      uint64_t* pt = reinterpret_cast<uint64_t*>(pf->cand_tmp.p);
      size_t b1 = 0, b2 = 0;
      CK(cub::DeviceRadixSort::SortPairs(nullptr, b1, pv, pt, pf->key.p, pf->key_tmp.p, (int)count, 0, 64,
                                         ctx->st));
      CK(cub::DeviceRadixSort::SortPairs(nullptr, b2, pf->key_tmp.p, pf->key.p, pt, pv, (int)count, 0, 32,
                                         ctx->st));
      CK(pf->sort_tmp.alloc(std::max<size_t>(std::max(b1, b2), 1)));
      b1 = b2 = pf->sort_tmp.n;
      ctx->stats.kernel_launches += 2;
      CK(cub::DeviceRadixSort::SortPairs(pf->sort_tmp.p, b1, pv, pt, pf->key.p, pf->key_tmp.p, (int)count, 0, 64,
                                         ctx->st));
      CK(cub::DeviceRadixSort::SortPairs(pf->sort_tmp.p, b2, pf->key_tmp.p, pf->key.p, pt, pv, (int)count, 0, 32,
                                         ctx->st));
      CK(pf->h_cand.alloc(count));
      CK(cpy(ctx, pf->h_cand.p, pf->cand.p, sizeof(int2) * count, cudaMemcpyDeviceToHost, ctx->st));
    }
    has.assign(std::max(n, 1), 0);
    CK(cpy(ctx, has.data(), pf->has.p, std::max(n, 1), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  st.ms_candidates = ms_since(t1);
  // layout: candidate groups contiguous (longer first inside each), only candidate tiles
  const auto t2 = clk::now();
  ctx->ms_layout_marks = ctx->ms_layout_upload = 0;
  if (count > cap) {
    st.fallback_full = 1;
    if (swe_status s = engine_relayout(ctx, nullptr, nullptr)) return s;
  } else {
    // groups: single linkage over the candidate pairs in key order (nearest
    // embeddings first), a join skipped when the two groups would together
    // exceed kGroupCap sequences.  Unbounded components of the candidate
    // graph chain most of a data set together; groups of about a family's
    // size put each family's candidate pairs into few tiles.  Without
    // embeddings every sequence is its own group.
    constexpr int kGroupCap = 128;
    std::vector<int> label(std::max(n, 1));  // each sequence's group: its smallest index
    if (group) {
      capped_linkage(n, reinterpret_cast<const int*>(pf->h_cand.p), (int64_t)count, kGroupCap, label.data());
    } else {
      for (int i = 0; i < n; ++i) label[i] = i;
    }
    // groups in order of their mean length (longest first), so that the
    // column blocks and packs that straddle two groups still hold sequences
    // of similar lengths
    std::vector<int64_t> gsum(n, 0), gcnt(n, 0);
    for (int i = 0; i < n; ++i) {
      const int r = label[i];
      gsum[r] += ctx->len[i];
      gcnt[r] += 1;
    }
    std::vector<int64_t> key(n);
    for (int i = 0; i < n; ++i) {
      const int r = label[i];
      const int64_t mean = (gsum[r] + gcnt[r] / 2) / std::max<int64_t>(gcnt[r], 1);
      // no candidate at all: after every group (any order works for them)
      key[i] = has[i] ? (((int64_t)INT32_MAX - mean) << 32 | (int64_t)r) : INT64_MAX;
    }
    st.ms_groups = ms_since(t2);
    if (swe_status s = engine_relayout_dev(ctx, &key, pf->cand.p, (long long)count)) return s;
  }
  st.tiles_kept = (int64_t)ctx->tiles.size();
  st.tiles_all = ctx->tiles_all;
  st.tile_cells = ctx->stats.tile_cells;
  st.ms_layout = ms_since(t2);
  st.ms_marks = ctx->ms_layout_marks;
  st.ms_upload = ctx->ms_layout_upload;
  const auto t3 = clk::now();
  if (swe_status s = score_pass(ctx)) return s;
  st.ms_score = ms_since(t3);
  st.ms_total = ms_since(t0);
  if (out) *out = st;
  return SWE_OK;
}

swe_status swe_gemm_bf16(int device, const void* A, const void* B, int M, int N, int K, const float* bias, int act,
                         float* C) {
  if (!A || !B || !C) return SWE_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return SWE_ERR_CUDA;
  DevBuf<unsigned> status;
  if (status.alloc(1) != cudaSuccess) return SWE_ERR_OOM;
  if (cudaMemset(status.p, 0, sizeof(unsigned)) != cudaSuccess) return SWE_ERR_CUDA;
  GemmEpi e{};
  e.bias = bias;
  e.act = act;
  e.out_f32 = C;
  e.status = status.p;
  e.wait_limit = 1u << 22;
  if (launch_gemm_bf16_tn((const __nv_bfloat16*)A, (const __nv_bfloat16*)B, M, N, K, e, 0) != cudaSuccess)
    return SWE_ERR_INVALID;
  if (cudaDeviceSynchronize() != cudaSuccess) return SWE_ERR_CUDA;
  unsigned s = 0;
  if (cudaMemcpy(&s, status.p, sizeof(s), cudaMemcpyDeviceToHost) != cudaSuccess) return SWE_ERR_CUDA;
  return s ? SWE_ERR_TIMEOUT : SWE_OK;
}

}  // extern "C"
