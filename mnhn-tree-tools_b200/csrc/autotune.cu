// Tile-plan autotuner of the 16x2 score kernel (swe_autotune).
//
// A plan is (row packs per tile, threads per CTA, lane-split width max_w).
// All plans produce the same matrix; the tuner times each candidate on a
// length-stratified sample of the caller's sequences in a scratch context of
// the same device, verifies the matrices are identical, and sets the fastest
// plan on the caller's context.  Plans are cached in a text file keyed by the
// device, its SM count, the sample size class and the length histogram.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine_ctx.cuh"
#include "swgpu.h"

namespace {

constexpr int TUNE_SAMPLE = 4096;
constexpr double TUNE_MARGIN = 0.98;  // a plan must beat the default by 2 % to replace it

struct Plan {
  int pb, threads, max_w;
};

// device | SMs | floor(log2(sample pairs)) | sixteen 64-symbol length bins in twentieths
std::string tune_key(int device, const std::vector<size_t>& lens, int sample) {
  cudaDeviceProp prop;
  std::string name = "unknown";
  int sms = 0;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
    name = prop.name;
    sms = prop.multiProcessorCount;
  } else {
    cudaGetLastError();
  }
  for (char& c : name)
    if (c == ' ' || c == '|') c = '_';
  int bins[16] = {0};
  for (size_t L : lens) bins[std::min<size_t>(L / 64, 15)]++;
  std::string key = name + "|sm" + std::to_string(sms) + "|p" +
                    std::to_string((int)std::floor(std::log2(std::max(1.0, 0.5 * sample * (sample - 1.0))))) + "|h";
  for (int b = 0; b < 16; ++b) {
    const int tw = lens.empty() ? 0 : (int)std::lround(20.0 * bins[b] / (double)lens.size());
    key += (b ? "." : "") + std::to_string(tw);
  }
  return key.substr(0, 159);
}

bool cache_lookup(const char* path, const std::string& key, Plan* plan) {
  if (!path) return false;
  FILE* f = fopen(path, "r");
  if (!f) return false;
  char k[256];
  Plan p{};
  bool found = false;
  while (fscanf(f, "%255s %d %d %d", k, &p.pb, &p.threads, &p.max_w) == 4)
    if (key == k && p.pb > 0 && p.pb <= 256 && p.threads > 0 && p.threads <= 256 && p.threads % 32 == 0 &&
        p.max_w > 0 && p.max_w <= swgpu::FAST_MAX_W) {
      *plan = p;
      found = true;  // the last line for a key wins
    }
  fclose(f);
  return found;
}

void cache_store(const char* path, const std::string& key, const Plan& p) {
  if (!path) return;
  FILE* f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s %d %d %d\n", key.c_str(), p.pb, p.threads, p.max_w);
  fclose(f);
}

void apply(swe_ctx* c, const Plan& p) {
  c->packs_per_block = p.pb;
  c->threads = p.threads;
  c->max_w = p.max_w;
}

}  // namespace

extern "C" swe_status swe_autotune(swe_ctx* ctx, const char* const* seqs, const size_t* lens, int n,
                                   const char* cache_path, int flags, swe_tune_result* out) {
  if (!ctx || !out || n < 0 || (n > 0 && (!seqs || !lens))) return SWE_ERR_INVALID;
  memset(out, 0, sizeof(*out));
  // length-stratified sample: every k-th sequence in length order
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return lens[a] < lens[b]; });
  const int S = std::min(n, TUNE_SAMPLE);
  std::vector<const char*> sp(S);
  std::vector<size_t> sl(S);
  for (int k = 0; k < S; ++k) {
    const int i = idx[(size_t)((double)k * n / S)];
    sp[k] = seqs[i];
    sl[k] = lens[i];
  }
  const std::string key = tune_key(ctx->device, sl, S);
  snprintf(out->key, sizeof(out->key), "%s", key.c_str());
  out->sample = S;

  Plan best{ctx->packs_per_block, ctx->threads, ctx->max_w};
  bool have = false;
  if (!(flags & SWE_TUNE_FORCE) && cache_lookup(cache_path, key, &best)) {
    out->from_cache = 1;
    have = true;
  }
  if (!have && S >= 2) {
    swe_opts o{};
    o.device = ctx->device;
    swe_ctx* tmp = nullptr;
    if (swe_status s = swe_create(&tmp, &o)) return s;
    swe_status st = swe_upload(tmp, sp.data(), sl.data(), S);
    const Plan def{32, 256, swgpu::FAST_MAX_W};
    std::vector<Plan> cands{def};
    for (int pb : {16, 32, 64})
      for (int th : {128, 256})
        for (int w : {16, 20, 24})
          if (!(pb == def.pb && th == def.threads && w == def.max_w)) cands.push_back(Plan{pb, th, w});
    std::vector<uint32_t> ref, got;
    double best_ms = 0;
    for (size_t c = 0; st == SWE_OK && c < cands.size(); ++c) {
      apply(tmp, cands[c]);
      if (swgpu::engine_relayout(tmp, nullptr, nullptr) != SWE_OK) {  // e.g. a plan that does not fit
        if (c == 0) st = SWE_ERR_CUDA;
        continue;
      }
      double ms = 1e30;
      for (int rep = 0; st == SWE_OK && rep < 3; ++rep) {
        st = swe_score_all_pairs(tmp);
        if (st == SWE_OK && rep > 0) ms = std::min(ms, tmp->stats.ms_fast_kernel);
      }
      if (st != SWE_OK) break;
      std::vector<uint32_t>& dst = c == 0 ? ref : got;
      dst.assign((size_t)S * S, 0);
      st = swe_copy_distances(tmp, dst.data());
      if (st != SWE_OK) break;
      if (c > 0 && got != ref) {
        st = swgpu::fail(ctx, SWE_ERR_STATE, "autotune: a tile plan changed the distances");
        break;
      }
      out->candidates += 1;
      if (c == 0) {
        out->ms_default = best_ms = ms;
        out->sample_cells = tmp->stats.cells;
        best = cands[0];
      } else if (ms < best_ms) {
        best_ms = ms;
        best = cands[c];
      }
    }
    if (st != SWE_OK && ctx->err.empty()) ctx->err = std::string("autotune: ") + swe_last_error(tmp);
    swe_destroy(tmp);
    if (st != SWE_OK) return st;
    if (best_ms > TUNE_MARGIN * out->ms_default) {  // within timing noise of the default: keep the default
      best = cands[0];
      best_ms = out->ms_default;
    }
    out->ms_best = best_ms;
    cache_store(cache_path, key, best);
  }
  out->packs_per_block = best.pb;
  out->threads = best.threads;
  out->max_w = best.max_w;
  apply(ctx, best);
  if (ctx->n > 0 && ctx->metric == 0) {
    if (swe_status s = swgpu::select_device(ctx)) return s;
    return swgpu::engine_relayout(ctx, nullptr, nullptr);
  }
  return SWE_OK;
}
