// swgpu engine: context, upload, score pass, eps neighbourhoods.
//
// Replaces the reference's inline OpenCL runtime (dbscan.c:97-298) and the
// per-point region_query launches (dbscan.c:471-522): the sequences go to the
// device once, one score pass fills the n x n distance matrix in HBM, and
// every later eps threshold reads that matrix instead of re-scoring.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <memory>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "engine_ctx.cuh"

using namespace swgpu;

namespace swgpu {

swe_status fail(swe_ctx* ctx, swe_status s, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return s;
}

swe_status cuda_fail(swe_ctx* ctx, cudaError_t e, const char* what) {
  const swe_status s = (e == cudaErrorMemoryAllocation) ? SWE_ERR_OOM : SWE_ERR_CUDA;
  return fail(ctx, s, std::string(what) + ": " + cudaGetErrorString(e));
}

swe_status check_kernel_status(swe_ctx* ctx, unsigned status) {
  if (status & KST_TIMEOUT) return fail(ctx, SWE_ERR_TIMEOUT, "device-side wait timed out");
  if (status & KST_RERUN_OVERFLOW) return fail(ctx, SWE_ERR_RERUN, "32-bit rerun queue overflowed");
  if (status & KST_BAD_TILE) return fail(ctx, SWE_ERR_STATE, "invalid tile descriptor");
  if (status & KST_REPLAY_OVERFLOW) return fail(ctx, SWE_ERR_STATE, "device DBSCAN replay: malformed neighbour bitmap");
  return SWE_OK;
}

}  // namespace swgpu

namespace {

void drop_graph(swe_ctx* ctx) {
  if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
  ctx->graph = nullptr;
}

// Builds the code table: A C G T N NUL -> 0..5, the most frequent other
// symbol -> 6, the remaining symbols by descending frequency -> 7, 8, ...
void build_code_table(const uint64_t* freq, int* code_of) {
  for (int c = 0; c < 256; ++c) code_of[c] = -1;
  code_of[(unsigned char)'A'] = CODE_A;
  code_of[(unsigned char)'C'] = CODE_C;
  code_of[(unsigned char)'G'] = CODE_G;
  code_of[(unsigned char)'T'] = CODE_T;
  code_of[(unsigned char)'N'] = CODE_N;
  code_of[0] = CODE_NUL;
  std::vector<int> rest;
  for (int c = 0; c < 256; ++c)
    if (code_of[c] < 0 && freq[c] > 0) rest.push_back(c);
  std::stable_sort(rest.begin(), rest.end(), [&](int a, int b) { return freq[a] > freq[b]; });
  int next = CODE_EXTRA;
  for (int c : rest) code_of[c] = next++;
  // symbols that never occur get the remaining codes, so queries can be encoded
  for (int c = 0; c < 256; ++c)
    if (code_of[c] < 0) code_of[c] = next++;
}

}  // namespace

namespace swgpu {

cudaError_t cpy(swe_ctx* ctx, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t st) {
  if (kind == cudaMemcpyHostToDevice) ctx->stats.h2d_bytes += (int64_t)bytes;
  else if (kind == cudaMemcpyDeviceToHost) ctx->stats.d2h_bytes += (int64_t)bytes;
  return cudaMemcpyAsync(dst, src, bytes, kind, st);
}

swe_status select_device(swe_ctx* ctx) {
  CK(cudaSetDevice(ctx->device));
  return SWE_OK;
}

}  // namespace swgpu

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* swe_strerror(swe_status s) {
  switch (s) {
    case SWE_OK: return "ok";
    case SWE_ERR_INVALID: return "invalid argument";
    case SWE_ERR_CUDA: return "CUDA error";
    case SWE_ERR_OOM: return "out of memory";
    case SWE_ERR_NO_DEVICE: return "no usable CUDA device";
    case SWE_ERR_TIMEOUT: return "device-side wait timed out";
    case SWE_ERR_RERUN: return "32-bit rerun queue overflowed";
    case SWE_ERR_STATE: return "call out of order";
    case SWE_ERR_IO: return "file could not be read or written";
    case SWE_ERR_SWEEP: return "adaptive sweep cannot reach one cluster";
  }
  return "unknown status";
}

const char* swe_last_error(const swe_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

void swe_free(void* p) { free(p); }

swe_status swe_create(swe_ctx** out, const swe_opts* opts) {
  if (!out) return SWE_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return SWE_ERR_NO_DEVICE;
  }
  const int dev = opts ? opts->device : 0;
  if (dev < 0 || dev >= ndev) return SWE_ERR_INVALID;
  swe_ctx* ctx = new (std::nothrow) swe_ctx();
  if (!ctx) return SWE_ERR_OOM;
  ctx->device = dev;
  if (opts && opts->sat_limit > 0) ctx->sat_limit = opts->sat_limit;
  if (opts && opts->packs_per_block > 0) ctx->packs_per_block = std::min(opts->packs_per_block, 256);
  if (opts && opts->threads > 0) {
    if (opts->threads % 32 != 0 || opts->threads > 256) {
      delete ctx;
      return SWE_ERR_INVALID;
    }
    ctx->threads = opts->threads;
  }
  if (opts && opts->inject_timeout) ctx->inject_timeout = 1;
  if (opts && opts->threshold_path >= 0 && opts->threshold_path <= 6) ctx->threshold_path = opts->threshold_path;
  if (opts && opts->kmer_batch_kb > 0) ctx->kmer_batch_bytes = (size_t)opts->kmer_batch_kb << 10;
  if (opts && opts->max_w > 0) ctx->max_w = std::min(opts->max_w, FAST_MAX_W);
  if (opts && opts->dbscan_replay >= 0 && opts->dbscan_replay <= 2) ctx->dbscan_replay = opts->dbscan_replay;
  cudaError_t e = cudaSetDevice(dev);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking);
  for (auto& ev : ctx->ev)
    if (e == cudaSuccess) e = cudaEventCreate(&ev);
  for (auto& ev : ctx->tev)
    if (e == cudaSuccess) e = cudaEventCreate(&ev);
  cudaDeviceProp prop;
  if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, dev);
  if (e == cudaSuccess) {
    ctx->num_sms = prop.multiProcessorCount;
    e = ctx->d_ctr.alloc(4);
  }
  if (e != cudaSuccess) {
    delete ctx;
    return e == cudaErrorMemoryAllocation ? SWE_ERR_OOM : SWE_ERR_CUDA;
  }
  *out = ctx;
  return SWE_OK;
}

static swe_status build_layout(swe_ctx* ctx, const std::vector<int64_t>* key, const CandSource* cand);

swe_status swe_set_partition(swe_ctx* ctx, int part, int nparts) {
  if (!ctx || nparts < 1 || part < 0 || part >= nparts) return SWE_ERR_INVALID;
  if (ctx->part == part && ctx->nparts == nparts) return SWE_OK;
  ctx->part = part;
  ctx->nparts = nparts;
  if (ctx->metric != 0 || ctx->n == 0 || ctx->n_sets == 0) return SWE_OK;  // applies at the next upload
  if (swe_status s = select_device(ctx)) return s;
  return build_layout(ctx, nullptr, nullptr);
}

int64_t swe_distance_bytes(const swe_ctx* ctx) {
  if (!ctx || ctx->n_sets == 0) return 0;
  return (int64_t)ctx->set_base[ctx->n_sets] * ctx->dist_bytes;
}

swe_status swe_distance_copy(swe_ctx* ctx, void* dev_buf, int to_engine) {
  if (!ctx || (!dev_buf && swe_distance_bytes(ctx) > 0)) return SWE_ERR_INVALID;
  const size_t bytes = (size_t)swe_distance_bytes(ctx);
  if (bytes == 0) return SWE_OK;
  if (swe_status s = select_device(ctx)) return s;
  void* D = ctx->dist_bytes == 2 ? (void*)ctx->d_D16.p : (void*)ctx->d_D32.p;
  if (!D) return fail(ctx, SWE_ERR_STATE, "no distance storage");
  CK(cudaMemcpyAsync(to_engine ? D : dev_buf, to_engine ? dev_buf : D, bytes, cudaMemcpyDeviceToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (to_engine) {
    ctx->bits_T = LLONG_MIN;  // cached neighbour bitmaps no longer match
    ctx->bits_set = -1;
  }
  return SWE_OK;
}

void swe_destroy(swe_ctx* ctx) { delete ctx; }

// Layout view of the device tables for the kernels.
static DistLayout layout(const swe_ctx* ctx) {
  DistLayout L;
  L.orig = ctx->d_order.p;
  L.pos = ctx->d_pos.p;
  L.set_of = ctx->d_setof.p;
  L.set_first = ctx->d_set_first.p;
  L.set_n = ctx->d_set_n.p;
  L.set_nfast = ctx->d_set_nfast.p;
  L.set_base = ctx->d_set_base.p;
  L.D16 = ctx->d_D16.p;
  L.D32 = ctx->d_D32.p;
  return L;
}

// ---------------------------------------------------------------------------
// The split pass's exchange: tile rectangles of one group
// ---------------------------------------------------------------------------
static void part_tiles(const swe_ctx* ctx, int part, std::vector<TileRect>* rects, std::vector<long long>* pre) {
  rects->clear();
  pre->assign(1, 0);
  for (size_t t = 0; t < ctx->part_rects.size(); ++t)
    if (ctx->part_owner[t] == part) {
      const TileRect& R = ctx->part_rects[t];
      rects->push_back(R);
      pre->push_back(pre->back() + (long long)R.nra * R.nb);
    }
}

extern "C" int64_t swe_partition_bytes(const swe_ctx* ctx, int part) {
  if (!ctx || part < 0 || part >= ctx->nparts || ctx->metric != 0) return -1;
  long long entries = 0;
  for (size_t t = 0; t < ctx->part_rects.size(); ++t)
    if (ctx->part_owner[t] == part) entries += (long long)ctx->part_rects[t].nra * ctx->part_rects[t].nb;
  return entries * ctx->dist_bytes;
}

static swe_status part_upload(swe_ctx* ctx, int part, long long* entries, int* ntiles) {
  std::vector<TileRect> rects;
  std::vector<long long> pre;
  part_tiles(ctx, part, &rects, &pre);
  CK(ctx->d_part_rects.alloc(std::max<size_t>(rects.size(), 1)));
  CK(ctx->d_part_pre.alloc(pre.size()));
  if (!rects.empty())
    CK(cpy(ctx, ctx->d_part_rects.p, rects.data(), sizeof(TileRect) * rects.size(), cudaMemcpyHostToDevice,
           ctx->st));
  CK(cpy(ctx, ctx->d_part_pre.p, pre.data(), sizeof(long long) * pre.size(), cudaMemcpyHostToDevice, ctx->st));
  *entries = pre.back();
  *ntiles = (int)rects.size();
  return SWE_OK;
}

extern "C" swe_status swe_partition_pack(swe_ctx* ctx, void* dev_buf) {
  if (!ctx) return SWE_ERR_INVALID;
  if (swe_status s = need_sequences(ctx)) return s;
  if (!ctx->scored) return fail(ctx, SWE_ERR_STATE, "no scored dataset");
  if (swe_status s = select_device(ctx)) return s;
  long long entries = 0;
  int ntiles = 0;
  if (swe_status s = part_upload(ctx, ctx->part, &entries, &ntiles)) return s;
  if (entries > 0 && !dev_buf) return SWE_ERR_INVALID;
  ctx->stats.kernel_launches += ntiles > 0;
  CK(launch_tile_pack(layout(ctx), ctx->d_part_rects.p, ctx->d_part_pre.p, ntiles, dev_buf, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return SWE_OK;
}

extern "C" swe_status swe_partition_unpack(swe_ctx* ctx, int part, const void* dev_buf, int64_t offset,
                                           int64_t bytes) {
  if (!ctx || part < 0 || part >= ctx->nparts || offset < 0 || bytes < 0) return SWE_ERR_INVALID;
  if (swe_status s = need_sequences(ctx)) return s;
  if (!ctx->scored) return fail(ctx, SWE_ERR_STATE, "no scored dataset");
  const int db = ctx->dist_bytes;
  if (offset % db || bytes % db) return fail(ctx, SWE_ERR_INVALID, "offset and size must be whole distances");
  if (offset + bytes > swe_partition_bytes(ctx, part)) return fail(ctx, SWE_ERR_INVALID, "beyond the group's blocks");
  if (bytes == 0) return SWE_OK;
  if (!dev_buf) return SWE_ERR_INVALID;
  if (swe_status s = select_device(ctx)) return s;
  long long entries = 0;
  int ntiles = 0;
  if (swe_status s = part_upload(ctx, part, &entries, &ntiles)) return s;
  ctx->stats.kernel_launches += 1;
  CK(launch_tile_unpack(layout(ctx), ctx->d_part_rects.p, ctx->d_part_pre.p, ntiles, dev_buf, offset / db,
                        (offset + bytes) / db, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->bits_T = LLONG_MIN;  // cached neighbour bitmaps no longer match
  ctx->bits_set = -1;
  return SWE_OK;
}

// Sorted order, packs, row blocks, tiles and every device array that depends
// on them.  key (optional, per original index): packed-path sequences of a set
// are ordered by (key, longer first) instead of longer first.  cand
// (optional): only tiles holding one of these pairs (original indices) are
// kept, and the distance matrix starts out at the largest value (no pair
// scored means no neighbour).
static swe_status build_layout(swe_ctx* ctx, const std::vector<int64_t>* key, const CandSource* cand) {
  // per set: packed-path sequences in the chosen order (longest first by
  // default), then the 32-bit-path ones
  const int n = ctx->n, n_sets = ctx->n_sets;
  drop_graph(ctx);
  ctx->scored = false;
  ctx->bits_T = LLONG_MIN;
  ctx->bits_set = -1;
  ctx->masked = cand != nullptr;
  ctx->set_nfast.assign(n_sets, 0);
  ctx->set_base.assign(n_sets + 1, 0);
  ctx->order.assign(n, 0);
  ctx->pos.assign(n, 0);
  ctx->set_of.assign(n, 0);
  ctx->exc.clear();
  ctx->exc_pre.assign(1, 0);
  int nfast_total = 0;
  for (int k = 0; k < n_sets; ++k) {
    const int f = ctx->set_first[k], nk = ctx->set_first[k + 1] - f;
    std::vector<int> fast, slow;
    for (int i = f; i < f + nk; ++i) (ctx->is_exc[i] ? slow : fast).push_back(i);
    if (key)
      std::stable_sort(fast.begin(), fast.end(), [&](int a, int b) {
        return (*key)[a] != (*key)[b] ? (*key)[a] < (*key)[b] : ctx->len[a] > ctx->len[b];
      });
    else
      std::stable_sort(fast.begin(), fast.end(), [&](int a, int b) { return ctx->len[a] > ctx->len[b]; });
    int p = 0;
    for (int i : fast) ctx->order[f + p++] = i;
    for (int i : slow) ctx->order[f + p++] = i;
    for (int q = 0; q < nk; ++q) {
      ctx->pos[ctx->order[f + q]] = q;
      ctx->set_of[ctx->order[f + q]] = k;
    }
    ctx->set_nfast[k] = (int)fast.size();
    nfast_total += (int)fast.size();
    ctx->set_base[k + 1] = ctx->set_base[k] + (long long)nk * nk;
    for (int q = (int)fast.size(); q < nk; ++q) {
      ctx->exc.push_back(f + q);
      ctx->exc_pre.push_back(ctx->exc_pre.back() + nk);
    }
  }
  ctx->nfast = nfast_total;

  // packs of two neighbouring sorted sequences of one set; blocks of up to PB
  // packs of one set, each starting on an 8-row (16-byte) boundary so a block
  // is one bulk copy
  const int PB = cand ? std::min(ctx->pf_packs_per_block, ctx->packs_per_block) : ctx->packs_per_block;
  ctx->layout_pb = PB;
  std::vector<int> pack_first, pack_off, pack_rows, block_first, block_npacks, block_rows, block_set;
  std::vector<uint8_t> pack_pair;
  int64_t row = 0;
  int max_block_rows = 8;
  for (int k = 0; k < n_sets; ++k) {
    const int f = ctx->set_first[k], nf = ctx->set_nfast[k];
    const int npk = (nf + 1) / 2;
    for (int b = 0; b < npk; b += PB) {
      row = (row + 7) & ~int64_t(7);
      const int64_t start = row;
      block_first.push_back((int)pack_first.size());
      block_npacks.push_back(std::min(PB, npk - b));
      block_set.push_back(k);
      for (int pl = b; pl < std::min(npk, b + PB); ++pl) {
        const int g = f + 2 * pl;
        const bool pair = 2 * pl + 1 < nf;
        // a row count that is a multiple of 4: the 16x2 kernel processes four rows per step
        const int R = (std::max(ctx->len[ctx->order[g]], pair ? ctx->len[ctx->order[g + 1]] : 0) + 3) & ~3;
        pack_first.push_back(g);
        pack_pair.push_back(pair ? 1 : 0);
        pack_off.push_back((int)row);
        pack_rows.push_back(R);
        row += R;
      }
      block_rows.push_back((int)(row - start));
      max_block_rows = std::max(max_block_rows, (int)((row - start + 7) & ~int64_t(7)));
      if (row > INT_MAX / 2) return fail(ctx, SWE_ERR_INVALID, "dataset too large for one upload");
    }
  }
  row = (row + 7) & ~int64_t(7);
  const int npacks = (int)pack_first.size();
  ctx->npacks = npacks;
  ctx->nblocks = (int)block_first.size();
  ctx->max_block_rows = max_block_rows;

  // tiles: blocks of column sequences against the row blocks of the same set
  // that hold a later sequence.  A column block's lane split follows its
  // longest sequence.  With candidate pairs, only the tiles holding one are kept.
  const int cta_warps = ctx->threads / 32;
  ctx->tiles.clear();
  std::vector<double> cost;
  std::vector<swgpu::TileRect> rects;  // each tile's rectangle of the sorted matrix (the split pass's exchange)
  double tile_cells = 0;
  long long tiles_all = 0;
  for (int q0 = 0, k = 0; k < n_sets; ++k) {
    const int f = ctx->set_first[k], nf = ctx->set_nfast[k];
    int q1 = q0;
    while (q1 < ctx->nblocks && block_set[q1] == k) ++q1;
    std::vector<int> cb_of(nf, 0);  // position -> column block index (within the set)
    struct ColBlock {
      int b0, nb, W, lpb;
    };
    std::vector<ColBlock> cbs;
    for (int b0 = 0; b0 < nf;) {
      int lpb = 8, nb = 0, L = 0;
      for (int it = 0; it < 3; ++it) {  // the split depends on the block's longest sequence
        nb = std::min(nf - b0, cta_warps * (32 / lpb));
        L = 0;
        for (int x = b0; x < b0 + nb; ++x) L = std::max(L, ctx->len[ctx->order[f + x]]);
        const int need = L <= 8 * ctx->max_w ? 8 : (L <= 16 * ctx->max_w ? 16 : 32);
        if (need <= lpb) break;
        lpb = need;
      }
      for (int x = b0; x < b0 + nb; ++x) cb_of[x] = (int)cbs.size();
      cbs.push_back(ColBlock{b0, nb, (L + lpb - 1) / lpb, lpb});
      b0 += nb;
    }
    std::vector<uint8_t> mark;
    const auto tm0 = std::chrono::steady_clock::now();
    if (cand && cand->dev) {
      // on the device: the candidates stay where the candidate kernel wrote them
      const int lo = f, hi = ctx->set_first[k + 1], nq = std::max(q1 - q0, 1);
      mark.assign(cbs.size() * (size_t)nq, 0);
      if (k == 0) {  // the new positions of every set, once
        CK(ctx->d_pos.alloc(std::max<size_t>(ctx->pos.size(), 1)));
        CK(cpy(ctx, ctx->d_pos.p, ctx->pos.data(), sizeof(int) * ctx->pos.size(), cudaMemcpyHostToDevice, ctx->st));
      }
      CK(ctx->d_cbof.alloc(std::max(nf, 1)));
      CK(ctx->d_mark.alloc(std::max<size_t>(mark.size(), 1)));
      if (nf > 0) CK(cpy(ctx, ctx->d_cbof.p, cb_of.data(), sizeof(int) * nf, cudaMemcpyHostToDevice, ctx->st));
      CK(cudaMemsetAsync(ctx->d_mark.p, 0, std::max<size_t>(mark.size(), 1), ctx->st));
      ctx->stats.kernel_launches += 1;
      CK(launch_mark_tiles(cand->dev, cand->count, ctx->d_pos.p, lo, hi, nf, ctx->d_cbof.p, nq, PB, ctx->d_mark.p,
                           ctx->st));
      CK(cpy(ctx, mark.data(), ctx->d_mark.p, mark.size(), cudaMemcpyDeviceToHost, ctx->st));
      CK(cudaStreamSynchronize(ctx->st));
    } else if (cand) {
      mark.assign(cbs.size() * (size_t)std::max(q1 - q0, 1), 0);
      const int lo = f, hi = ctx->set_first[k + 1], nq = q1 - q0;
      auto mark_range = [&](std::vector<uint8_t>* mk, size_t c0, size_t c1) {
        for (size_t c = c0; c < c1; ++c) {
          const int2 pr = (*cand->host)[c];
          if (pr.x < lo || pr.x >= hi || pr.y < lo || pr.y >= hi) continue;
          int px = ctx->pos[pr.x], py = ctx->pos[pr.y];
          if (px >= nf || py >= nf || px == py) continue;  // 32-bit-path pairs are all scored anyway
          if (px > py) std::swap(px, py);
          const int q = (py / 2) / PB;  // row block of the later sequence, within the set
          (*mk)[(size_t)cb_of[px] * nq + q] = 1;
        }
      };
      // threads mark private copies over slices of the candidates, then OR them
      const size_t C = cand->host->size();
      const int T = (int)std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 1 + C / 200000);
      std::vector<std::vector<uint8_t>> priv(T - 1, std::vector<uint8_t>(mark.size(), 0));
      std::vector<std::thread> th;
      for (int t = 1; t < T; ++t) th.emplace_back(mark_range, &priv[t - 1], C * t / T, C * (t + 1) / T);
      mark_range(&mark, 0, C / T);
      for (auto& x : th) x.join();
      for (const auto& pm : priv)
        for (size_t i = 0; i < mark.size(); ++i) mark[i] |= pm[i];
    }
    ctx->ms_layout_marks += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tm0).count();
    for (size_t c = 0; c < cbs.size(); ++c) {
      const ColBlock& cb = cbs[c];
      for (int q = q0; q < q1; ++q) {
        const int lastpk = block_first[q] + block_npacks[q] - 1;
        const int maxA = pack_first[lastpk] - f + (pack_pair[lastpk] ? 1 : 0);
        if (maxA > cb.b0) {
          ++tiles_all;
          if (cand && !mark[c * (q1 - q0) + (q - q0)]) continue;
          ctx->tiles.push_back(FastTile{f + cb.b0, cb.nb, q, cb.W | (cb.lpb << 8), k});
          const int pkl = block_first[q] + block_npacks[q] - 1;
          rects.push_back(swgpu::TileRect{pack_first[block_first[q]],
                                          2 * block_npacks[q] - (pack_pair[pkl] ? 0 : 1), f + cb.b0, cb.nb, k});
          const double cc = (double)cb.nb * cb.lpb * cb.W * block_rows[q];
          cost.push_back(cc);
          tile_cells += 2.0 * cc;
        }
      }
    }
    q0 = q1;
  }
  ctx->tiles_all = tiles_all;
  {
    std::vector<int> idx(ctx->tiles.size());
    cost_order(cost.data(), (int64_t)cost.size(), idx.data());
    std::vector<FastTile> sorted(ctx->tiles.size());
    std::vector<double> sorted_cost(ctx->tiles.size());
    ctx->part_rects.resize(ctx->tiles.size());
    for (size_t k = 0; k < idx.size(); ++k) {
      sorted[k] = ctx->tiles[idx[k]], sorted_cost[k] = cost[idx[k]];
      ctx->part_rects[k] = rects[idx[k]];
    }
    ctx->tiles.swap(sorted);
    ctx->part_owner.assign(ctx->tiles.size(), 0);
    if (ctx->nparts > 1) {  // this process's share of the tiles
      lpt_partition(sorted_cost.data(), (int64_t)sorted_cost.size(), ctx->nparts, ctx->part_owner.data());
      std::vector<FastTile> mine;
      tile_cells = 0;
      for (size_t k = 0; k < ctx->tiles.size(); ++k)
        if (ctx->part_owner[k] == ctx->part) mine.push_back(ctx->tiles[k]), tile_cells += 2.0 * sorted_cost[k];
      ctx->tiles.swap(mine);
    }
  }
  ctx->max_cols = cta_warps * 4;
  ctx->smem = fast_smem_bytes(ctx->max_block_rows, ctx->max_cols, PB);

  // statistics
  {
    double cells = 0;
    int64_t pairs = 0;
    for (int k = 0; k < n_sets; ++k) {
      double sum = 0, sq = 0;
      for (int i = ctx->set_first[k]; i < ctx->set_first[k + 1]; ++i) {
        sum += ctx->len[i];
        sq += (double)ctx->len[i] * ctx->len[i];
      }
      cells += (sum * sum - sq) / 2.0;
      const int64_t nk = ctx->set_first[k + 1] - ctx->set_first[k];
      pairs += nk * (nk - 1) / 2;
    }
    ctx->stats.cells = cells;
    ctx->stats.tile_cells = tile_cells;
    ctx->stats.n_sequences = n;
    ctx->stats.n_fast = nfast_total;
    ctx->stats.n_exceptional = (int64_t)ctx->exc.size();
    ctx->stats.unique_pairs = pairs;
    ctx->stats.n_tiles = (int64_t)ctx->tiles.size();
  }

  // device copies
  const auto tu0 = std::chrono::steady_clock::now();
  std::vector<int> set_n(n_sets);
  for (int k = 0; k < n_sets; ++k) set_n[k] = ctx->set_first[k + 1] - ctx->set_first[k];
  cudaStream_t st = ctx->st;
  auto up = [&](auto& buf, const auto& vec) -> cudaError_t {
    cudaError_t e = buf.alloc(std::max<size_t>(vec.size(), 1));
    if (e == cudaSuccess && !vec.empty())
      e = cpy(ctx, buf.p, vec.data(), sizeof(vec[0]) * vec.size(), cudaMemcpyHostToDevice, st);
    return e;
  };
  CK(up(ctx->d_order, ctx->order));
  CK(up(ctx->d_pos, ctx->pos));
  CK(up(ctx->d_setof, ctx->set_of));
  CK(up(ctx->d_set_first, ctx->set_first));
  CK(up(ctx->d_set_n, set_n));
  CK(up(ctx->d_set_nfast, ctx->set_nfast));
  CK(up(ctx->d_set_base, ctx->set_base));
  CK(up(ctx->d_exc, ctx->exc));
  CK(up(ctx->d_exc_pre, ctx->exc_pre));
  CK(up(ctx->d_pack_first, pack_first));
  CK(up(ctx->d_pack_pair, pack_pair));
  CK(up(ctx->d_pack_off, pack_off));
  CK(up(ctx->d_pack_rows, pack_rows));
  CK(up(ctx->d_block_first, block_first));
  CK(up(ctx->d_block_npacks, block_npacks));
  CK(up(ctx->d_tiles, ctx->tiles));
  CK(ctx->d_sel.alloc(std::max<int64_t>(row, 8)));
  // rows outside the packs (block alignment) hold the pad selector 0xF7F7
  CK(cudaMemsetAsync(ctx->d_sel.p, 0xF7, sizeof(uint16_t) * std::max<int64_t>(row, 8), st));
  ctx->stats.kernel_launches += 1;
  CK(launch_build_sel(ctx->d_codes.p, ctx->d_off.p, ctx->d_len.p, ctx->d_order.p, ctx->d_pack_first.p,
                      ctx->d_pack_pair.p, ctx->d_pack_off.p, ctx->d_pack_rows.p, npacks, ctx->d_sel.p, st));

  // distance storage: one sorted n_s x n_s matrix per set
  ctx->dist_bytes = ctx->max_len <= 16383 ? 2 : 4;
  ctx->stats.dist_bytes = ctx->dist_bytes;
  const size_t nn = (size_t)ctx->set_base[n_sets];
  // 16 bytes of slack after the last row: the threshold pass copies 16-byte
  // aligned windows around each row
  if (ctx->dist_bytes == 2) {
    ctx->d_D32.release();
    if (ctx->d_D16.n < nn + 8 || ctx->d_D16.n > 2 * (nn + 8)) ctx->d_D16.release();
    CK(ctx->d_D16.alloc(nn + 8));
  } else {
    ctx->d_D16.release();
    if (ctx->d_D32.n < nn + 4 || ctx->d_D32.n > 2 * (nn + 4)) ctx->d_D32.release();
    CK(ctx->d_D32.alloc(nn + 4));
  }

  // 32-bit path resources: rerun queue (only when the guard can fire) and
  // per-warp boundary columns for sequences longer than one 512-column chunk
  ctx->rerun_possible = (long long)ctx->sat_limit <= 4LL * ctx->max_fast_len + 8;
  double tile_pairs = 0;
  for (const auto& t : ctx->tiles) tile_pairs += 2.0 * t.nb * PB;
  ctx->rerun_cap = ctx->rerun_possible ? (unsigned)std::min(tile_pairs, (double)(1u << 26)) : 1024u;
  CK(ctx->d_rerun.alloc(std::max(ctx->rerun_cap, 1u)));
  ctx->gen_grid = ctx->num_sms * 4;
  ctx->scratch_stride = 0;
  if (ctx->max_len > GEN_CHUNK) {
    ctx->scratch_stride = (long long)ctx->max_len + 1;
    const long long warps = (long long)ctx->gen_grid * 8;
    const long long budget = 1LL << 31;  // bytes
    if (warps * ctx->scratch_stride * 4 > budget)
      ctx->gen_grid = (int)std::max<long long>(ctx->num_sms, budget / (ctx->scratch_stride * 4 * 8));
    CK(ctx->d_scratch.alloc((size_t)ctx->gen_grid * 8 * ctx->scratch_stride));
  }

  // launch shapes
  CK(fast_set_smem_limit(ctx->smem));
  const int occ = std::max(1, fast_occupancy(ctx->threads, ctx->smem));
  ctx->fast_grid = std::max(1, std::min<int>(ctx->num_sms * occ, (int)std::max<size_t>(ctx->tiles.size(), 1)));
  CK(cudaStreamSynchronize(st));
  ctx->ms_layout_upload += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tu0).count();
  return SWE_OK;
}


// Uploads n sequences forming n_sets independent sets: set k is the original
// indices [set_first[k], set_first[k+1]).  Pairs are scored only inside a set.
static swe_status upload_sets(swe_ctx* ctx, const char* const* seqs, const size_t* lens, int n,
                              const int* set_first_in, int n_sets) {
  if (!ctx) return SWE_ERR_INVALID;
  if (n < 0 || (n > 0 && (!seqs || !lens))) return fail(ctx, SWE_ERR_INVALID, "bad sequence arrays");
  if (n_sets < 1 || !set_first_in || set_first_in[0] != 0 || set_first_in[n_sets] != n)
    return fail(ctx, SWE_ERR_INVALID, "set offsets must run from 0 to n");
  for (int k = 0; k < n_sets; ++k)
    if (set_first_in[k + 1] < set_first_in[k]) return fail(ctx, SWE_ERR_INVALID, "set offsets must not decrease");
  if (swe_status s = select_device(ctx)) return s;
  drop_graph(ctx);
  ctx->scored = false;
  ctx->bits_T = LLONG_MIN;
  ctx->bits_set = -1;
  ctx->metric = 0;
  ctx->dims = 0;
  ctx->d_points.release();
  ctx->n = n;
  ctx->len.assign(n, 0);
  ctx->off.assign(n, 0);
  ctx->is_exc.assign(n, 0);
  ctx->stats = swe_stats{};

  // alphabet over the effective symbols s[1..len]
  uint64_t freq[256] = {0};
  int64_t total = 0;
  int max_len = 0;
  for (int i = 0; i < n; ++i) {
    if (!seqs[i] && lens[i] > 0) return fail(ctx, SWE_ERR_INVALID, "null sequence pointer");
    if (lens[i] > (size_t)(INT_MAX / 8)) return fail(ctx, SWE_ERR_INVALID, "sequence too long");
    const int L = (int)lens[i];
    ctx->len[i] = L;
    max_len = std::max(max_len, L);
    const unsigned char* s = reinterpret_cast<const unsigned char*>(seqs[i]);
    for (int r = 0; r < L; ++r) freq[s[r + 1]]++;
    ctx->off[i] = total;
    total += (L + 15) & ~15;
  }
  ctx->max_len = max_len;
  build_code_table(freq, ctx->code_of);
  ctx->upload_gen++;
  ctx->first_code.assign(std::max(n, 1), 0);
  for (int i = 0; i < n; ++i) ctx->first_code[i] = (uint8_t)ctx->code_of[(unsigned char)(seqs[i] ? seqs[i][0] : 0)];
  ctx->codes.assign((size_t)std::max<int64_t>(total, 16), 0);
  int max_fast = 0;
  for (int i = 0; i < n; ++i) {
    const int L = ctx->len[i];
    const unsigned char* s = reinterpret_cast<const unsigned char*>(seqs[i]);
    uint8_t* dst = ctx->codes.data() + ctx->off[i];
    bool fast = (L >= 1 && L <= FAST_MAX_LEN);
    for (int r = 0; r < L; ++r) {
      const int c = ctx->code_of[s[r + 1]];
      dst[r] = (uint8_t)c;
      if (c >= FAST_CODES) fast = false;
    }
    if (fast) max_fast = std::max(max_fast, L);
    else ctx->is_exc[i] = 1;
  }
  ctx->max_fast_len = max_fast;

  ctx->n_sets = n_sets;
  ctx->set_first.assign(set_first_in, set_first_in + n_sets + 1);
  cudaStream_t st = ctx->st;
  auto up = [&](auto& buf, const auto& vec) -> cudaError_t {
    cudaError_t e = buf.alloc(std::max<size_t>(vec.size(), 1));
    if (e == cudaSuccess && !vec.empty())
      e = cpy(ctx, buf.p, vec.data(), sizeof(vec[0]) * vec.size(), cudaMemcpyHostToDevice, st);
    return e;
  };
  CK(up(ctx->d_codes, ctx->codes));
  CK(up(ctx->d_first, ctx->first_code));
  CK(up(ctx->d_off, ctx->off));
  CK(up(ctx->d_len, ctx->len));
  return build_layout(ctx, nullptr, nullptr);
}

swe_status swe_upload(swe_ctx* ctx, const char* const* seqs, const size_t* lens, int n) {
  const int sets[2] = {0, n < 0 ? 0 : n};
  return upload_sets(ctx, seqs, lens, n, sets, 1);
}

swe_status swe_upload_sets(swe_ctx* ctx, const char* const* seqs, const size_t* lens, int n,
                           const int* set_first, int n_sets) {
  return upload_sets(ctx, seqs, lens, n, set_first, n_sets);
}

int swe_set_count(const swe_ctx* ctx) { return ctx ? ctx->n_sets : 0; }

static swe_status build_score_graph(swe_ctx* ctx) {
  cudaStream_t st = ctx->st;
  const DistLayout L = layout(ctx);
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaMemsetAsync(ctx->d_ctr.p, 0, 4 * sizeof(unsigned), st);
  if (e == cudaSuccess && (ctx->masked || ctx->nparts > 1)) {
    // pairs outside the scored tiles read as the largest value (0xFF bytes)
    const size_t nn = (size_t)ctx->set_base[ctx->n_sets];
    e = ctx->d_D16.p ? cudaMemsetAsync(ctx->d_D16.p, 0xFF, nn * sizeof(uint16_t), st)
                     : cudaMemsetAsync(ctx->d_D32.p, 0xFF, nn * sizeof(uint32_t), st);
  }
  ctx->graph_kernels = 1;
  if (e == cudaSuccess) e = launch_diag(L, ctx->n, st);
  // inside a capture only an external record becomes a real event node
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->ev[0], st, cudaEventRecordExternal);
  if (e == cudaSuccess && !ctx->tiles.empty()) {
    FastParams p{};
    p.codes = ctx->d_codes.p;
    p.code_off = ctx->d_off.p;
    p.len = ctx->d_len.p;
    p.L = L;
    p.sel = ctx->d_sel.p;
    p.pack_first = ctx->d_pack_first.p;
    p.pack_pair = ctx->d_pack_pair.p;
    p.pack_row_off = ctx->d_pack_off.p;
    p.pack_rows = ctx->d_pack_rows.p;
    p.block_first = ctx->d_block_first.p;
    p.block_npacks = ctx->d_block_npacks.p;
    p.max_packs_per_block = ctx->layout_pb;
    p.tiles = ctx->d_tiles.p;
    p.ntiles = (int)ctx->tiles.size();
    p.tile_counter = ctx->d_ctr.p;
    p.rerun = ctx->d_rerun.p;
    p.rerun_count = ctx->d_ctr.p + 2;
    p.rerun_cap = ctx->rerun_cap;
    p.sat_limit = ctx->sat_limit;
    p.status = ctx->d_ctr.p + 1;
    p.max_block_rows = ctx->max_block_rows;
    p.max_cols_per_cta = ctx->max_cols;
    p.wait_limit = ctx->inject_timeout ? (1u << 10) : (1u << 24);
    p.inject_timeout = ctx->inject_timeout;
    e = launch_fast(p, ctx->fast_grid, ctx->threads, ctx->smem, st);
    ctx->graph_kernels++;
  }
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->ev[1], st, cudaEventRecordExternal);
  GenParams g{};
  g.codes = ctx->d_codes.p;
  g.code_off = ctx->d_off.p;
  g.len = ctx->d_len.p;
  g.n = ctx->n;
  g.L = L;
  g.scratch = ctx->d_scratch.p;
  g.scratch_stride = ctx->scratch_stride;
  g.nwarps_total = ctx->gen_grid * 8;
  g.status = ctx->d_ctr.p + 1;
  if (e == cudaSuccess && !ctx->exc.empty()) {
    GenParams x = g;
    x.mode = GEN_EXC_CROSS;
    x.exc = ctx->d_exc.p;
    x.exc_pre = ctx->d_exc_pre.p;
    x.nexc = (int)ctx->exc.size();
    e = launch_generic(x, ctx->gen_grid, st);
    ctx->graph_kernels++;
  }
  if (e == cudaSuccess && ctx->rerun_possible) {
    GenParams r = g;
    r.mode = GEN_PAIRS;
    r.pairs = ctx->d_rerun.p;
    r.npairs_dev = ctx->d_ctr.p + 2;
    e = launch_generic(r, ctx->gen_grid, st);
    ctx->graph_kernels++;
  }
  cudaGraph_t graph = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(st, &graph);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->graph, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    ctx->graph = nullptr;
    return cuda_fail(ctx, e, "building the score-pass graph");
  }
  return SWE_OK;
}

swe_status swe_score_all_pairs(swe_ctx* ctx) {
  if (!ctx) return SWE_ERR_INVALID;
  if (ctx->metric != 0) return SWE_OK;  // point distances are computed by the upload
  if (swe_status s = select_device(ctx)) return s;
  if (ctx->masked)  // back from a prefiltered pass: every tile again, longest first
    if (swe_status s = build_layout(ctx, nullptr, nullptr)) return s;
  return score_pass(ctx);
}

}  // extern "C"

namespace swgpu {

swe_status engine_relayout(swe_ctx* ctx, const std::vector<int64_t>* key, const std::vector<int2>* cand) {
  if (!cand) return build_layout(ctx, key, nullptr);
  CandSource src;
  src.host = cand;
  src.count = (long long)cand->size();
  return build_layout(ctx, key, &src);
}

swe_status engine_relayout_dev(swe_ctx* ctx, const std::vector<int64_t>* key, const int2* cand, long long count) {
  CandSource src;
  src.dev = cand;
  src.count = count;
  return build_layout(ctx, key, &src);
}

swe_status score_pass(swe_ctx* ctx) {
  ctx->bits_T = LLONG_MIN;
  ctx->bits_set = -1;
  if (ctx->n == 0) {
    ctx->scored = true;
    return SWE_OK;
  }
  if (!ctx->graph)
    if (swe_status s = build_score_graph(ctx)) return s;
  CK(cudaEventRecord(ctx->ev[2], ctx->st));
  CK(cudaGraphLaunch(ctx->graph, ctx->st));
  ctx->stats.kernel_launches += ctx->graph_kernels;
  CK(cudaEventRecord(ctx->ev[3], ctx->st));
  unsigned ctr[4];
  CK(cpy(ctx, ctr, ctx->d_ctr.p, sizeof(ctr), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  float ms = 0, msf = 0;
  CK(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
  CK(cudaEventElapsedTime(&msf, ctx->ev[0], ctx->ev[1]));
  ctx->stats.ms_score_pass = ms;
  ctx->stats.ms_fast_kernel = msf;
  ctx->stats.reruns = std::min(ctr[2], ctx->rerun_cap);
  if (swe_status s = check_kernel_status(ctx, ctr[1])) return s;
  ctx->scored = true;
  return SWE_OK;
}

}  // namespace swgpu

extern "C" {

static const uint16_t* set_D16(const swe_ctx* ctx, int s) {
  return ctx->d_D16.p ? ctx->d_D16.p + ctx->set_base[s] : nullptr;
}
static const uint32_t* set_D32(const swe_ctx* ctx, int s) {
  return ctx->d_D32.p ? ctx->d_D32.p + ctx->set_base[s] : nullptr;
}

swe_status swe_copy_set_rows(swe_ctx* ctx, int s, int row0, int row1, uint32_t* out) {
  if (!ctx) return SWE_ERR_INVALID;
  if (!ctx->scored) return fail(ctx, SWE_ERR_STATE, "no scored dataset");
  if (s < 0 || s >= ctx->n_sets) return fail(ctx, SWE_ERR_INVALID, "no such set");
  if (swe_status st = select_device(ctx)) return st;
  const int first = ctx->set_first[s], ns = ctx->set_first[s + 1] - first;
  if (row0 < 0 || row1 < row0 || row1 > ns) return fail(ctx, SWE_ERR_INVALID, "bad row range");
  if (ns == 0 || row1 == row0) return SWE_OK;
  if (!out) return SWE_ERR_INVALID;
  // rows in original order, in chunks of about 64 Mi entries
  const int rows = (int)std::max<long long>(1, std::min<long long>(row1 - row0, (64LL << 20) / ns));
  DevBuf<uint32_t> tmp;
  CK(tmp.alloc((size_t)rows * ns));
  for (int r0 = row0; r0 < row1; r0 += rows) {
    const int r1 = std::min(row1, r0 + rows);
    ctx->stats.kernel_launches += 1;
    CK(launch_unpermute_set(set_D16(ctx, s), set_D32(ctx, s), ctx->d_pos.p + first, ns, r0, r1, tmp.p, ctx->st));
    CK(cpy(ctx, out + (size_t)(r0 - row0) * ns, tmp.p, sizeof(uint32_t) * (size_t)(r1 - r0) * ns,
           cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  return SWE_OK;
}

swe_status swe_copy_set_distances(swe_ctx* ctx, int s, uint32_t* out) {
  if (!ctx) return SWE_ERR_INVALID;
  if (s < 0 || s >= ctx->n_sets) return fail(ctx, SWE_ERR_INVALID, "no such set");
  return swe_copy_set_rows(ctx, s, 0, ctx->set_first[s + 1] - ctx->set_first[s], out);
}

swe_status swe_copy_distances(swe_ctx* ctx, uint32_t* out) {
  if (!ctx) return SWE_ERR_INVALID;
  if (ctx->n_sets > 1) return fail(ctx, SWE_ERR_STATE, "several sets uploaded: use swe_copy_set_distances");
  if (ctx->n == 0) return SWE_OK;
  return swe_copy_set_distances(ctx, 0, out);
}

swe_status swe_block_stats(swe_ctx* ctx, int set, int r0, int r1, int c0, int c1, double mean, uint64_t* row_sum,
                           uint64_t* row_sqdev, uint32_t* min, uint32_t* max) {
  if (!ctx) return SWE_ERR_INVALID;
  if (!ctx->scored) return fail(ctx, SWE_ERR_STATE, "no scored dataset");
  if (swe_status s = need_sequences(ctx)) return s;
  if (set < 0 || set >= ctx->n_sets) return fail(ctx, SWE_ERR_INVALID, "no such set");
  const int first = ctx->set_first[set], ns = ctx->set_first[set + 1] - first;
  if (r0 < 0 || r1 < r0 || r1 > ns || c0 < 0 || c1 < c0 || c1 > ns) return fail(ctx, SWE_ERR_INVALID, "bad block");
  if (swe_status st = select_device(ctx)) return st;
  const int rows = r1 - r0;
  DevBuf<unsigned long long> dsum, dsq;
  DevBuf<unsigned> mm;
  CK(dsum.alloc(std::max(rows, 1)));
  CK(dsq.alloc(std::max(rows, 1)));
  CK(mm.alloc(2));
  const unsigned init[2] = {0xFFFFFFFFu, 0u};
  CK(cpy(ctx, mm.p, init, sizeof(init), cudaMemcpyHostToDevice, ctx->st));
  ctx->stats.kernel_launches += 1;
  CK(launch_block_stats(set_D16(ctx, set), set_D32(ctx, set), ctx->d_pos.p + first, ns, r0, r1, c0, c1, mean,
                        dsum.p, dsq.p, mm.p, mm.p + 1, ctx->st));
  unsigned hm[2] = {0, 0};
  if (row_sum && rows) CK(cpy(ctx, row_sum, dsum.p, sizeof(uint64_t) * rows, cudaMemcpyDeviceToHost, ctx->st));
  if (row_sqdev && rows) CK(cpy(ctx, row_sqdev, dsq.p, sizeof(uint64_t) * rows, cudaMemcpyDeviceToHost, ctx->st));
  CK(cpy(ctx, hm, mm.p, sizeof(hm), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (min) *min = hm[0];
  if (max) *max = hm[1];
  return SWE_OK;
}

}  // extern "C"

// Groups of one set against thresholds T[0..count) (all >= 0), THR_MAX per
// group; threshold j's bitmap starts at word *bits_words + j * n_s * wpr and its
// counts at *count_ints + j * n_s.  Advances both offsets past the set.
static void add_set_groups(const swe_ctx* ctx, int s, const long long* T, int count, std::vector<ThrGroup>* groups,
                           std::vector<unsigned>* thr, long long* bits_words, long long* count_ints) {
  const int first = ctx->set_first[s], ns = ctx->set_first[s + 1] - first;
  const int wpr = (ns + 63) / 64;
  for (int j0 = 0; j0 < count; j0 += THR_MAX) {
    ThrGroup g;
    g.dist_base = ctx->set_base[s];
    g.bits_base = *bits_words + (long long)j0 * ns * wpr;
    g.counts_base = *count_ints + (long long)j0 * ns;
    g.pos_first = first;
    g.n_s = ns;
    g.wpr = wpr;
    g.thr_first = (int)thr->size();
    g.nthr = std::min(THR_MAX, count - j0);
    for (int j = j0; j < j0 + g.nthr; ++j) thr->push_back((unsigned)std::min<long long>(T[j], 0xFFFFFFFFLL));
    if (ns > 0) groups->push_back(g);
  }
  *bits_words += (long long)count * ns * wpr;
  *count_ints += (long long)count * ns;
}

// One threshold launch over `groups`, bracketed by ev[2] / ev[3].
static swe_status launch_groups(swe_ctx* ctx, const std::vector<ThrGroup>& groups, const std::vector<unsigned>& thr,
                                uint64_t* d_bits, int* d_counts) {
  std::vector<long long> pre(groups.size() + 1, 0);
  int maxn = 0;
  for (size_t g = 0; g < groups.size(); ++g) {
    pre[g + 1] = pre[g] + groups[g].n_s;
    maxn = std::max(maxn, groups[g].n_s);
  }
  CK(cudaEventRecord(ctx->ev[2], ctx->st));
  if (pre.back() > 0) {
    CK(ctx->d_groups.alloc(groups.size()));
    CK(ctx->d_rowpre.alloc(pre.size()));
    CK(ctx->d_thr.alloc(std::max<size_t>(thr.size(), 1)));
    CK(cpy(ctx, ctx->d_groups.p, groups.data(), sizeof(ThrGroup) * groups.size(), cudaMemcpyHostToDevice, ctx->st));
    CK(cpy(ctx, ctx->d_rowpre.p, pre.data(), sizeof(long long) * pre.size(), cudaMemcpyHostToDevice, ctx->st));
    CK(cpy(ctx, ctx->d_thr.p, thr.data(), sizeof(unsigned) * thr.size(), cudaMemcpyHostToDevice, ctx->st));
    ThrParams p{};
    p.D16 = ctx->d_D16.p;
    p.D32 = ctx->d_D32.p;
    p.pos = ctx->d_pos.p;
    p.groups = ctx->d_groups.p;
    p.ngroups = (int)groups.size();
    p.row_pre = ctx->d_rowpre.p;
    p.thr = ctx->d_thr.p;
    p.bits = d_bits;
    p.counts = d_counts;
    CK(ctx->d_thr_status.alloc(1));
    CK(ctx->h_thr_status.alloc(1));
    CK(cudaMemsetAsync(ctx->d_thr_status.p, 0, sizeof(unsigned), ctx->st));
    p.status = ctx->d_thr_status.p;
    p.wait_limit = 1u << 22;
    p.order = ctx->d_order.p;
    int H = ctx->threshold_path == 0 ? transposed_height(maxn) : 0;
    if (ctx->threshold_path == 5 || ctx->threshold_path == 6) {  // test hooks: smaller blocks than automatic
      H = std::min(transposed_height(maxn), ctx->threshold_path == 5 ? 16 : 8);
      if (H < 8) H = 0;
    }
    if (H > 0) {  // transposed two-pass threshold: scratch of H-bit words, item prefix sums
      std::vector<ThrGroup> tg(groups);
      std::vector<long long> pre1(groups.size() + 1, 0), pre2(groups.size() + 1, 0);
      long long tb = 0;
      for (size_t g = 0; g < tg.size(); ++g) {
        ThrGroup& G = tg[g];
        G.nblk = (G.n_s + H - 1) / H;
        G.blk_stride = transposed_block_stride(G.n_s, H);
        G.tb_base = tb;
        tb += (long long)G.nthr * G.nblk * G.blk_stride;
        const int ic = transposed_item_cols();
        pre1[g + 1] = pre1[g] + (long long)G.nblk * ((G.n_s + ic - 1) / ic);
        pre2[g + 1] = pre2[g] + (long long)G.nthr * G.nblk;
      }
      CK(ctx->d_tbits.alloc((size_t)std::max<long long>(tb, 16)));
      CK(ctx->d_tpre.alloc(2 * pre1.size()));
      CK(cpy(ctx, ctx->d_groups.p, tg.data(), sizeof(ThrGroup) * tg.size(), cudaMemcpyHostToDevice, ctx->st));
      CK(cpy(ctx, ctx->d_tpre.p, pre1.data(), sizeof(long long) * pre1.size(), cudaMemcpyHostToDevice, ctx->st));
      CK(cpy(ctx, ctx->d_tpre.p + pre1.size(), pre2.data(), sizeof(long long) * pre2.size(), cudaMemcpyHostToDevice,
             ctx->st));
      p.tbits = ctx->d_tbits.p;
      CK(cudaEventRecord(ctx->ev[2], ctx->st));
      ctx->stats.kernel_launches += 2;
      bool aligned16 = ctx->threshold_path != 5 && ctx->threshold_path != 6;  // test hooks keep the scalar pass
      for (const ThrGroup& G : groups) aligned16 = aligned16 && G.dist_base % 8 == 0 && G.n_s % 8 == 0;
      CK(launch_threshold_transposed(p, H, maxn, aligned16, ctx->d_tpre.p, pre1.back(), ctx->d_tpre.p + pre1.size(),
                                     pre2.back(), ctx->st));
      CK(cudaEventRecord(ctx->ev[3], ctx->st));
      CK(cpy(ctx, ctx->h_thr_status.p, ctx->d_thr_status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->st));
      return SWE_OK;
    }
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    ctx->stats.kernel_launches += 1;
    ThrPlan plan = threshold_plan(maxn, ctx->dist_bytes);  // path 4 (and sets too large for path 0)
    if (ctx->threshold_path == 1) {
      plan.staged = 0, plan.nbuf = 0, plan.stage_pos = 0, plan.block = 256, plan.smem = 0;
    } else if (ctx->threshold_path == 2 && plan.staged) {
      plan.stage_pos = 1;
      plan.smem = plan.nbuf * plan.rowbuf + (size_t)maxn * 4;
      if (plan.smem > 220 * 1024) plan.stage_pos = 0, plan.smem = plan.nbuf * plan.rowbuf;
    } else if (ctx->threshold_path == 3 && plan.staged) {
      plan.nbuf = 1;
      plan.smem = plan.rowbuf;
    }
    CK(launch_threshold(p, pre.back(), plan, ctx->st));
    CK(cudaEventRecord(ctx->ev[3], ctx->st));
    CK(cpy(ctx, ctx->h_thr_status.p, ctx->d_thr_status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->st));
  } else {
    CK(cudaEventRecord(ctx->ev[3], ctx->st));
    CK(ctx->h_thr_status.alloc(1));
    ctx->h_thr_status.p[0] = 0;
  }
  return SWE_OK;
}

// Status word of the last threshold launch; valid once the stream has been
// synchronised after launch_groups.
static swe_status thr_status(swe_ctx* ctx) { return check_kernel_status(ctx, ctx->h_thr_status.p[0]); }

// Neighbour bitmap of set s for threshold T on the host (pinned), cached per
// (set, T).  Rows and columns are in the set's original index order.
static swe_status ensure_bitmap(swe_ctx* ctx, int s, long long T) {
  if (ctx->bits_T == T && ctx->bits_set == s) return SWE_OK;
  const int first = ctx->set_first[s], n = ctx->set_first[s + 1] - first;
  ctx->wpr = (n + 63) / 64;
  const size_t words = (size_t)n * (size_t)ctx->wpr;
  CK(ctx->h_bits.alloc(std::max<size_t>(words, 1)));
  CK(ctx->h_counts.alloc(std::max(n, 1)));
  if (T < 0 || n == 0) {
    if (words) memset(ctx->h_bits.p, 0, words * 8);
    if (n) memset(ctx->h_counts.p, 0, sizeof(int) * n);
    ctx->bits_T = T;
    ctx->bits_set = s;
    return SWE_OK;
  }
  CK(ctx->d_bits.alloc(words));
  CK(ctx->d_counts.alloc(n));
  std::vector<ThrGroup> groups;
  std::vector<unsigned> thr;
  long long bw = 0, ci = 0;
  add_set_groups(ctx, s, &T, 1, &groups, &thr, &bw, &ci);
  if (swe_status st = launch_groups(ctx, groups, thr, ctx->d_bits.p, ctx->d_counts.p)) return st;
  CK(cpy(ctx, ctx->h_bits.p, ctx->d_bits.p, words * 8, cudaMemcpyDeviceToHost, ctx->st));
  CK(cpy(ctx, ctx->h_counts.p, ctx->d_counts.p, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (swe_status st = thr_status(ctx)) return st;
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
  ctx->stats.ms_last_neighbors = ms;
  ctx->stats.last_neighbor_launches = 1;
  ctx->bits_T = T;
  ctx->bits_set = s;
  return SWE_OK;
}

// The single-set calls refuse uploads of several sets.
static swe_status need_one_set(swe_ctx* ctx) {
  if (ctx->n_sets != 1) return fail(ctx, SWE_ERR_STATE, "several sets uploaded: use the per-set calls");
  return SWE_OK;
}

extern "C" {

static swe_status check_set(swe_ctx* ctx, int s) {
  if (!ctx->scored) return fail(ctx, SWE_ERR_STATE, "no scored dataset");
  if (s < 0 || s >= ctx->n_sets) return fail(ctx, SWE_ERR_INVALID, "no such set");
  return select_device(ctx);
}

swe_status swe_neighbors_set(swe_ctx* ctx, int set, float eps, int64_t** row_ptr, int** cols) {
  if (!ctx || !row_ptr || !cols) return SWE_ERR_INVALID;
  if (swe_status s = check_set(ctx, set)) return s;
  const long long T = ctx_threshold(ctx, eps);
  if (swe_status s = ensure_bitmap(ctx, set, T)) return s;
  const int n = ctx->set_first[set + 1] - ctx->set_first[set];
  int64_t* rp = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
  if (!rp) return fail(ctx, SWE_ERR_OOM, "row_ptr");
  rp[0] = 0;
  for (int i = 0; i < n; ++i) rp[i + 1] = rp[i] + ctx->h_counts.p[i];
  const int64_t E = rp[n];
  int* cl = (int*)malloc(sizeof(int) * std::max<int64_t>(E, 1));
  if (!cl) {
    free(rp);
    return fail(ctx, SWE_ERR_OOM, "cols");
  }
  if (E > 0) {
    swe_status s = SWE_OK;
    cudaError_t e = ctx->d_row_ptr.alloc(n + 1);
    if (e == cudaSuccess) e = ctx->d_cols.alloc(E);
    if (e == cudaSuccess)
      e = cpy(ctx, ctx->d_row_ptr.p, rp, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, ctx->st);
    ctx->stats.kernel_launches += 1;
    if (e == cudaSuccess)
      e = launch_csr_fill(ctx->d_bits.p, n, ctx->wpr, ctx->d_row_ptr.p, ctx->d_cols.p, ctx->st);
    if (e == cudaSuccess) e = cpy(ctx, cl, ctx->d_cols.p, sizeof(int) * E, cudaMemcpyDeviceToHost, ctx->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    if (e != cudaSuccess) s = cuda_fail(ctx, e, "neighbour lists");
    if (s) {
      free(rp);
      free(cl);
      return s;
    }
  }
  *row_ptr = rp;
  *cols = cl;
  return SWE_OK;
}

swe_status swe_neighbors(swe_ctx* ctx, float eps, int64_t** row_ptr, int** cols) {
  if (!ctx || !row_ptr || !cols) return SWE_ERR_INVALID;
  if (swe_status s = need_one_set(ctx)) return s;
  return swe_neighbors_set(ctx, 0, eps, row_ptr, cols);
}

swe_status swe_dbscan_set(swe_ctx* ctx, int set, float eps, int minpts, split_set* out) {
  if (!ctx || !out) return SWE_ERR_INVALID;
  out->n_clusters = 0;
  out->clusters = nullptr;
  if (swe_status s = check_set(ctx, set)) return s;
  if (eps == -1) eps = 0.015f;  // dbscan.c:980-984
  if (minpts == -1) minpts = 5; // dbscan.c:985-989
  const long long T = ctx_threshold(ctx, eps);
  if (swe_status s = ensure_bitmap(ctx, set, T)) return s;
  const int n = ctx->set_first[set + 1] - ctx->set_first[set];
  const int rc = dbscan_replay_bitmap(n, ctx->h_bits.p, ctx->wpr, ctx->h_counts.p, minpts, out);
  if (rc) return fail(ctx, (swe_status)rc, "dbscan replay");
  return SWE_OK;
}

swe_status swe_dbscan(swe_ctx* ctx, float eps, int minpts, split_set* out) {
  if (!ctx || !out) return SWE_ERR_INVALID;
  out->n_clusters = 0;
  out->clusters = nullptr;
  if (swe_status s = need_one_set(ctx)) return s;
  return swe_dbscan_set(ctx, 0, eps, minpts, out);
}

swe_status swe_adaptive_set(swe_ctx* ctx, int set, float eps_start, float eps_inc, int minpts, const char* prefix,
                            FILE* log, split_set** out_sets, int* out_n_sets) {
  if (!ctx) return SWE_ERR_INVALID;
  if (swe_status s = check_set(ctx, set)) return s;
  DbscanProvider prov;
  prov.run = [ctx, set, minpts](const float* e, int c, split_set* o) {
    return engine_dbscan_batch(ctx, set, e, c, minpts, o);
  };
  prov.batch = engine_batch_size(ctx, set);
  prov.key = [ctx](float e) { return ctx_sweep_key(ctx, e); };
  prov.speculate = true;
  std::vector<split_set> kept;
  std::string err;
  const long long fixed = ctx_fixed_point(ctx);
  const int n = ctx->set_first[set + 1] - ctx->set_first[set];
  const int rc = adaptive_sweep(n, eps_start, eps_inc, minpts, prefix, log ? log : stdout, prov, true, fixed,
                                &kept, &err);
  if (rc) {
    for (auto& s : kept) free_split_set_and_associated_clusters(s);
    return fail(ctx, (swe_status)rc, err);
  }
  if (out_n_sets) *out_n_sets = (int)kept.size();
  if (out_sets) {
    split_set* arr = (split_set*)malloc(sizeof(split_set) * std::max<size_t>(kept.size(), 1));
    if (!arr) {
      for (auto& s : kept) free_split_set_and_associated_clusters(s);
      return fail(ctx, SWE_ERR_OOM, "split set array");
    }
    for (size_t k = 0; k < kept.size(); ++k) arr[k] = kept[k];
    *out_sets = arr;
    if (out_n_sets) *out_n_sets = (int)kept.size();
  } else {
    for (auto& s : kept) free_split_set_and_associated_clusters(s);
  }
  return SWE_OK;
}

swe_status swe_adaptive(swe_ctx* ctx, float eps_start, float eps_inc, int minpts, const char* prefix,
                        FILE* log, split_set** out_sets, int* out_n_sets) {
  if (!ctx) return SWE_ERR_INVALID;
  if (swe_status s = need_one_set(ctx)) return s;
  return swe_adaptive_set(ctx, 0, eps_start, eps_inc, minpts, prefix, log, out_sets, out_n_sets);
}

}  // extern "C"

namespace {

// f(i) for i in [0, n) on up to hardware_concurrency threads, dynamic order.
template <class F>
void parallel_for(int n, F&& f) {
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int T = std::min(hw, n);
  if (T <= 1) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> th;
  th.reserve(T);
  for (int t = 0; t < T; ++t)
    th.emplace_back([&]() {
      for (;;) {
        const int i = next.fetch_add(1);
        if (i >= n) break;
        f(i);
      }
    });
  for (auto& t : th) t.join();
}

// One distinct threshold of one set in a round.
struct SweepJob {
  int set;
  long long T;
  long long bits_off;   // words into the round's bitmap buffer (-1: no launch, empty neighbourhoods)
  long long count_off;  // ints into the round's count buffer
  split_set res;
  int rc;
  int replay = -1;      // its instance in the round's device replay launch (-1: none)
  long long cs_off = 0; // ints into the round's cluster-start buffer
};

// The DBSCAN replays of a round's launched jobs in one device launch over the
// bitmaps the threshold pass left in d_bbits / d_bcounts (largest sets first);
// members, cluster starts and counts come back to the pinned buffers.
swe_status device_replays(swe_ctx* ctx, std::vector<SweepJob>& jobs, const std::vector<int>& order, int minpts,
                          long long ci, const int* job_n = nullptr) {
  std::vector<ReplayJob> rj;
  long long cs_total = 0, vis_total = 0, q_total = 0;
  for (int q : order) {
    SweepJob& j = jobs[q];
    if (j.bits_off < 0) continue;
    // points of the instance: its set's size (or job_n[q] for caller bitmaps)
    const int ns = job_n ? job_n[q] : ctx->set_first[j.set + 1] - ctx->set_first[j.set];
    ReplayJob r{j.bits_off, j.count_off, cs_total, vis_total, q_total, ns, 0};
    j.replay = (int)rj.size();
    j.cs_off = cs_total;
    cs_total += ns + 1;
    if (ns > RP_SMEM_NS) {
      vis_total += 2LL * ((ns + 31) / 32);
      q_total += (ns + 63) / 64;
    }
    rj.push_back(r);
  }
  if (rj.empty()) return SWE_OK;
  const size_t nj = rj.size();
  CK(ctx->d_rjobs.alloc(nj));
  CK(ctx->d_rmembers.alloc((size_t)std::max(ci, 1LL)));
  CK(ctx->d_rfrontier.alloc((size_t)std::max(ci, 1LL)));
  CK(ctx->d_rcstart.alloc((size_t)cs_total));
  CK(ctx->d_rncl.alloc(nj));
  CK(ctx->d_rvis.alloc((size_t)std::max(vis_total, 1LL)));
  CK(ctx->d_rqueued.alloc((size_t)std::max(q_total, 1LL)));
  CK(ctx->d_rstatus.alloc(1));
  CK(ctx->h_rmembers.alloc((size_t)std::max(ci, 1LL)));
  CK(ctx->h_rcstart.alloc((size_t)cs_total));
  CK(ctx->h_rncl.alloc(nj));
  CK(ctx->h_rstatus.alloc(1));
  CK(cpy(ctx, ctx->d_rjobs.p, rj.data(), sizeof(ReplayJob) * nj, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemsetAsync(ctx->d_rstatus.p, 0, sizeof(unsigned), ctx->st));
  ctx->stats.kernel_launches += 1;
  CK(launch_dbscan_replay(ctx->d_rjobs.p, (int)nj, ctx->d_bbits.p, ctx->d_bcounts.p, minpts, ctx->d_rmembers.p,
                          ctx->d_rfrontier.p, ctx->d_rcstart.p, ctx->d_rncl.p, ctx->d_rvis.p, ctx->d_rqueued.p,
                          ctx->d_rstatus.p, ctx->st));
  if (ci > 0)
    CK(cpy(ctx, ctx->h_rmembers.p, ctx->d_rmembers.p, sizeof(int) * ci, cudaMemcpyDeviceToHost, ctx->st));
  CK(cpy(ctx, ctx->h_rcstart.p, ctx->d_rcstart.p, sizeof(int) * cs_total, cudaMemcpyDeviceToHost, ctx->st));
  CK(cpy(ctx, ctx->h_rncl.p, ctx->d_rncl.p, sizeof(int) * nj, cudaMemcpyDeviceToHost, ctx->st));
  CK(cpy(ctx, ctx->h_rstatus.p, ctx->d_rstatus.p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->st));
  return SWE_OK;
}

// The split set of a device replay instance (malloc'd like the host replay's).
int replay_result(const swe_ctx* ctx, const SweepJob& j, split_set* out) {
  const int nc = ctx->h_rncl.p[j.replay];
  const int* cs = ctx->h_rcstart.p + j.cs_off;
  const int* mem = ctx->h_rmembers.p + j.count_off;
  out->n_clusters = 0;
  out->clusters = (cluster*)malloc(sizeof(cluster) * (size_t)std::max(nc, 1));
  if (!out->clusters) return SWE_ERR_OOM;
  for (int c = 0; c < nc; ++c) {
    cluster& cl = out->clusters[c];
    cl.n_members = cs[c + 1] - cs[c];
    cl.id = c;
    cl.members = (int*)malloc(sizeof(int) * (size_t)std::max(cl.n_members, 1));
    if (!cl.members) {
      free_split_set_and_associated_clusters(*out);
      out->n_clusters = 0;
      out->clusters = nullptr;
      return SWE_ERR_OOM;
    }
    memcpy(cl.members, mem + cs[c], sizeof(int) * (size_t)cl.n_members);
    out->n_clusters = c + 1;
  }
  return 0;
}

}  // namespace

extern "C" {

swe_status swe_adaptive_sets(swe_ctx* ctx, float eps_start, float eps_inc, int minpts, int max_steps,
                             const char* prefix, swe_sweep_result* results) {
  if (!ctx || !results || max_steps < 0) return SWE_ERR_INVALID;
  if (!ctx->scored) return fail(ctx, SWE_ERR_STATE, "no scored dataset");
  if (swe_status s = select_device(ctx)) return s;
  const auto t0 = std::chrono::steady_clock::now();
  const int S = ctx->n_sets;
  for (int k = 0; k < S; ++k) results[k] = swe_sweep_result{};
  const long long fixed = ctx_fixed_point(ctx);
  const int mp = minpts == -1 ? 5 : minpts;    // dbscan.c:985-989
  const int batch = max_steps > 0 ? std::min(8, max_steps) : 8;
  std::vector<std::unique_ptr<SweepMachine>> m(S);
  std::vector<std::string> logs(S);
  for (int k = 0; k < S; ++k) {
    m[k].reset(new SweepMachine(ctx->set_first[k + 1] - ctx->set_first[k], eps_start, eps_inc, minpts, max_steps,
                                batch, true, fixed));
    m[k]->set_key([ctx](float e) { return ctx_sweep_key(ctx, e); });
    m[k]->set_speculate(true);
  }
  auto finish_set = [&](int k) {
    std::vector<split_set> kept;
    std::string pre;
    if (prefix) pre = std::string(prefix) + std::to_string(k) + "_";
    m[k]->finish(prefix ? pre.c_str() : nullptr, &kept);
    logs[k] += m[k]->take_log();
    swe_sweep_result& r = results[k];
    r.status = m[k]->status();
    r.truncated = m[k]->truncated() ? 1 : 0;
    r.steps = m[k]->steps();
    r.n_layers = (int)kept.size();
    r.layers = (split_set*)malloc(sizeof(split_set) * std::max<size_t>(kept.size(), 1));
    r.log = (char*)malloc(logs[k].size() + 1);
    if (r.layers) {
      for (size_t i = 0; i < kept.size(); ++i) r.layers[i] = kept[i];
    } else {
      for (auto& x : kept) free_split_set_and_associated_clusters(x);
      r.n_layers = 0;
      r.status = SWE_ERR_OOM;
    }
    if (r.log) memcpy(r.log, logs[k].c_str(), logs[k].size() + 1);
    r.done_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  };
  std::vector<int> active;
  for (int k = 0; k < S; ++k) {
    logs[k] += m[k]->take_log();
    if (m[k]->done()) finish_set(k);
    else active.push_back(k);
  }
  const long long budget_words = (1LL << 30) / 8;  // bitmaps of one launch: 1 GiB
  const bool dev_replay = ctx->dbscan_replay != 1;
  double kernel_ms = 0;
  int launches = 0;
  while (!active.empty()) {
    // largest sets first: their replays start first and their bitmaps are copied first
    std::stable_sort(active.begin(), active.end(), [&](int x, int y) {
      return ctx->set_first[x + 1] - ctx->set_first[x] > ctx->set_first[y + 1] - ctx->set_first[y];
    });
    size_t a = 0;
    while (a < active.size()) {
      // sets [a, b) of the active list share one launch
      std::vector<ThrGroup> groups;
      std::vector<unsigned> thr;
      std::vector<SweepJob> jobs;
      std::vector<size_t> job_first;
      long long bw = 0, ci = 0;
      size_t b = a;
      for (; b < active.size(); ++b) {
        const int k = active[b];
        const int ns = ctx->set_first[k + 1] - ctx->set_first[k], wpr = (ns + 63) / 64;
        std::vector<long long> launchT;
        std::vector<long long> uniq;
        for (float e : m[k]->request()) {
          const long long T = ctx_threshold(ctx, e == -1 ? 0.015f : e);  // dbscan.c:980-984
          if (std::find(uniq.begin(), uniq.end(), T) == uniq.end()) uniq.push_back(T);
        }
        for (long long T : uniq)
          if (T >= 0 && ns > 0) launchT.push_back(T);
        const long long words = (long long)launchT.size() * ns * wpr;
        if (b > a && bw + words > budget_words) break;
        job_first.push_back(jobs.size());
        long long off = bw, coff = ci;
        for (long long T : uniq) {
          SweepJob j{k, T, -1, -1, split_set{0, nullptr}, 0};
          if (T >= 0 && ns > 0) {
            j.bits_off = off;
            j.count_off = coff;
            off += (long long)ns * wpr;
            coff += ns;
          }
          jobs.push_back(j);
        }
        add_set_groups(ctx, k, launchT.data(), (int)launchT.size(), &groups, &thr, &bw, &ci);
      }
      job_first.push_back(jobs.size());
      // the bitmaps come back in chunks (in the sets' memory order, largest
      // first); a replay waits for the chunk that completes its bitmap
      constexpr int NCH = 16;
      std::vector<cudaEvent_t> chunk_ev(NCH, nullptr);
      struct EventGuard {
        std::vector<cudaEvent_t>& ev;
        ~EventGuard() {
          for (auto e : ev)
            if (e) cudaEventDestroy(e);
        }
      } guard{chunk_ev};
      // the chunk whose range [total*c/NCH, total*(c+1)/NCH) holds pos
      auto chunk_of = [&](long long pos, long long total) -> int {
        int c = 0;
        while (c + 1 < NCH && total * (c + 1) / NCH <= pos) ++c;
        return c;
      };
      // order-faithful replays, one per (set, distinct threshold), largest sets first
      std::vector<int> order(jobs.size());
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return ctx->set_first[jobs[x].set + 1] - ctx->set_first[jobs[x].set] >
               ctx->set_first[jobs[y].set + 1] - ctx->set_first[jobs[y].set];
      });
      if (bw > 0 && dev_replay) {
        // the bitmaps stay on the device: one replay launch, the clusters come back
        CK(ctx->d_bbits.alloc((size_t)bw));
        CK(ctx->d_bcounts.alloc((size_t)ci));
        if (swe_status st = launch_groups(ctx, groups, thr, ctx->d_bbits.p, ctx->d_bcounts.p)) return st;
        if (swe_status st = device_replays(ctx, jobs, order, mp, ci)) return st;
        CK(cudaStreamSynchronize(ctx->st));
        if (swe_status st = thr_status(ctx)) return st;
        if (swe_status st = check_kernel_status(ctx, ctx->h_rstatus.p[0])) return st;
      } else if (bw > 0) {
        CK(ctx->d_bbits.alloc((size_t)bw));
        CK(ctx->d_bcounts.alloc((size_t)ci));
        CK(ctx->h_bbits.alloc((size_t)bw));
        CK(ctx->h_bcounts.alloc((size_t)ci));
        if (swe_status st = launch_groups(ctx, groups, thr, ctx->d_bbits.p, ctx->d_bcounts.p)) return st;
        for (int c = 0; c < NCH; ++c) {
          const long long w0 = bw * c / NCH, w1 = bw * (c + 1) / NCH;
          const long long c0 = ci * c / NCH, c1 = ci * (c + 1) / NCH;
          if (w1 > w0)
            CK(cpy(ctx, ctx->h_bbits.p + w0, ctx->d_bbits.p + w0, sizeof(uint64_t) * (w1 - w0),
                   cudaMemcpyDeviceToHost, ctx->st));
          if (c1 > c0)
            CK(cpy(ctx, ctx->h_bcounts.p + c0, ctx->d_bcounts.p + c0, sizeof(int) * (c1 - c0),
                   cudaMemcpyDeviceToHost, ctx->st));
          CK(cudaEventCreateWithFlags(&chunk_ev[c], cudaEventDisableTiming));
          CK(cudaEventRecord(chunk_ev[c], ctx->st));
        }
      }
      parallel_for((int)jobs.size(), [&](int q) {
        SweepJob& j = jobs[order[q]];
        const int ns = ctx->set_first[j.set + 1] - ctx->set_first[j.set], wpr = (ns + 63) / 64;
        if (j.replay >= 0) {
          j.rc = replay_result(ctx, j, &j.res);
        } else if (j.bits_off >= 0) {
          const int c = std::max(chunk_of(j.bits_off + (long long)ns * wpr - 1, bw), chunk_of(j.count_off + ns - 1, ci));
          if (cudaEventSynchronize(chunk_ev[c]) != cudaSuccess) {
            j.rc = SWE_ERR_CUDA;
            return;
          }
          j.rc = dbscan_replay_bitmap(ns, ctx->h_bbits.p + j.bits_off, wpr, ctx->h_bcounts.p + j.count_off, mp,
                                      &j.res);
        } else {  // no neighbour at all, not even the point itself
          std::vector<uint64_t> zb((size_t)ns * wpr + 1, 0);
          std::vector<int> zc((size_t)ns + 1, 0);
          j.rc = dbscan_replay_bitmap(ns, zb.data(), wpr, zc.data(), mp, &j.res);
        }
      });
      if (bw > 0) {
        CK(cudaStreamSynchronize(ctx->st));
        swe_status st = thr_status(ctx);
        if (st) {
          for (auto& j : jobs) free_split_set_and_associated_clusters(j.res);
          return st;
        }
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
        kernel_ms += ms;
        ++launches;
      }
      // advance every set of the launch
      parallel_for((int)(b - a), [&](int x) {
        const int k = active[a + x];
        const std::vector<float>& req = m[k]->request();
        std::vector<split_set> out(req.size(), split_set{0, nullptr});
        std::vector<bool> used(job_first[x + 1] - job_first[x], false);
        int rc = 0;
        for (size_t q = job_first[x]; q < job_first[x + 1]; ++q) rc = rc ? rc : jobs[q].rc;
        if (rc) {
          for (size_t q = job_first[x]; q < job_first[x + 1]; ++q) free_split_set_and_associated_clusters(jobs[q].res);
          m[k]->abort(rc, "dbscan replay failed");
        } else {
          for (size_t e = 0; e < req.size(); ++e) {
            const long long T = ctx_threshold(ctx, req[e] == -1 ? 0.015f : req[e]);
            size_t q = job_first[x];
            while (jobs[q].T != T) ++q;
            const size_t u = q - job_first[x];
            out[e] = used[u] ? copy_split_set(jobs[q].res) : jobs[q].res;
            used[u] = true;
          }
          for (size_t q = job_first[x]; q < job_first[x + 1]; ++q)
            if (!used[q - job_first[x]]) free_split_set_and_associated_clusters(jobs[q].res);
          m[k]->consume(out.data());
        }
        logs[k] += m[k]->take_log();
        if (m[k]->done()) finish_set(k);
      });
      a = b;
    }
    std::vector<int> still;
    for (int k : active)
      if (!m[k]->done()) still.push_back(k);
    active.swap(still);
  }
  ctx->stats.ms_last_neighbors = kernel_ms;
  ctx->stats.last_neighbor_launches = launches;
  return SWE_OK;
}

swe_status swe_dbscan_bitmaps_device(swe_ctx* ctx, int n_inst, const int* n, const uint64_t* bits,
                                     const int64_t* bits_off, int64_t bits_words, const int* counts,
                                     const int64_t* counts_off, int64_t counts_len, int minpts, split_set* out) {
  if (!ctx || n_inst < 0 || (n_inst > 0 && (!n || !bits_off || !counts_off || !out)) || bits_words < 0 ||
      counts_len < 0)
    return SWE_ERR_INVALID;
  for (int k = 0; k < n_inst; ++k) {
    out[k] = split_set{0, nullptr};
    const long long wpr = (n[k] + 63) / 64;
    if (n[k] < 0 || bits_off[k] < 0 || counts_off[k] < 0 || bits_off[k] + (long long)n[k] * wpr > bits_words ||
        counts_off[k] + n[k] > counts_len)
      return SWE_ERR_INVALID;
  }
  if (n_inst == 0) return SWE_OK;
  if (swe_status s = select_device(ctx)) return s;
  const int mp = minpts == -1 ? 5 : minpts;  // dbscan.c:985-989
  // one SweepJob per instance; members / frontiers at fresh offsets
  std::vector<SweepJob> jobs((size_t)n_inst);
  std::vector<int> order((size_t)n_inst);
  long long ci = 0;
  for (int k = 0; k < n_inst; ++k) {
    jobs[k] = SweepJob{0, 0, n[k] > 0 ? (long long)bits_off[k] : -1, ci, split_set{0, nullptr}, 0};
    ci += n[k];
    order[k] = k;
  }
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return n[x] > n[y]; });
  // counts regrouped at the members' offsets
  std::vector<int> cnt((size_t)std::max<long long>(ci, 1));
  for (int k = 0; k < n_inst; ++k)
    if (n[k] > 0) memcpy(cnt.data() + jobs[k].count_off, counts + counts_off[k], sizeof(int) * (size_t)n[k]);
  CK(ctx->d_bbits.alloc((size_t)std::max<int64_t>(bits_words, 1)));
  CK(ctx->d_bcounts.alloc((size_t)std::max<long long>(ci, 1)));
  if (bits_words > 0)
    CK(cpy(ctx, ctx->d_bbits.p, bits, sizeof(uint64_t) * (size_t)bits_words, cudaMemcpyHostToDevice, ctx->st));
  if (ci > 0) CK(cpy(ctx, ctx->d_bcounts.p, cnt.data(), sizeof(int) * (size_t)ci, cudaMemcpyHostToDevice, ctx->st));
  if (swe_status st = device_replays(ctx, jobs, order, mp, ci, n)) return st;
  CK(cudaStreamSynchronize(ctx->st));
  if (swe_status st = check_kernel_status(ctx, ctx->h_rstatus.p[0])) return st;
  for (int k = 0; k < n_inst; ++k) {
    int rc = 0;
    if (jobs[k].replay >= 0) rc = replay_result(ctx, jobs[k], &out[k]);
    else out[k].clusters = (cluster*)malloc(sizeof(cluster));  // no points: no cluster
    if (rc || !out[k].clusters) {
      for (int x = 0; x <= k; ++x) {
        free_split_set_and_associated_clusters(out[x]);
        out[x] = split_set{0, nullptr};
      }
      return SWE_ERR_OOM;
    }
  }
  return SWE_OK;
}

void swe_free_sweep_results(swe_sweep_result* results, int n) {
  if (!results) return;
  for (int k = 0; k < n; ++k) {
    for (int i = 0; i < results[k].n_layers; ++i) free_split_set_and_associated_clusters(results[k].layers[i]);
    free(results[k].layers);
    free(results[k].log);
    results[k].layers = nullptr;
    results[k].log = nullptr;
    results[k].n_layers = 0;
  }
}

swe_status swe_score_one_to_many(swe_ctx* ctx, const char* q, size_t qlen, unsigned* out) {
  if (!ctx || (!q && qlen > 0) || (!out && ctx->n > 0)) return SWE_ERR_INVALID;
  if (swe_status s = need_sequences(ctx)) return s;
  if (swe_status s = select_device(ctx)) return s;
  if (ctx->n == 0) return SWE_OK;
  if (qlen > (size_t)(INT_MAX / 8)) return fail(ctx, SWE_ERR_INVALID, "query too long");
  const int L = (int)qlen;
  std::vector<uint8_t> qc((size_t)std::max(L, 1) + 15, 0);
  for (int r = 0; r < L; ++r) qc[r] = (uint8_t)ctx->code_of[(unsigned char)q[r + 1]];
  CK(ctx->d_q.alloc(qc.size()));
  CK(ctx->d_out.alloc(ctx->n));
  long long need_stride = std::min<long long>(L, ctx->max_len) > GEN_CHUNK ? std::max<long long>(L, ctx->max_len) + 1 : 0;
  int grid = ctx->gen_grid;
  int* scratch = ctx->d_scratch.p;
  long long stride = ctx->scratch_stride;
  if (need_stride > stride) {
    grid = ctx->num_sms;
    CK(ctx->d_small_scratch.alloc((size_t)grid * 8 * need_stride));
    scratch = ctx->d_small_scratch.p;
    stride = need_stride;
  }
  CK(cpy(ctx, ctx->d_q.p, qc.data(), qc.size(), cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemsetAsync(ctx->d_ctr.p + 1, 0, sizeof(unsigned), ctx->st));
  GenParams g{};
  g.mode = GEN_QUERY;
  g.codes = ctx->d_codes.p;
  g.code_off = ctx->d_off.p;
  g.len = ctx->d_len.p;
  g.n = ctx->n;
  g.qcodes = ctx->d_q.p;
  g.qlen = L;
  g.out = ctx->d_out.p;
  g.scratch = scratch;
  g.scratch_stride = stride;
  g.nwarps_total = grid * 8;
  g.status = ctx->d_ctr.p + 1;
  ctx->stats.kernel_launches += 1;
  CK(launch_generic(g, grid, ctx->st));
  CK(cpy(ctx, out, ctx->d_out.p, sizeof(unsigned) * ctx->n, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return SWE_OK;
}

swe_status swe_score_pairs(swe_ctx* ctx, const int* a, const int* b, int64_t npairs, unsigned* out) {
  if (!ctx || npairs < 0 || (npairs > 0 && (!a || !b || !out))) return SWE_ERR_INVALID;
  if (swe_status s = need_sequences(ctx)) return s;
  if (npairs == 0) return SWE_OK;
  if (swe_status s = select_device(ctx)) return s;
  std::vector<int2> pr(npairs);
  for (int64_t k = 0; k < npairs; ++k) {
    if (a[k] < 0 || a[k] >= ctx->n || b[k] < 0 || b[k] >= ctx->n)
      return fail(ctx, SWE_ERR_INVALID, "pair index out of range");
    pr[k] = make_int2(a[k], b[k]);
  }
  CK(ctx->d_pairs.alloc(npairs));
  CK(ctx->d_out.alloc(npairs));
  CK(cpy(ctx, ctx->d_pairs.p, pr.data(), sizeof(int2) * npairs, cudaMemcpyHostToDevice, ctx->st));
  GenParams g{};
  g.mode = GEN_PAIRS_OUT;
  g.codes = ctx->d_codes.p;
  g.code_off = ctx->d_off.p;
  g.len = ctx->d_len.p;
  g.n = ctx->n;
  g.pairs = ctx->d_pairs.p;
  g.npairs = npairs;
  g.out = ctx->d_out.p;
  g.scratch = ctx->d_scratch.p;
  g.scratch_stride = ctx->scratch_stride;
  g.nwarps_total = ctx->gen_grid * 8;
  g.status = ctx->d_ctr.p + 1;
  ctx->stats.kernel_launches += 1;
  CK(launch_generic(g, ctx->gen_grid, ctx->st));
  CK(cpy(ctx, out, ctx->d_out.p, sizeof(unsigned) * npairs, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return SWE_OK;
}

swe_status swe_measure_mix_peak(int device, double* cells_per_s, double* lane_instr_per_s) {
  if (!cells_per_s || !lane_instr_per_s) return SWE_ERR_INVALID;
  swe_ctx* ctx = nullptr;
  swe_opts o{};
  o.device = device;
  if (swe_status s = swe_create(&ctx, &o)) return s;
  struct Guard {
    swe_ctx* c;
    ~Guard() { swe_destroy(c); }
  } guard{ctx};
  const int block = 256, grid = ctx->num_sms * 8, iters = 4096;
  DevBuf<uint32_t> sink;
  CK(sink.alloc((size_t)grid * block));
  CK(launch_mix_probe(sink.p, grid, block, 64, ctx->st));  // warm-up
  CK(cudaEventRecord(ctx->ev[0], ctx->st));
  CK(launch_mix_probe(sink.p, grid, block, iters, ctx->st));
  CK(cudaEventRecord(ctx->ev[1], ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
  const double updates = (double)grid * block * iters * 8.0;  // packed cell updates (8 chains)
  *cells_per_s = 2.0 * updates / (ms * 1e-3);
  *lane_instr_per_s = 4.5 * updates / (ms * 1e-3);  // PRMT, 2 adds, 3-input max, half a max
  return SWE_OK;
}

swe_status swe_timer_start(swe_ctx* ctx) {
  if (!ctx) return SWE_ERR_INVALID;
  if (swe_status s = select_device(ctx)) return s;
  CK(cudaEventRecord(ctx->tev[0], ctx->st));
  return SWE_OK;
}

swe_status swe_timer_stop(swe_ctx* ctx, double* ms) {
  if (!ctx || !ms) return SWE_ERR_INVALID;
  if (swe_status s = select_device(ctx)) return s;
  CK(cudaEventRecord(ctx->tev[1], ctx->st));
  CK(cudaEventSynchronize(ctx->tev[1]));
  float f = 0;
  CK(cudaEventElapsedTime(&f, ctx->tev[0], ctx->tev[1]));
  *ms = f;
  return SWE_OK;
}

swe_status swe_get_stats(const swe_ctx* ctx, swe_stats* out) {
  if (!ctx || !out) return SWE_ERR_INVALID;
  *out = ctx->stats;
  return SWE_OK;
}

}  // extern "C"

namespace swgpu {

int engine_batch_size(const swe_ctx* ctx, int set) {
  const double ns = ctx->set_first[set + 1] - ctx->set_first[set];
  const double bytes = ns * std::floor((ns + 63) / 64) * 8.0;
  const double budget = 2.0 * 1024 * 1024 * 1024;  // device and pinned host bytes for one batch
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  return (int)std::max(1.0, std::min({8.0, (double)hw, budget / std::max(bytes, 1.0)}));
}

int engine_dbscan_batch(swe_ctx* ctx, int set, const float* eps, int count, int minpts, split_set* out) {
  for (int k = 0; k < count; ++k) out[k] = split_set{0, nullptr};
  if (swe_status s = check_set(ctx, set)) return s;
  const auto t_begin = std::chrono::steady_clock::now();
  if (minpts == -1) minpts = 5;  // dbscan.c:985-989
  const int first = ctx->set_first[set], n = ctx->set_first[set + 1] - first;
  const int wpr = (n + 63) / 64;
  const size_t words = (size_t)n * (size_t)wpr;
  // distinct thresholds (eps == -1 means 0.015, dbscan.c:980-984)
  std::vector<long long> uniq;
  std::vector<int> slot(count);
  for (int k = 0; k < count; ++k) {
    const long long T = ctx_threshold(ctx, eps[k] == -1 ? 0.015f : eps[k]);
    const auto it = std::find(uniq.begin(), uniq.end(), T);
    slot[k] = (int)(it - uniq.begin());
    if (it == uniq.end()) uniq.push_back(T);
  }
  const int U = (int)uniq.size();
  CK(ctx->h_bbits.alloc(std::max<size_t>(words * U, 1)));
  CK(ctx->h_bcounts.alloc(std::max<size_t>((size_t)n * U, 1)));
  // thresholds >= 0 first (one launch reads the matrix once for all of them)
  std::vector<int> launch_idx, none_idx, launch_of(U, -1);
  std::vector<long long> launchT;
  for (int u = 0; u < U; ++u) {
    if (uniq[u] >= 0 && n > 0) {
      launch_of[u] = (int)launch_idx.size();
      launch_idx.push_back(u);
      launchT.push_back(uniq[u]);
    } else {
      none_idx.push_back(u);
    }
  }
  for (int u : none_idx) {  // no neighbour at all, not even the point itself
    if (words) memset(ctx->h_bbits.p + words * u, 0, words * 8);
    if (n) memset(ctx->h_bcounts.p + (size_t)n * u, 0, sizeof(int) * n);
  }
  const int UL = (int)launch_idx.size();
  // one event per bitmap copy: each replay starts as soon as its bitmap is on the host
  std::vector<cudaEvent_t> ready(UL, nullptr);
  struct EventGuard {
    std::vector<cudaEvent_t>& ev;
    ~EventGuard() {
      for (auto e : ev)
        if (e) cudaEventDestroy(e);
    }
  } guard{ready};
  if (UL > 0) {
    CK(ctx->d_bbits.alloc(words * UL));
    CK(ctx->d_bcounts.alloc((size_t)n * UL));
    std::vector<ThrGroup> groups;
    std::vector<unsigned> thr;
    long long bw = 0, ci = 0;
    add_set_groups(ctx, set, launchT.data(), UL, &groups, &thr, &bw, &ci);
    if (swe_status st = launch_groups(ctx, groups, thr, ctx->d_bbits.p, ctx->d_bcounts.p)) return st;
    for (int j = 0; j < UL; ++j) {
      const int u = launch_idx[j];
      CK(cudaEventCreateWithFlags(&ready[j], cudaEventDisableTiming));
      CK(cpy(ctx, ctx->h_bcounts.p + (size_t)n * u, ctx->d_bcounts.p + (size_t)n * j, sizeof(int) * n,
             cudaMemcpyDeviceToHost, ctx->st));
      CK(cpy(ctx, ctx->h_bbits.p + words * u, ctx->d_bbits.p + words * j, words * 8, cudaMemcpyDeviceToHost,
             ctx->st));
      CK(cudaEventRecord(ready[j], ctx->st));
    }
  }
  // one order-faithful replay per distinct threshold, in parallel, each after its copy
  std::vector<split_set> res(U, split_set{0, nullptr});
  std::vector<int> rc(U, 0);
  std::vector<double> replay_ms(U, 0.0);
  std::vector<std::thread> th;
  for (int u = 0; u < U; ++u)
    th.emplace_back([&, u]() {
      if (launch_of[u] >= 0 && cudaEventSynchronize(ready[launch_of[u]]) != cudaSuccess) {
        rc[u] = SWE_ERR_CUDA;
        return;
      }
      const auto t0 = std::chrono::steady_clock::now();
      rc[u] = dbscan_replay_bitmap(n, ctx->h_bbits.p + words * u, wpr, ctx->h_bcounts.p + (size_t)n * u, minpts,
                                   &res[u]);
      replay_ms[u] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    });
  for (auto& t : th) t.join();
  CK(cudaStreamSynchronize(ctx->st));
  float ms = 0;
  if (UL > 0) {
    if (swe_status st = thr_status(ctx)) {
      for (auto& s : res) free_split_set_and_associated_clusters(s);
      return st;
    }
    CK(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
  }
  ctx->stats.ms_last_neighbors = ms;
  ctx->stats.last_neighbor_launches = UL > 0 ? 1 : 0;
  int bad = 0;
  for (int u = 0; u < U; ++u) bad = bad ? bad : rc[u];
  if (bad) {
    for (auto& s : res) free_split_set_and_associated_clusters(s);
    return fail(ctx, (swe_status)bad, bad == SWE_ERR_CUDA ? "bitmap copy" : "dbscan replay");
  }
  ctx->stats.ms_last_replay = U ? *std::max_element(replay_ms.begin(), replay_ms.end()) : 0.0;
  ctx->stats.ms_last_batch =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count();
  std::vector<bool> used(U, false);
  for (int k = 0; k < count; ++k) {
    const int u = slot[k];
    out[k] = used[u] ? copy_split_set(res[u]) : res[u];
    used[u] = true;
  }
  return SWE_OK;
}

long long eps_threshold(float eps) {
  if (!(eps >= 0.0f)) return -1;  // negative or NaN: not even the point itself
  if (eps >= 9.0e18f) return LLONG_MAX / 2;
  return (long long)std::floor((double)eps);
}

// Distance of one pair of raw strings (the drop-in score()); codes are the
// raw bytes, which keeps equality exact without a code table.
swe_status score_raw(swe_ctx* ctx, const char* A, size_t la, const char* B, size_t lb, unsigned* out) {
  if (!ctx || !out || (!A && la) || (!B && lb)) return SWE_ERR_INVALID;
  if (la > (size_t)(INT_MAX / 8) || lb > (size_t)(INT_MAX / 8)) return fail(ctx, SWE_ERR_INVALID, "too long");
  if (swe_status s = select_device(ctx)) return s;
  const int64_t oa = 0, ob = ((int64_t)la + 15) & ~int64_t(15);
  std::vector<uint8_t> buf((size_t)(ob + lb + 16), 0);
  for (size_t r = 0; r < la; ++r) buf[oa + r] = (uint8_t)A[r + 1];
  for (size_t r = 0; r < lb; ++r) buf[ob + r] = (uint8_t)B[r + 1];
  const int64_t offs[2] = {oa, ob};
  const int lens[2] = {(int)la, (int)lb};
  const int2 pr = make_int2(0, 1);
  CK(ctx->d_q.alloc(buf.size()));
  CK(ctx->d_small_off.alloc(2));
  CK(ctx->d_small_len.alloc(2));
  CK(ctx->d_pairs.alloc(1));
  CK(ctx->d_out.alloc(1));
  const long long need = std::min(la, lb) > (size_t)GEN_CHUNK ? (long long)std::max(la, lb) + 1 : 1;
  CK(ctx->d_small_scratch.alloc((size_t)8 * need));
  CK(cpy(ctx, ctx->d_q.p, buf.data(), buf.size(), cudaMemcpyHostToDevice, ctx->st));
  CK(cpy(ctx, ctx->d_small_off.p, offs, sizeof(offs), cudaMemcpyHostToDevice, ctx->st));
  CK(cpy(ctx, ctx->d_small_len.p, lens, sizeof(lens), cudaMemcpyHostToDevice, ctx->st));
  CK(cpy(ctx, ctx->d_pairs.p, &pr, sizeof(pr), cudaMemcpyHostToDevice, ctx->st));
  GenParams g{};
  g.mode = GEN_PAIRS_OUT;
  g.codes = ctx->d_q.p;
  g.code_off = ctx->d_small_off.p;
  g.len = ctx->d_small_len.p;
  g.n = 2;
  g.pairs = ctx->d_pairs.p;
  g.npairs = 1;
  g.out = ctx->d_out.p;
  g.scratch = ctx->d_small_scratch.p;
  g.scratch_stride = need;
  g.nwarps_total = 8;
  g.status = ctx->d_ctr.p + 1;
  ctx->stats.kernel_launches += 1;
  CK(launch_generic(g, 1, ctx->st));
  CK(cpy(ctx, out, ctx->d_out.p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return SWE_OK;
}

}  // namespace swgpu
