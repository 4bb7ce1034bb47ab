// Engine context shared by the engine's translation units (no public ABI).
#pragma once
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <string>
#include <vector>

#include "host_internal.h"
#include "sw_device.cuh"
#include "sw_kernels.cuh"
#include "dbscan_kernels.cuh"

namespace swgpu {

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    if (p && count <= n) return cudaSuccess;
    release();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e == cudaSuccess) n = count;
    else p = nullptr;
    return e;
  }
};

template <typename T>
struct HostPinned {
  T* p = nullptr;
  size_t n = 0;
  HostPinned() = default;
  HostPinned(const HostPinned&) = delete;
  HostPinned& operator=(const HostPinned&) = delete;
  ~HostPinned() { release(); }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    if (p && count <= n) return cudaSuccess;
    release();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e == cudaSuccess) n = count;
    else p = nullptr;
    return e;
  }
};

// Candidate pairs that restrict a layout to the tiles holding one: a host
// vector, or `count` pairs on the device (original indices, bit 31 of .x a
// flag the layout ignores).
struct CandSource {
  const std::vector<int2>* host = nullptr;
  const int2* dev = nullptr;
  long long count = 0;
};

struct PrefilterState;
void prefilter_destroy(PrefilterState* pf);
struct KmerState;
void kmer_state_destroy(KmerState* km);
struct PcaState;
void pca_state_destroy(PcaState* ps);
struct Staging;
void staging_destroy(Staging* sg);

}  // namespace swgpu

struct swe_ctx {
  int device = 0;
  cudaStream_t st = nullptr;
  int num_sms = 148;
  int sat_limit = 32000;
  int packs_per_block = 32;     // row-sequence pairs per tile of the full layout
  int pf_packs_per_block = 8;   // the same for candidate-tile layouts (sparser work, finer tiles)
  int layout_pb = 32;           // the value the current layout was built with
  int threads = 256;
  int max_w = swgpu::FAST_MAX_W;
  double ms_layout_marks = 0, ms_layout_upload = 0;  // host time of build_layout's tile marks and uploads  // lane-split rule: a column sequence gets the fewest lanes holding <= max_w columns each
  int inject_timeout = 0;
  int part = 0, nparts = 1;     // this context scores tile group `part` of `nparts` (swe_set_partition)
  int threshold_path = 0;
  int dbscan_replay = 0;        // swe_adaptive_sets: 0 / 2 = device replays, 1 = host threads
  size_t kmer_batch_bytes = 0;  // k-mer calls' device batch (0 = their defaults)
  int graph_kernels = 0;
  std::string err;

  // what the upload holds: 0 = sequences (Smith-Waterman distances), else
  // points with SWE_METRIC_L1 / SWE_METRIC_L2 float distances
  int metric = 0;
  int dims = 0;
  uint32_t point_max_bits = 0;      // bit pattern of the largest point distance
  swgpu::DevBuf<float> d_points;    // dims x n_pad, dimension-major

  // dataset (host)
  int n = 0;
  int max_len = 0;
  int max_fast_len = 0;
  int nfast = 0;
  std::vector<int> len;
  std::vector<int64_t> off;
  std::vector<uint8_t> codes;
  int code_of[256];
  std::vector<int> order, exc;
  std::vector<uint8_t> is_exc;
  int npacks = 0;
  int max_block_rows = 0;
  int max_cols = 0;
  size_t smem = 0;
  int fast_grid = 0;
  std::vector<swgpu::FastTile> tiles;
  std::vector<swgpu::TileRect> part_rects;  // every tile of the layout (all groups), in cost order
  std::vector<int> part_owner;              // its group under swe_set_partition
  long long tiles_all = 0;  // tiles of the full layout (before a candidate mask)
  bool masked = false;      // only candidate tiles are scored; other pairs read as the largest value

  // sets (independent datasets in one upload) and the sorted layout
  int n_sets = 0;
  std::vector<int> set_first, set_nfast;  // set_first has n_sets + 1 entries
  std::vector<long long> set_base;        // n_sets + 1 entries
  std::vector<int> pos, set_of;           // per original index
  std::vector<long long> exc_pre;

  int upload_gen = 0;               // bumped by every upload
  std::vector<uint8_t> first_code;  // code of s[0] per sequence (k-mer features)

  // dataset (device)
  swgpu::DevBuf<uint8_t> d_codes, d_first;
  swgpu::DevBuf<int64_t> d_off;
  swgpu::DevBuf<int> d_len, d_order, d_exc, d_pack_off, d_pack_rows;
  swgpu::DevBuf<uint8_t> d_isexc;
  swgpu::DevBuf<int> d_pos, d_setof, d_set_first, d_set_n, d_set_nfast, d_pack_first, d_block_first, d_block_npacks;
  swgpu::DevBuf<long long> d_set_base, d_exc_pre;
  swgpu::DevBuf<uint8_t> d_pack_pair;
  int nblocks = 0;
  swgpu::DevBuf<uint16_t> d_sel;
  swgpu::DevBuf<swgpu::FastTile> d_tiles;
  swgpu::DevBuf<unsigned> d_ctr;  // [0] tile counter, [1] status, [2] rerun count
  swgpu::DevBuf<int2> d_rerun;
  unsigned rerun_cap = 0;
  bool rerun_possible = false;
  swgpu::DevBuf<int> d_scratch;
  long long scratch_stride = 0;
  int gen_grid = 0;

  // distances
  swgpu::DevBuf<uint16_t> d_D16;
  swgpu::DevBuf<uint32_t> d_D32;
  int dist_bytes = 2;
  bool scored = false;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t tev[2] = {nullptr, nullptr};

  // neighbour bitmaps
  int wpr = 0;
  swgpu::DevBuf<uint64_t> d_bits;
  swgpu::DevBuf<int> d_counts;
  swgpu::HostPinned<uint64_t> h_bits;
  swgpu::HostPinned<int> h_counts;
  long long bits_T = LLONG_MIN;
  int bits_set = -1;
  // threshold launches: groups, their row prefix and thresholds
  swgpu::DevBuf<swgpu::ThrGroup> d_groups;
  swgpu::DevBuf<long long> d_rowpre;
  swgpu::DevBuf<unsigned> d_thr, d_thr_status;
  swgpu::DevBuf<uint8_t> d_tbits;   // H-bit words of the transposed threshold pass
  swgpu::DevBuf<int> d_cbof;         // column block of each sorted position (device tile marking)
  swgpu::DevBuf<uint8_t> d_mark;     // tiles that hold a candidate pair
  swgpu::DevBuf<swgpu::TileRect> d_part_rects;  // one group's tile rectangles (split-pass exchange)
  swgpu::DevBuf<long long> d_part_pre;
  swgpu::DevBuf<long long> d_tpre;  // its two item prefix arrays
  swgpu::HostPinned<unsigned> h_thr_status;
  // batched sweeps: one bitmap slot per distinct threshold
  swgpu::DevBuf<uint64_t> d_bbits;
  swgpu::DevBuf<int> d_bcounts;
  swgpu::HostPinned<uint64_t> h_bbits;
  swgpu::HostPinned<int> h_bcounts;
  // device DBSCAN replays of a round: jobs, members, frontiers, cluster starts and counts, scratch
  swgpu::DevBuf<swgpu::ReplayJob> d_rjobs;
  swgpu::DevBuf<int> d_rmembers, d_rfrontier, d_rcstart, d_rncl;
  swgpu::DevBuf<uint32_t> d_rvis;
  swgpu::DevBuf<uint64_t> d_rqueued;
  swgpu::DevBuf<unsigned> d_rstatus;
  swgpu::HostPinned<int> h_rmembers, h_rcstart, h_rncl;
  swgpu::HostPinned<unsigned> h_rstatus;

  // small transfers
  swgpu::DevBuf<uint8_t> d_q;
  swgpu::DevBuf<unsigned> d_out;
  swgpu::DevBuf<int2> d_pairs;
  swgpu::DevBuf<int64_t> d_small_off;
  swgpu::DevBuf<int> d_small_len;
  swgpu::DevBuf<int> d_small_scratch;
  swgpu::DevBuf<long long> d_row_ptr;
  swgpu::DevBuf<int> d_cols;

  swe_stats stats{};

  // learned prefilter (null until first used)
  swgpu::PrefilterState* pf = nullptr;
  // k-mer tables: device buffers and pinned staging (null until first used)
  swgpu::KmerState* km = nullptr;
  // kmer2pca: the resident table and its buffers (null until first used)
  swgpu::PcaState* pca = nullptr;
  // pinned staging chunks of the chunked transfers (null until first used)
  swgpu::Staging* stage = nullptr;

  ~swe_ctx() {
    cudaSetDevice(device);
    swgpu::prefilter_destroy(pf);
    swgpu::kmer_state_destroy(km);
    swgpu::pca_state_destroy(pca);
    swgpu::staging_destroy(stage);
    if (graph) cudaGraphExecDestroy(graph);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (auto& e : tev)
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }
};

namespace swgpu {

swe_status fail(swe_ctx* ctx, swe_status s, const std::string& msg);
swe_status cuda_fail(swe_ctx* ctx, cudaError_t e, const char* what);
swe_status check_kernel_status(swe_ctx* ctx, unsigned status);
// Stream-ordered copy that also counts the bytes crossing PCIe.
cudaError_t cpy(swe_ctx* ctx, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t st);
swe_status select_device(swe_ctx* ctx);
// SWE_ERR_STATE unless the upload holds sequences (calls that score
// sequences refuse a point upload).
swe_status need_sequences(swe_ctx* ctx);
// Neighbour threshold of eps for the current upload, compared with the stored
// distance as an unsigned integer: floor(eps) for Smith-Waterman distances,
// the bit pattern of eps*eps (L2) or eps (L1) for point distances (their bit
// patterns order like the non-negative floats they hold); -1 = no neighbour.
long long ctx_threshold(const swe_ctx* ctx, float eps);
// A threshold at or above which every larger eps gives the same neighbours
// (-1 when there is none), and the key of eps that a sweep compares with it
// (-1 where thresholds do not grow with eps: negative eps under L2).
long long ctx_fixed_point(const swe_ctx* ctx);
long long ctx_sweep_key(const swe_ctx* ctx, float eps);
// Rebuilds the sorted layout (see build_layout in engine.cu) and runs one
// score pass over the current layout.
swe_status engine_relayout(swe_ctx* ctx, const std::vector<int64_t>* key, const std::vector<int2>* cand);
// The same with the candidate pairs (original indices, bit 31 of .x ignored)
// left on the device: the tiles holding one are marked by a kernel.
swe_status engine_relayout_dev(swe_ctx* ctx, const std::vector<int64_t>* key, const int2* cand, long long count);
swe_status score_pass(swe_ctx* ctx);
long long eps_threshold(float eps);

}  // namespace swgpu

#define CK(call)                                                      \
  do {                                                                \
    cudaError_t e_ = (call);                                          \
    if (e_ != cudaSuccess) return swgpu::cuda_fail(ctx, e_, #call);   \
  } while (0)
