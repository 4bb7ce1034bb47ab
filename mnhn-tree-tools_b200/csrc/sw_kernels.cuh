// Kernel parameter blocks and launchers shared by the engine (host) and the
// kernel translation unit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace swgpu {

constexpr int FAST_MAX_W = 24;     // columns per lane in the 16x2 kernel
constexpr int FAST_MAX_LEN = 768;  // 32 lanes x 24 columns
constexpr int GEN_W = 16;          // columns per lane in the 32-bit kernel (chunk = 512)
constexpr int GEN_CHUNK = 32 * GEN_W;

// Distance storage.  An upload holds one or more independent sets (contiguous
// ranges of original indices).  Inside a set, sequences are ordered by
// length (packed-path sequences longest first, then the 32-bit-path ones), and
// the set's n_s x n_s matrix is stored in that sorted order, so a tile of
// neighbouring sorted sequences writes contiguous runs.  A global sorted
// index g = set_first[s] + position runs over all sets.
struct DistLayout {
  const int* orig;            // global sorted index -> original index
  const int* pos;             // original index -> position in its set's sorted order
  const int* set_of;          // original index -> set
  const int* set_first;       // set -> first index (original and global sorted alike)
  const int* set_n;           // set -> size
  const int* set_nfast;       // set -> sequences on the packed path (positions 0..nfast-1)
  const long long* set_base;  // set -> offset of its matrix in D
  uint16_t* D16;              // one of D16 / D32 is non-null
  uint32_t* D32;
};

__device__ __forceinline__ void store_dist(const DistLayout& L, long long idx, unsigned d) {
  if (L.D16) L.D16[idx] = (uint16_t)d;
  else L.D32[idx] = d;
}

// Tile of the 16x2 all-pairs kernel: `nb` column sequences (global sorted
// indices b0..b0+nb-1, all in set `set`) against row block `q`.
// wl = W | (lanes per column sequence << 8).
struct FastTile {
  int b0, nb, q, wl, set;
};

// The rectangle of the sorted matrix a tile writes (both triangles): rows
// ra0 .. ra0+nra-1 x columns b0 .. b0+nb-1 (global sorted positions, one set).
struct TileRect {
  int ra0, nra, b0, nb, set;
};
// Copies between a packed buffer of tile rectangles (tile after tile, row
// after row, each entry one stored distance) and the matrix: pack reads rows
// ra x columns b; unpack writes entries [e0, e1) of the buffer to both
// triangles.  pre[t] = first entry of tile t (ntiles + 1 values).
cudaError_t launch_tile_pack(const DistLayout& L, const TileRect* rects, const long long* pre, int ntiles,
                             void* out, cudaStream_t st);
// Tiles of one set that hold a candidate pair: for pair (x, y) of original
// indices in [lo, hi) with packed-path positions px < py (pos[]), sets
// mark[cb_of[px] * nq + (py / 2) / PB] (the tile of column block cb_of[px]
// and the row block of py).
cudaError_t launch_mark_tiles(const int2* cand, long long count, const int* pos, int lo, int hi, int nf,
                              const int* cb_of, int nq, int PB, uint8_t* mark, cudaStream_t st);
cudaError_t launch_tile_unpack(const DistLayout& L, const TileRect* rects, const long long* pre, int ntiles,
                               const void* in, long long e0, long long e1, cudaStream_t st);

struct FastParams {
  const uint8_t* codes;      // effective symbol codes, all sequences
  const int64_t* code_off;   // per original index
  const int* len;            // per original index
  DistLayout L;
  const uint16_t* sel;       // row selectors, packs back to back
  const int* pack_first;     // [npacks] global sorted index of a pack's first sequence
  const uint8_t* pack_pair;  // [npacks] 1 when the pack has a second sequence (pack_first + 1)
  const int* pack_row_off;   // [npacks] start row of each pack (blocks 8-row aligned)
  const int* pack_rows;      // [npacks] rows of each pack (a multiple of 4)
  const int* block_first;    // [nblocks] first pack of each row block
  const int* block_npacks;   // [nblocks] packs in each row block
  int max_packs_per_block;   // PB
  const FastTile* tiles;
  int ntiles;
  unsigned* tile_counter;
  int2* rerun;               // global sorted index pairs whose 16-bit maximum reached sat_limit
  unsigned* rerun_count;
  unsigned rerun_cap;
  int sat_limit;
  unsigned* status;
  int max_block_rows;        // shared-memory sizing (rows, already 8-aligned)
  int max_cols_per_cta;      // shared-memory sizing (column sequences per tile)
  unsigned wait_limit;       // attempts of the bounded mbarrier wait
  int inject_timeout;        // test hook: the first tile's copy is never issued, so its wait runs out
};

// Generic 32-bit kernel: one warp per pair, any length, any symbols.
enum GenMode : int {
  GEN_PAIRS = 0,     // explicit pairs of global sorted indices; results to the matrix
  GEN_EXC_CROSS = 1, // every 32-bit-path sequence against every sequence of its set
  GEN_QUERY = 2,     // external query against original indices [0, n); results to out[]
  GEN_PAIRS_OUT = 3, // explicit pairs of original indices; results to out[]
};

struct GenParams {
  int mode;
  const uint8_t* codes;
  const int64_t* code_off;
  const int* len;
  int n;
  DistLayout L;                 // GEN_PAIRS / GEN_EXC_CROSS
  const int2* pairs;            // GEN_PAIRS / GEN_PAIRS_OUT
  long long npairs;             // used when npairs_dev == nullptr
  const unsigned* npairs_dev;   // device-resident pair count (rerun queue)
  const int* exc;               // GEN_EXC_CROSS: global sorted indices, ascending
  const long long* exc_pre;     // GEN_EXC_CROSS: [nexc+1] prefix sums of the sets' sizes
  int nexc;
  const uint8_t* qcodes;        // GEN_QUERY: effective query codes
  int qlen;
  unsigned* out;                // GEN_QUERY / GEN_PAIRS_OUT
  int* scratch;                 // per-warp boundary column, scratch_stride ints each
  long long scratch_stride;
  int nwarps_total;
  unsigned* status;
};

// Launchers (stream-ordered; no synchronisation).
cudaError_t launch_build_sel(const uint8_t* codes, const int64_t* code_off, const int* len, const int* orig,
                             const int* pack_first, const uint8_t* pack_pair, const int* pack_row_off,
                             const int* pack_rows, int npacks, uint16_t* sel, cudaStream_t st);
cudaError_t launch_fast(const FastParams& p, int grid, int block, size_t smem, cudaStream_t st);
size_t fast_smem_bytes(int max_block_rows, int max_cols_per_cta, int packs_per_block);
cudaError_t fast_set_smem_limit(size_t bytes);
int fast_occupancy(int block, size_t smem);
cudaError_t launch_generic(const GenParams& p, int grid, cudaStream_t st);
// Zero self-distances of every sequence.
cudaError_t launch_diag(const DistLayout& L, int n, cudaStream_t st);
// Rows [r0, r1) of one set's matrix in original index order, widened to 32
// bits (out holds (r1 - r0) x n_s entries).
cudaError_t launch_unpermute_set(const uint16_t* D16set, const uint32_t* D32set, const int* pos, int n_s, int r0,
                                 int r1, uint32_t* out, cudaStream_t st);
// Threshold pass over several sets and several thresholds at once.  A group
// is one set against up to THR_MAX thresholds; each row of the set's matrix is
// read once and yields one bitmap row per threshold.  Bits of group g,
// threshold u, row i (original order inside the set), word w are at
// bits[bits_base + (u * n_s + i) * wpr + w]; its popcount at
// counts[counts_base + u * n_s + i].  A threshold t keeps d <= t.
constexpr int THR_MAX = 32;
struct ThrGroup {
  long long dist_base;    // offset of the set's matrix in D (elements)
  long long bits_base;    // words
  long long counts_base;  // ints
  int pos_first;          // the set's slice of the position table
  int n_s, wpr;
  int thr_first, nthr;    // thresholds thr[thr_first .. thr_first + nthr), nthr <= THR_MAX
  // transposed pass (launch_threshold_transposed): threshold u's bit blocks
  // start at byte tb_base + u * nblk * blk_stride of the scratch, one block of
  // blk_stride bytes per H consecutive sorted rows
  long long tb_base;
  int nblk, blk_stride;
};
struct ThrParams {
  const uint16_t* D16;      // one of D16 / D32 is non-null
  const uint32_t* D32;
  const int* pos;
  const int* order;          // sorted position (+ set_first) -> original index
  uint8_t* tbits;            // scratch of the transposed pass
  const ThrGroup* groups;
  int ngroups;
  const long long* row_pre;  // [ngroups + 1] prefix sums of the groups' n_s
  const unsigned* thr;
  uint64_t* bits;
  int* counts;
  unsigned* status;          // KST_TIMEOUT when a bounded wait gave up
  unsigned wait_limit;       // attempts of the bounded mbarrier wait
};
// Shared-memory plan of a threshold launch whose largest set has max_n_s
// sequences: rows arrive by bulk copy into nbuf row buffers (double-buffered
// when two fit), the set's position table is staged too when it fits, and
// rows too long for shared memory are read from global memory (staged == 0).
struct ThrPlan {
  int staged, nbuf, stage_pos, block;
  size_t rowbuf, smem;
};
ThrPlan threshold_plan(int max_n_s, int dist_bytes);
cudaError_t launch_threshold(const ThrParams& p, long long total_rows, const ThrPlan& plan, cudaStream_t st);
// Transposed two-pass threshold.  Pass 1 streams each block of H consecutive
// sorted rows once and writes, per threshold and sorted column, an H-bit word
// (bit t = row t of the block is a neighbour).  Pass 2 stages one such block
// in shared memory and gathers the words through the position table into
// original column order: one random shared-memory read serves H rows.
// transposed_height: H (32, 16 or 8) for the largest set, 0 when even an
// 8-row block does not fit in shared memory.
int transposed_height(int max_n_s);
int transposed_block_stride(int n_s, int H);  // bytes, 16-byte multiple
int transposed_item_cols();                   // columns of one pass-1 item
// aligned16: every group's dist_base and n_s are multiples of 8 (rows start
// on 16-byte boundaries), so a 16-bit matrix can take the vector pack kernel.
cudaError_t launch_threshold_transposed(const ThrParams& p, int H, int max_n_s, bool aligned16,
                                        const long long* d_item_pre1, long long items1, const long long* d_item_pre2,
                                        long long items2, cudaStream_t st);
// Block [r0, r1) x [c0, c1) (original indices) of one set's matrix: per row the
// sum of the distances and the sum of floor((d - mean)^2) (each square rounded
// once in double), over the block the minimum and maximum (atomicMin / Max on
// *bmin / *bmax, which the caller initialises).
cudaError_t launch_block_stats(const uint16_t* D16set, const uint32_t* D32set, const int* pos, int n_s, int r0,
                               int r1, int c0, int c1, double mean, unsigned long long* row_sum,
                               unsigned long long* row_sqdev, unsigned* bmin, unsigned* bmax, cudaStream_t st);
// CSR from a bitmap: ascending column indices per row at row_ptr[i].
cudaError_t launch_csr_fill(const uint64_t* bits, int n, int words_per_row, const long long* row_ptr,
                            int* cols, cudaStream_t st);
// Throughput probe of the 16x2 per-cell instruction mix over independent
// chains; each thread runs `iters` cells on each of 8 chains.
cudaError_t launch_mix_probe(uint32_t* sink, int grid, int block, int iters, cudaStream_t st);

}  // namespace swgpu
