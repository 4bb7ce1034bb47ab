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

// Tile of the 16x2 all-pairs kernel: up to `nb` column sequences (sorted
// positions b0..b0+nb-1) against A-block `q` (packs q*PB .. q*PB+PB-1).
// wl = W | (lanes per column sequence << 8).
struct FastTile {
  int b0, nb, q, wl;
};

struct FastParams {
  const uint8_t* codes;      // effective symbol codes, all sequences
  const int64_t* code_off;   // per original index
  const int* len;            // per original index
  const int* order;          // sorted fast position -> original index
  int nfast;                 // number of fast sequences
  const uint16_t* sel;       // row selectors, packs back to back
  const int* pack_row_off;   // [npacks+1] start row of each pack (blocks 8-row aligned)
  const int* pack_rows;      // [npacks] rows of each pack
  int npacks;
  int packs_per_block;       // PB
  const FastTile* tiles;
  int ntiles;
  unsigned* tile_counter;
  uint16_t* D16;             // n x n output (one of D16 / D32 is non-null)
  uint32_t* D32;
  int n;
  int2* rerun;               // pairs whose 16-bit maximum reached sat_limit
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
  GEN_PAIRS = 0,     // explicit (a, b) list; results to the matrix
  GEN_EXC_CROSS = 1, // every exceptional sequence against every sequence
  GEN_QUERY = 2,     // external query against sequences [0, n); results to out[]
  GEN_PAIRS_OUT = 3, // explicit (a, b) list; results to out[]
};

struct GenParams {
  int mode;
  const uint8_t* codes;
  const int64_t* code_off;
  const int* len;
  int n;
  const int2* pairs;            // GEN_PAIRS / GEN_PAIRS_OUT
  long long npairs;             // used when npairs_dev == nullptr
  const unsigned* npairs_dev;   // device-resident pair count (rerun queue)
  const int* exc;               // GEN_EXC_CROSS
  int nexc;
  const uint8_t* is_exc;
  const uint8_t* qcodes;        // GEN_QUERY: effective query codes
  int qlen;
  uint16_t* D16;
  uint32_t* D32;
  unsigned* out;                // GEN_QUERY / GEN_PAIRS_OUT
  int* scratch;                 // per-warp boundary column, scratch_stride ints each
  long long scratch_stride;
  int nwarps_total;
  unsigned* status;
};

// Launchers (stream-ordered; no synchronisation).
cudaError_t launch_build_sel(const uint8_t* codes, const int64_t* code_off, const int* len,
                             const int* order, int nfast, const int* pack_row_off, int npacks,
                             uint16_t* sel, cudaStream_t st);
cudaError_t launch_fast(const FastParams& p, int grid, int block, size_t smem, cudaStream_t st);
size_t fast_smem_bytes(int max_block_rows, int max_cols_per_cta, int packs_per_block);
cudaError_t fast_set_smem_limit(size_t bytes);
int fast_occupancy(int block, size_t smem);
cudaError_t launch_generic(const GenParams& p, int grid, cudaStream_t st);
cudaError_t launch_diag(uint16_t* D16, uint32_t* D32, int n, cudaStream_t st);
// Neighbour bitmap for threshold T: bit k of row i set iff D[i][k] <= T.
cudaError_t launch_bitmap(const uint16_t* D16, const uint32_t* D32, int n, long long T,
                          uint64_t* bits, int words_per_row, int* counts, cudaStream_t st);
// CSR from a bitmap: ascending column indices per row at row_ptr[i].
cudaError_t launch_csr_fill(const uint64_t* bits, int n, int words_per_row, const long long* row_ptr,
                            int* cols, cudaStream_t st);
// Throughput probe of the 16x2 cell instruction mix (PRMT + 3 add-max + max)
// over independent chains; each thread runs `iters` cells on each of 8 chains.
cudaError_t launch_mix_probe(uint32_t* sink, int grid, int block, int iters, cudaStream_t st);

}  // namespace swgpu
