// Smith-Waterman distance kernels for B200 (sm_100a).
//
// Scoring follows the reference exactly (smith-waterman.c:16-80): linear gap
// 3, +4 on symbol equality, -4 otherwise, local floor 0, and the distance
// 4*max(len_a, len_b) - max H.  Sequences arrive as "effective" symbol codes:
// position r holds the reference's A[r+1] (the first base never takes part and
// the terminating NUL does, smith-waterman.c:56-58).
//
// Kernels:
//   fast_all_pairs_kernel  packed 16x2 warp wavefront (two row sequences per
//                          lane word, one column sequence per lane segment),
//                          persistent over a cost-ordered tile list;
//   generic_kernel         32-bit warp wavefront, one pair per warp, any
//                          length (512-column chunks) and any symbol;
//   threshold_kernel       eps thresholds of the distance matrices of many
//                          sets at once into neighbour bitmaps plus per-row
//                          counts (each row read once for all thresholds);
//   unpermute_kernel       a set's matrix back in original index order;
//   csr_fill_kernel        bitmap -> ascending CSR column lists.
#include <algorithm>
#include <mutex>

#include "sw_device.cuh"
#include "sw_kernels.cuh"
#include "sw_wavefront32.cuh"  // sw32_warp

namespace swgpu {

// ---------------------------------------------------------------------------
// 16x2 wavefront over one column sequence (a lane segment of `lpb` lanes).
//
// Lane li of the segment owns columns [li*W, li*W+W) of the column sequence B
// and, at step s, computes row g = s - li of the row stream (two row
// sequences per 16-bit half, packs back to back).  Its left boundary arrives
// from lane li-1 by shuffle; the diagonal boundary is the left boundary of the
// previous step.
//
// Each column keeps E = H - 3 of the previous row, so one stored value feeds
// all three uses of a cell: left and up need H - 3 = E, and the diagonal needs
// H + s = E + d with d = s + 3 from the PRMT table.  Per cell:
//   t = E_diag + d               (packed add, FMA pipe)
//   H = max(t, E_left, E_up, 0)  (3-input packed max, ALU pipe)
//   E = H - 3                    (packed add, FMA pipe)
// i.e. H = max(0, diag + s, left - 3, up - 3).
//
// The running maximum is taken over t, two cells per 3-input max: the largest
// H of a matrix is always reached on a diagonal step (a gap step only lowers
// the score), so max(0, max t) = max H, and t - unlike H - is off the
// left-neighbour dependency chain.
//
// A step processes four rows (pack row counts are multiples of 4), which
// spreads the per-step selector load, pack-boundary test and loop cost over
// four rows (measured on B200: 9.77 -> 10.17 Tcell/s against two rows per
// step; eight rows per step lost more to row padding and registers than it
// saved).  The shuffle of each row's boundary value stays.  Pad columns (beyond len B) and
// pad rows (code 7) only ever see mismatches, so they can never raise the
// maximum above the real cells' maximum.
// ---------------------------------------------------------------------------
template <int W>
__device__ __forceinline__ void fast_row(uint32_t (&E)[W], const uint32_t (&tlo)[W], const uint32_t (&thi)[W],
                                         uint32_t sel, uint32_t ed, uint32_t el, uint32_t& mx) {
  const uint32_t M3 = 0xFFFDFFFDu;
  uint32_t tprev = 0u;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const uint32_t d = prmt(tlo[k], thi[k], sel);
    const uint32_t t = vadd(ed, d);
    const uint32_t h = vmax3_0(t, el, E[k]);
    ed = E[k];
    el = vadd(h, M3);
    E[k] = el;
    if (k & 1) mx = vmax3_0(mx, tprev, t);
    else if (k == W - 1) mx = vmax0(mx, t);
    tprev = t;
  }
}

template <int W>
__device__ __forceinline__ void fast_segment(const uint16_t* __restrict__ sel0, int total_rows,
                                             const int* __restrict__ pstart, int npk,
                                             const uint8_t* __restrict__ bcodes, int lenB, int lpb,
                                             int li, unsigned* __restrict__ smax) {
  const uint32_t M3 = 0xFFFDFFFDu;  // -3 in both halves (E of a zero cell)
  uint32_t tlo[W], thi[W], E[W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const int col = li * W + k;
    const int c = (col < lenB) ? (int)bcodes[col] : 0xFF;
    uint32_t lo = 0xFFFFFFFFu, hi = 0xFFFFFFFFu;  // -1 (mismatch: -4 + 3)
    if (c < 4) lo ^= (0xF8u << (8 * c));           // 0x07 (match: +4 + 3)
    else if (c < 8) hi ^= (0xF8u << (8 * (c - 4)));
    tlo[k] = lo;
    thi[k] = hi;
    E[k] = M3;
  }
  uint32_t mx = 0u, last_a = M3, last_b = M3, last_c = M3, last_d = M3, diag = M3;
  int pk = -1, next = 0;
  const bool lead = (li == 0);
  const int steps = total_rows / 4 + lpb;
  // four selectors per 64-bit word: rows 4q .. 4q+3
  const uint2* sp = reinterpret_cast<const uint2*>(sel0) - li;
  for (int s = 0; s < steps; ++s) {
    uint32_t la = __shfl_up_sync(0xFFFFFFFFu, last_a, 1, lpb);
    uint32_t lb = __shfl_up_sync(0xFFFFFFFFu, last_b, 1, lpb);
    uint32_t lc = __shfl_up_sync(0xFFFFFFFFu, last_c, 1, lpb);
    uint32_t ld = __shfl_up_sync(0xFFFFFFFFu, last_d, 1, lpb);
    la = lead ? M3 : la;  // column 0 boundary: H = 0
    lb = lead ? M3 : lb;
    lc = lead ? M3 : lc;
    ld = lead ? M3 : ld;
    const int g = 4 * (s - li);  // first of the four rows
    if (g == next) {  // first row of a new pack (or the end of the stream)
      if (pk >= 0) {
        atomicMax(&smax[2 * pk], mx & 0xFFFFu);
        atomicMax(&smax[2 * pk + 1], mx >> 16);
      }
      ++pk;
      mx = 0u;
      diag = M3;
#pragma unroll
      for (int k = 0; k < W; ++k) E[k] = M3;
      next = (pk < npk) ? pstart[pk + 1] : 0x7FFFFFFF;
    }
    const uint2 sel4 = sp[s];
    fast_row<W>(E, tlo, thi, sel4.x & 0xFFFFu, diag, la, mx);
    last_a = E[W - 1];
    fast_row<W>(E, tlo, thi, sel4.x >> 16, la, lb, mx);  // a row's diagonal is the left of the row above
    last_b = E[W - 1];
    fast_row<W>(E, tlo, thi, sel4.y & 0xFFFFu, lb, lc, mx);
    last_c = E[W - 1];
    fast_row<W>(E, tlo, thi, sel4.y >> 16, lc, ld, mx);
    last_d = E[W - 1];
    diag = ld;
  }
}

// Shared selector buffer: SEL_FRONT pad rows before row 0 (lanes that have not
// started read rows down to -4*(lanes-1) = -124) and SEL_TAIL after the last
// row (lanes that have finished read up to rows + 4*lanes - 1).
constexpr int SEL_FRONT = 128, SEL_TAIL = 160;

__host__ __device__ inline size_t fast_sel_bytes(int max_block_rows) {
  return ((size_t)(SEL_FRONT + max_block_rows + SEL_TAIL) * 2 + 15) & ~(size_t)15;
}

size_t fast_smem_bytes(int max_block_rows, int max_cols_per_cta, int packs_per_block) {
  return fast_sel_bytes(max_block_rows) + (size_t)max_cols_per_cta * packs_per_block * 2 * 4 +
         (size_t)(packs_per_block + 1) * 4 + 16;
}

template <int W>
__device__ __forceinline__ void fast_dispatch_one(const uint16_t* sel0, int rows, const int* pstart,
                                                  int npk, const uint8_t* bc, int lenB, int lpb,
                                                  int li, unsigned* smax) {
  fast_segment<W>(sel0, rows, pstart, npk, bc, lenB, lpb, li, smax);
}

__device__ __noinline__ void fast_dispatch(int W, const uint16_t* sel0, int rows, const int* pstart,
                                           int npk, const uint8_t* bc, int lenB, int lpb, int li,
                                           unsigned* smax) {
  switch (W) {
#define SWGPU_CASE(w) \
  case w: fast_dispatch_one<w>(sel0, rows, pstart, npk, bc, lenB, lpb, li, smax); break;
    SWGPU_CASE(1) SWGPU_CASE(2) SWGPU_CASE(3) SWGPU_CASE(4) SWGPU_CASE(5) SWGPU_CASE(6)
    SWGPU_CASE(7) SWGPU_CASE(8) SWGPU_CASE(9) SWGPU_CASE(10) SWGPU_CASE(11) SWGPU_CASE(12)
    SWGPU_CASE(13) SWGPU_CASE(14) SWGPU_CASE(15) SWGPU_CASE(16) SWGPU_CASE(17) SWGPU_CASE(18)
    SWGPU_CASE(19) SWGPU_CASE(20) SWGPU_CASE(21) SWGPU_CASE(22) SWGPU_CASE(23) SWGPU_CASE(24)
#undef SWGPU_CASE
    default: break;
  }
}

__global__ void __launch_bounds__(256, 2) fast_all_pairs_kernel(FastParams p) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_tile;
  __shared__ int s_ok;
  const int PB = p.max_packs_per_block;
  uint16_t* s_sel = reinterpret_cast<uint16_t*>(smem);
  unsigned* s_max = reinterpret_cast<unsigned*>(smem + fast_sel_bytes(p.max_block_rows));
  int* s_pstart = reinterpret_cast<int*>(s_max + (size_t)p.max_cols_per_cta * PB * 2);
  const int tid = threadIdx.x, bd = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31, nwarps = bd >> 5;

  if (tid == 0) mbar_init(&bar, 1);
  for (int i = tid; i < SEL_FRONT; i += bd) s_sel[i] = SEL_PAD;
  __syncthreads();
  uint32_t phase = 0;

  for (;;) {
    if (tid == 0) s_tile = (int)atomicAdd(p.tile_counter, 1u);
    __syncthreads();
    const int t = s_tile;
    if (t >= p.ntiles) break;
    const FastTile tile = p.tiles[t];
    const int W = tile.wl & 0xFF, lpb = tile.wl >> 8;
    const int pk0 = p.block_first[tile.q];
    const int npk = p.block_npacks[tile.q];
    bool bad = (W < 1 || W > FAST_MAX_W || (lpb != 8 && lpb != 16 && lpb != 32) || npk <= 0 || npk > PB ||
                tile.nb < 1 || tile.nb > p.max_cols_per_cta || tile.nb > nwarps * (32 / max(lpb, 1)));
    int row0 = 0, rows = 0, rows8 = 0;
    if (!bad) {
      row0 = p.pack_row_off[pk0];
      rows = p.pack_row_off[pk0 + npk - 1] + p.pack_rows[pk0 + npk - 1] - row0;
      rows8 = (rows + 7) & ~7;
      bad = rows8 > p.max_block_rows || (row0 & 7) != 0;
    }
    if (bad) {
      if (tid == 0) atomicOr(p.status, KST_BAD_TILE);
      __syncthreads();
      continue;
    }
    // test hook: tile 0's copy is never issued, so nothing completes its phase
    const bool skip_copy = p.inject_timeout && t == 0;
    if (tid == 0 && !skip_copy) {
      // order earlier generic-proxy reads of s_sel before the async-proxy write
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive_expect_tx(&bar, (uint32_t)rows8 * 2u);
      bulk_g2s(s_sel + SEL_FRONT, p.sel + row0, (uint32_t)rows8 * 2u, &bar);
    }
    for (int i = tid; i <= npk; i += bd)
      s_pstart[i] = (i < npk ? p.pack_row_off[pk0 + i] : row0 + rows) - row0;
    for (int i = tid; i < tile.nb * npk * 2; i += bd) s_max[i] = 0u;
    if (tid == 0) {
      bool ok = mbar_wait_bounded(&bar, phase, p.wait_limit);
      if (!ok) {
        atomicOr(p.status, KST_TIMEOUT);
        if (!skip_copy) mbar_wait_bounded(&bar, phase, p.wait_limit);  // let the copy in flight land
      }
      s_ok = ok ? 1 : 0;
    }
    phase ^= 1u;
    __syncthreads();
    if (!s_ok) return;
    for (int i = tid; i < SEL_TAIL; i += bd) s_sel[SEL_FRONT + rows + i] = SEL_PAD;
    __syncthreads();

    const int spw = 32 / lpb;  // column sequences per warp
    if (warp * spw < tile.nb) {
      const int j = min(warp * spw + lane / lpb, tile.nb - 1);  // idle segments repeat the last one
      const int b = p.L.orig[tile.b0 + j];
      fast_dispatch(W, s_sel + SEL_FRONT, rows, s_pstart, npk, p.codes + p.code_off[b], p.len[b], lpb,
                    lane % lpb, s_max + (size_t)j * npk * 2);
    }
    __syncthreads();

    // epilogue: this tile's distances.  Row sequences of a block and column
    // sequences of a tile are consecutive in the set's sorted order, so the
    // first pass (row sequence fastest) writes contiguous runs of row b of the
    // set's matrix and the second pass (column sequence fastest) contiguous
    // runs of row a.
    const int s = tile.set;
    const int first = p.L.set_first[s], ns = p.L.set_n[s];
    const long long base = p.L.set_base[s];
    const int nr = npk * 2;
    for (int i = tid; i < tile.nb * nr; i += bd) {
      const int j = i / nr, r = i - j * nr;
      const int pk = pk0 + (r >> 1);
      if ((r & 1) && !p.pack_pair[pk]) continue;
      const int ga = p.pack_first[pk] + (r & 1), gb = tile.b0 + j;
      const int a = p.L.orig[ga], b = p.L.orig[gb];
      const unsigned m = s_max[i];
      if ((int)m >= p.sat_limit) {
        const unsigned slot = atomicAdd(p.rerun_count, 1u);
        if (slot < p.rerun_cap) p.rerun[slot] = make_int2(ga, gb);
        else atomicOr(p.status, KST_RERUN_OVERFLOW);
        continue;
      }
      store_dist(p.L, base + (long long)(gb - first) * ns + (ga - first),
                 4u * (unsigned)max(p.len[a], p.len[b]) - m);
    }
    for (int i = tid; i < tile.nb * nr; i += bd) {
      const int r = i / tile.nb, j = i - r * tile.nb;
      const int pk = pk0 + (r >> 1);
      if ((r & 1) && !p.pack_pair[pk]) continue;
      const unsigned m = s_max[j * nr + r];
      if ((int)m >= p.sat_limit) continue;  // queued for the 32-bit rerun above
      const int ga = p.pack_first[pk] + (r & 1), gb = tile.b0 + j;
      const int a = p.L.orig[ga], b = p.L.orig[gb];
      store_dist(p.L, base + (long long)(ga - first) * ns + (gb - first),
                 4u * (unsigned)max(p.len[a], p.len[b]) - m);
    }
    __syncthreads();
  }
}

cudaError_t fast_set_smem_limit(size_t bytes) {
  return cudaFuncSetAttribute(fast_all_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)bytes);
}

int fast_occupancy(int block, size_t smem) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fast_all_pairs_kernel, block, smem) !=
      cudaSuccess) {
    cudaGetLastError();  // do not leave the query's error for the next launch check
    return 0;
  }
  return nb;
}

cudaError_t launch_fast(const FastParams& p, int grid, int block, size_t smem, cudaStream_t st) {
  fast_all_pairs_kernel<<<grid, block, smem, st>>>(p);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Row selector stream: one 16-bit PRMT selector per row of each pack.
// ---------------------------------------------------------------------------
// Rows of a pack beyond both sequences (the even-row padding) get the pad
// selector; rows between blocks are filled with it by the host's memset.
__global__ void build_sel_kernel(const uint8_t* __restrict__ codes, const int64_t* __restrict__ code_off,
                                 const int* __restrict__ len, const int* __restrict__ orig,
                                 const int* __restrict__ pack_first, const uint8_t* __restrict__ pack_pair,
                                 const int* __restrict__ pack_row_off, const int* __restrict__ pack_rows,
                                 int npacks, uint16_t* sel) {
  for (int pk = blockIdx.x; pk < npacks; pk += gridDim.x) {
    const int a = orig[pack_first[pk]];
    const int b = pack_pair[pk] ? orig[pack_first[pk] + 1] : -1;
    const int la = len[a], lb = b >= 0 ? len[b] : 0;
    const uint8_t* ca = codes + code_off[a];
    const uint8_t* cb = b >= 0 ? codes + code_off[b] : nullptr;
    const int r0 = pack_row_off[pk], R = pack_rows[pk];
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
      const int x = r < la ? (int)ca[r] : CODE_ROWPAD;
      const int y = r < lb ? (int)cb[r] : CODE_ROWPAD;
      sel[r0 + r] = make_sel(x, y);
    }
  }
}

cudaError_t launch_build_sel(const uint8_t* codes, const int64_t* code_off, const int* len, const int* orig,
                             const int* pack_first, const uint8_t* pack_pair, const int* pack_row_off,
                             const int* pack_rows, int npacks, uint16_t* sel, cudaStream_t st) {
  if (npacks <= 0) return cudaSuccess;
  build_sel_kernel<<<min(npacks, 65535), 128, 0, st>>>(codes, code_off, len, orig, pack_first, pack_pair,
                                                       pack_row_off, pack_rows, npacks, sel);
  return cudaGetLastError();
}

__global__ void __launch_bounds__(256) generic_kernel(GenParams p) {
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  long long total = 0;
  if (p.mode == GEN_PAIRS || p.mode == GEN_PAIRS_OUT)
    total = p.npairs_dev ? (long long)*p.npairs_dev : p.npairs;
  else if (p.mode == GEN_EXC_CROSS)
    total = p.exc_pre[p.nexc];
  else
    total = p.n;
  int* scratch = p.scratch ? p.scratch + (long long)gw * p.scratch_stride : nullptr;
  for (long long w = gw; w < total; w += p.nwarps_total) {
    int ia = -1, ib = -1;  // original indices
    int ga = -1, gb = -1;  // global sorted indices (matrix modes)
    const uint8_t *A, *B;
    int la, lb;
    if (p.mode == GEN_PAIRS_OUT) {
      const int2 pr = p.pairs[w];
      ia = pr.x;
      ib = pr.y;
    } else if (p.mode == GEN_PAIRS) {
      const int2 pr = p.pairs[w];
      ga = pr.x;
      gb = pr.y;
    } else if (p.mode == GEN_EXC_CROSS) {
      // exceptional sequence e pairs with every sequence of its set
      int lo = 0, hi = p.nexc - 1;
      while (lo < hi) {  // last e with exc_pre[e] <= w
        const int mid = (lo + hi + 1) >> 1;
        if (p.exc_pre[mid] <= w) lo = mid;
        else hi = mid - 1;
      }
      ga = p.exc[lo];
      const int s = p.L.set_of[p.L.orig[ga]];
      const int first = p.L.set_first[s];
      gb = first + (int)(w - p.exc_pre[lo]);
      // a pair of two exceptional sequences belongs to the lower one
      if (gb - first >= p.L.set_nfast[s] && gb < ga) continue;
    } else {
      ib = (int)w;
    }
    if (ga >= 0) {
      ia = p.L.orig[ga];
      ib = p.L.orig[gb];
    }
    if (p.mode == GEN_QUERY) {
      A = p.qcodes;
      la = p.qlen;
    } else {
      A = p.codes + p.code_off[ia];
      la = p.len[ia];
    }
    B = p.codes + p.code_off[ib];
    lb = p.len[ib];
    // keep the shorter sequence on the column side (fewer chunks)
    const uint8_t* R = A;
    const uint8_t* Cc = B;
    int lr = la, lc = lb;
    if (lc > lr) {
      R = B;
      Cc = A;
      lr = lb;
      lc = la;
    }
    const int best = sw32_warp(R, lr, Cc, lc, scratch, lane);
    if (lane == 0) {
      const unsigned d = 4u * (unsigned)max(la, lb) - (unsigned)best;
      if (p.mode == GEN_QUERY || p.mode == GEN_PAIRS_OUT) {
        p.out[w] = d;
      } else {
        const int s = p.L.set_of[ia];
        const int first = p.L.set_first[s], ns = p.L.set_n[s];
        const long long base = p.L.set_base[s];
        store_dist(p.L, base + (long long)(ga - first) * ns + (gb - first), d);
        store_dist(p.L, base + (long long)(gb - first) * ns + (ga - first), d);
      }
    }
  }
}

cudaError_t launch_generic(const GenParams& p, int grid, cudaStream_t st) {
  generic_kernel<<<grid, 256, 0, st>>>(p);
  return cudaGetLastError();
}

// Self-distances are 0 (a sequence aligns with itself on the diagonal).
__global__ void diag_kernel(DistLayout L, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int s = L.set_of[i], q = L.pos[i];
    store_dist(L, L.set_base[s] + (long long)q * L.set_n[s] + q, 0u);
  }
}

cudaError_t launch_diag(const DistLayout& L, int n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  diag_kernel<<<min((n + 255) / 256, 4096), 256, 0, st>>>(L, n);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Threshold pass over groups (set x up to 32 thresholds), persistent over the
// global row list of all groups.  Each CTA walks rows blockIdx.x + k*grid:
// one thread brings the row's bytes into shared memory with a bulk copy (TMA
// engine) completed on an mbarrier, the next row's copy in flight while the
// current one is processed.  Each warp then gathers two columns per lane
// through the set's position table (staged in shared memory when it fits)
// and produces one 64-bit word per threshold with two ballots; lane u keeps
// threshold u's word and count, so a row is read once for all thresholds.
// ---------------------------------------------------------------------------
constexpr size_t THRESHOLD_SMEM_MAX = 220 * 1024;
constexpr int THR_BLOCK = 512;

ThrPlan threshold_plan(int max_n_s, int dist_bytes) {
  ThrPlan pl{};
  pl.rowbuf = ((size_t)max_n_s * (size_t)dist_bytes + 32 + 15) & ~(size_t)15;
  const size_t posb = (size_t)max_n_s * 4;
  pl.block = THR_BLOCK;
  // Positions stay in global memory (L1-resident): staging them costs more in
  // occupancy than it saves in loads (0.66 vs 0.50 ms for a 20,000-sequence set
  // on B200).
  (void)posb;
  if (2 * pl.rowbuf <= THRESHOLD_SMEM_MAX) {
    pl.staged = 1, pl.nbuf = 2, pl.stage_pos = 0;
  } else if (pl.rowbuf <= THRESHOLD_SMEM_MAX) {
    pl.staged = 1, pl.nbuf = 1, pl.stage_pos = 0;
  } else {
    pl.staged = 0, pl.nbuf = 0, pl.stage_pos = 0, pl.block = 256;
  }
  pl.smem = pl.staged ? pl.nbuf * pl.rowbuf + (pl.stage_pos ? posb : 0) : 0;
  return pl;
}

__device__ __forceinline__ int thr_find_group(const ThrParams& p, long long r) {
  int lo = 0, hi = p.ngroups - 1;  // last group with row_pre[g] <= r
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (p.row_pre[mid] <= r) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One row: words of threshold `lane` for every 64-column word this warp owns,
// two words per iteration so that four gathers are in flight per lane.
template <typename DT>
__device__ __forceinline__ int thr_row(const ThrParams& p, const ThrGroup& G, int i, const DT* src, const int* ps,
                                       const unsigned* s_thr, int lane, int warp, int nwarps) {
  const int ns = G.n_s, nthr = G.nthr;
  uint64_t* brow = p.bits + G.bits_base + (long long)i * G.wpr;
  const long long plane = (long long)ns * G.wpr;  // words between thresholds
  int cnt = 0;
  for (int w = warp; w < G.wpr; w += 2 * nwarps) {
    const int wb = w + nwarps;  // second word (warp-uniform validity)
    const int c0 = w * 64 + lane, c1 = c0 + 32, c2 = wb * 64 + lane, c3 = c2 + 32;
    const unsigned d0 = c0 < ns ? (unsigned)src[ps[c0]] : 0xFFFFFFFFu;
    const unsigned d1 = c1 < ns ? (unsigned)src[ps[c1]] : 0xFFFFFFFFu;
    const unsigned d2 = c2 < ns ? (unsigned)src[ps[c2]] : 0xFFFFFFFFu;
    const unsigned d3 = c3 < ns ? (unsigned)src[ps[c3]] : 0xFFFFFFFFu;
    uint64_t ma = 0, mb = 0;
    for (int u = 0; u < nthr; ++u) {
      const unsigned t = s_thr[u];
      const uint32_t a0 = __ballot_sync(0xFFFFFFFFu, c0 < ns && d0 <= t);
      const uint32_t a1 = __ballot_sync(0xFFFFFFFFu, c1 < ns && d1 <= t);
      const uint32_t b0 = __ballot_sync(0xFFFFFFFFu, c2 < ns && d2 <= t);
      const uint32_t b1 = __ballot_sync(0xFFFFFFFFu, c3 < ns && d3 <= t);
      if (lane == u) {
        ma = (uint64_t)a0 | ((uint64_t)a1 << 32);
        mb = (uint64_t)b0 | ((uint64_t)b1 << 32);
      }
    }
    if (lane < nthr) {
      brow[lane * plane + w] = ma;
      cnt += __popcll(ma);
      if (wb < G.wpr) {
        brow[lane * plane + wb] = mb;
        cnt += __popcll(mb);
      }
    }
  }
  return cnt;
}

template <typename DT, bool STAGE_POS>
__global__ void __launch_bounds__(THR_BLOCK) threshold_bulk_kernel(ThrParams p, const DT* __restrict__ D,
                                                                   long long total, int nbuf, unsigned rowbuf) {
  extern __shared__ __align__(16) uint8_t th_smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_group[2], s_off[2];
  __shared__ unsigned s_thr[THR_MAX];
  __shared__ int s_cnt[THR_BLOCK / 32][THR_MAX];
  __shared__ int s_ok, s_cur;
  int* pos_s = reinterpret_cast<int*>(th_smem + (size_t)nbuf * rowbuf);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;

  // thread 0: bulk copy of row r into buffer b (16-byte aligned window around the row)
  auto issue = [&](int b, long long r) {
    const int g = thr_find_group(p, r);
    const ThrGroup& G = p.groups[g];
    const int i = (int)(r - p.row_pre[g]);
    const uintptr_t a = reinterpret_cast<uintptr_t>(D + G.dist_base + (long long)p.pos[G.pos_first + i] * G.n_s);
    const uintptr_t a16 = a & ~(uintptr_t)15;
    const unsigned off = (unsigned)(a - a16);
    const unsigned bytes = (off + (unsigned)G.n_s * (unsigned)sizeof(DT) + 15u) & ~15u;
    s_group[b] = g;
    s_off[b] = (int)(off / sizeof(DT));
    mbar_arrive_expect_tx(&bar[b], bytes);
    bulk_g2s(th_smem + (size_t)b * rowbuf, reinterpret_cast<const void*>(a16), bytes, &bar[b]);
  };

  if (tid == 0) {
    for (int b = 0; b < nbuf; ++b) mbar_init(&bar[b], 1);
    s_cur = -1;
  }
  __syncthreads();
  if (tid == 0)
    for (int b = 0; b < nbuf; ++b) {
      const long long r = blockIdx.x + (long long)b * gridDim.x;
      if (r < total) issue(b, r);
    }
  for (long long it = 0;; ++it) {
    const long long r = blockIdx.x + it * gridDim.x;
    if (r >= total) break;
    const int b = (int)(it % nbuf);
    const unsigned parity = (unsigned)((it / nbuf) & 1);
    if (tid == 0) s_ok = mbar_wait_bounded(&bar[b], parity, p.wait_limit) ? 1 : 0;
    __syncthreads();
    if (!s_ok) {  // CTA-uniform
      if (tid == 0) {
        atomicOr(p.status, KST_TIMEOUT);
        // let every copy this CTA issued land before it leaves
        for (int k = 0; k < nbuf; ++k) {
          const long long it2 = it + k;
          if (blockIdx.x + it2 * gridDim.x < total)
            mbar_wait_bounded(&bar[it2 % nbuf], (unsigned)((it2 / nbuf) & 1), p.wait_limit);
        }
      }
      break;
    }
    const int g = s_group[b];
    const ThrGroup G = p.groups[g];
    const int i = (int)(r - p.row_pre[g]);
    if (g != s_cur) {  // CTA-uniform: thresholds (and positions) of a new group
      if (tid < G.nthr) s_thr[tid] = p.thr[G.thr_first + tid];
      if (STAGE_POS)
        for (int k = tid; k < G.n_s; k += blockDim.x) pos_s[k] = p.pos[G.pos_first + k];
      __syncthreads();
      if (tid == 0) s_cur = g;
    }
    const DT* src = reinterpret_cast<const DT*>(th_smem + (size_t)b * rowbuf) + s_off[b];
    const int* ps = STAGE_POS ? pos_s : p.pos + G.pos_first;
    const int cnt = thr_row<DT>(p, G, i, src, ps, s_thr, lane, warp, nwarps);
    if (lane < G.nthr) s_cnt[warp][lane] = cnt;
    __syncthreads();  // buffer b, s_cnt and s_cur are complete
    if (tid < G.nthr) {
      int c = 0;
      for (int k = 0; k < nwarps; ++k) c += s_cnt[k][tid];
      p.counts[G.counts_base + (long long)tid * G.n_s + i] = c;
    }
    if (tid == 0) {
      const long long rn = r + (long long)nbuf * gridDim.x;
      if (rn < total) issue(b, rn);
    }
  }
}

// Rows longer than shared memory: gathered straight from global memory.
template <typename DT>
__global__ void __launch_bounds__(256) threshold_global_kernel(ThrParams p, const DT* __restrict__ D,
                                                               long long total) {
  __shared__ unsigned s_thr[THR_MAX];
  __shared__ int s_cnt[8][THR_MAX];
  __shared__ int s_group;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (long long r = blockIdx.x; r < total; r += gridDim.x) {
    if (threadIdx.x == 0) s_group = thr_find_group(p, r);
    __syncthreads();
    const ThrGroup G = p.groups[s_group];
    const int i = (int)(r - p.row_pre[s_group]);
    if (threadIdx.x < G.nthr) s_thr[threadIdx.x] = p.thr[G.thr_first + threadIdx.x];
    __syncthreads();
    const int* ps = p.pos + G.pos_first;
    const DT* row = D + G.dist_base + (long long)ps[i] * G.n_s;
    const int cnt = thr_row<DT>(p, G, i, row, ps, s_thr, lane, warp, nwarps);
    if (lane < G.nthr) s_cnt[warp][lane] = cnt;
    __syncthreads();
    if (threadIdx.x < G.nthr) {
      int c = 0;
      for (int k = 0; k < nwarps; ++k) c += s_cnt[k][threadIdx.x];
      p.counts[G.counts_base + (long long)threadIdx.x * G.n_s + i] = c;
    }
    __syncthreads();  // s_group, s_thr and s_cnt are reused by the next row
  }
}

template <typename DT>
static cudaError_t launch_threshold_t(const ThrParams& p, const DT* D, long long total, const ThrPlan& pl,
                                      cudaStream_t st) {
  int dev = 0, sms = 148, occ = 1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  if (!pl.staged) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, threshold_global_kernel<DT>, 256, 0);
    if (e != cudaSuccess) return e;
    const long long grid = std::min<long long>(total, (long long)sms * std::max(occ, 1));
    threshold_global_kernel<DT><<<(int)grid, 256, 0, st>>>(p, D, total);
    return cudaGetLastError();
  }
  auto kern = pl.stage_pos ? threshold_bulk_kernel<DT, true> : threshold_bulk_kernel<DT, false>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, pl.block, pl.smem);
  if (e != cudaSuccess) return e;
  const long long grid = std::min<long long>(total, (long long)sms * std::max(occ, 1));
  kern<<<(int)grid, pl.block, pl.smem, st>>>(p, D, total, pl.nbuf, (unsigned)pl.rowbuf);
  return cudaGetLastError();
}

cudaError_t launch_threshold(const ThrParams& p, long long total_rows, const ThrPlan& plan, cudaStream_t st) {
  if (total_rows <= 0 || p.ngroups <= 0) return cudaSuccess;
  if (p.D16) return launch_threshold_t<uint16_t>(p, p.D16, total_rows, plan, st);
  return launch_threshold_t<uint32_t>(p, p.D32, total_rows, plan, st);
}

// ---------------------------------------------------------------------------
// Transposed two-pass threshold (the default when an H-row block fits in
// shared memory).  The matrix is stored with rows and columns in sorted
// order; neighbour bits are wanted in original order.  Gathering each element
// through the position table costs a random shared-memory read per element;
// here it costs one per H elements:
//   pass 1 (thr_pack_kernel): for a block of H consecutive sorted rows, thread
//     k reads the H values of sorted column k (each step one coalesced row
//     segment) and writes, per threshold, the H-bit word of that column;
//   pass 2 (thr_unpack_kernel): one CTA stages a block's words of one
//     threshold in shared memory; lane l of a warp takes original column j
//     and reads word[pos[j]] (H rows at once), then a 32 x 32 bit transpose
//     across the warp turns the 32 lanes' words into 32-column bit runs of the
//     H rows, which go out through a shared-memory stage in row runs.
// ---------------------------------------------------------------------------
template <int H>
struct HWord;
template <>
struct HWord<8> {
  using T = uint8_t;
};
template <>
struct HWord<16> {
  using T = uint16_t;
};
template <>
struct HWord<32> {
  using T = uint32_t;
};

constexpr int TP1_THREADS = 256;
constexpr int TP1_COLS = 8;  // columns per thread per item: items of 2,048 columns
constexpr int TP1_ITEM_COLS = TP1_THREADS * TP1_COLS;
constexpr int TP2_THREADS = 512;  // two CTAs per SM where two blocks fit in shared memory
constexpr int TP2_SLICES = 4;  // 32-column slices per warp per chunk
constexpr int TP2_CHUNK_WORDS = (TP2_THREADS / 32) * TP2_SLICES;
constexpr int TP2_STAGE_PITCH = TP2_CHUNK_WORDS + 1;  // odd pitch: lane t's stage row in its own bank
constexpr size_t TP_BLOCK_MAX = 200 * 1024;

int transposed_height(int max_n_s) {
  for (int H = 32; H >= 8; H >>= 1)
    if ((size_t)transposed_block_stride(max_n_s, H) <= TP_BLOCK_MAX) return H;
  return 0;
}

int transposed_block_stride(int n_s, int H) { return (int)((((size_t)n_s * (size_t)(H / 8)) + 15) & ~(size_t)15); }
int transposed_item_cols() { return TP1_ITEM_COLS; }

__device__ __forceinline__ int tp_find_group(const long long* pre, int ngroups, long long item) {
  int lo = 0, hi = ngroups - 1;  // last group with pre[g] <= item
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// An item is (group, block B, 2,048 columns); thread t of the CTA takes
// columns c0 + t + 256 c, c < 8.  The item decodes in 32-bit arithmetic (a
// group has far fewer than 2^31 items).
template <int H, typename DT>
__global__ void __launch_bounds__(TP1_THREADS) thr_pack_kernel(ThrParams p, const DT* __restrict__ D,
                                                               const long long* __restrict__ item_pre) {
  using W = typename HWord<H>::T;
  const long long items = item_pre[p.ngroups];
  for (long long item = blockIdx.x; item < items; item += gridDim.x) {
    const int g = tp_find_group(item_pre, p.ngroups, item);
    const ThrGroup G = p.groups[g];
    const int ns = G.n_s;
    const int nch = (ns + TP1_ITEM_COLS - 1) / TP1_ITEM_COLS;
    const int r = (int)(item - item_pre[g]);
    const int B = r / nch, ch = r - B * nch;
    const int rows = min(H, ns - B * H);
    const DT* blk = D + G.dist_base + (long long)B * H * ns;
    uint8_t* out = p.tbits + G.tb_base + (long long)B * G.blk_stride;
    const long long plane = (long long)G.nblk * G.blk_stride;
    // CPI columns per iteration: CPI * H loads in flight per thread (32 or more)
    constexpr int CPI = H == 32 ? 1 : 32 / H;
#pragma unroll 1
    for (int c = 0; c < TP1_COLS; c += CPI) {
      unsigned v[CPI][H];
#pragma unroll
      for (int x = 0; x < CPI; ++x) {
        const int k = ch * TP1_ITEM_COLS + (c + x) * TP1_THREADS + threadIdx.x;
        const DT* q = blk + (k < ns ? k : 0);  // one pointer walks down the column
#pragma unroll
        for (int t = 0; t < H; ++t) {
          v[x][t] = (t < rows && k < ns) ? (unsigned)*q : 0xFFFFFFFFu;
          q += ns;
        }
      }
#pragma unroll
      for (int x = 0; x < CPI; ++x) {
        const int k = ch * TP1_ITEM_COLS + (c + x) * TP1_THREADS + threadIdx.x;
        if (k >= ns) break;
        for (int u = 0; u < G.nthr; ++u) {
          const unsigned th = p.thr[G.thr_first + u];
          unsigned w = 0;
#pragma unroll
          for (int t = 0; t < H; ++t) w |= (v[x][t] <= th ? 1u : 0u) << t;
          reinterpret_cast<W*>(out + (long long)u * plane)[k] = (W)w;
        }
      }
    }
  }
}

// The same pass for 16-bit matrices whose rows start on 16-byte boundaries
// (every group's dist_base and n_s multiples of 8): thread t of an item takes
// the 8 consecutive columns c0 + 8 t .. +7, one 16-byte load per row, and
// compares two columns per DPX instruction (__vibmin_u16x2 sets a <= b for
// both halves), so a pair of elements costs one compare and two predicated
// ORs.  Items are (group, block B, 2,048 columns) as in thr_pack_kernel.
template <int H>
__global__ void __launch_bounds__(TP1_THREADS) thr_pack_vec_kernel(ThrParams p, const uint16_t* __restrict__ D,
                                                                   const long long* __restrict__ item_pre) {
  using W = typename HWord<H>::T;
  const long long items = item_pre[p.ngroups];
  for (long long item = blockIdx.x; item < items; item += gridDim.x) {
    const int g = tp_find_group(item_pre, p.ngroups, item);
    const ThrGroup G = p.groups[g];
    const int ns = G.n_s;
    const int nch = (ns + TP1_ITEM_COLS - 1) / TP1_ITEM_COLS;
    const int r = (int)(item - item_pre[g]);
    const int B = r / nch, ch = r - B * nch;
    const int rows = min(H, ns - B * H);
    const int k0 = ch * TP1_ITEM_COLS + 8 * threadIdx.x;  // ns is a multiple of 8: all 8 columns or none
    if (k0 >= ns) continue;
    const uint16_t* col = D + G.dist_base + (long long)B * H * ns + k0;
    W* out = reinterpret_cast<W*>(p.tbits + G.tb_base + (long long)B * G.blk_stride) + k0;
    const long long plane_w = (long long)G.nblk * G.blk_stride / (long long)sizeof(W);
    for (int u = 0; u < G.nthr; ++u) {
      const unsigned th = min(p.thr[G.thr_first + u], 0xFFFFu);
      const unsigned th2 = th | (th << 16);
      unsigned w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      const uint4* q = reinterpret_cast<const uint4*>(col);
      const long long step = ns / 8;  // uint4 per row
      // eight rows' loads in flight before any of them is used (not more:
      // the registers of all H rows at once would cut the CTAs per SM)
#pragma unroll 1
      for (int t0 = 0; t0 < H; t0 += 8) {
        uint4 v[8];
#pragma unroll
        for (int x = 0; x < 8; ++x)
          v[x] = (t0 + x < rows) ? q[(long long)(t0 + x) * step] : make_uint4(~0u, ~0u, ~0u, ~0u);
#pragma unroll
        for (int x = 0; x < 8; ++x) {
          const unsigned vv[4] = {v[x].x, v[x].y, v[x].z, v[x].w};
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            bool hi, lo;
            __vibmin_u16x2(vv[j], th2, &hi, &lo);
            w[2 * j] |= (lo ? 1u : 0u) << (t0 + x);
            w[2 * j + 1] |= (hi ? 1u : 0u) << (t0 + x);
          }
        }
      }
      W* o = out + (long long)u * plane_w;
#pragma unroll
      for (int j = 0; j < 8; ++j) o[j] = (W)w[j];
    }
  }
}

// 32 x 32 bit transpose across a warp: lane l holds word x (bit t = element
// (t, l)); afterwards lane t holds the word whose bit l is element (t, l).
// Five rounds of exchanging half-blocks with the lane j apart.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, int lane) {
#pragma unroll
  for (int j = 16; j >= 1; j >>= 1) {
    const uint32_t m = j == 16 ? 0x0000FFFFu : j == 8 ? 0x00FF00FFu : j == 4 ? 0x0F0F0F0Fu : j == 2 ? 0x33333333u
                                                                                                   : 0x55555555u;
    const uint32_t o = __shfl_xor_sync(0xFFFFFFFFu, x, j);
    x = (lane & j) ? ((x & ~m) | ((o >> j) & m)) : ((x & m) | ((o << j) & ~m));
  }
  return x;
}

template <int H>
__global__ void __launch_bounds__(TP2_THREADS) thr_unpack_kernel(ThrParams p, const long long* __restrict__ item_pre,
                                                                 int blk_bytes_max) {
  using W = typename HWord<H>::T;
  extern __shared__ __align__(16) uint8_t tp_smem[];
  W* blk = reinterpret_cast<W*>(tp_smem);
  uint32_t* stage = reinterpret_cast<uint32_t*>(tp_smem + blk_bytes_max);  // H rows x TP2_STAGE_PITCH
  __shared__ int s_cnt[H], s_row[H];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = TP2_THREADS / 32;
  const long long items = item_pre[p.ngroups];
  for (long long item = blockIdx.x; item < items; item += gridDim.x) {
    const int g = tp_find_group(item_pre, p.ngroups, item);
    const ThrGroup G = p.groups[g];
    const int ns = G.n_s;
    const int r = (int)(item - item_pre[g]);
    const int u = r / G.nblk, B = r - u * G.nblk;
    const uint4* src = reinterpret_cast<const uint4*>(p.tbits + G.tb_base + (long long)u * G.nblk * G.blk_stride +
                                                      (long long)B * G.blk_stride);
    const int rows = min(H, ns - B * H);
    const int* ps = p.pos + G.pos_first;
    // the first chunk's positions and the block's original row indices are
    // in flight while the block is staged
    int qn[TP2_SLICES];
#pragma unroll
    for (int s = 0; s < TP2_SLICES; ++s) {
      const int j = (warp * TP2_SLICES + s) * 32 + lane;
      qn[s] = j < ns ? ps[j] : -1;
    }
    if (tid < rows) s_row[tid] = p.order[G.pos_first + B * H + tid] - G.pos_first;
    for (int q = tid; q < G.blk_stride / 16; q += TP2_THREADS) reinterpret_cast<uint4*>(tp_smem)[q] = src[q];
    if (tid < H) s_cnt[tid] = 0;
    __syncthreads();
    const int words32 = 2 * G.wpr;  // every 32-bit half of the row's 64-bit words, padding included
    uint64_t* plane_bits = p.bits + G.bits_base + (long long)u * ns * G.wpr;
    int cnt = 0;
    for (int cw0 = 0; cw0 < words32; cw0 += TP2_CHUNK_WORDS) {
      // this chunk's positions were loaded one chunk ahead; the next chunk's go out now
      int q[TP2_SLICES];
#pragma unroll
      for (int s = 0; s < TP2_SLICES; ++s) {
        q[s] = qn[s];
        const int j = (cw0 + TP2_CHUNK_WORDS + warp * TP2_SLICES + s) * 32 + lane;
        qn[s] = j < ns ? ps[j] : -1;
      }
      unsigned w[TP2_SLICES];
#pragma unroll
      for (int s = 0; s < TP2_SLICES; ++s) w[s] = q[s] >= 0 ? (unsigned)blk[q[s]] : 0u;
#pragma unroll
      for (int s = 0; s < TP2_SLICES; ++s) {
        const uint32_t mine = warp_transpose32(w[s], lane);  // lane t: row t's bits of the 32 columns
        if (lane < H) {
          stage[lane * TP2_STAGE_PITCH + warp * TP2_SLICES + s] = mine;
          cnt += __popc(mine);
        }
      }
      __syncthreads();
      const int nw = min(TP2_CHUNK_WORDS, words32 - cw0);
      for (int t = warp; t < rows; t += nwarps) {
        const int i = s_row[t];  // original row inside the set
        uint32_t* dst = reinterpret_cast<uint32_t*>(plane_bits + (long long)i * G.wpr) + cw0;
        for (int x = lane; x < nw; x += 32) dst[x] = stage[t * TP2_STAGE_PITCH + x];
      }
      __syncthreads();  // the stage is rewritten by the next chunk
    }
    if (lane < rows) atomicAdd(&s_cnt[lane], cnt);
    __syncthreads();
    if (tid < rows) p.counts[G.counts_base + (long long)u * ns + s_row[tid]] = s_cnt[tid];
    __syncthreads();  // blk, s_cnt and s_row are reused by the next item
  }
}

// Launch shapes are looked up once per kernel (and shared-memory size) so
// that the second pass follows the first without host work in between.
template <int H>
static cudaError_t launch_transposed_h(const ThrParams& p, int max_n_s, bool aligned16, const long long* pre1,
                                       long long items1, const long long* pre2, long long items2, cudaStream_t st) {
  static std::mutex mu;
  static int sms = 0, occ16 = 0, occ32 = 0;
  static size_t smem_set = 0;
  static int occ2_at = 0;
  std::lock_guard<std::mutex> lock(mu);  // contexts on several host threads share the cache
  cudaError_t e = cudaSuccess;
  if (!sms) {
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ16, thr_pack_kernel<H, uint16_t>, TP1_THREADS, 0);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ32, thr_pack_kernel<H, uint32_t>, TP1_THREADS, 0);
    if (e != cudaSuccess) {
      sms = 0;
      return e;
    }
  }
  static int occv = 0;
  if (!occv) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occv, thr_pack_vec_kernel<H>, TP1_THREADS, 0);
    if (e != cudaSuccess) {
      occv = 0;
      return e;
    }
  }
  const int occ1 = std::max(p.D16 ? occ16 : occ32, 1);
  if (p.D16 && aligned16)
    thr_pack_vec_kernel<H><<<(int)std::min<long long>(items1, (long long)sms * std::max(occv, 1)), TP1_THREADS, 0,
                             st>>>(p, p.D16, pre1);
  else if (p.D16)
    thr_pack_kernel<H, uint16_t><<<(int)std::min<long long>(items1, (long long)sms * occ1), TP1_THREADS, 0, st>>>(
        p, p.D16, pre1);
  else
    thr_pack_kernel<H, uint32_t><<<(int)std::min<long long>(items1, (long long)sms * occ1), TP1_THREADS, 0, st>>>(
        p, p.D32, pre1);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int blk_max = transposed_block_stride(max_n_s, H);
  const size_t smem = (size_t)blk_max + (size_t)H * TP2_STAGE_PITCH * 4;
  if (smem > smem_set) {  // the attribute only ever grows
    e = cudaFuncSetAttribute(thr_unpack_kernel<H>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    smem_set = smem;
    occ2_at = 0;
  }
  static size_t occ2_smem = 0;
  if (!occ2_at || occ2_smem != smem) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2_at, thr_unpack_kernel<H>, TP2_THREADS, smem);
    if (e != cudaSuccess) return e;
    occ2_smem = smem;
  }
  const int occ2 = occ2_at;
  thr_unpack_kernel<H><<<(int)std::min<long long>(items2, (long long)sms * std::max(occ2, 1)), TP2_THREADS, smem,
                         st>>>(p, pre2, blk_max);
  return cudaGetLastError();
}

cudaError_t launch_threshold_transposed(const ThrParams& p, int H, int max_n_s, bool aligned16,
                                        const long long* d_item_pre1, long long items1, const long long* d_item_pre2,
                                        long long items2, cudaStream_t st) {
  if (items1 <= 0 || items2 <= 0 || p.ngroups <= 0) return cudaSuccess;
  if (H == 32) return launch_transposed_h<32>(p, max_n_s, aligned16, d_item_pre1, items1, d_item_pre2, items2, st);
  if (H == 16) return launch_transposed_h<16>(p, max_n_s, aligned16, d_item_pre1, items1, d_item_pre2, items2, st);
  if (H == 8) return launch_transposed_h<8>(p, max_n_s, aligned16, d_item_pre1, items1, d_item_pre2, items2, st);
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// Tile rectangles for the split pass's exchange: one entry per thread,
// grid-stride; the tile of an entry by binary search over the prefix array.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int tile_of_entry(const long long* pre, int ntiles, long long e) {
  int lo = 0, hi = ntiles - 1;  // last tile with pre[t] <= e
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= e) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(256) tile_pack_kernel(DistLayout L, const TileRect* __restrict__ rects,
                                                        const long long* __restrict__ pre, int ntiles,
                                                        void* __restrict__ out) {
  const long long total = pre[ntiles];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int t = tile_of_entry(pre, ntiles, e);
    const TileRect R = rects[t];
    const long long k = e - pre[t];
    const int r = (int)(k / R.nb), c = (int)(k - (long long)r * R.nb);
    const int first = L.set_first[R.set], ns = L.set_n[R.set];
    const long long idx = L.set_base[R.set] + (long long)(R.ra0 + r - first) * ns + (R.b0 + c - first);
    if (L.D16) static_cast<uint16_t*>(out)[e] = L.D16[idx];
    else static_cast<uint32_t*>(out)[e] = L.D32[idx];
  }
}

__global__ void __launch_bounds__(256) tile_unpack_kernel(DistLayout L, const TileRect* __restrict__ rects,
                                                          const long long* __restrict__ pre, int ntiles,
                                                          const void* __restrict__ in, long long e0, long long e1) {
  for (long long e = e0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < e1;
       e += (long long)gridDim.x * blockDim.x) {
    const int t = tile_of_entry(pre, ntiles, e);
    const TileRect R = rects[t];
    const long long k = e - pre[t];
    const int r = (int)(k / R.nb), c = (int)(k - (long long)r * R.nb);
    const int first = L.set_first[R.set], ns = L.set_n[R.set];
    const long long a = R.ra0 + r - first, b = R.b0 + c - first;
    const unsigned v = L.D16 ? (unsigned)static_cast<const uint16_t*>(in)[e - e0]
                             : static_cast<const uint32_t*>(in)[e - e0];
    store_dist(L, L.set_base[R.set] + a * ns + b, v);
    store_dist(L, L.set_base[R.set] + b * ns + a, v);
  }
}

__global__ void __launch_bounds__(256) mark_tiles_kernel(const int2* __restrict__ cand, long long count,
                                                         const int* __restrict__ pos, int lo, int hi, int nf,
                                                         const int* __restrict__ cb_of, int nq, int PB,
                                                         uint8_t* __restrict__ mark) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < count;
       c += (long long)gridDim.x * blockDim.x) {
    const int2 pr = cand[c];
    const int x = pr.x & 0x7FFFFFFF, y = pr.y;
    if (x < lo || x >= hi || y < lo || y >= hi) continue;
    int px = pos[x], py = pos[y];
    if (px >= nf || py >= nf || px == py) continue;  // 32-bit-path pairs are scored anyway
    if (px > py) {
      const int t = px;
      px = py;
      py = t;
    }
    mark[(size_t)cb_of[px] * nq + (py / 2) / PB] = 1;
  }
}

cudaError_t launch_mark_tiles(const int2* cand, long long count, const int* pos, int lo, int hi, int nf,
                              const int* cb_of, int nq, int PB, uint8_t* mark, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((count + 255) / 256, 148LL * 8);
  mark_tiles_kernel<<<(int)blocks, 256, 0, st>>>(cand, count, pos, lo, hi, nf, cb_of, nq, PB, mark);
  return cudaGetLastError();
}

cudaError_t launch_tile_pack(const DistLayout& L, const TileRect* rects, const long long* pre, int ntiles,
                             void* out, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  tile_pack_kernel<<<148 * 8, 256, 0, st>>>(L, rects, pre, ntiles, out);
  return cudaGetLastError();
}

cudaError_t launch_tile_unpack(const DistLayout& L, const TileRect* rects, const long long* pre, int ntiles,
                               const void* in, long long e0, long long e1, cudaStream_t st) {
  if (ntiles <= 0 || e1 <= e0) return cudaSuccess;
  tile_unpack_kernel<<<148 * 8, 256, 0, st>>>(L, rects, pre, ntiles, in, e0, e1);
  return cudaGetLastError();
}

// Set matrix in original index order, widened to 32 bits.
template <typename DT>
__global__ void __launch_bounds__(256) unpermute_kernel(const DT* __restrict__ Dset, const int* __restrict__ pos,
                                                        int ns, int r0, int r1, uint32_t* __restrict__ out) {
  for (int i = r0 + blockIdx.x; i < r1; i += gridDim.x) {
    const DT* row = Dset + (long long)pos[i] * ns;
    for (int k = threadIdx.x; k < ns; k += blockDim.x) out[(size_t)(i - r0) * ns + k] = (uint32_t)row[pos[k]];
  }
}

cudaError_t launch_unpermute_set(const uint16_t* D16set, const uint32_t* D32set, const int* pos, int n_s, int r0,
                                 int r1, uint32_t* out, cudaStream_t st) {
  if (n_s <= 0 || r1 <= r0) return cudaSuccess;
  const int grid = min(r1 - r0, 148 * 8);
  if (D16set) unpermute_kernel<uint16_t><<<grid, 256, 0, st>>>(D16set, pos, n_s, r0, r1, out);
  else unpermute_kernel<uint32_t><<<grid, 256, 0, st>>>(D32set, pos, n_s, r0, r1, out);
  return cudaGetLastError();
}

// Statistics of a block of one set's matrix (original indices): one CTA per
// row of [r0, r1) over the columns [c0, c1).
template <typename DT>
__global__ void __launch_bounds__(256) block_stats_kernel(const DT* __restrict__ Dset, const int* __restrict__ pos,
                                                          int ns, int r0, int r1, int c0, int c1, double mean,
                                                          unsigned long long* __restrict__ row_sum,
                                                          unsigned long long* __restrict__ row_sqdev,
                                                          unsigned* bmin, unsigned* bmax) {
  __shared__ unsigned long long s_sum[8], s_sq[8];
  __shared__ unsigned s_min[8], s_max[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int i = r0 + blockIdx.x; i < r1; i += gridDim.x) {
    const DT* row = Dset + (long long)pos[i] * ns;
    unsigned long long sum = 0, sq = 0;
    unsigned mn = 0xFFFFFFFFu, mx = 0u;
    for (int k = c0 + threadIdx.x; k < c1; k += blockDim.x) {
      const unsigned v = row[pos[k]];
      sum += v;
      const double d = (double)v - mean;
      sq += (unsigned long long)floor(__dmul_rn(d, d));  // no contraction into a later add
      mn = min(mn, v);
      mx = max(mx, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
      sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
      sq += __shfl_xor_sync(0xFFFFFFFFu, sq, o);
      mn = min(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
      mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    }
    if (lane == 0) s_sum[warp] = sum, s_sq[warp] = sq, s_min[warp] = mn, s_max[warp] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < nwarps; ++w) {
        sum += s_sum[w];
        sq += s_sq[w];
        mn = min(mn, s_min[w]);
        mx = max(mx, s_max[w]);
      }
      if (row_sum) row_sum[i - r0] = sum;
      if (row_sqdev) row_sqdev[i - r0] = sq;
      if (c1 > c0) {
        atomicMin(bmin, mn);
        atomicMax(bmax, mx);
      }
    }
    __syncthreads();  // s_* are reused by the next row
  }
}

cudaError_t launch_block_stats(const uint16_t* D16set, const uint32_t* D32set, const int* pos, int n_s, int r0,
                               int r1, int c0, int c1, double mean, unsigned long long* row_sum,
                               unsigned long long* row_sqdev, unsigned* bmin, unsigned* bmax, cudaStream_t st) {
  if (n_s <= 0 || r1 <= r0) return cudaSuccess;
  const int grid = min(r1 - r0, 148 * 8);
  if (D16set)
    block_stats_kernel<uint16_t><<<grid, 256, 0, st>>>(D16set, pos, n_s, r0, r1, c0, c1, mean, row_sum, row_sqdev,
                                                       bmin, bmax);
  else
    block_stats_kernel<uint32_t><<<grid, 256, 0, st>>>(D32set, pos, n_s, r0, r1, c0, c1, mean, row_sum, row_sqdev,
                                                       bmin, bmax);
  return cudaGetLastError();
}

__global__ void __launch_bounds__(256) csr_fill_kernel(const uint64_t* __restrict__ bits, int n, int wpr,
                                                       const long long* __restrict__ row_ptr,
                                                       int* __restrict__ cols) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    long long pos = row_ptr[i];
    const uint64_t* rb = bits + (size_t)i * (size_t)wpr;
    for (int w0 = 0; w0 < wpr; w0 += 32) {
      const int w = w0 + lane;
      uint64_t word = w < wpr ? rb[w] : 0ull;
      const int c = __popcll(word);
      int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      long long q = pos + incl - c;
      while (word) {
        const int bit = __ffsll((long long)word) - 1;
        cols[q++] = w * 64 + bit;
        word &= word - 1;
      }
      pos += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
  }
}

cudaError_t launch_csr_fill(const uint64_t* bits, int n, int words_per_row, const long long* row_ptr,
                            int* cols, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int grid = min((n + 7) / 8, 148 * 16);
  csr_fill_kernel<<<grid, 256, 0, st>>>(bits, n, words_per_row, row_ptr, cols);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Instruction-mix probe: the per-cell sequence of fast_segment (PRMT, three
// add-max, one max) on 8 independent chains per thread, so that issue rate,
// not latency, limits it.  Writes one word per thread so nothing is elided.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) mix_probe_kernel(uint32_t* sink, int iters) {
  constexpr int C = 8;
  const uint32_t t = threadIdx.x + blockIdx.x * blockDim.x;
  uint32_t h[C], x[C], m[C], tlo[C], thi[C];
  uint32_t sel = make_sel(t & 3, (t >> 2) & 3);
  const uint32_t M3 = 0xFFFDFFFDu;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    h[c] = (t * (c + 3)) & 0x00FF00FFu;
    x[c] = (t * (c + 7)) & 0x00FF00FFu;
    m[c] = 0u;
    // a distinct table per chain, as each column has its own in the kernel,
    // so no chain can reuse another chain's permute
    tlo[c] = (0xFF07FFFFu ^ t) + 0x01010101u * (uint32_t)c;
    thi[c] = (0xFFFF07FFu + t) ^ (0x00010000u * (uint32_t)c);
  }
  // per packed cell update, as in fast_segment: PRMT, add, 3-input max, add,
  // and half a 3-input max for the running maximum (two chains share one)
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const uint32_t d = prmt(tlo[c], thi[c], sel);
      const uint32_t t = vadd(h[c], d);
      const uint32_t hn = vmax3_0(t, x[c], h[c]);
      x[c] = vadd(hn, M3);
      h[c] = hn;
      if (c & 1) m[c] = vmax3_0(m[c], x[c - 1], t);
    }
    sel ^= 0x0101u;
  }
  uint32_t acc = 0;
#pragma unroll
  for (int c = 0; c < C; ++c) acc ^= m[c] ^ h[c] ^ x[c];
  sink[t] = acc;
}

cudaError_t launch_mix_probe(uint32_t* sink, int grid, int block, int iters, cudaStream_t st) {
  mix_probe_kernel<<<grid, block, 0, st>>>(sink, iters);
  return cudaGetLastError();
}

}  // namespace swgpu
