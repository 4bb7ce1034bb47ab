// k-mer frequency tables and their text form on the GPU: the work of
// fasta2kmer (fasta2kmer.c:8-44) over frequencies_from_dataset and
// write_kmer_base (kmers.c:157-389).
//
// Counting.  The reference tests every table entry against every window of a
// sequence (4^k * len byte compares per sequence).  Here a CTA takes one
// sequence, each thread rolls a k-mer index over a contiguous run of windows
// and adds one to that entry, so the work is len, not 4^k * len:
//   kmer_shared_kernel   tables of <= 65536 entries: 16-bit counters packed two
//                        to a 32-bit word in shared memory, written out as the
//                        int16 row in 16-byte stores
//   kmer_packed_kernel   larger tables: the same packed counters, in the row
//                        itself (zeroed first) with global atomics
//   kmer_wide_kernel     sequences with >= 65536 windows, where a 16-bit
//                        counter could carry into its neighbour: 32-bit
//                        counters, then kmer_narrow_kernel keeps the low 16
//                        bits (the reference's short arithmetic)
// Text.  kmer_tsv_len_kernel measures each segment of a row (up to 65536
// counts), kmer_scan_kernel turns the lengths into offsets, and
// kmer_tsv_write_kernel prints the digits, one warp per segment.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "staging.cuh"

namespace swgpu {
namespace {

constexpr int KM_THREADS = 256;
constexpr int64_t KM_SHARED_MAX = 65536;   // entries a CTA's shared table holds (128 KB)
constexpr int64_t KM_CARRY = 65536;        // windows from which a 16-bit counter can carry
constexpr int64_t KM_SEG = 65536;          // counts per text segment
constexpr size_t KM_OUT_CAP = size_t(1) << 30;    // bytes of int16 rows per device batch
constexpr size_t KM_TEXT_CAP = size_t(256) << 20; // bytes of text per device batch

// Symbol codes: 'A' 'C' 'G' 'T' -> 0..3 (gen_dna_string_from_binary,
// kmers.c:26-63), or the 20 letters of gen_protein_kmers (kmers.c:136-140) ->
// 0..19; any other byte -> -1 (it equals no k-mer symbol).
__device__ void load_codes(int8_t* tab, bool protein) {
  for (int c = threadIdx.x; c < 256; c += blockDim.x) {
    int v = -1;
    if (!protein) {
      v = c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : c == 'T' ? 3 : -1;
    } else {
      const char letters[21] = "ACDEFGHIKLMNPQRSTVWY";
      for (int j = 0; j < 20; ++j)
        if (letters[j] == c) v = j;
    }
    tab[c] = (int8_t)v;
  }
}

// Calls f(index) for every counted window of s that belongs to this thread.
// Windows 0 .. nwin-1 are split into one contiguous run per thread; the index
// rolls from window to window.  DNA: symbol p of the window in bits 2p..2p+1.
// Protein: base-20 number, symbol 0 most significant (top = 20^(k-1)).  A
// window holding a byte without code is not counted.
template <bool PROTEIN, class F>
__device__ __forceinline__ void for_each_window(const uint8_t* __restrict__ s, int64_t nwin, int k,
                                                const int8_t* tab, uint64_t top, F&& f) {
  const int64_t per = (nwin + blockDim.x - 1) / blockDim.x;
  const int64_t w0 = (int64_t)threadIdx.x * per;
  const int64_t w1 = w0 + per < nwin ? w0 + per : nwin;
  if (w0 >= w1) return;
  uint64_t code = 0;
  int64_t bad = -1;  // last position holding a byte without code
  auto sym = [&](int64_t q) -> uint64_t {
    const int c = tab[s[q]];
    if (c < 0) {
      bad = q;
      return 0;
    }
    return (uint64_t)c;
  };
  for (int p = 0; p < k - 1; ++p) {
    const uint64_t c = sym(w0 + p);
    if (PROTEIN) code = code * 20 + c;
    else code |= c << (2 * p);
  }
  for (int64_t w = w0; w < w1; ++w) {
    const uint64_t c = sym(w + k - 1);
    if (PROTEIN) code = code * 20 + c;
    else code |= c << (2 * (k - 1));
    if (bad < w) f(code);
    if (PROTEIN) {
      const int lead = tab[s[w]];
      code -= (uint64_t)(lead < 0 ? 0 : lead) * top;
    } else {
      code >>= 2;
    }
  }
}

__device__ __forceinline__ void packed_add(uint32_t* words, uint64_t idx) {
  atomicAdd(words + (idx >> 1), 1u << ((unsigned)(idx & 1) << 4));
}

template <bool PROTEIN>
__global__ void __launch_bounds__(KM_THREADS) kmer_shared_kernel(const uint8_t* __restrict__ seqs,
                                                                 const int64_t* __restrict__ off,
                                                                 const int64_t* __restrict__ len, int64_t n, int k,
                                                                 uint64_t top, int64_t nk,
                                                                 int16_t* __restrict__ out) {
  extern __shared__ uint4 km_table[];
  __shared__ int8_t tab[256];
  load_codes(tab, PROTEIN);
  uint32_t* words = reinterpret_cast<uint32_t*>(km_table);
  const int64_t nwords = nk >> 1;  // nk is even for every k >= 1
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    const int64_t L = len[i];
    const int64_t nwin = L > k ? L - k : 0;
    if (nwin >= KM_CARRY) continue;  // kmer_wide_kernel's row (uniform over the CTA)
    for (int64_t w = threadIdx.x; w < nwords; w += blockDim.x) words[w] = 0;
    __syncthreads();
    for_each_window<PROTEIN>(seqs + off[i], nwin, k, tab, top, [&](uint64_t idx) { packed_add(words, idx); });
    __syncthreads();
    int16_t* row = out + i * nk;
    if ((nk & 7) == 0) {
      uint4* dst = reinterpret_cast<uint4*>(row);
      for (int64_t v = threadIdx.x; v < (nk >> 3); v += blockDim.x) dst[v] = km_table[v];
    } else {
      uint32_t* dst = reinterpret_cast<uint32_t*>(row);
      for (int64_t v = threadIdx.x; v < nwords; v += blockDim.x) dst[v] = words[v];
    }
    __syncthreads();
  }
}

// Rows zeroed beforehand; sequences with fewer than KM_CARRY windows.
template <bool PROTEIN>
__global__ void __launch_bounds__(KM_THREADS) kmer_packed_kernel(const uint8_t* __restrict__ seqs,
                                                                 const int64_t* __restrict__ off,
                                                                 const int64_t* __restrict__ len, int64_t n, int k,
                                                                 uint64_t top, int64_t nk,
                                                                 int16_t* __restrict__ out) {
  __shared__ int8_t tab[256];
  load_codes(tab, PROTEIN);
  __syncthreads();
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    const int64_t L = len[i];
    const int64_t nwin = L > k ? L - k : 0;
    if (nwin >= KM_CARRY) continue;
    uint32_t* words = reinterpret_cast<uint32_t*>(out + i * nk);
    for_each_window<PROTEIN>(seqs + off[i], nwin, k, tab, top, [&](uint64_t idx) { packed_add(words, idx); });
  }
}

// 32-bit counters (zeroed beforehand) for the rows in list[0..nlist).
template <bool PROTEIN>
__global__ void __launch_bounds__(KM_THREADS) kmer_wide_kernel(const uint8_t* __restrict__ seqs,
                                                               const int64_t* __restrict__ off,
                                                               const int64_t* __restrict__ len,
                                                               const int64_t* __restrict__ list, int64_t nlist, int k,
                                                               uint64_t top, int64_t nk,
                                                               uint32_t* __restrict__ counts) {
  __shared__ int8_t tab[256];
  load_codes(tab, PROTEIN);
  __syncthreads();
  for (int64_t j = blockIdx.x; j < nlist; j += gridDim.x) {
    const int64_t i = list[j];
    const int64_t L = len[i];
    const int64_t nwin = L > k ? L - k : 0;
    uint32_t* c = counts + j * nk;
    for_each_window<PROTEIN>(seqs + off[i], nwin, k, tab, top, [&](uint64_t idx) { atomicAdd(c + idx, 1u); });
  }
}

__global__ void kmer_narrow_kernel(const uint32_t* __restrict__ counts, const int64_t* __restrict__ list,
                                   int64_t nlist, int64_t nk, int16_t* __restrict__ out) {
  const int64_t total = nlist * nk;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / nk, b = e - j * nk;
    out[list[j] * nk + b] = (int16_t)(uint16_t)(counts[e] & 0xFFFFu);
  }
}

// ---- text ----------------------------------------------------------------

// Characters of printf("%hi") for a short.
__device__ __forceinline__ int short_len(int v) {
  const int a = v < 0 ? -v : v;
  return (v < 0) + (a >= 10000 ? 5 : a >= 1000 ? 4 : a >= 100 ? 3 : a >= 10 ? 2 : 1);
}

__device__ __forceinline__ int uint_len(uint64_t a) {
  int n = 1;
  while (a >= 10) a /= 10, ++n;
  return n;
}

// Writes the decimal digits of a (len characters) ending before end.
__device__ __forceinline__ void put_digits(char* end, uint64_t a, int len) {
  for (int q = 0; q < len; ++q) {
    *--end = (char)('0' + (int)(a % 10));
    a /= 10;
  }
}

struct SegGeom {
  int64_t first_seg;  // global index of the batch's first segment
  int64_t nseg;       // segments in the batch
  int64_t spr;        // segments per row
  int64_t nk;         // counts per row
  int64_t elem0;      // row-major index of the batch's first count
};

__device__ __forceinline__ void seg_bounds(const SegGeom& g, int64_t s, int64_t* row, int64_t* c0, int64_t* c1,
                                           int64_t* local0) {
  const int64_t gs = g.first_seg + s;
  *row = gs / g.spr;
  const int64_t part = gs - *row * g.spr;
  *c0 = part * KM_SEG;
  *c1 = *c0 + KM_SEG < g.nk ? *c0 + KM_SEG : g.nk;
  *local0 = *row * g.nk + *c0 - g.elem0;
}

__device__ __forceinline__ int prefix_len(int64_t row) { return 9 + uint_len((uint64_t)row) + 1; }  // "sequence_<i>\t"

__global__ void kmer_tsv_len_kernel(const int16_t* __restrict__ counts, SegGeom g, uint32_t* __restrict__ seg_len) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t s = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); s < g.nseg; s += warps) {
    int64_t row, c0, c1, l0;
    seg_bounds(g, s, &row, &c0, &c1, &l0);
    uint32_t t = 0;
    for (int64_t c = c0 + lane; c < c1; c += 32) t += short_len(counts[l0 + (c - c0)]) + 1;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
    if (lane == 0) seg_len[s] = t + (c0 == 0 ? prefix_len(row) : 0);
  }
}

// Exclusive prefix sums of n lengths into off[0..n] (off[n] = total); one CTA.
__global__ void __launch_bounds__(1024) kmer_scan_kernel(const uint32_t* __restrict__ len, int64_t n,
                                                         int64_t* __restrict__ off) {
  __shared__ int64_t part[32];
  __shared__ int64_t carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t b = 0; b < n; b += blockDim.x) {
    const int64_t i = b + threadIdx.x;
    const int64_t v = i < n ? (int64_t)len[i] : 0;
    int64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) part[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int64_t p = lane < (int)(blockDim.x >> 5) ? part[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xFFFFFFFFu, p, o);
        if (lane >= o) p += y;
      }
      part[lane] = p;  // inclusive over warps
    }
    __syncthreads();
    const int64_t before = carry + (warp > 0 ? part[warp - 1] : 0);
    if (i < n) off[i] = before + x - v;
    __syncthreads();
    if (threadIdx.x == 0) carry += part[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) off[n] = carry;
}

__global__ void kmer_tsv_write_kernel(const int16_t* __restrict__ counts, SegGeom g, const int64_t* __restrict__ off,
                                      char* __restrict__ text) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t s = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); s < g.nseg; s += warps) {
    int64_t row, c0, c1, l0;
    seg_bounds(g, s, &row, &c0, &c1, &l0);
    int64_t pos = off[s];
    if (c0 == 0) {
      const int pl = prefix_len(row);
      if (lane < 9) text[pos + lane] = "sequence_"[lane];
      if (lane == 0) {
        put_digits(text + pos + pl - 1, (uint64_t)row, pl - 10);
        text[pos + pl - 1] = '\t';
      }
      pos += pl;
    }
    for (int64_t cb = c0; cb < c1; cb += 32) {
      const int64_t c = cb + lane;
      const bool on = c < c1;
      const int v = on ? (int)counts[l0 + (c - c0)] : 0;
      const int l = on ? short_len(v) + 1 : 0;
      int x = l;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
      }
      if (on) {
        char* p = text + pos + (x - l);
        const int dl = l - 1;
        if (v < 0) p[0] = '-';
        put_digits(p + dl, (uint64_t)(v < 0 ? -v : v), dl - (v < 0));
        p[dl] = c == g.nk - 1 ? '\n' : '\t';
      }
      pos += __shfl_sync(0xFFFFFFFFu, x, 31);
    }
  }
}

int grid_for(const swe_ctx* ctx, int64_t units, int per_sm) {
  const int64_t cap = (int64_t)ctx->num_sms * per_sm;
  return (int)std::max<int64_t>(1, std::min(units, cap));
}

}  // namespace

// Device buffers kept by a context between k-mer calls.
struct KmerState {
  DevBuf<int16_t> d_out, d_cnt;
  DevBuf<uint8_t> d_seq;
  DevBuf<int64_t> d_off, d_len, d_list, d_segoff;
  DevBuf<uint32_t> d_wide, d_seglen;
  DevBuf<char> d_text;
};

void kmer_state_destroy(KmerState* km) { delete km; }

void staging_destroy(Staging* sg) { delete sg; }

swe_status staging_ready(swe_ctx* ctx, size_t chunk, Staging** out) {
  if (!ctx->stage) {
    ctx->stage = new (std::nothrow) Staging();
    if (!ctx->stage) return fail(ctx, SWE_ERR_OOM, "staging buffers");
    for (auto& e : ctx->stage->ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  for (auto& p : ctx->stage->pin) CK(p.alloc(chunk));
  *out = ctx->stage;
  return SWE_OK;
}

namespace {

// Device buffers above 1 GB (very long k-mers, very many rows) are given back
// after a call instead of being kept for the next one.
void trim_kmer_state(KmerState* km) {
  constexpr size_t KEEP = size_t(1) << 30;
  if (km->d_out.n * sizeof(int16_t) > KEEP) km->d_out.release();
  if (km->d_cnt.n * sizeof(int16_t) > KEEP) km->d_cnt.release();
  if (km->d_text.n > KEEP) km->d_text.release();
  if (km->d_wide.n * sizeof(uint32_t) > KEEP) km->d_wide.release();
  if (km->d_seq.n > KEEP) km->d_seq.release();
}

// The context's k-mer buffers and its staging chunks.
swe_status kmer_state(swe_ctx* ctx, size_t chunk, KmerState** out, Staging** sg) {
  if (!ctx->km) {
    ctx->km = new (std::nothrow) KmerState();
    if (!ctx->km) return fail(ctx, SWE_ERR_OOM, "k-mer state");
  }
  *out = ctx->km;
  return staging_ready(ctx, chunk, sg);
}

}  // namespace
}  // namespace swgpu

using namespace swgpu;

extern "C" {

int64_t swe_kmer_count(int k, int protein) {
  if (k < 1 || k > (protein ? SWE_KMER_MAX_PROTEIN : SWE_KMER_MAX_DNA)) return 0;
  int64_t n = 1;
  for (int i = 0; i < k; ++i) n *= protein ? 20 : 4;
  return n;
}

swe_status swe_kmer_counts(swe_ctx* ctx, const char* const* seqs, const int64_t* len, int64_t n, int k, int protein,
                           int16_t* const* rows) {
  if (!ctx) return SWE_ERR_INVALID;
  const int64_t nk = swe_kmer_count(k, protein);
  if (nk == 0) return fail(ctx, SWE_ERR_INVALID, "k-mer length out of range");
  if (n < 0 || (n > 0 && (!seqs || !len || !rows))) return fail(ctx, SWE_ERR_INVALID, "bad k-mer input");
  if (n == 0) return SWE_OK;
  for (int64_t i = 0; i < n; ++i)
    if (len[i] < 0 || (len[i] > 0 && !seqs[i]) || !rows[i]) return fail(ctx, SWE_ERR_INVALID, "bad k-mer input");
  if (swe_status st = select_device(ctx)) return st;
  const size_t chunk = stage_chunk(ctx);
  KmerState* km = nullptr;
  Staging* sg = nullptr;
  if (swe_status st = kmer_state(ctx, chunk, &km, &sg)) return st;
  uint64_t top = 1;
  for (int i = 0; i < k - 1; ++i) top *= protein ? 20 : 4;

  const size_t out_cap = ctx->kmer_batch_bytes ? ctx->kmer_batch_bytes : KM_OUT_CAP;
  const size_t row_bytes = (size_t)nk * sizeof(int16_t);
  const int64_t rows_per_batch = std::max<int64_t>(1, (int64_t)(out_cap / row_bytes));
  const bool shared_table = nk <= KM_SHARED_MAX;
  const size_t smem = ((size_t)nk * sizeof(int16_t) + 15) & ~size_t(15);
  if (shared_table && smem > 48 * 1024) {
    CK(cudaFuncSetAttribute(kmer_shared_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CK(cudaFuncSetAttribute(kmer_shared_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  const int shared_per_sm = (int)std::max<size_t>(1, std::min<size_t>(8, (200u << 10) / std::max<size_t>(smem, 1)));

  std::vector<int64_t> b_off, b_len, longs;
  for (int64_t r0 = 0, nb = 0; r0 < n; r0 += nb) {
    // this batch's rows (at most out_cap bytes of rows and of sequences, at
    // least one row)
    b_off.clear();
    b_len.clear();
    longs.clear();
    int64_t bytes = 0;
    for (nb = 0; r0 + nb < n && nb < rows_per_batch; ++nb) {
      const int64_t L = len[r0 + nb];
      if (nb > 0 && bytes + L > (int64_t)out_cap) break;
      b_off.push_back(bytes);
      b_len.push_back(L);
      bytes += L;
      if (L - k >= KM_CARRY) longs.push_back(nb);
    }
    CK(km->d_seq.alloc((size_t)std::max<int64_t>(bytes, 1)));
    CK(km->d_off.alloc(nb));
    CK(km->d_len.alloc(nb));
    CK(km->d_out.alloc((size_t)nb * nk));
    // the batch's sequences, packed back to back
    swe_status st = staged_h2d(ctx, sg, chunk, km->d_seq.p, (size_t)bytes, [&](char* dst, size_t a, size_t b) {
      split_copy(a, b, [&](size_t x, size_t y) {
        int64_t i = std::upper_bound(b_off.begin(), b_off.end(), (int64_t)x) - b_off.begin() - 1;
        for (size_t p = x; p < y; ++i) {
          const size_t s0 = (size_t)b_off[i], s1 = s0 + (size_t)b_len[i];
          if (s1 <= p) continue;
          const size_t e = std::min(y, s1);
          memcpy(dst + (p - a), seqs[r0 + i] + (p - s0), e - p);
          p = e;
        }
      });
    });
    if (st) return st;
    CK(cpy(ctx, km->d_off.p, b_off.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, ctx->st));
    CK(cpy(ctx, km->d_len.p, b_len.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, ctx->st));

    if (shared_table) {
      const int grid = grid_for(ctx, nb, shared_per_sm);
      ctx->stats.kernel_launches += 1;
      if (protein)
        kmer_shared_kernel<true><<<grid, KM_THREADS, smem, ctx->st>>>(km->d_seq.p, km->d_off.p, km->d_len.p, nb, k,
                                                                      top, nk, km->d_out.p);
      else
        kmer_shared_kernel<false><<<grid, KM_THREADS, smem, ctx->st>>>(km->d_seq.p, km->d_off.p, km->d_len.p, nb, k,
                                                                       top, nk, km->d_out.p);
      CK(cudaGetLastError());
    } else {
      CK(cudaMemsetAsync(km->d_out.p, 0, (size_t)nb * row_bytes, ctx->st));
      const int grid = grid_for(ctx, nb, 8);
      ctx->stats.kernel_launches += 1;
      if (protein)
        kmer_packed_kernel<true><<<grid, KM_THREADS, 0, ctx->st>>>(km->d_seq.p, km->d_off.p, km->d_len.p, nb, k, top,
                                                                   nk, km->d_out.p);
      else
        kmer_packed_kernel<false><<<grid, KM_THREADS, 0, ctx->st>>>(km->d_seq.p, km->d_off.p, km->d_len.p, nb, k,
                                                                    top, nk, km->d_out.p);
      CK(cudaGetLastError());
    }
    // sequences long enough for a 16-bit counter to carry
    if (!longs.empty()) {
      const int64_t per = std::max<int64_t>(1, (int64_t)(2 * out_cap / (nk * sizeof(uint32_t))));
      CK(km->d_list.alloc(longs.size()));
      CK(cpy(ctx, km->d_list.p, longs.data(), sizeof(int64_t) * longs.size(), cudaMemcpyHostToDevice, ctx->st));
      for (size_t j0 = 0; j0 < longs.size(); j0 += (size_t)per) {
        const int64_t nl = std::min<int64_t>(per, (int64_t)(longs.size() - j0));
        CK(km->d_wide.alloc((size_t)nl * nk));
        CK(cudaMemsetAsync(km->d_wide.p, 0, sizeof(uint32_t) * nl * nk, ctx->st));
        ctx->stats.kernel_launches += 2;
        if (protein)
          kmer_wide_kernel<true><<<grid_for(ctx, nl, 8), KM_THREADS, 0, ctx->st>>>(
              km->d_seq.p, km->d_off.p, km->d_len.p, km->d_list.p + j0, nl, k, top, nk, km->d_wide.p);
        else
          kmer_wide_kernel<false><<<grid_for(ctx, nl, 8), KM_THREADS, 0, ctx->st>>>(
              km->d_seq.p, km->d_off.p, km->d_len.p, km->d_list.p + j0, nl, k, top, nk, km->d_wide.p);
        CK(cudaGetLastError());
        kmer_narrow_kernel<<<grid_for(ctx, (nl * nk + 255) / 256, 8), 256, 0, ctx->st>>>(
            km->d_wide.p, km->d_list.p + j0, nl, nk, km->d_out.p);
        CK(cudaGetLastError());
      }
    }
    // rows back into the caller's row buffers
    st = staged_d2h(ctx, sg, chunk, km->d_out.p, (size_t)nb * row_bytes, [&](const char* src, size_t a, size_t b) {
      split_copy(a, b, [&](size_t x, size_t y) {
        for (size_t p = x; p < y;) {
          const size_t r = p / row_bytes, in = p - r * row_bytes;
          const size_t e = std::min(y, (r + 1) * row_bytes);
          memcpy(reinterpret_cast<char*>(rows[r0 + (int64_t)r]) + in, src + (p - a), e - p);
          p = e;
        }
      });
      return true;
    });
    if (st) return st;
  }
  CK(cudaStreamSynchronize(ctx->st));
  trim_kmer_state(km);
  return SWE_OK;
}

swe_status swe_kmer_tsv(swe_ctx* ctx, const int16_t* const* rows, int64_t n, int64_t nk, swe_text_sink sink,
                        void* user) {
  if (!ctx) return SWE_ERR_INVALID;
  if (n < 0 || nk < 0 || (n > 0 && (!rows || !sink))) return fail(ctx, SWE_ERR_INVALID, "bad k-mer table");
  if (n == 0) return SWE_OK;
  if (nk == 0) return fail(ctx, SWE_ERR_INVALID, "k-mer table without columns");
  for (int64_t i = 0; i < n; ++i)
    if (!rows[i]) return fail(ctx, SWE_ERR_INVALID, "bad k-mer table");
  if (swe_status st = select_device(ctx)) return st;
  const size_t chunk = stage_chunk(ctx);
  KmerState* km = nullptr;
  Staging* sg = nullptr;
  if (swe_status st = kmer_state(ctx, chunk, &km, &sg)) return st;

  const int64_t spr = (nk + KM_SEG - 1) / KM_SEG;
  const int64_t seg_cols = std::min(nk, KM_SEG);
  const int64_t seg_worst = 7 * seg_cols + 32;  // "-32768\t" per count, plus the row label
  const size_t text_cap = ctx->kmer_batch_bytes ? ctx->kmer_batch_bytes : KM_TEXT_CAP;
  const int64_t segs_per_batch = std::max<int64_t>(1, (int64_t)text_cap / seg_worst);
  const int64_t nseg_all = n * spr;
  const size_t row_bytes = (size_t)nk * sizeof(int16_t);

  for (int64_t s0 = 0; s0 < nseg_all; s0 += segs_per_batch) {
    const int64_t ns = std::min(segs_per_batch, nseg_all - s0);
    // the batch covers counts [e0, e1) of the row-major table
    const int64_t r_first = s0 / spr, r_last = (s0 + ns - 1) / spr;
    const int64_t e0 = r_first * nk + (s0 - r_first * spr) * KM_SEG;
    const int64_t last_part = (s0 + ns - 1) - r_last * spr;
    const int64_t e1 = r_last * nk + std::min(nk, (last_part + 1) * KM_SEG);
    const size_t bytes = (size_t)(e1 - e0) * sizeof(int16_t);
    const size_t base = (size_t)e0 * sizeof(int16_t);
    CK(km->d_cnt.alloc((size_t)(e1 - e0)));
    swe_status st = staged_h2d(ctx, sg, chunk, km->d_cnt.p, bytes, [&](char* dst, size_t a, size_t b) {
      split_copy(base + a, base + b, [&](size_t x, size_t y) {
        for (size_t p = x; p < y;) {
          const size_t r = p / row_bytes, in = p - r * row_bytes;
          const size_t e = std::min(y, (r + 1) * row_bytes);
          memcpy(dst + (p - base - a), reinterpret_cast<const char*>(rows[r]) + in, e - p);
          p = e;
        }
      });
    });
    if (st) return st;
    CK(km->d_seglen.alloc((size_t)ns));
    CK(km->d_segoff.alloc((size_t)ns + 1));
    SegGeom g{s0, ns, spr, nk, e0};
    const int warps_per_block = 8;
    const int grid = grid_for(ctx, (ns + warps_per_block - 1) / warps_per_block, 16);
    ctx->stats.kernel_launches += 3;
    kmer_tsv_len_kernel<<<grid, 32 * warps_per_block, 0, ctx->st>>>(km->d_cnt.p, g, km->d_seglen.p);
    CK(cudaGetLastError());
    kmer_scan_kernel<<<1, 1024, 0, ctx->st>>>(km->d_seglen.p, ns, km->d_segoff.p);
    CK(cudaGetLastError());
    int64_t total = 0;
    CK(cpy(ctx, &total, km->d_segoff.p + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    CK(km->d_text.alloc((size_t)std::max<int64_t>(total, 1)));
    kmer_tsv_write_kernel<<<grid, 32 * warps_per_block, 0, ctx->st>>>(km->d_cnt.p, g, km->d_segoff.p, km->d_text.p);
    CK(cudaGetLastError());
    st = staged_d2h(ctx, sg, chunk, km->d_text.p, (size_t)total,
                    [&](const char* src, size_t a, size_t b) { return sink(src, b - a, user) == 0; });
    if (st) return st;
  }
  CK(cudaStreamSynchronize(ctx->st));
  trim_kmer_state(km);
  return SWE_OK;
}

}  // extern "C"
