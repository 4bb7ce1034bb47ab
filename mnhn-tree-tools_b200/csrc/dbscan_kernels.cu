// Order-faithful DBSCAN replays on the device: many independent instances
// (one per split set and eps threshold) in one launch, one warp each.
//
// Each instance replays the reference's sequential traversal (dbscan_SW,
// dbscan.c:950-1047, with expand_cluster, dbscan.c:783-948) on the eps-neighbour
// bitmap rows the threshold pass left in device memory, with the host replay's
// rules (csrc/dbscan_replay.cpp):
//   * seeds in index order; a seed opens a cluster only if minpts < |N(seed)|;
//   * the frontier starts as N(seed) in ascending order; a frontier point seen
//     unvisited is marked visited and, when |N(q)| >= minpts, appends the
//     members of N(q) never queued in this cluster, in ascending order;
//   * a frontier point joins the cluster unless an earlier cluster holds it.
// The warp takes 32 consecutive seeds at a time (the first core seed among the
// unvisited ones opens the next cluster; the unvisited ones before it are
// marked visited) and 32 consecutive frontier points at a time: their
// visited / in-cluster tests touch only their own bits (a frontier holds each
// point once), so they run in parallel, members are appended in lane order,
// and the expansions run in lane order, each scanning its bitmap row with the
// 32 lanes (lane l owns words l, l+32, ... of the queued bitmap) and appending
// the fresh bits with a warp prefix sum, so the frontier stays in the order
// the sequential traversal builds.
//
// Output per instance: members in cluster order (cluster c holds
// members[cstart[c] .. cstart[c+1])), cstart, the cluster count.  No wait or
// spin anywhere; a frontier that would outgrow its set (impossible for
// well-formed bitmaps) raises KST_REPLAY_OVERFLOW and ends the instance.
#include "dbscan_kernels.cuh"
#include "sw_device.cuh"

namespace swgpu {

namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr int RP_WARPS = 4;  // warps (instances) per CTA

// Appends the set bits of `word` (bitmap word w of a row, lane order = word
// order) to F at *fsz, ascending.  Returns false when the frontier would
// outgrow ns or a bit lies beyond it.
__device__ __forceinline__ bool append_bits(int* __restrict__ F, int& fsz, uint64_t word, int w, int ns, int lane) {
  if (!__ballot_sync(FULL, word != 0)) return true;
  const int cnt = __popcll(word);
  int x = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  const int total = __shfl_sync(FULL, x, 31);
  const bool ok = fsz + total <= ns && (word == 0 || (long long)w * 64 + 63 - __clzll(word) < ns);
  if (!__all_sync(FULL, ok)) return false;
  int at = fsz + x - cnt;
  while (word) {
    F[at++] = w * 64 + __ffsll((long long)word) - 1;
    word &= word - 1;
  }
  fsz += total;
  return true;
}

}  // namespace

__global__ void __launch_bounds__(RP_WARPS * 32) dbscan_replay_kernel(
    const ReplayJob* __restrict__ jobs, int njobs, const uint64_t* __restrict__ bits, const int* __restrict__ counts,
    int minpts, int* __restrict__ members, int* __restrict__ frontier, int* __restrict__ cstart,
    int* __restrict__ ncl, uint32_t* __restrict__ g_vis, uint64_t* __restrict__ g_queued, unsigned* status) {
  extern __shared__ uint8_t rp_smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int j = blockIdx.x * RP_WARPS + wib;
  if (j >= njobs) return;
  const ReplayJob jb = jobs[j];
  const int ns = jb.ns, wpr = (ns + 63) >> 6, vw = (ns + 31) >> 5;
  const uint64_t* __restrict__ B = bits + jb.bits;
  const int* __restrict__ C = counts + jb.counts;
  int* __restrict__ M = members + jb.counts;
  int* __restrict__ F = frontier + jb.counts;
  int* __restrict__ CS = cstart + jb.cstart;
  // visited and in-cluster bits, queued words: this warp's shared-memory slice
  // for sets up to RP_SMEM_NS points, else the instance's global scratch.
  // Visited / in-cluster bits are only touched by atomics (coherent in both
  // spaces); each queued word only by its owning lane.
  uint32_t* V;
  uint64_t* Q;
  if (ns <= RP_SMEM_NS) {
    uint8_t* base = rp_smem + (size_t)wib * RP_SMEM_PER_WARP;
    Q = reinterpret_cast<uint64_t*>(base);
    V = reinterpret_cast<uint32_t*>(base + (RP_SMEM_NS / 64) * 8);
  } else {
    Q = g_queued + jb.q;
    V = g_vis + jb.vis;
  }
  uint32_t* IC = V + vw;
  for (int w = lane; w < 2 * vw; w += 32) atomicExch(&V[w], 0u);
  __syncwarp();
  const unsigned lt = (1u << lane) - 1u;
  int nmem = 0, ncls = 0;
  bool ok = true;
  for (int base = 0; base < ns && ok; base += 32) {
    const int i = base + lane;
    const int ci = i < ns ? C[i] : 0;
    int start = 0;
    while (start < 32 && ok) {
      const uint32_t vword = atomicOr(&V[base >> 5], 0u);
      const bool unv = i < ns && lane >= start && !((vword >> lane) & 1u);
      const unsigned umask = __ballot_sync(FULL, unv);
      const unsigned cmask = __ballot_sync(FULL, unv && minpts < ci);
      if (!cmask) {
        if (lane == 0 && umask) atomicOr(&V[base >> 5], umask);
        __syncwarp();
        break;
      }
      const int c = __ffs((int)cmask) - 1;
      if (lane == 0) atomicOr(&V[base >> 5], umask & ((2u << c) - 1u));  // up to and including the seed
      const int s = base + c;
      // the cluster of seed s: the seed first, then its frontier's members
      const int cl0 = nmem;
      if (lane == 0) {
        M[nmem] = s;
        atomicOr(&IC[s >> 5], 1u << (s & 31));
        CS[ncls] = cl0;
      }
      nmem += 1;
      ++ncls;
      int fsz = 0;
      const uint64_t* __restrict__ R = B + (long long)s * wpr;
      for (int w0 = 0; w0 < wpr && ok; w0 += 32) {
        const int w = w0 + lane;
        const uint64_t word = w < wpr ? R[w] : 0ull;
        if (w < wpr) Q[w] = word;
        ok = append_bits(F, fsz, word, w, ns, lane);
      }
      __syncwarp();
      for (int f = 0; f < fsz && ok;) {
        // the next (up to) 32 frontier points; points appended while they are
        // processed come after them
        const int k = min(32, fsz - f);
        const int q = lane < k ? F[f + lane] : -1;
        bool exp = false, inc = false;
        if (q >= 0) {
          const uint32_t bit = 1u << (q & 31);
          const bool newly = !(atomicOr(&V[q >> 5], bit) & bit);
          exp = newly && C[q] >= minpts;
          inc = !(atomicOr(&IC[q >> 5], bit) & bit);
        }
        const unsigned im = __ballot_sync(FULL, inc);
        if (inc) M[nmem + __popc(im & lt)] = q;
        nmem += __popc(im);
        unsigned em = __ballot_sync(FULL, exp);
        while (em && ok) {
          const int jl = __ffs((int)em) - 1;
          em &= em - 1;
          const int qq = __shfl_sync(FULL, q, jl);
          const uint64_t* __restrict__ RQ = B + (long long)qq * wpr;
          // row words in groups of four chunks, loads first
          for (int w0 = 0; w0 < wpr && ok; w0 += 128) {
            uint64_t rw[4];
#pragma unroll
            for (int g = 0; g < 4; ++g) {
              const int w = w0 + 32 * g + lane;
              rw[g] = w < wpr ? RQ[w] : 0ull;
            }
#pragma unroll
            for (int g = 0; g < 4; ++g) {
              const int w = w0 + 32 * g + lane;
              if (w0 + 32 * g >= wpr) break;
              uint64_t fresh = 0;
              if (w < wpr) {
                const uint64_t qw = Q[w];
                fresh = rw[g] & ~qw;
                if (fresh) Q[w] = qw | fresh;
              }
              ok = ok && append_bits(F, fsz, fresh, w, ns, lane);
            }
          }
        }
        __syncwarp();
        f += k;
      }
      start = c + 1;
    }
  }
  if (!ok) {
    if (lane == 0) atomicOr(status, KST_REPLAY_OVERFLOW);
    ncls = 0;
    nmem = 0;
  }
  if (lane == 0) {
    CS[ncls] = nmem;
    ncl[j] = ncls;
  }
}

cudaError_t launch_dbscan_replay(const ReplayJob* jobs, int njobs, const uint64_t* bits, const int* counts,
                                 int minpts, int* members, int* frontier, int* cstart, int* ncl, uint32_t* g_vis,
                                 uint64_t* g_queued, unsigned* status, cudaStream_t st) {
  if (njobs <= 0) return cudaSuccess;
  const size_t smem = (size_t)RP_WARPS * RP_SMEM_PER_WARP;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(dbscan_replay_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int grid = (njobs + RP_WARPS - 1) / RP_WARPS;
  dbscan_replay_kernel<<<grid, RP_WARPS * 32, smem, st>>>(jobs, njobs, bits, counts, minpts, members, frontier,
                                                         cstart, ncl, g_vis, g_queued, status);
  return cudaGetLastError();
}

}  // namespace swgpu
