// Device DBSCAN replays (dbscan_kernels.cu): many order-faithful instances in
// one launch, one warp each.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace swgpu {

// One instance: the eps-neighbour bitmap rows of one set at one threshold.
struct ReplayJob {
  long long bits;    // word offset of its ns x ceil(ns/64) bitmap rows
  long long counts;  // int offset of its neighbour counts; also of its members and frontier (ns each)
  long long cstart;  // int offset of its cluster starts (ns + 1 slots)
  long long vis;     // uint32 word offset of its visited + in-cluster bits in global scratch (sets above RP_SMEM_NS)
  long long q;       // uint64 word offset of its queued words in global scratch (sets above RP_SMEM_NS)
  int ns;            // points of the set
  int pad;
};

// Sets up to this many points keep their traversal state in shared memory.
constexpr int RP_SMEM_NS = 16384;
constexpr int RP_SMEM_PER_WARP = (RP_SMEM_NS / 64) * 8 + 2 * (RP_SMEM_NS / 32) * 4;

// minpts as the reference takes it (-1 already replaced by its default).
// members / frontier: sum of ns ints; cstart: sum of (ns + 1); ncl: one per job.
cudaError_t launch_dbscan_replay(const ReplayJob* jobs, int njobs, const uint64_t* bits, const int* counts,
                                 int minpts, int* members, int* frontier, int* cstart, int* ncl, uint32_t* g_vis,
                                 uint64_t* g_queued, unsigned* status, cudaStream_t st);

}  // namespace swgpu
