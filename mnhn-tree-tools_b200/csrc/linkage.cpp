// Capped single linkage of the prefiltered layout (host code).
//
// The candidate pairs of a prefiltered pass arrive sorted by how close their
// embeddings are; joining them in that order, and refusing any join that
// would make a group larger than `cap`, gathers each family's reads into a
// few consecutive packs and column blocks.  The groups depend only on the
// order of the pairs: a join happens when the two reads are in different
// groups whose sizes add up to at most `cap`.
//
// Every read keeps the label of its group's current representative, so the
// test of a pair is two independent loads instead of two pointer chases.  A
// join relabels the smaller group (ties: the second pair member's) through
// its member list, so a read is relabelled at most log2(cap) times.  The
// reported label of a group is its smallest read index.
//
// Joins are rare (at most n - 1 of millions of pairs), and a pair that
// cannot join at some point never can later: groups only grow, so reads in
// one group stay together and a size sum above the cap stays above it.  The
// pairs therefore go in batches: a branch-free pass tests every pair of the
// batch against the groups as they are at the batch's start, and only the
// pairs it lets through are tested again, in order, as the joins happen.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "host_internal.h"
#include "swgpu.h"

namespace swgpu {

void capped_linkage(int n, const int* pairs, int64_t count, int cap, int* label) {
  if (n <= 0) return;
  std::vector<int> rep(n), next(n, -1), tail(n), size(n, 1), low(n);
  for (int i = 0; i < n; ++i) rep[i] = tail[i] = low[i] = i;
  constexpr int64_t kBatch = 4096;
  uint8_t live[kBatch];
  for (int64_t c0 = 0; c0 < count; c0 += kBatch) {
    const int64_t nb = std::min(kBatch, count - c0);
    const int* pb = pairs + 2 * c0;
    for (int64_t c = 0; c < nb; ++c) {  // against the groups at the batch's start
      const int a = pb[2 * c], b = pb[2 * c + 1];
      const bool valid = (unsigned)a < (unsigned)n && (unsigned)b < (unsigned)n;
      const int ra = rep[valid ? a : 0], rb = rep[valid ? b : 0];
      live[c] = (uint8_t)(valid & (ra != rb) & (size[ra] + size[rb] <= cap));
    }
    for (int64_t c = 0; c < nb; ++c) {
      if (!live[c]) continue;
      int ra = rep[pb[2 * c]], rb = rep[pb[2 * c + 1]];
      if (ra == rb || size[ra] + size[rb] > cap) continue;
      if (size[ra] < size[rb]) std::swap(ra, rb);  // rb, the smaller group, joins ra
      for (int m = rb; m >= 0; m = next[m]) rep[m] = ra;
      next[tail[ra]] = rb;  // a group's list starts at its representative
      tail[ra] = tail[rb];
      size[ra] += size[rb];
      low[ra] = std::min(low[ra], low[rb]);
    }
  }
  for (int i = 0; i < n; ++i) label[i] = low[rep[i]];
}

}  // namespace swgpu

extern "C" void swe_capped_linkage(int n, const int* pairs, int64_t count, int cap, int* label) {
  if (!label || n <= 0 || count < 0 || (count > 0 && !pairs)) return;
  swgpu::capped_linkage(n, pairs, count, cap, label);
}
