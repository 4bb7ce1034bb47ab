// Order-faithful DBSCAN replay over eps-neighbour bitmaps.
//
// The reference's dbscan_SW (dbscan.c:950-1047) is sequential and
// order-dependent, so its labels are reproduced by replaying its traversal on
// neighbourhoods the GPU produced:
//   * seeds in index order; a seed opens a cluster only if minpts < |N(seed)|
//     (strict, dbscan.c:1011);
//   * expand_cluster (dbscan.c:783-948) walks a frontier that starts as N(seed)
//     in ascending order; a frontier point visited for the first time is
//     expanded when |N(q)| >= minpts (dbscan.c:847), appending the members of
//     N(q) that were never queued in this cluster, in ascending order
//     (dbscan.c:894-920);
//   * points visited earlier (as seeds or in earlier clusters) are never
//     queried again (dbscan.c:835-838);
//   * a frontier point joins the cluster unless an earlier cluster holds it
//     (dbscan.c:934-940); cluster ids are the seed order.
// The "already queued" set is a bitmap, so appending the new members of N(q)
// costs one and-not over the row's words.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "host_internal.h"

namespace swgpu {

int dbscan_replay_bitmap(int n, const uint64_t* bits, int wpr, const int* counts, int minpts,
                         split_set* out) {
  out->n_clusters = 0;
  out->clusters = nullptr;
  std::vector<uint8_t> visited(n > 0 ? n : 1, 0), in_cluster(n > 0 ? n : 1, 0);
  std::vector<uint64_t> queued(wpr > 0 ? wpr : 1, 0);
  std::vector<int> frontier;
  frontier.reserve(n > 0 ? n : 1);
  std::vector<int> members;
  std::vector<cluster> clusters;
  auto fail = [&]() {
    for (auto& c : clusters) free(c.members);
    return (int)SWE_ERR_OOM;
  };
  for (int i = 0; i < n; ++i) {
    if (visited[i]) continue;
    visited[i] = 1;
    if (!(minpts < counts[i])) continue;
    frontier.clear();
    members.clear();
    const uint64_t* row = bits + (size_t)i * (size_t)wpr;
    for (int w = 0; w < wpr; ++w) {
      uint64_t word = row[w];
      queued[w] = word;
      while (word) {
        frontier.push_back(w * 64 + __builtin_ctzll(word));
        word &= word - 1;
      }
    }
    members.push_back(i);
    in_cluster[i] = 1;
    for (size_t f = 0; f < frontier.size(); ++f) {
      const int q = frontier[f];
      if (!visited[q]) {
        visited[q] = 1;
        if (counts[q] >= minpts) {
          const uint64_t* rq = bits + (size_t)q * (size_t)wpr;
          // blocks of 8 words: most rows add nothing new once the cluster's
          // core is queued, so a branch-free test of the block comes first
          for (int w0 = 0; w0 < wpr; w0 += 8) {
            const int w1 = w0 + 8 < wpr ? w0 + 8 : wpr;
            uint64_t any = 0;
            for (int w = w0; w < w1; ++w) any |= rq[w] & ~queued[w];
            if (!any) continue;
            for (int w = w0; w < w1; ++w) {
              uint64_t fresh = rq[w] & ~queued[w];
              if (!fresh) continue;
              queued[w] |= fresh;
              while (fresh) {
                frontier.push_back(w * 64 + __builtin_ctzll(fresh));
                fresh &= fresh - 1;
              }
            }
          }
        }
      }
      if (!in_cluster[q]) {
        members.push_back(q);
        in_cluster[q] = 1;
      }
    }
    cluster c;
    c.n_members = (int)members.size();
    c.id = (int)clusters.size();
    c.members = (int*)malloc(sizeof(int) * members.size());
    if (!c.members) return fail();
    memcpy(c.members, members.data(), sizeof(int) * members.size());
    clusters.push_back(c);
  }
  out->clusters = (cluster*)malloc(sizeof(cluster) * (clusters.empty() ? 1 : clusters.size()));
  if (!out->clusters) return fail();
  if (!clusters.empty()) memcpy(out->clusters, clusters.data(), sizeof(cluster) * clusters.size());
  out->n_clusters = (int)clusters.size();
  return 0;
}

}  // namespace swgpu

extern "C" swe_status swe_dbscan_bitmap(int n, const uint64_t* bits, int words_per_row, const int* counts,
                                        int minpts, split_set* out) {
  if (!out || n < 0 || (n > 0 && (!bits || !counts || words_per_row < (n + 63) / 64))) return SWE_ERR_INVALID;
  if (minpts == -1) minpts = 5;  // dbscan.c:985-989
  return (swe_status)swgpu::dbscan_replay_bitmap(n, bits, words_per_row, counts, minpts, out);
}
