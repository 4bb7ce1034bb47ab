// Split-set files, cluster FASTA files and layer relations with the
// reference's byte formats and side effects (cluster_io.c:407-501, 564-729).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "host_internal.h"

extern "C" {

void free_split_set_and_associated_clusters(split_set s) {
  for (int i = 0; i < s.n_clusters; ++i) free(s.clusters[i].members);
  free(s.clusters);
}

// cluster_io.c:638-669.  Opened with O_WRONLY|O_CREAT and no O_TRUNC, as in
// the reference: an existing longer file keeps its tail.
void store_split_set(char* filename, split_set s) {
  static const char tag[] = "SPLIT_SET";
  const int fd = open(filename, O_WRONLY | O_CREAT, S_IRUSR | S_IWUSR | S_IRGRP | S_IROTH);
  size_t check = 0, count = 0;
  auto put = [&](const void* p, size_t k) {
    if (fd >= 0) {
      const ssize_t w = write(fd, p, k);
      if (w > 0) check += (size_t)w;
    }
    count += k;
  };
  std::vector<char> buf;
  put(tag, 9);
  put(&s.n_clusters, sizeof(int));
  for (int i = 0; i < s.n_clusters; ++i) {
    put(&s.clusters[i].n_members, sizeof(int));
    put(&s.clusters[i].id, sizeof(int));
    if (s.clusters[i].n_members > 0) put(s.clusters[i].members, sizeof(int) * (size_t)s.clusters[i].n_members);
  }
  if (check != count) printf("There was an error in creating the binary clusterfile %s", filename);
  if (fd >= 0) close(fd);
}

// cluster_io.c:595-636.  Where the reference exits on a file that is not a
// split set, this prints the same message and returns an empty set.
split_set read_split_set(char* filename) {
  split_set s{0, nullptr};
  const int fd = open(filename, O_RDONLY);
  char buffer[10] = {0};
  if (fd < 0 || read(fd, buffer, 9) != 9 || strcmp(buffer, "SPLIT_SET") != 0) {
    printf("Error %s is not a split_set\n", filename);
    if (fd >= 0) close(fd);
    return s;
  }
  size_t check = 9, count = 9;
  auto get = [&](void* p, size_t k) {
    const ssize_t r = read(fd, p, k);
    if (r > 0) check += (size_t)r;
    count += k;
    return r == (ssize_t)k;
  };
  int nc = 0;
  if (!get(&nc, sizeof(int)) || nc < 0) nc = 0;
  s.clusters = (cluster*)malloc(sizeof(cluster) * (size_t)(nc > 0 ? nc : 1));
  s.n_clusters = nc;
  for (int i = 0; i < nc; ++i) {
    int nm = 0, id = 0;
    get(&nm, sizeof(int));
    get(&id, sizeof(int));
    if (nm < 0) nm = 0;
    s.clusters[i].n_members = nm;
    s.clusters[i].id = id;
    s.clusters[i].members = (int*)malloc(sizeof(int) * (size_t)(nm > 0 ? nm : 1));
    if (nm > 0) get(s.clusters[i].members, sizeof(int) * (size_t)nm);
  }
  if (check != count) printf("There was an error reading the binary clusterfile %s", filename);
  close(fd);
  return s;
}

// cluster_io.c:672-699: ">sequence_<idx>" headers and 50 characters per line.
// (The reference's loop bound strlen-1 underflows for an empty sequence; an
// empty sequence is written as an empty line here.)
void create_single_cluster_file(char* filename, cluster cl, dataset ds) {
  FILE* f = fopen(filename, "w");
  if (!f) return;
  for (int j = 0; j < cl.n_members; ++j) {
    const int m = cl.members[j];
    fprintf(f, ">sequence_%i\n", m);
    const char* s = ds.sequences[m];
    const size_t L = strlen(s);
    for (size_t k = 0; k < L; ++k) {
      if (k != 0 && k % 50 == 0) fputc('\n', f);
      fputc(s[k], f);
    }
    fputc('\n', f);
  }
  fclose(f);
}

// cluster_io.c:701-720: files <prefix>-%03d.
void create_cluster_files(char* prefix, split_set s, dataset ds) {
  for (int i = 0; i < s.n_clusters; ++i) {
    char idx[32];
    snprintf(idx, sizeof idx, "%03d", i);
    std::string name = std::string(prefix) + "-" + idx;
    create_single_cluster_file(const_cast<char*>(name.c_str()), s.clusters[i], ds);
  }
}

// cluster_io.c:564-593.
cluster data_not_in_clusters(split_set s, dataset ds) {
  cluster out;
  const int n = ds.n_values;
  std::vector<uint8_t> seen(n > 0 ? n : 1, 0);
  for (int i = 0; i < s.n_clusters; ++i)
    for (int j = 0; j < s.clusters[i].n_members; ++j) {
      const int m = s.clusters[i].members[j];
      if (m >= 0 && m < n) seen[m] = 1;
    }
  int count = 0;
  for (int i = 0; i < n; ++i) count += !seen[i];
  out.id = -1;
  out.n_members = count;
  out.members = count > 0 ? (int*)malloc(sizeof(int) * (size_t)count) : nullptr;
  int k = 0;
  for (int i = 0; i < n && out.members; ++i)
    if (!seen[i]) out.members[k++] = i;
  return out;
}

static int cmp_int(const void* a, const void* b) {
  const int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

// cluster_io.c:446-501.  The larger cluster (a on ties) is sorted in place
// when it has more than 20 members; the sort is visible to the caller.
cluster intersection_of_clusters(cluster a, cluster b) {
  const cluster big = (a.n_members >= b.n_members) ? a : b;
  const cluster small = (a.n_members >= b.n_members) ? b : a;
  cluster out;
  out.id = -1;
  std::vector<int> hit;
  if (big.n_members > 20) {
    qsort(big.members, (size_t)big.n_members, sizeof(int), cmp_int);
    for (int i = 0; i < small.n_members; ++i) {
      const int t = small.members[i];
      int lo = 0, hi = big.n_members - 1;
      while (lo <= hi) {
        const int mid = (lo + hi) / 2;
        if (big.members[mid] < t) lo = mid + 1;
        else if (big.members[mid] > t) hi = mid - 1;
        else {
          hit.push_back(t);
          break;
        }
      }
    }
  } else {
    for (int i = 0; i < small.n_members; ++i)
      for (int j = 0; j < big.n_members; ++j)
        if (small.members[i] == big.members[j]) hit.push_back(small.members[i]);
  }
  out.n_members = (int)hit.size();
  out.members = hit.empty() ? nullptr : (int*)malloc(sizeof(int) * hit.size());
  if (out.members) memcpy(out.members, hit.data(), sizeof(int) * hit.size());
  return out;
}

// True when no index appears twice in the set (no duplicate inside a cluster,
// no overlap between clusters) and all indices are >= 0; *max_id receives the
// largest index.
static bool partition_like(const split_set& s, std::vector<uint8_t>& seen, int* max_id) {
  for (int c = 0; c < s.n_clusters; ++c)
    for (int k = 0; k < s.clusters[c].n_members; ++k) {
      const int m = s.clusters[c].members[k];
      if (m < 0) return false;
      if ((size_t)m >= seen.size()) seen.resize((size_t)m + 1 + seen.size() / 2, 0);
      if (seen[m]) return false;
      seen[m] = 1;
      if (m > *max_id) *max_id = m;
    }
  return true;
}

// cluster_io.c:407-444.  The reference calls intersection_of_clusters for
// every (new, ancient) pair, which sorts the larger cluster of the pair in
// place when it has more than 20 members (cluster_io.c:467-469).  For split
// sets that are partitions (every DBSCAN result is) the same connections and
// the same sorted clusters come from one pass over the members: ancient
// cluster j ends up sorted iff some new cluster is no larger than it, new
// cluster i iff some ancient cluster is smaller.  Other inputs use the
// pairwise computation.
cluster_connections* generate_split_set_relation(split_set ancient, split_set new_set) {
  cluster_connections* c =
      (cluster_connections*)malloc(sizeof(cluster_connections) * (size_t)(new_set.n_clusters > 0 ? new_set.n_clusters : 1));
  int max_id = -1;
  std::vector<uint8_t> seen_a, seen_n;
  if (ancient.n_clusters > 0 && new_set.n_clusters > 0 && partition_like(ancient, seen_a, &max_id) &&
      partition_like(new_set, seen_n, &max_id)) {
    std::vector<int> anc_of((size_t)max_id + 1, -1);
    int min_a = INT_MAX, min_n = INT_MAX;
    for (int j = 0; j < ancient.n_clusters; ++j) {
      min_a = std::min(min_a, ancient.clusters[j].n_members);
      for (int k = 0; k < ancient.clusters[j].n_members; ++k) anc_of[ancient.clusters[j].members[k]] = j;
    }
    for (int i = 0; i < new_set.n_clusters; ++i) min_n = std::min(min_n, new_set.clusters[i].n_members);
    std::vector<int> cnt(ancient.n_clusters, 0), touched;
    for (int i = 0; i < new_set.n_clusters; ++i) {
      touched.clear();
      for (int k = 0; k < new_set.clusters[i].n_members; ++k) {
        const int j = anc_of[new_set.clusters[i].members[k]];
        if (j < 0) continue;
        if (cnt[j]++ == 0) touched.push_back(j);
      }
      std::sort(touched.begin(), touched.end());
      std::vector<int> conn;
      for (int j : touched) {
        if ((double)cnt[j] > (double)ancient.clusters[j].n_members * (double)0.8) conn.push_back(j);
        cnt[j] = 0;
      }
      c[i].n_connections = (int)conn.size();
      c[i].connections = conn.empty() ? nullptr : (int*)malloc(sizeof(int) * conn.size());
      if (c[i].connections) memcpy(c[i].connections, conn.data(), sizeof(int) * conn.size());
    }
    for (int j = 0; j < ancient.n_clusters; ++j)
      if (ancient.clusters[j].n_members > 20 && ancient.clusters[j].n_members >= min_n)
        qsort(ancient.clusters[j].members, (size_t)ancient.clusters[j].n_members, sizeof(int), cmp_int);
    for (int i = 0; i < new_set.n_clusters; ++i)
      if (new_set.clusters[i].n_members > 20 && new_set.clusters[i].n_members > min_a)
        qsort(new_set.clusters[i].members, (size_t)new_set.clusters[i].n_members, sizeof(int), cmp_int);
    return c;
  }
  for (int i = 0; i < new_set.n_clusters; ++i) {
    std::vector<int> conn;
    for (int j = 0; j < ancient.n_clusters; ++j) {
      cluster inter = intersection_of_clusters(ancient.clusters[j], new_set.clusters[i]);
      if ((double)inter.n_members > (double)ancient.clusters[j].n_members * (double)0.8) conn.push_back(j);
      free(inter.members);
    }
    c[i].n_connections = (int)conn.size();
    c[i].connections = conn.empty() ? nullptr : (int*)malloc(sizeof(int) * conn.size());
    if (c[i].connections) memcpy(c[i].connections, conn.data(), sizeof(int) * conn.size());
  }
  return c;
}

}  // extern "C"
