// Adaptive-eps sweep (the reference's adaptive_dbscan, dbscan.c:1117-1380),
// run in eps order over any DBSCAN provider.
//
// Output lines, their order and the float arithmetic follow the reference:
//   * eps_start is halved (float) while the first result has one cluster, at
//     most 20 times (dbscan.c:1211-1231);
//   * the sweep uses eps_{k+1} = eps_k + inc accumulated in float, starting
//     from eps_start + inc (dbscan.c:1077-1080, 1267);
//   * the sweep stops at the first one-cluster result (dbscan.c:1105-1111);
//   * a layer is kept when its cluster count is strictly below the last kept
//     layer's (dbscan.c:1307-1339); the logged eps is one inc above the eps
//     that produced it (dbscan.c:1323-1324);
//   * layer relations sort clusters in place (cluster_io.c:467-469) before
//     the split sets are stored as <prefix>%04d (dbscan.c:1346-1354).
// The reference ends the process with _exit(1) on a failed start search; here
// the same message is printed and SWE_ERR_SWEEP is returned.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "host_internal.h"

namespace swgpu {

float layer_eps(float eps_start, int i, float eps_inc) {
  // The reference build contracts this multiply-add into one fused
  // multiply-add (gcc -O2 on an FMA-capable x86-64), so the value is rounded once.
  return std::fmaf((float)(i + 1), eps_inc, eps_start);
}

static int not_covered_count(const split_set& s, int n) {
  std::vector<uint8_t> seen(n > 0 ? n : 1, 0);
  for (int c = 0; c < s.n_clusters; ++c)
    for (int k = 0; k < s.clusters[c].n_members; ++k) {
      const int m = s.clusters[c].members[k];
      if (m >= 0 && m < n) seen[m] = 1;
    }
  int cnt = 0;
  for (int i = 0; i < n; ++i) cnt += !seen[i];
  return cnt;
}

static float coverage(int not_covered, int n) { return 1.f - (float)not_covered / (float)n; }

split_set copy_split_set(const split_set& s) {
  split_set c;
  c.n_clusters = s.n_clusters;
  c.clusters = (cluster*)malloc(sizeof(cluster) * (size_t)(s.n_clusters > 0 ? s.n_clusters : 1));
  for (int i = 0; i < s.n_clusters; ++i) {
    c.clusters[i] = s.clusters[i];
    const size_t k = (size_t)(s.clusters[i].n_members > 0 ? s.clusters[i].n_members : 1);
    c.clusters[i].members = (int*)malloc(sizeof(int) * k);
    if (s.clusters[i].n_members > 0)
      memcpy(c.clusters[i].members, s.clusters[i].members, sizeof(int) * (size_t)s.clusters[i].n_members);
  }
  return c;
}

int adaptive_sweep(int n, float eps_start, float eps_inc, int minpts, const char* prefix, FILE* log,
                   const DbscanProvider& prov, bool dbscan_sw_warnings, long long fixed_point,
                   std::vector<split_set>* kept, std::string* err) {
  std::vector<split_set> sets;
  auto cleanup = [&]() {
    for (auto& s : sets) free_split_set_and_associated_clusters(s);
    sets.clear();
  };
  // dbscan.c:980-989, printed when the reference's dbscanner would run
  auto warn = [&](float eps) {
    if (!dbscan_sw_warnings) return;
    if (eps == -1) {
      fprintf(log, "Warning @dbscan: epsilon value is: %f\n", eps);
      fprintf(log, "Warning @dbscan: epsilon was changed to: %f\n", 0.015f);
    }
    if (minpts == -1) {
      fprintf(log, "Warning @dbscan: minpts value is: %i\n", minpts);
      fprintf(log, "Warning @dbscan: minpts was changed to: %i\n", 5);
    }
  };
  auto fn = [&](float eps, split_set* o) {
    warn(eps);
    return prov.run(&eps, 1, o);
  };
  fprintf(log,
          "Performing adaptive clustering with parameters: \n"
          "minpts: %i\n"
          "epsilon_start: %f\n"
          "epsilon_inc: %f\n",
          minpts, eps_start, eps_inc);
  split_set first;
  int rc = fn(eps_start, &first);
  if (rc) {
    *err = "dbscan failed";
    return rc;
  }
  fprintf(log, "Initial set obtained with %i clusters\n", first.n_clusters);
  int counter = 0;
  while (first.n_clusters == 1) {
    if (counter == 20 || eps_start == 0) {
      fprintf(log, "Error did not find a sufficient starting position in 20 tries \n");
      free_split_set_and_associated_clusters(first);
      *err = "no starting eps with more than one cluster";
      return SWE_ERR_SWEEP;
    }
    eps_start = eps_start / 2;
    fprintf(log, "Trying new starting point \n");
    free_split_set_and_associated_clusters(first);
    rc = fn(eps_start, &first);
    if (rc) {
      *err = "dbscan failed";
      return rc;
    }
    counter++;
  }
  fprintf(log, "Sarting with %i clusters\n", first.n_clusters);
  fprintf(log, "Coverage at initial point: %f\n", coverage(not_covered_count(first, n), n));
  sets.push_back(first);

  float eps_now = eps_start + eps_inc;
  int stop = -1;
  const int batch = prov.batch > 0 ? prov.batch : 1;
  while (stop < 0) {
    // the next eps values of the sweep, evaluated together; a value past the
    // largest distance (every later eps gives the same result) or an increment
    // too small to move eps ends the batch, since the reference would loop
    // forever after it
    std::vector<float> eps;
    bool terminal = false;
    while ((int)eps.size() < batch) {
      const float e = eps_now;
      eps_now = eps_now + eps_inc;
      eps.push_back(e);
      if ((fixed_point >= 0 && eps_threshold(e) >= fixed_point) || !(eps_now > e)) {
        terminal = true;
        break;
      }
    }
    std::vector<split_set> res(eps.size());
    rc = prov.run(eps.data(), (int)eps.size(), res.data());
    if (rc) {
      cleanup();
      *err = "dbscan failed";
      return rc;
    }
    size_t k = 0;
    for (; k < eps.size(); ++k) {
      warn(eps[k]);
      sets.push_back(res[k]);
      if (res[k].n_clusters == 1) {
        stop = (int)sets.size() - 1;
        break;
      }
    }
    for (size_t j = k + 1; j < eps.size(); ++j) free_split_set_and_associated_clusters(res[j]);
    if (stop < 0 && terminal) {
      cleanup();
      *err = "the sweep can never reach one cluster";
      return SWE_ERR_SWEEP;
    }
  }

  std::vector<split_set> keep;
  std::vector<cluster_connections*> conns;
  keep.push_back(sets[0]);
  for (int i = 1; i <= stop; ++i) {
    split_set ns = sets[i];
    if (ns.n_clusters < keep.back().n_clusters) {
      const int count = (int)keep.size();
      fprintf(log, "Layer %i has %i clusters\n", count, ns.n_clusters);
      fprintf(log, "  Coverage at layer %i: %f\n", count, coverage(not_covered_count(ns, n), n));
      fprintf(log, "  Epsilon at layer %i: %f\n", count, layer_eps(eps_start, i, eps_inc));
      conns.push_back(generate_split_set_relation(keep.back(), ns));
      keep.push_back(ns);
    } else {
      free_split_set_and_associated_clusters(ns);
    }
  }
  sets.clear();
  fprintf(log, "Connections found: \n");
  if (prefix) {
    for (size_t i = 0; i < keep.size(); ++i) {
      std::string name = std::string(prefix);
      char buf[32];
      snprintf(buf, sizeof buf, "%04d", (int)i);
      name += buf;
      store_split_set(const_cast<char*>(name.c_str()), keep[i]);
    }
  }
  for (int i = (int)keep.size() - 1; i > 0; --i) {
    fprintf(log, "Layer %i:\n", i);
    for (int j = 0; j < keep[i].n_clusters; ++j) {
      fprintf(log, "  Cluster %i connected to: \n  ", j);
      for (int k = 0; k < conns[i - 1][j].n_connections; ++k) fprintf(log, "%i ", conns[i - 1][j].connections[k]);
      fprintf(log, "\n");
    }
  }
  for (int i = (int)keep.size() - 1; i > 0; --i) {
    for (int j = 0; j < keep[i].n_clusters; ++j) free(conns[i - 1][j].connections);
    free(conns[i - 1]);
  }
  *kept = std::move(keep);
  return 0;
}

}  // namespace swgpu
