// Reference-named entry points (mnhn_dropin.h) on top of the engine.
//
// One process-wide context (device $SWGPU_DEVICE, default 0) serves the
// drop-in calls.  dbscan_SW scores all pairs of a dataset once and keeps the
// distance matrix while later calls pass the same sequences (same count,
// lengths and bytes), so the reference's adaptive driver calling dbscan_SW
// once per eps re-scores nothing.
#include <climits>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "host_internal.h"

namespace {

std::mutex g_mu;
swe_ctx* g_ctx = nullptr;
int g_status = 0;
bool g_have = false;
uint64_t g_fp = 0;

swe_ctx* default_ctx() {
  if (g_ctx) return g_ctx;
  swe_opts o{};
  const char* dev = getenv("SWGPU_DEVICE");
  o.device = dev ? atoi(dev) : 0;
  const swe_status s = swe_create(&g_ctx, &o);
  if (s != SWE_OK) {
    fprintf(stderr, "swgpu: cannot open the GPU engine: %s\n", swe_strerror(s));
    g_status = s;
    g_ctx = nullptr;
  }
  return g_ctx;
}

uint64_t fingerprint(const dataset& ds) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](const void* p, size_t k) {
    const unsigned char* b = (const unsigned char*)p;
    for (size_t i = 0; i < k; ++i) {
      h ^= b[i];
      h *= 1099511628211ull;
    }
  };
  mix(&ds.n_values, sizeof ds.n_values);
  for (int i = 0; i < ds.n_values; ++i) {
    mix(&ds.sequence_lengths[i], sizeof(size_t));
    mix(ds.sequences[i], ds.sequence_lengths[i] + 1);
  }
  return h;
}

// Uploads and scores `ds` unless the context already holds its distances.
int ensure_scored(swe_ctx* ctx, const dataset& ds) {
  const uint64_t fp = fingerprint(ds);
  if (g_have && fp == g_fp) return SWE_OK;
  g_have = false;
  swe_status s = swe_upload(ctx, ds.sequences, ds.sequence_lengths, ds.n_values);
  if (s == SWE_OK) s = swe_score_all_pairs(ctx);
  if (s != SWE_OK) {
    fprintf(stderr, "swgpu: scoring failed: %s (%s)\n", swe_strerror(s), swe_last_error(ctx));
    return s;
  }
  g_have = true;
  g_fp = fp;
  return SWE_OK;
}

uint64_t fingerprint_points(const dataset& ds, int metric) {
  uint64_t h = 0x9E3779B97F4A7C15ull ^ (uint64_t)metric;
  auto mix = [&](const void* p, size_t k) {
    const unsigned char* b = (const unsigned char*)p;
    for (size_t i = 0; i < k; ++i) {
      h ^= b[i];
      h *= 1099511628211ull;
    }
  };
  mix(&ds.n_values, sizeof ds.n_values);
  mix(&ds.n_dimensions, sizeof ds.n_dimensions);
  for (int d = 0; d < ds.n_dimensions && ds.n_values > 0; ++d) mix(ds.values[d], sizeof(float) * ds.n_values);
  return h;
}

// Uploads the points of `ds` (values[dimension][point]) with their L1 / L2
// distances unless the context already holds them.
int ensure_points(swe_ctx* ctx, const dataset& ds, int metric) {
  const uint64_t fp = fingerprint_points(ds, metric);
  if (g_have && fp == g_fp) return SWE_OK;
  g_have = false;
  const int dims = ds.n_values > 0 ? ds.n_dimensions : 0;
  const swe_status s = swe_upload_points(ctx, ds.values, dims, ds.n_values, metric);
  if (s != SWE_OK) {
    fprintf(stderr, "swgpu: point distances failed: %s (%s)\n", swe_strerror(s), swe_last_error(ctx));
    return s;
  }
  g_have = true;
  g_fp = fp;
  return SWE_OK;
}

// dbscan_L1 / dbscan_L2 body without the lock (dbscan.c:950-1047 with the
// region queries of dbscan.c:563-779).
split_set dbscan_points_locked(const dataset& ds, float epsilon, int minpts, int metric) {
  split_set out{0, nullptr};
  if (epsilon == -1) {  // dbscan.c:980-984
    printf("Warning @dbscan: epsilon value is: %f\n", epsilon);
    epsilon = 0.015f;
    printf("Warning @dbscan: epsilon was changed to: %f\n", epsilon);
  }
  if (minpts == -1) {  // dbscan.c:985-989
    printf("Warning @dbscan: minpts value is: %i\n", minpts);
    minpts = 5;
    printf("Warning @dbscan: minpts was changed to: %i\n", minpts);
  }
  swe_ctx* ctx = default_ctx();
  if (!ctx) return out;
  int s = ensure_points(ctx, ds, metric);
  if (s == SWE_OK) s = swe_dbscan(ctx, epsilon, minpts, &out);
  if (s != SWE_OK) {
    fprintf(stderr, "swgpu: dbscan_L%d failed: %s\n", metric, swe_strerror((swe_status)s));
    g_status = s;
    out.n_clusters = 0;
    out.clusters = nullptr;
  }
  return out;
}

// dbscan_SW body without the lock (also the engine provider of adaptive_dbscan).
split_set dbscan_locked(const dataset& ds, float epsilon, int minpts) {
  split_set out{0, nullptr};
  if (epsilon == -1) {  // dbscan.c:980-984
    printf("Warning @dbscan: epsilon value is: %f\n", epsilon);
    epsilon = 0.015f;
    printf("Warning @dbscan: epsilon was changed to: %f\n", epsilon);
  }
  if (minpts == -1) {  // dbscan.c:985-989
    printf("Warning @dbscan: minpts value is: %i\n", minpts);
    minpts = 5;
    printf("Warning @dbscan: minpts was changed to: %i\n", minpts);
  }
  swe_ctx* ctx = default_ctx();
  if (!ctx) return out;
  int s = ensure_scored(ctx, ds);
  if (s == SWE_OK) s = swe_dbscan(ctx, epsilon, minpts, &out);
  if (s != SWE_OK) {
    fprintf(stderr, "swgpu: dbscan_SW failed: %s\n", swe_strerror((swe_status)s));
    g_status = s;
    out.n_clusters = 0;
    out.clusters = nullptr;
  }
  return out;
}

}  // namespace

namespace swgpu {

std::mutex& dropin_mutex() { return g_mu; }
swe_ctx* dropin_ctx() { return default_ctx(); }
int dropin_scored(swe_ctx* ctx, const dataset& ds) { return ensure_scored(ctx, ds); }
void dropin_forget() { g_have = false; }
void dropin_set_status(int s) { g_status = s; }

}  // namespace swgpu

extern "C" {

int swgpu_last_dropin_status(void) { return g_status; }

unsigned int score(char* A, char* B, size_t len_a, size_t len_b, int* work) {
  (void)work;
  std::lock_guard<std::mutex> lk(g_mu);
  swe_ctx* ctx = default_ctx();
  if (!ctx) return UINT_MAX;
  unsigned d = UINT_MAX;
  const swe_status s = swgpu::score_raw(ctx, A, len_a, B, len_b, &d);
  if (s != SWE_OK) {
    fprintf(stderr, "swgpu: score failed: %s\n", swe_strerror(s));
    g_status = s;
    return UINT_MAX;
  }
  return d;
}

dataset dataset_from_fasta(FILE* in) {
  dataset ds;
  std::string err;
  if (swgpu::fasta_read(in, &ds, &err) != 0) fprintf(stderr, "swgpu: %s\n", err.c_str());
  return ds;
}

void free_sequences_from_dataset(dataset ds) {
  for (int i = 0; i < ds.n_values; ++i) free(ds.sequences[i]);
  free(ds.sequence_lengths);
  free(ds.sequences);
}

split_set dbscan_SW(dataset ds, float epsilon, int minpts) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_status = 0;
  return dbscan_locked(ds, epsilon, minpts);
}

split_set dbscan_L1(dataset ds, float epsilon, int minpts) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_status = 0;
  return dbscan_points_locked(ds, epsilon, minpts, SWE_METRIC_L1);
}

split_set dbscan_L2(dataset ds, float epsilon, int minpts) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_status = 0;
  return dbscan_points_locked(ds, epsilon, minpts, SWE_METRIC_L2);
}

void adaptive_dbscan(split_set (*dbscanner)(dataset, float, int), dataset ds, float epsilon_start,
                     float epsilon_inc, int minpts, char* split_files_prefix, int n_threads) {
  (void)n_threads;  // layers are always produced in eps order
  std::lock_guard<std::mutex> lk(g_mu);
  g_status = 0;
  swgpu::DbscanProvider prov;
  long long fixed = -1;
  bool engine = false;
  if (dbscanner == &dbscan_SW || dbscanner == nullptr) {
    // one score pass; the sweep's DBSCAN runs share it (dbscan_SW's warnings
    // are printed by the sweep for each run it consumes)
    swe_ctx* ctx = default_ctx();
    if (!ctx) return;
    if (int s = ensure_scored(ctx, ds)) {
      g_status = s;
      return;
    }
    prov.run = [ctx, minpts](const float* e, int c, split_set* o) {
      return swgpu::engine_dbscan_batch(ctx, 0, e, c, minpts, o);
    };
    prov.batch = swgpu::engine_batch_size(ctx, 0);
    prov.speculate = true;
    size_t mx = 0;
    for (int i = 0; i < ds.n_values; ++i) mx = ds.sequence_lengths[i] > mx ? ds.sequence_lengths[i] : mx;
    fixed = 4LL * (long long)mx;
    engine = true;
  } else if (dbscanner == &dbscan_L1 || dbscanner == &dbscan_L2) {
    // the point distances once; the sweep's DBSCAN runs share them
    swe_ctx* ctx = default_ctx();
    if (!ctx) return;
    if (int s = ensure_points(ctx, ds, dbscanner == &dbscan_L1 ? SWE_METRIC_L1 : SWE_METRIC_L2)) {
      g_status = s;
      return;
    }
    prov.run = [ctx, minpts](const float* e, int c, split_set* o) {
      return swgpu::engine_dbscan_batch(ctx, 0, e, c, minpts, o);
    };
    prov.batch = swgpu::engine_batch_size(ctx, 0);
    prov.key = [ctx](float e) { return swgpu::engine_sweep_key(ctx, e); };
    prov.speculate = true;
    fixed = swgpu::engine_fixed_point(ctx);
    engine = true;
  } else {
    prov.run = [&ds, dbscanner, minpts](const float* e, int c, split_set* o) {
      for (int k = 0; k < c; ++k) o[k] = dbscanner(ds, e[k], minpts);
      return 0;
    };
  }
  std::vector<split_set> kept;
  std::string err;
  const int rc = swgpu::adaptive_sweep(ds.n_values, epsilon_start, epsilon_inc, minpts, split_files_prefix,
                                       stdout, prov, engine, fixed, &kept, &err);
  for (auto& s : kept) free_split_set_and_associated_clusters(s);
  if (rc) {
    if (rc != SWE_ERR_SWEEP) fprintf(stderr, "swgpu: adaptive_dbscan failed: %s\n", err.c_str());
    g_status = rc;
  }
}

}  // extern "C"
