// Host-side pieces shared by the engine, the adaptive driver and the drop-in
// layer.  No CUDA types here.
#pragma once
#include <cstdint>
#include <cstdio>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "mnhn_dropin.h"
#include "swgpu.h"

namespace swgpu {

// kmer2pca's eigen-decomposition pieces (pca_eigen.cpp).  A diagonal matrix is
// solved directly, with dsyev's order of equal eigenvalues (false if A is not
// diagonal).  pca_vectors_from_tridiagonal: the unit eigenvectors of the
// n_vectors largest eigenvalues (eigenvalues: all of them, ascending) of the
// tridiagonal T (d, e) of a Householder reduction whose reflector k
// (k = 0 .. n-3) acts on indices k+1 .. n-1 and is stored in A[k][k+1 ..]
// (first entry 1) with factor tau[k]; largest first, each signed so that its
// largest-magnitude entry is positive.
bool pca_eigen_diagonal(const double* A, int64_t n, int64_t n_vectors, double* eigenvalues, double* vectors);
void pca_vectors_from_tridiagonal(const double* A, const double* tau, const double* d, const double* e, int64_t n,
                                  const double* eigenvalues, int64_t n_vectors, double* vectors);

// Integer form of the reference's neighbour test (float)d <= eps
// (dbscan.c:548-551): d <= T with T = floor(eps) for eps >= 0, and no
// neighbour at all (T = -1) for negative or NaN eps.  Exact while d < 2^24.
long long eps_threshold(float eps);

// Order-faithful replay of dbscan_SW (dbscan.c:950-1047, expand_cluster
// dbscan.c:783-948) over per-point neighbour bitmaps: bit k of row i is set
// iff k is an eps-neighbour of i; counts[i] is the popcount of row i.
// The split set is malloc'd reference-style.  Returns 0 or SWE_ERR_OOM.
int dbscan_replay_bitmap(int n, const uint64_t* bits, int words_per_row, const int* counts, int minpts,
                         split_set* out);

// DBSCAN runs for `count` eps values (split sets malloc'd, in the given
// order); returns an swe_status.  `batch` is how many eps values the provider
// prefers per call: the sweep evaluates that many upcoming eps values at once
// and discards the ones past the one-cluster stop.
struct DbscanProvider {
  std::function<int(const float* eps, int count, split_set* out)> run;
  int batch = 1;
  // the sweep key of an eps (see SweepMachine::set_key); empty = eps_threshold
  std::function<long long(float)> key;
  // run without side effects, so the sweep may evaluate eps values
  // speculatively (SweepMachine::set_speculate)
  bool speculate = false;
};

// Adaptive sweep of dbscan.c:1117-1380 as a state machine: request() holds
// the eps values to evaluate next, consume() takes their DBSCAN results
// (ownership passes in), and once done() finish() selects the layers, writes
// the split-set files and the rest of the log.  Log text accumulates in the
// machine (take_log()).  Driving many machines at once lets one threshold
// launch serve the pending requests of many independent sets.
//
// With `dbscan_sw_warnings` the warnings dbscan_SW prints for eps == -1 or
// minpts == -1 (dbscan.c:980-989) are logged for every DBSCAN result the
// sweep consumes, where the reference's dbscanner calls would print them.
// `fixed_point` (when >= 0) is a threshold at or above which every eps gives
// the same result, used to stop sweeps that could never reach one cluster
// (the reference loops forever there); an eps is compared with it through its
// key (eps_threshold unless set_key gives another).  max_steps > 0 bounds the DBSCAN runs
// of the sweep phase (after the starting eps); a sweep that reaches the bound
// before a one-cluster result keeps the layers found so far (truncated()).
// max_steps == 0 is the reference's unbounded sweep.
class SweepMachine {
 public:
  SweepMachine(int n, float eps_start, float eps_inc, int minpts, int max_steps, int batch, bool dbscan_sw_warnings,
               long long fixed_point);
  ~SweepMachine();
  SweepMachine(const SweepMachine&) = delete;
  SweepMachine& operator=(const SweepMachine&) = delete;
  void set_key(std::function<long long(float)> key) {
    key_ = std::move(key);
    if (phase_ == FIRST) request_start();
  }
  // With speculation the request for a starting eps also holds the sweep
  // batch that follows it when that start gives more than one cluster (the
  // usual case): one round less.  The results of a start with one cluster are
  // discarded.  Only for providers without side effects (the engine).
  void set_speculate(bool on);
  bool done() const { return phase_ == DONE; }
  const std::vector<float>& request() const { return req_; }
  void consume(split_set* res);
  void abort(int status, const char* why);
  void finish(const char* prefix, std::vector<split_set>* kept);
  std::string take_log();
  int status() const { return status_; }
  const std::string& error() const { return err_; }
  bool truncated() const { return truncated_; }
  int steps() const { return steps_; }

 private:
  enum Phase { FIRST, HALVING, SWEEP, DONE };
  void say(const char* fmt, ...) __attribute__((format(printf, 2, 3)));
  void warn(float eps);
  void fail(int status, const char* why);
  void next_sweep_batch();
  std::vector<float> sweep_batch(float* eps_now, bool* terminal) const;
  void request_start();
  void consume_sweep(split_set* res, size_t count);
  int n_;
  float eps_start_, eps_inc_;
  int minpts_, max_steps_, batch_;
  bool warnings_;
  long long fixed_;
  std::function<long long(float)> key_;
  bool speculate_ = false;
  float spec_now_ = 0;     // eps_now_ after the speculative batch
  bool spec_terminal_ = false;
  Phase phase_ = FIRST;
  std::vector<float> req_;
  std::vector<split_set> sets_;
  float eps_now_ = 0;
  int counter_ = 0, steps_ = 0, stop_ = -1, status_ = 0;
  bool terminal_ = false, truncated_ = false;
  std::string log_, err_;
};

// One sweep driven to the end over a DBSCAN provider, log lines written to
// `log` as they are produced.  Kept layers are returned in `kept` (ownership
// passes to the caller).
int adaptive_sweep(int n, float eps_start, float eps_inc, int minpts, const char* prefix, FILE* log,
                   const DbscanProvider& prov, bool dbscan_sw_warnings, long long fixed_point,
                   std::vector<split_set>* kept, std::string* err, int max_steps = 0);

int not_covered_count(const split_set& s, int n);
float coverage(int not_covered, int n);

// The engine's batched DBSCAN over its scored matrix: the GPU builds one
// neighbour bitmap per distinct threshold and host threads replay them in
// parallel.  Semantics of swe_dbscan_set for each eps.
int engine_dbscan_batch(swe_ctx* ctx, int set, const float* eps, int count, int minpts, split_set* out);
int engine_batch_size(const swe_ctx* ctx, int set);
// The sweep's fixed point and eps key for the current upload (see
// SweepMachine): Smith-Waterman or point distances.
long long engine_fixed_point(const swe_ctx* ctx);
long long engine_sweep_key(const swe_ctx* ctx, float eps);

// Tile groups of nearly equal cost for a multi-process score pass: tiles in
// the given order (descending cost) go one by one to the least loaded group
// (the lowest index on ties), so every process derives the same groups.
void lpt_partition(const double* cost, int64_t n, int nparts, int* owner);

// The score pass's tile order: order[0..n) = the indices of cost[] by
// descending cost, equal costs in index order (what std::stable_sort with
// "greater" gives).
void cost_order(const double* cost, int64_t n, int* order);

// Single linkage over `count` pairs (pairs[2c], pairs[2c+1]) taken in order,
// a join skipped when the two groups together would exceed `cap` members;
// label[i] = the smallest index of i's group.
void capped_linkage(int n, const int* pairs, int64_t count, int cap, int* label);

// Deep copy of a split set (malloc'd like the original).
split_set copy_split_set(const split_set& s);

// FASTA loading with dataset_from_fasta semantics (dataset.c:264-344).
int fasta_read(FILE* in, dataset* out, std::string* err);

// Distance of one pair of raw strings on the GPU (the drop-in score()).
swe_status score_raw(swe_ctx* ctx, const char* A, size_t la, const char* B, size_t lb, unsigned* out);

// The eps printed for kept layer i (dbscan.c:1323-1324):
// epsilon_start + (i+1) * (float)epsilon_inc, evaluated in float.
float layer_eps(float eps_start, int i, float eps_inc);

// The drop-in layer's process-wide context (dropin.cpp): its lock, the
// context itself (null without a device), "make sure ds is uploaded and
// scored" (cached by content), forgetting that cache after another upload,
// and the status swgpu_last_dropin_status() reports.
std::mutex& dropin_mutex();
swe_ctx* dropin_ctx();
int dropin_scored(swe_ctx* ctx, const dataset& ds);
void dropin_forget();
void dropin_set_status(int s);

}  // namespace swgpu
