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
#include <algorithm>
#include <cmath>
#include <cstdarg>
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

int not_covered_count(const split_set& s, int n) {
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

float coverage(int not_covered, int n) { return 1.f - (float)not_covered / (float)n; }

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

void SweepMachine::say(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  const int k = vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (k > 0) log_.append(buf, (size_t)std::min<int>(k, (int)sizeof buf - 1));
}

// dbscan.c:980-989, printed where the reference's dbscanner call would print them
void SweepMachine::warn(float eps) {
  if (!warnings_) return;
  if (eps == -1) {
    say("Warning @dbscan: epsilon value is: %f\n", eps);
    say("Warning @dbscan: epsilon was changed to: %f\n", 0.015f);
  }
  if (minpts_ == -1) {
    say("Warning @dbscan: minpts value is: %i\n", minpts_);
    say("Warning @dbscan: minpts was changed to: %i\n", 5);
  }
}

SweepMachine::SweepMachine(int n, float eps_start, float eps_inc, int minpts, int max_steps, int batch,
                           bool dbscan_sw_warnings, long long fixed_point)
    : n_(n), eps_start_(eps_start), eps_inc_(eps_inc), minpts_(minpts), max_steps_(max_steps),
      batch_(batch > 0 ? batch : 1), warnings_(dbscan_sw_warnings), fixed_(fixed_point) {
  say("Performing adaptive clustering with parameters: \n"
      "minpts: %i\n"
      "epsilon_start: %f\n"
      "epsilon_inc: %f\n",
      minpts, eps_start, eps_inc);
  phase_ = FIRST;
  request_start();
}

SweepMachine::~SweepMachine() {
  for (auto& s : sets_) free_split_set_and_associated_clusters(s);
}

void SweepMachine::fail(int status, const char* why) {
  status_ = status;
  err_ = why;
  req_.clear();
  phase_ = DONE;
}

std::vector<float> SweepMachine::sweep_batch(float* eps_now, bool* terminal) const {
  // the next eps values of the sweep, evaluated together; a value past the
  // largest distance (every later eps gives the same result) or an increment
  // too small to move eps ends the batch, since the reference would loop
  // forever after it
  std::vector<float> out;
  *terminal = false;
  int room = batch_;
  if (max_steps_ > 0) room = std::min(room, max_steps_ - steps_);
  while ((int)out.size() < room) {
    const float e = *eps_now;
    *eps_now = *eps_now + eps_inc_;
    out.push_back(e);
    if ((fixed_ >= 0 && (key_ ? key_(e) : eps_threshold(e)) >= fixed_) || !(*eps_now > e)) {
      *terminal = true;
      break;
    }
  }
  return out;
}

void SweepMachine::next_sweep_batch() { req_ = sweep_batch(&eps_now_, &terminal_); }

void SweepMachine::set_speculate(bool on) {
  speculate_ = on;
  if (phase_ == FIRST && req_.size() == 1) request_start();
}

void SweepMachine::request_start() {
  req_.assign(1, eps_start_);
  if (!speculate_) return;
  // the batch next_sweep_batch would request after this start
  spec_now_ = eps_start_ + eps_inc_;
  const std::vector<float> more = sweep_batch(&spec_now_, &spec_terminal_);
  req_.insert(req_.end(), more.begin(), more.end());
}

void SweepMachine::consume(split_set* res) {
  const size_t count = req_.size();
  if (phase_ == FIRST || phase_ == HALVING) {
    warn(req_[0]);
    split_set first = res[0];
    if (phase_ == FIRST) say("Initial set obtained with %i clusters\n", first.n_clusters);
    if (first.n_clusters == 1) {
      for (size_t j = 1; j < count; ++j) free_split_set_and_associated_clusters(res[j]);  // speculative
      if (counter_ == 20 || eps_start_ == 0) {
        say("Error did not find a sufficient starting position in 20 tries \n");
        free_split_set_and_associated_clusters(first);
        fail(SWE_ERR_SWEEP, "no starting eps with more than one cluster");
        return;
      }
      eps_start_ = eps_start_ / 2;
      say("Trying new starting point \n");
      free_split_set_and_associated_clusters(first);
      counter_++;
      phase_ = HALVING;
      request_start();
      return;
    }
    say("Sarting with %i clusters\n", first.n_clusters);
    say("Coverage at initial point: %f\n", coverage(not_covered_count(first, n_), n_));
    sets_.push_back(first);
    eps_now_ = eps_start_ + eps_inc_;
    phase_ = SWEEP;
    if (max_steps_ > 0 && steps_ >= max_steps_) {
      for (size_t j = 1; j < count; ++j) free_split_set_and_associated_clusters(res[j]);
      truncated_ = true;
      stop_ = 0;
      req_.clear();
      phase_ = DONE;
      return;
    }
    if (count > 1) {  // the speculative batch is this sweep's first batch
      req_.erase(req_.begin());
      eps_now_ = spec_now_;
      terminal_ = spec_terminal_;
      consume_sweep(res + 1, count - 1);
      return;
    }
    next_sweep_batch();
    return;
  }
  if (phase_ != SWEEP) return;
  consume_sweep(res, count);
}

void SweepMachine::consume_sweep(split_set* res, size_t count) {
  size_t k = 0;
  for (; k < count; ++k) {
    warn(req_[k]);
    sets_.push_back(res[k]);
    ++steps_;
    if (res[k].n_clusters == 1) {
      stop_ = (int)sets_.size() - 1;
      break;
    }
  }
  for (size_t j = k + 1; j < count; ++j) free_split_set_and_associated_clusters(res[j]);
  if (stop_ >= 0) {
    req_.clear();
    phase_ = DONE;
    return;
  }
  if (max_steps_ > 0 && (steps_ >= max_steps_ || terminal_)) {
    // the step budget ends the sweep: the layers found so far are kept
    truncated_ = true;
    stop_ = (int)sets_.size() - 1;
    req_.clear();
    phase_ = DONE;
    return;
  }
  if (terminal_) {
    fail(SWE_ERR_SWEEP, "the sweep can never reach one cluster");
    return;
  }
  next_sweep_batch();
}

void SweepMachine::abort(int status, const char* why) { fail(status, why); }

void SweepMachine::finish(const char* prefix, std::vector<split_set>* kept) {
  kept->clear();
  if (status_ || stop_ < 0) return;
  std::vector<split_set> keep;
  std::vector<cluster_connections*> conns;
  keep.push_back(sets_[0]);
  for (int i = 1; i <= stop_; ++i) {
    split_set ns = sets_[i];
    if (ns.n_clusters < keep.back().n_clusters) {
      const int count = (int)keep.size();
      say("Layer %i has %i clusters\n", count, ns.n_clusters);
      say("  Coverage at layer %i: %f\n", count, coverage(not_covered_count(ns, n_), n_));
      say("  Epsilon at layer %i: %f\n", count, layer_eps(eps_start_, i, eps_inc_));
      conns.push_back(generate_split_set_relation(keep.back(), ns));
      keep.push_back(ns);
    } else {
      free_split_set_and_associated_clusters(ns);
    }
  }
  for (size_t i = (size_t)stop_ + 1; i < sets_.size(); ++i) free_split_set_and_associated_clusters(sets_[i]);
  sets_.clear();
  say("Connections found: \n");
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
    say("Layer %i:\n", i);
    for (int j = 0; j < keep[i].n_clusters; ++j) {
      say("  Cluster %i connected to: \n  ", j);
      for (int k = 0; k < conns[i - 1][j].n_connections; ++k) say("%i ", conns[i - 1][j].connections[k]);
      say("\n");
    }
  }
  for (int i = (int)keep.size() - 1; i > 0; --i) {
    for (int j = 0; j < keep[i].n_clusters; ++j) free(conns[i - 1][j].connections);
    free(conns[i - 1]);
  }
  *kept = std::move(keep);
}

std::string SweepMachine::take_log() {
  std::string out;
  out.swap(log_);
  return out;
}

int adaptive_sweep(int n, float eps_start, float eps_inc, int minpts, const char* prefix, FILE* log,
                   const DbscanProvider& prov, bool dbscan_sw_warnings, long long fixed_point,
                   std::vector<split_set>* kept, std::string* err, int max_steps) {
  SweepMachine m(n, eps_start, eps_inc, minpts, max_steps, prov.batch, dbscan_sw_warnings, fixed_point);
  if (prov.key) m.set_key(prov.key);
  if (prov.speculate) m.set_speculate(true);
  auto flush = [&]() {
    const std::string t = m.take_log();
    if (!t.empty()) fwrite(t.data(), 1, t.size(), log);
  };
  while (!m.done()) {
    flush();
    const std::vector<float>& eps = m.request();
    std::vector<split_set> res(eps.size(), split_set{0, nullptr});
    const int rc = prov.run(eps.data(), (int)eps.size(), res.data());
    if (rc) {
      for (auto& s : res) free_split_set_and_associated_clusters(s);
      m.abort(rc, "dbscan failed");
      break;
    }
    m.consume(res.data());
  }
  if (m.status()) {
    flush();
    *err = m.error();
    return m.status();
  }
  m.finish(prefix, kept);
  flush();
  return 0;
}

void lpt_partition(const double* cost, int64_t n, int nparts, int* owner) {
  std::vector<double> load((size_t)std::max(nparts, 1), 0.0);
  for (int64_t t = 0; t < n; ++t) {
    int best = 0;
    for (int p = 1; p < nparts; ++p)
      if (load[p] < load[best]) best = p;
    owner[t] = best;
    load[best] += cost[t];
  }
}

void cost_order(const double* cost, int64_t n, int* order) {
  if (n <= 0) return;
  // Tile costs are products of small integers, so as 64-bit integers they
  // sort exactly; key = max - cost turns "descending, ties in index order"
  // into an ascending stable sort, done as an LSD radix sort over 11-bit
  // digits (three passes for the 100,000-read workload's 4.9M tiles instead
  // of a comparison sort).  Anything else takes the comparison sort.
  uint64_t top = 0;
  bool integral = n < ((int64_t)1 << 31);
  for (int64_t i = 0; i < n && integral; ++i) {
    const double c = cost[i];
    if (!(c >= 0.0 && c < 9007199254740992.0) || c != std::floor(c)) integral = false;
    else top = std::max(top, (uint64_t)c);
  }
  if (!integral) {
    for (int64_t i = 0; i < n; ++i) order[i] = (int)i;
    std::stable_sort(order, order + n, [&](int a, int b) { return cost[a] > cost[b]; });
    return;
  }
  constexpr int kBits = 11;
  constexpr uint64_t kMask = (1u << kBits) - 1;
  std::vector<int64_t> count((size_t)1 << kBits);
  if (top < ((uint64_t)1 << 32)) {
    // key in the high half, index in the low half: one array moves per pass,
    // and the low half keeps equal keys in index order
    std::vector<uint64_t> v((size_t)n), v2((size_t)n);
    for (int64_t i = 0; i < n; ++i) v[i] = ((top - (uint64_t)cost[i]) << 32) | (uint64_t)i;
    for (int shift = 32; shift < 64 && (top >> (shift - 32)) != 0; shift += kBits) {
      std::fill(count.begin(), count.end(), 0);
      for (int64_t i = 0; i < n; ++i) ++count[(v[i] >> shift) & kMask];
      int64_t sum = 0;
      for (auto& c : count) {
        const int64_t k = c;
        c = sum;
        sum += k;
      }
      for (int64_t i = 0; i < n; ++i) v2[count[(v[i] >> shift) & kMask]++] = v[i];
      v.swap(v2);
    }
    for (int64_t i = 0; i < n; ++i) order[i] = (int)(uint32_t)v[i];
    return;
  }
  std::vector<uint64_t> key((size_t)n), key2((size_t)n);
  std::vector<int> tmp((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    key[i] = top - (uint64_t)cost[i];
    order[i] = (int)i;
  }
  for (int shift = 0; shift < 64 && (top >> shift) != 0; shift += kBits) {
    std::fill(count.begin(), count.end(), 0);
    for (int64_t i = 0; i < n; ++i) ++count[(key[i] >> shift) & kMask];
    int64_t sum = 0;
    for (auto& c : count) {
      const int64_t k = c;
      c = sum;
      sum += k;
    }
    for (int64_t i = 0; i < n; ++i) {
      const int64_t dst = count[(key[i] >> shift) & kMask]++;
      key2[dst] = key[i];
      tmp[dst] = order[i];
    }
    key.swap(key2);
    std::copy(tmp.begin(), tmp.end(), order);
  }
}

}  // namespace swgpu

extern "C" swe_status swe_adaptive_matrix(int n, const uint32_t* D, float eps_start, float eps_inc, int minpts,
                                          const char* prefix, FILE* log, int speculate, int batch,
                                          split_set** out_sets, int* out_n_sets) {
  if (n < 0 || (n > 0 && !D) || batch < 1) return SWE_ERR_INVALID;
  const int wpr = (n + 63) / 64;
  const size_t words = (size_t)n * (size_t)wpr;
  uint32_t dmax = 0;
  for (size_t i = 0; i < (size_t)n * (size_t)n; ++i) dmax = D[i] > dmax ? D[i] : dmax;
  swgpu::DbscanProvider prov;
  prov.batch = batch;
  prov.speculate = speculate != 0;
  prov.run = [&](const float* eps, int count, split_set* out) -> int {
    std::vector<uint64_t> bits(std::max<size_t>(words, 1));
    std::vector<int> counts(std::max(n, 1));
    for (int k = 0; k < count; ++k) {
      const long long T = swgpu::eps_threshold(eps[k] == -1 ? 0.015f : eps[k]);  // dbscan.c:980-984
      std::fill(bits.begin(), bits.end(), 0);
      for (int i = 0; i < n; ++i) {
        int c = 0;
        for (int j = 0; j < n && T >= 0; ++j)
          if ((long long)D[(size_t)i * n + j] <= T) {
            bits[(size_t)i * wpr + (j >> 6)] |= 1ull << (j & 63);
            ++c;
          }
        counts[i] = c;
      }
      const int rc = swgpu::dbscan_replay_bitmap(n, bits.data(), wpr, counts.data(), minpts == -1 ? 5 : minpts,
                                                 &out[k]);
      if (rc) return rc;
    }
    return 0;
  };
  std::vector<split_set> kept;
  std::string err;
  const int rc = swgpu::adaptive_sweep(n, eps_start, eps_inc, minpts, prefix, log ? log : stdout, prov, true,
                                       (long long)dmax, &kept, &err);
  if (out_n_sets) *out_n_sets = (int)kept.size();
  if (rc) {
    for (auto& s : kept) free_split_set_and_associated_clusters(s);
    return (swe_status)rc;
  }
  if (out_sets) {
    split_set* arr = (split_set*)malloc(sizeof(split_set) * std::max<size_t>(kept.size(), 1));
    if (!arr) {
      for (auto& s : kept) free_split_set_and_associated_clusters(s);
      return SWE_ERR_OOM;
    }
    for (size_t k = 0; k < kept.size(); ++k) arr[k] = kept[k];
    *out_sets = arr;
  } else {
    for (auto& s : kept) free_split_set_and_associated_clusters(s);
  }
  return SWE_OK;
}

extern "C" void swe_cost_order(const double* cost, int64_t n, int* order) {
  if (!cost || !order || n <= 0) return;
  swgpu::cost_order(cost, n, order);
}

extern "C" void swe_lpt_partition(const double* cost, int64_t n, int nparts, int* owner) {
  if (!cost || !owner || n <= 0 || nparts < 1) return;
  swgpu::lpt_partition(cost, n, nparts, owner);
}
