// Reference-named callers of score() around the hot path, on the engine:
// the distance statistics of comparison.c (compareSW, silhouette,
// compare_norms), the distance filter of filter.c (find_satellite) and the
// dataset writers/loaders those tools use (dataset.c).
//
// Two datasets are scored as one upload (ds_one's sequences, then ds_two's):
// one score pass gives every distance the reference computes pair by pair,
// and swe_block_stats reduces the needed block of the matrix on the GPU.
// Every result equals the reference's single-threaded result; with
// n_threads > 1 the reference sums per-thread partial results in an order
// that depends on scheduling, and its `int` partial sums can overflow on
// large inputs (comparison.c:120, 203), neither of which happens here.
#include <cmath>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "host_internal.h"

namespace {

using swgpu::dropin_ctx;
using swgpu::dropin_scored;
using swgpu::dropin_set_status;

// ds_one followed by ds_two (sequence pointers borrowed).
struct Joined {
  std::vector<char*> seqs;
  std::vector<size_t> lens;
  dataset ds;
  Joined(const dataset& a, const dataset& b) {
    for (int i = 0; i < a.n_values; ++i) seqs.push_back(a.sequences[i]), lens.push_back(a.sequence_lengths[i]);
    for (int i = 0; i < b.n_values; ++i) seqs.push_back(b.sequences[i]), lens.push_back(b.sequence_lengths[i]);
    memset(&ds, 0, sizeof ds);
    ds.sequences = seqs.data();
    ds.sequence_lengths = lens.data();
    ds.n_values = a.n_values + b.n_values;
  }
};

bool failed(swe_ctx* ctx, int s, const char* what) {
  if (s == SWE_OK) return false;
  fprintf(stderr, "swgpu: %s failed: %s (%s)\n", what, swe_strerror((swe_status)s), ctx ? swe_last_error(ctx) : "");
  dropin_set_status(s);
  return true;
}

// Row sums of rows [0, n1) of the joined matrix over columns [c0, c1), the
// sums of floor((d - mean)^2), and the block's extremes.
bool joined_stats(const dataset& a, const dataset& b, int c0, int c1, double mean, std::vector<uint64_t>* sum,
                  std::vector<uint64_t>* sq, uint32_t* mn, uint32_t* mx) {
  swe_ctx* ctx = dropin_ctx();
  if (!ctx) return false;
  Joined j(a, b);
  if (failed(ctx, dropin_scored(ctx, j.ds), "scoring")) return false;
  sum->assign(std::max(a.n_values, 1), 0);
  sq->assign(std::max(a.n_values, 1), 0);
  const int s = swe_block_stats(ctx, 0, 0, a.n_values, c0, c1, mean, sum->data(), sq->data(), mn, mx);
  return !failed(ctx, s, "block statistics");
}

}  // namespace

extern "C" {

// comparison.c:84-112: n1 x n2 matrix, row i = ds_one[i] (malloc'd).
unsigned long* smith_waterman_distances_matrix(dataset ds_one, dataset ds_two) {
  std::lock_guard<std::mutex> lk(swgpu::dropin_mutex());
  const int n1 = ds_one.n_values, n2 = ds_two.n_values;
  unsigned long* m = (unsigned long*)malloc(sizeof(unsigned long) * (size_t)n1 * (size_t)n2);
  if (!m || n1 == 0 || n2 == 0) return m;
  swe_ctx* ctx = dropin_ctx();
  if (!ctx) return m;
  Joined j(ds_one, ds_two);
  if (failed(ctx, dropin_scored(ctx, j.ds), "scoring")) return m;
  const int n = n1 + n2;
  const int chunk = std::max(1, std::min(n1, (int)((64LL << 20) / n)));
  std::vector<uint32_t> rows((size_t)chunk * n);
  for (int r0 = 0; r0 < n1; r0 += chunk) {
    const int r1 = std::min(n1, r0 + chunk);
    if (failed(ctx, swe_copy_set_rows(ctx, 0, r0, r1, rows.data()), "copying distances")) return m;
    for (int i = r0; i < r1; ++i)
      for (int k = 0; k < n2; ++k) m[(size_t)i * n2 + k] = rows[(size_t)(i - r0) * n + n1 + k];
  }
  return m;
}

// comparison.c:156-193: mean distance over ds_one x ds_two.
double mean_from_smith_waterman_datasets(dataset ds_one, dataset ds_two, size_t n_threads) {
  (void)n_threads;
  std::lock_guard<std::mutex> lk(swgpu::dropin_mutex());
  std::vector<uint64_t> sum, sq;
  uint32_t mn, mx;
  const int n = ds_one.n_values + ds_two.n_values;
  double total = 0.;
  if (ds_one.n_values > 0 && ds_two.n_values > 0 &&
      joined_stats(ds_one, ds_two, ds_one.n_values, n, 0.0, &sum, &sq, &mn, &mx)) {
    uint64_t t = 0;
    for (int i = 0; i < ds_one.n_values; ++i) t += sum[i];
    total = (double)t;
  }
  return total / ((double)ds_one.n_values * (double)ds_two.n_values);
}

// comparison.c:241-280: sqrt(sum over ds_one x ds_two of the integer part of
// (d - mean)^2) / (n1 + n2) (the reference accumulates into an int, which
// drops each term's fraction).
double sigma_from_smith_waterman_datasets(double mean, dataset ds_one, dataset ds_two, size_t n_threads) {
  (void)n_threads;
  std::lock_guard<std::mutex> lk(swgpu::dropin_mutex());
  std::vector<uint64_t> sum, sq;
  uint32_t mn, mx;
  const int n = ds_one.n_values + ds_two.n_values;
  double total = 0.;
  if (ds_one.n_values > 0 && ds_two.n_values > 0 &&
      joined_stats(ds_one, ds_two, ds_one.n_values, n, mean, &sum, &sq, &mn, &mx)) {
    uint64_t t = 0;
    for (int i = 0; i < ds_one.n_values; ++i) t += sq[i];
    total = (double)t;
  }
  return sqrt(total) / (ds_one.n_values + ds_two.n_values);
}

// comparison.c:20-82, 282-323: mean over ds_one of the silhouette s(i) with
// a = mean distance to ds_one (the point itself included in the sum, n1 - 1
// in the divisor) and b = mean distance to ds_two.
double silhouette_from_smith_waterman_datasets(dataset ds_one, dataset ds_two, size_t n_threads) {
  (void)n_threads;
  std::lock_guard<std::mutex> lk(swgpu::dropin_mutex());
  const int n1 = ds_one.n_values, n2 = ds_two.n_values, n = n1 + n2;
  std::vector<uint64_t> in, out, sq;
  uint32_t mn, mx;
  if (n1 == 0) return 0. / (double)n1;
  if (!joined_stats(ds_one, ds_two, 0, n1, 0.0, &in, &sq, &mn, &mx)) return NAN;
  if (!joined_stats(ds_one, ds_two, n1, n, 0.0, &out, &sq, &mn, &mx)) return NAN;
  double s_mean = 0;
  for (int i = 0; i < n1; ++i) {
    const double a = (double)in[i] / ((double)n1 - 1.);
    const double b = (double)out[i] / ((double)n2);
    double s = 0;
    if (a < b) s = 1 - a / b;
    else if (a == b) s = 0;
    else if (a > b) s = b / a - 1;
    s_mean += s;
  }
  return s_mean / (double)n1;
}

// comparison.c:325-350, 388-403 (host arithmetic on a caller's matrix).
double mean_from_smith_waterman_distance_matrix(unsigned long* matrix, dataset ds_one, dataset ds_two) {
  double sum = 0.;
  for (size_t i = 0; i < (size_t)ds_one.n_values * ds_two.n_values; i++) sum += (double)matrix[i];
  return sum / ((double)ds_one.n_values * (double)ds_two.n_values);
}

double sigma_from_smith_waterman_distance_matrix(unsigned long* matrix, double mean, dataset ds_one,
                                                 dataset ds_two) {
  double sigma = 0.;
  for (size_t i = 0; i < (size_t)ds_one.n_values * ds_two.n_values; i++) {
    const double d = (double)matrix[i] - mean;
    sigma = std::fma(d, d, sigma);  // the reference build contracts this multiply-add
  }
  return sqrt(sigma) / ((double)ds_one.n_values + (double)ds_two.n_values);
}

void shortest_longest_distance_in_matrix(unsigned long* matrix, unsigned long* shortest, unsigned long* largest,
                                         dataset ds_one, dataset ds_two) {
  shortest[0] = ULONG_MAX;
  largest[0] = 0;
  for (size_t i = 0; i < (size_t)ds_one.n_values * ds_two.n_values; i++) {
    if (matrix[i] < shortest[0]) shortest[0] = matrix[i];
    if (matrix[i] > largest[0]) largest[0] = matrix[i];
  }
}

// comparison.c:352-386: every pair j < i with its SW distance and the L2 / L1
// distances of the projections in ds.values.
void print_SW_PCA_L_comparison(FILE* f, dataset ds) {
  std::lock_guard<std::mutex> lk(swgpu::dropin_mutex());
  fprintf(f, "i j SW L1 L2\n");
  const int n = ds.n_values;
  if (n < 2) return;
  swe_ctx* ctx = dropin_ctx();
  if (!ctx) return;
  if (failed(ctx, dropin_scored(ctx, ds), "scoring")) return;
  const int chunk = std::max(1, std::min(n, (int)((64LL << 20) / n)));
  std::vector<uint32_t> rows((size_t)chunk * n);
  for (int r0 = 0; r0 < n; r0 += chunk) {
    const int r1 = std::min(n, r0 + chunk);
    if (failed(ctx, swe_copy_set_rows(ctx, 0, r0, r1, rows.data()), "copying distances")) return;
    for (int i = r0; i < r1; ++i)
      for (int j = 0; j < i; ++j) {
        const double sw = (double)rows[(size_t)(i - r0) * n + j];
        double l2 = 0, l1 = 0;
        for (int k = 0; k < ds.n_dimensions; ++k) {
          const double b = (float)(ds.values[k][j] - ds.values[k][i]);
          l2 = std::fma(b, b, l2);  // the reference build contracts this multiply-add
          l1 += fabs(b);
        }
        l2 = sqrt(l2);
        fprintf(f, "%i %i %lf %lf %lf\n", i, j, sw, l2, l1);
      }
  }
}

// filter.c:18-50: sequences with size - minus <= len <= size + plus (size_t
// arithmetic, as in the reference).
dataset filter_ds_by_size(dataset in_set, size_t size, size_t plus, size_t minus) {
  dataset out;
  memset(&out, 0, sizeof out);
  out.sequences = (char**)malloc(sizeof(char*) * (size_t)std::max(in_set.n_values, 1));
  out.sequence_lengths = (size_t*)malloc(sizeof(size_t) * (size_t)std::max(in_set.n_values, 1));
  int counter = 0;
  for (int i = 0; i < in_set.n_values; i++) {
    const size_t L = in_set.sequence_lengths[i];
    if (L <= size + plus && L >= size - minus) {
      out.sequences[counter] = (char*)malloc(L + 1);
      memcpy(out.sequences[counter], in_set.sequences[i], L);
      out.sequences[counter][L] = 0;
      out.sequence_lengths[counter] = L;
      out.max_sequence_length = std::max(out.max_sequence_length, L);
      counter++;
    }
  }
  out.n_values = counter;
  return out;
}

// filter.c:52-140: the sequences whose distance to `target` is at most
// max_distance (one query against the dataset on the GPU).
dataset filter_by_SW_distance(dataset in_set, char* target, size_t target_length, unsigned int max_distance,
                              int n_threads) {
  (void)n_threads;
  std::lock_guard<std::mutex> lk(swgpu::dropin_mutex());
  dataset out;
  memset(&out, 0, sizeof out);
  const int n = in_set.n_values;
  out.sequences = (char**)malloc(sizeof(char*) * (size_t)std::max(n, 1));
  out.sequence_lengths = (size_t*)malloc(sizeof(size_t) * (size_t)std::max(n, 1));
  if (n == 0) return out;
  swe_ctx* ctx = dropin_ctx();
  if (!ctx) return out;
  swgpu::dropin_forget();  // the upload below replaces whatever the context had scored
  std::vector<unsigned> d(n, UINT_MAX);
  int s = swe_upload(ctx, in_set.sequences, in_set.sequence_lengths, n);
  if (s == SWE_OK) s = swe_score_one_to_many(ctx, target, target_length, d.data());
  if (failed(ctx, s, "filter_by_SW_distance")) return out;
  int counter = 0;
  for (int i = 0; i < n; i++) {
    if (max_distance >= (unsigned)(int)d[i]) {  // filter.c:62-67 compares the int score as unsigned
      const size_t L = in_set.sequence_lengths[i];
      out.sequences[counter] = (char*)malloc(L + 1);
      memcpy(out.sequences[counter], in_set.sequences[i], L);
      out.sequences[counter][L] = 0;
      out.sequence_lengths[counter] = L;
      out.max_sequence_length = std::max(out.max_sequence_length, L);
      counter++;
    }
  }
  out.n_values = counter;
  return out;
}

// dataset.c:85-110: ">sequence_<j>" records, 50 symbols per line.  A record
// of length 0 is written as its header and an empty line (the reference's
// loop bound underflows there).
void dataset_to_fasta(FILE* f, dataset ds) {
  for (int j = 0; j < ds.n_values; j++) {
    fprintf(f, ">sequence_%i\n", j);
    const size_t L = ds.sequence_lengths[j];
    if (L == 0) {
      fprintf(f, "\n");
      continue;
    }
    size_t k;
    for (k = 0; k < L - 1; k++) {
      if (k != 0 && k % 50 == 0) fprintf(f, "\n");
      fputc(ds.sequences[j][k], f);
    }
    if ((L - 1) != 0 && (L - 1) % 50 == 0) fprintf(f, "\n");
    fputc(ds.sequences[j][k], f);
    fprintf(f, "\n");
  }
}

// dataset.c:427-471: `dimensions` floats per sequence, read with "%f".
void load_projections_from_file_into_dataset(FILE* projections, size_t dimensions, dataset* ds) {
  ds->n_dimensions = (int)dimensions;
  ds->values = (float**)malloc(sizeof(float*) * std::max<size_t>(dimensions, 1));
  for (size_t i = 0; i < dimensions; i++) {
    ds->values[i] = (float*)malloc(sizeof(float) * (size_t)(ds->n_values + (8 - (ds->n_values % 8))));
    if (!ds->values[i]) {
      printf("Could not allocate memory to load projections \n");
      dropin_set_status(SWE_ERR_OOM);
      return;
    }
  }
  for (int i = 0; i < ds->n_values; i++) {
    size_t counter = 0;
    for (size_t j = 0; j < dimensions; j++) counter += fscanf(projections, "%f", ds->values[j] + i);
    if (counter != dimensions) {
      printf("Error reading projections file \n");
      dropin_set_status(SWE_ERR_IO);
      return;
    }
  }
}

}  // extern "C"
