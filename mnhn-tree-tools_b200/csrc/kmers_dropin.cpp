// fasta2kmer's calls (fasta2kmer.c:8-44) on the GPU: frequencies_from_dataset
// and write_kmer_base of kmers.c:292-385 over swe_kmer_counts / swe_kmer_tsv,
// and free_kmer_frequencies (kmers.c:387-396).  The table is allocated the
// reference's way (one malloc'd row per sequence) so that either side's free
// releases it.
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "host_internal.h"

namespace {

bool failed(swe_ctx* ctx, int s, const char* what) {
  if (s == SWE_OK) return false;
  fprintf(stderr, "swgpu: %s failed: %s (%s)\n", what, swe_strerror((swe_status)s), ctx ? swe_last_error(ctx) : "");
  swgpu::dropin_set_status(s);
  return true;
}

int write_to_file(const char* data, size_t size, void* user) {
  return fwrite(data, 1, size, static_cast<FILE*>(user)) == size ? 0 : 1;
}

}  // namespace

extern "C" {

kmer_frequencies frequencies_from_dataset(dataset ds, size_t kmer_length, int n_threads, int protein) {
  (void)n_threads;
  kmer_frequencies freq;
  memset(&freq, 0, sizeof freq);
  std::lock_guard<std::mutex> lk(swgpu::dropin_mutex());
  swgpu::dropin_set_status(SWE_OK);
  const int64_t nk = kmer_length > 64 ? 0 : swe_kmer_count((int)kmer_length, protein);
  if (nk == 0) {
    fprintf(stderr, "swgpu: k-mer length %zu is not supported (1..%d, protein 1..%d)\n", kmer_length,
            SWE_KMER_MAX_DNA, SWE_KMER_MAX_PROTEIN);
    swgpu::dropin_set_status(SWE_ERR_INVALID);
    return freq;
  }
  swe_ctx* ctx = swgpu::dropin_ctx();
  if (!ctx) return freq;
  const int n = ds.n_values > 0 ? ds.n_values : 0;
  short** rows = static_cast<short**>(malloc(sizeof(short*) * (n > 0 ? n : 1)));
  std::vector<int64_t> len(n);
  bool ok = rows != nullptr;
  for (int i = 0; ok && i < n; ++i) {
    rows[i] = static_cast<short*>(malloc(sizeof(short) * (size_t)nk));
    ok = rows[i] != nullptr;
    len[i] = (int64_t)strlen(ds.sequences[i]);  // kmers.c:162
    if (!ok) {
      for (int j = 0; j < i; ++j) free(rows[j]);
    }
  }
  if (!ok) {
    free(rows);
    fprintf(stderr, "swgpu: out of host memory for the k-mer table\n");
    swgpu::dropin_set_status(SWE_ERR_OOM);
    return freq;
  }
  const int s = swe_kmer_counts(ctx, ds.sequences, len.data(), n, (int)kmer_length, protein,
                                reinterpret_cast<int16_t* const*>(rows));
  if (failed(ctx, s, "k-mer counting")) {
    for (int i = 0; i < n; ++i) free(rows[i]);
    free(rows);
    return freq;
  }
  freq.frequencies = rows;
  freq.n_kmers = (size_t)nk;
  freq.n_seq = (size_t)n;
  return freq;
}

void write_kmer_base(FILE* f, kmer_frequencies freq) {
  std::lock_guard<std::mutex> lk(swgpu::dropin_mutex());
  swgpu::dropin_set_status(SWE_OK);
  if (freq.n_seq == 0) return;
  swe_ctx* ctx = swgpu::dropin_ctx();
  if (!ctx) return;
  const int s = swe_kmer_tsv(ctx, reinterpret_cast<const int16_t* const*>(freq.frequencies), (int64_t)freq.n_seq,
                             (int64_t)freq.n_kmers, write_to_file, f);
  failed(ctx, s, "k-mer table output");
}

void free_kmer_frequencies(kmer_frequencies freq) {
  for (size_t i = 0; i < freq.n_seq; ++i) free(freq.frequencies[i]);
  free(freq.frequencies);
}

}  // extern "C"
