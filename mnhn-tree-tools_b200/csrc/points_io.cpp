// Point-dataset files of the k-mer / PCA DBSCAN tools (cluster_dbscan_kmer.c,
// cluster_dbscan_pca.c, adaptive_clustering.c): the k-mer table loader of
// dataset.c:346-425, the value frees of dataset.c:629-649 and the cluster
// files with values of cluster_io.c:343-379, and kmer2pca's table reader
// (kmer2pca.c:255-268).
//
// load_kmer_from_file_into_dataset reads the reference's token stream (a
// label, then n_features numbers, per sample, whitespace anywhere) with strtof
// on host threads: the file is cut at whitespace, each piece counts its
// tokens, and token t of the stream is field t % (n_features + 1) of sample
// t / (n_features + 1), which is what the reference's fscanf("%s") /
// fscanf("%f") sequence assigns.  strtof gives the same float as fscanf("%f")
// for every number; a token that is not a number reads as 0 (the reference
// leaves the value unset and stops advancing).  swe_read_feature_table reads
// the same stream with strtod (fscanf("%lf")) into kmer2pca's row-major
// doubles and reports such a token, or a short file, as an error.
#include <errno.h>
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "host_internal.h"

namespace {

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// A token of `len` bytes that is an optional '-' and 1 .. max_digits decimal
// digits (every count of a k-mer table) as its integer value: what strtod /
// strtof return for it whenever the value is exactly representable
// (max_digits 15 for double, 7 for float).  False for any other token.
inline bool small_integer(const char* tok, size_t len, int max_digits, long long* out) {
  const char* c = tok;
  const char* end = tok + len;
  const bool neg = c < end && *c == '-';
  if (neg) ++c;
  const size_t nd = (size_t)(end - c);
  if (nd == 0 || nd > (size_t)max_digits) return false;
  long long v = 0;
  for (; c < end; ++c) {
    if (*c < '0' || *c > '9') return false;
    v = v * 10 + (*c - '0');
  }
  if (neg && v == 0) return false;  // "-0" is -0.0: left to strtod
  *out = neg ? -v : v;
  return true;
}

float* alloc_values(size_t n) {
  void* p = nullptr;
  const size_t padded = (n + 8) & ~size_t(7);  // whole 8-float vectors, as the reference's AVX loop reads
  if (posix_memalign(&p, 32, sizeof(float) * std::max<size_t>(padded, 8)) != 0) return nullptr;
  memset(p, 0, sizeof(float) * std::max<size_t>(padded, 8));
  return static_cast<float*>(p);
}


// Reads the token stream of a table file (a label, then n_features numbers,
// per sample, whitespace anywhere) on host threads and hands each number token
// to on_value(sample, feature, token, length); the token lies in a buffer
// where whitespace or a NUL follows it, so strtod / strtof can read it in
// place.  Returns the number of tokens found (at most (n_features + 1) *
// n_samples are used).
template <class F>
uint64_t read_fields(FILE* in_file, data_shape shape, F&& on_value) {
  rewind(in_file);
  std::vector<char> text;
  {
    // the whole file in one buffer: sized from the stream's length when it has
    // one, grown chunk by chunk otherwise (a pipe)
    size_t have = 0;
    if (fseeko(in_file, 0, SEEK_END) == 0) {
      const off_t size = ftello(in_file);
      if (size > 0) text.resize((size_t)size);
    }
    rewind(in_file);
    for (;;) {
      if (have == text.size()) text.resize(std::max<size_t>(text.size() * 2, size_t(1) << 16));
      const size_t got = fread(text.data() + have, 1, text.size() - have, in_file);
      have += got;
      if (got == 0) break;
    }
    text.resize(have);
  }
  text.push_back('\0');
  const size_t len = text.size() - 1;
  const size_t fields = shape.n_features + 1;
  const uint64_t want = (uint64_t)fields * shape.n_samples;
  if (want == 0) return 0;
  // pieces cut at whitespace
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int T = (int)std::max<size_t>(1, std::min<size_t>((size_t)std::min(hw, 16), len >> 20));
  std::vector<size_t> cut(T + 1, len);
  cut[0] = 0;
  for (int t = 1; t < T; ++t) {
    size_t p = std::max(cut[t - 1], len * t / T);
    while (p < len && !is_space(text[p])) ++p;
    cut[t] = p;
  }
  auto tokens = [&](size_t a, size_t b, auto&& on_token) {
    size_t p = a;
    uint64_t k = 0;
    while (p < b) {
      while (p < b && is_space(text[p])) ++p;
      if (p >= b) break;
      const size_t q0 = p;
      while (p < b && !is_space(text[p])) ++p;
      if (!on_token(k++, q0, p)) break;
    }
    return k;
  };
  std::vector<uint64_t> count(T, 0), first(T + 1, 0);
  {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t)
      th.emplace_back([&, t]() { count[t] = tokens(cut[t], cut[t + 1], [](uint64_t, size_t, size_t) { return true; }); });
    for (auto& x : th) x.join();
  }
  for (int t = 0; t < T; ++t) first[t + 1] = first[t] + count[t];
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t)
    th.emplace_back([&, t]() {
      // token g of the stream is field g % fields of sample g / fields
      uint64_t g = first[t], sample = g / fields, field = g % fields;
      tokens(cut[t], cut[t + 1], [&](uint64_t, size_t q0, size_t q1) {
        if (g >= want) return false;
        bool go = true;
        if (field != 0)  // field 0 is the label, read with "%s"
          go = on_value(sample, field - 1, (const char*)text.data() + q0, q1 - q0);
        ++g;
        if (++field == fields) {
          field = 0;
          ++sample;
        }
        return go;
      });
    });
  for (auto& x : th) x.join();
  return first[T];
}

}  // namespace

extern "C" {

data_shape shape_from_kmer_file(int infile) {
  data_shape s{0, 0};
  lseek(infile, 0, SEEK_SET);
  // dataset.c:370-378: the tabs of the first line, then the newlines from
  // the end of the first line on; read in 8 MB pieces
  std::vector<char> buf(size_t(8) << 20);
  bool first_line = true;
  for (;;) {
    const ssize_t got = read(infile, buf.data(), buf.size());
    if (got < 0) {
      if (errno == EINTR) continue;
      printf("Could not read file in order to read obtain data shape\n");
      swgpu::dropin_set_status(SWE_ERR_IO);
      return data_shape{0, 0};
    }
    if (got == 0) break;
    const char* p = buf.data();
    const char* end = p + got;
    if (first_line) {
      const char* nl = static_cast<const char*>(memchr(p, '\n', (size_t)(end - p)));
      s.n_features += (size_t)std::count(p, nl ? nl : end, '\t');
      if (!nl) continue;
      first_line = false;
      p = nl;
    }
    while ((p = static_cast<const char*>(memchr(p, '\n', (size_t)(end - p)))) != nullptr) {
      s.n_samples++;
      ++p;
    }
  }
  return s;
}

dataset load_kmer_from_file_into_dataset(FILE* in_file, data_shape shape) {
  dataset ds;
  memset(&ds, 0, sizeof ds);
  ds.n_dimensions = (int)shape.n_features;
  ds.n_values = (int)shape.n_samples;
  ds.values = static_cast<float**>(malloc(sizeof(float*) * std::max<size_t>(shape.n_features, 1)));
  for (size_t d = 0; d < shape.n_features; ++d) {
    ds.values[d] = alloc_values(shape.n_samples);
    if (!ds.values[d]) {
      printf("Error allocating aligned memory for kmers \n");
      swgpu::dropin_set_status(SWE_ERR_OOM);
      return ds;
    }
  }
  read_fields(in_file, shape, [&](uint64_t sample, uint64_t field, const char* tok, size_t len) {
    long long v;
    ds.values[field][sample] = small_integer(tok, len, 7, &v) ? (float)v : strtof(tok, nullptr);
    return true;
  });
  return ds;
}

int swe_read_feature_table(FILE* in_file, data_shape shape, double* data) {
  if (!in_file || (!data && shape.n_features * shape.n_samples > 0)) return SWE_ERR_INVALID;
  std::atomic<int> bad{0};
  const uint64_t got = read_fields(in_file, shape, [&](uint64_t sample, uint64_t field, const char* tok, size_t len) {
    long long iv;
    if (small_integer(tok, len, 15, &iv)) {
      data[sample * shape.n_features + field] = (double)iv;
      return true;
    }
    char* end = nullptr;
    const double v = strtod(tok, &end);
    if (end == tok) {
      bad.store(1, std::memory_order_relaxed);
      return false;
    }
    data[sample * shape.n_features + field] = v;
    return true;
  });
  if (bad.load() || got < (uint64_t)(shape.n_features + 1) * shape.n_samples) return SWE_ERR_IO;
  return SWE_OK;
}

void free_values_from_dataset(dataset ds) {
  for (int i = 0; i < ds.n_dimensions; i++) free(ds.values[i]);
  free(ds.values);
}

void free_dataset(dataset ds) {
  free_values_from_dataset(ds);
  free_sequences_from_dataset(ds);
}

void create_single_cluster_file_with_values(char* filename, cluster cl, dataset ds) {
  FILE* f = fopen(filename, "w");
  if (!f) {
    swgpu::dropin_set_status(SWE_ERR_IO);
    return;
  }
  for (int j = 0; j < cl.n_members; j++) {
    for (int k = 0; k < ds.n_dimensions - 1; k++) fprintf(f, "%f\t", ds.values[k][cl.members[j]]);
    if (ds.n_dimensions > 0) fprintf(f, "%f\n", ds.values[ds.n_dimensions - 1][cl.members[j]]);
    else fputc('\n', f);
  }
  fclose(f);
}

void create_cluster_files_with_values(char* prefix, split_set s, dataset ds) {
  std::vector<char> name(strlen(prefix) + 32);
  for (int i = 0; i < s.n_clusters; i++) {
    snprintf(name.data(), name.size(), "%s-%03d", prefix, i);
    create_single_cluster_file_with_values(name.data(), s.clusters[i], ds);
  }
}

}  // extern "C"
