// FASTA loader with the reference's dataset_from_fasta semantics
// (dataset.c:264-344):
//   * a line whose first byte is '>' starts a record (the header text is not kept);
//   * any other line contributes its first whitespace-delimited token
//     (sscanf "%s", dataset.c:316), upper-cased (dataset.c:326-328);
//   * a line without a token appends the previous token again, because the
//     reference's sscanf leaves its buffer unchanged (dataset.c:316-333);
//     before the first token that buffer is empty here (uninitialised in the
//     reference);
//   * sequence lines before the first '>' are skipped here (the reference
//     writes through record index -1).
// Tokens may be of any length (the reference's buffer holds 1999 characters).
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "host_internal.h"

namespace swgpu {

static bool is_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

int fasta_read(FILE* in, dataset* out, std::string* err) {
  memset(out, 0, sizeof(*out));
  if (!in) {
    if (err) *err = "no input stream";
    return SWE_ERR_IO;
  }
  rewind(in);
  std::vector<std::string> seqs;
  std::string token;
  char* line = nullptr;
  size_t cap = 0;
  ssize_t got;
  bool started = false;
  while ((got = getline(&line, &cap, in)) != -1) {
    if (line[0] == '>') {
      seqs.emplace_back();
      started = true;
      continue;
    }
    ssize_t p = 0;
    while (p < got && is_space(line[p])) ++p;
    ssize_t e = p;
    while (e < got && line[e] != 0 && !is_space(line[e])) ++e;
    if (e > p) {
      token.assign(line + p, (size_t)(e - p));
      for (auto& c : token)
        if (c >= 'a' && c <= 'z') c = (char)(c - 'a' + 'A');
    }
    if (!started) continue;
    seqs.back() += token;
  }
  free(line);
  const int n = (int)seqs.size();
  out->n_values = n;
  out->sequences = (char**)malloc(sizeof(char*) * (size_t)(n > 0 ? n : 1));
  out->sequence_lengths = (size_t*)malloc(sizeof(size_t) * (size_t)(n > 0 ? n : 1));
  if (!out->sequences || !out->sequence_lengths) {
    free(out->sequences);
    free(out->sequence_lengths);
    memset(out, 0, sizeof(*out));
    if (err) *err = "out of memory";
    return SWE_ERR_OOM;
  }
  size_t mx = 0;
  for (int i = 0; i < n; ++i) {
    const size_t L = seqs[i].size();
    out->sequences[i] = (char*)malloc(L + 1);
    if (!out->sequences[i]) {
      for (int k = 0; k < i; ++k) free(out->sequences[k]);
      free(out->sequences);
      free(out->sequence_lengths);
      memset(out, 0, sizeof(*out));
      if (err) *err = "out of memory";
      return SWE_ERR_OOM;
    }
    memcpy(out->sequences[i], seqs[i].data(), L);
    out->sequences[i][L] = 0;
    out->sequence_lengths[i] = L;
    if (L > mx) mx = L;
  }
  out->max_sequence_length = mx;
  return 0;
}

}  // namespace swgpu
