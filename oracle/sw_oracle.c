/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C restatement of the reference's CPU path for the all-pairs
 * Smith-Waterman neighbourhood engine of MNHN-Tree-Tools.  It exists to check
 * the GPU engine; it is never linked into, called by, or used as a fallback
 * for the product library.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it.
 *
 * Parity of this restatement is pinned against the reference itself: the
 * golden vectors under tests/golden/ were produced by the reference's own
 * score(), dataset_from_fasta(), dbscan_SW() and adaptive_dbscan() compiled
 * from its sources (oracle/Makefile target `ref`), and tests/test_oracle.py
 * checks this file against them.
 *
 * Every function names the reference lines it restates (paths are relative to
 * the reference project root).
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MATCH 4 /* smith-waterman.c:4 (SCORE) */
#define ORC_GAP 3   /* smith-waterman.c:5 (GAP)   */

/*
 * Linear-gap local alignment distance, smith-waterman.c:16-80.
 *
 * The reference walks i = 1..len_a over A and j = 1..len_b over B, so A[0]
 * and B[0] never take part and the C-string terminators A[len_a], B[len_b]
 * do (smith-waterman.c:56-58).  Cells follow
 *   H[i][j] = max(0, H[i-1][j-1] + s(A[i],B[j]), H[i][j-1] - 3, H[i-1][j] - 3)
 * with s = +4 on raw char equality and -4 otherwise (smith-waterman.c:7-14).
 * The result is 4*max(len_a,len_b) minus the largest cell
 * (smith-waterman.c:42-46,80).
 *
 * This restatement keeps one row of H (the reference keeps the whole matrix;
 * the values are the same).  A and B must be readable at [0..len].
 */
unsigned int orc_score(const char* A, const char* B, size_t len_a, size_t len_b) {
  int* row = (int*)calloc(len_a + 1, sizeof(int));
  int best = 0;
  for (size_t j = 1; j <= len_b; j++) {
    int diag = 0; /* H[j-1][0] */
    int left = 0; /* H[j][0]   */
    for (size_t i = 1; i <= len_a; i++) {
      int up = row[i];
      int h = diag + (A[i] == B[j] ? ORC_MATCH : -ORC_MATCH);
      if (left - ORC_GAP > h) h = left - ORC_GAP;
      if (up - ORC_GAP > h) h = up - ORC_GAP;
      if (h < 0) h = 0;
      row[i] = h;
      diag = up;
      left = h;
      if (h > best) best = h;
    }
  }
  free(row);
  int optimum = (int)((len_a > len_b ? len_a : len_b) * ORC_MATCH);
  return (unsigned int)(optimum - best);
}

/* ---------------------------------------------------------------------- */
/* All-pairs and one-to-many drivers (threaded over rows).                */
/* ---------------------------------------------------------------------- */

typedef struct {
  const char* const* seqs;
  const size_t* lens;
  int n;
  const int* rows; /* NULL: rows 0..n-1 */
  int nrows;
  uint32_t* out; /* nrows x n */
  int next;
  pthread_mutex_t lock;
} rows_job;

static void* rows_worker(void* arg) {
  rows_job* job = (rows_job*)arg;
  for (;;) {
    pthread_mutex_lock(&job->lock);
    int r = job->next++;
    pthread_mutex_unlock(&job->lock);
    if (r >= job->nrows) break;
    int i = job->rows ? job->rows[r] : r;
    uint32_t* out = job->out + (size_t)r * (size_t)job->n;
    /* region_query scores candidate k against the query point
       (dbscan.c:546-549): score(seq[k], seq[point], len[k], len[point]). */
    for (int k = 0; k < job->n; k++)
      out[k] = orc_score(job->seqs[k], job->seqs[i], job->lens[k], job->lens[i]);
  }
  return NULL;
}

/* Distances of the listed query rows to every sequence (out is nrows x n). */
int orc_score_rows(const char* const* seqs, const size_t* lens, int n, const int* rows,
                   int nrows, uint32_t* out, int n_threads) {
  if (n_threads < 1) n_threads = 1;
  rows_job job = {seqs, lens, n, rows, nrows, out, 0, PTHREAD_MUTEX_INITIALIZER};
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
  for (int t = 0; t < n_threads; t++) pthread_create(&th[t], NULL, rows_worker, &job);
  for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
  free(th);
  return 0;
}

/* Full n x n matrix, every ordered pair scored as the reference does. */
int orc_all_pairs(const char* const* seqs, const size_t* lens, int n, uint32_t* out,
                  int n_threads) {
  return orc_score_rows(seqs, lens, n, NULL, n, out, n_threads);
}

/* ---------------------------------------------------------------------- */
/* DBSCAN over a precomputed distance matrix.                              */
/* ---------------------------------------------------------------------- */

/* region_query, dbscan.c:525-561: ascending k with (float)d(k,point) <= eps,
   the point itself included. */
static int orc_region(const void* Dv, int n, int point, float eps, int* out) {
  const uint32_t* D = (const uint32_t*)Dv;
  int m = 0;
  for (int k = 0; k < n; k++) {
    float d = (float)D[(size_t)point * (size_t)n + (size_t)k];
    if (d <= eps) out[m++] = k;
  }
  return m;
}

/* region_query of dbscan_L1 / dbscan_L2 (dbscan.c:563-779) over a float
   matrix of point distances: d <= epsilon (L1), d <= epsilon*epsilon with
   the square rounded to float (L2, dbscan.c:578). */
static int orc_region_l1(const void* Dv, int n, int point, float eps, int* out) {
  const float* D = (const float*)Dv;
  int m = 0;
  for (int k = 0; k < n; k++)
    if (D[(size_t)point * (size_t)n + (size_t)k] <= eps) out[m++] = k;
  return m;
}

static int orc_region_l2(const void* Dv, int n, int point, float eps, int* out) {
  const float* D = (const float*)Dv;
  const float eps2 = eps * eps;
  int m = 0;
  for (int k = 0; k < n; k++)
    if (D[(size_t)point * (size_t)n + (size_t)k] <= eps2) out[m++] = k;
  return m;
}

typedef int (*orc_region_fn)(const void* D, int n, int point, float eps, int* out);
static int dbscan_core(const void* D, int n, float eps, int minpts, orc_region_fn region, int* members, int* sizes);

/* The pair distances of dbscan_L1 / dbscan_L2's region_query (dbscan.c:
   563-779, the AVX build with FMA): for query point p and point i, over the
   dimensions k in order from +0, L2 dist = fmaf(v_p - v_i, v_p - v_i, dist)
   (dbscan.c:661-665), L1 dist = dist + |v_p - v_i| (dbscan.c:672-675).  V is
   dimension-major (V[k*n + i], the reference's values[k][i]); D[p*n + i]
   receives the distance.  metric 1 = L1, 2 = L2. */
void orc_points_dist(const float* V, int dims, int n, int metric, float* D) {
  for (int p = 0; p < n; p++)
    for (int i = 0; i < n; i++) {
      float acc = 0.0f;
      for (int k = 0; k < dims; k++) {
        const float d = V[(size_t)k * (size_t)n + (size_t)p] - V[(size_t)k * (size_t)n + (size_t)i];
        acc = metric == 2 ? fmaf(d, d, acc) : acc + fabsf(d);
      }
      D[(size_t)p * (size_t)n + (size_t)i] = acc;
    }
}

/* dbscan_L1 / dbscan_L2 (dbscan.c:950-1047 with the region queries above)
   over that matrix; output as orc_dbscan. */
int orc_dbscan_points(const float* D, int n, float eps, int minpts, int metric, int* members, int* sizes) {
  return dbscan_core(D, n, eps, minpts, metric == 2 ? orc_region_l2 : orc_region_l1, members, sizes);
}

/*
 * dbscan_SW, dbscan.c:950-1047, with expand_cluster, dbscan.c:783-948.
 *
 *  - seeds are taken in index order; a seed opens a cluster only when
 *    minpts < |N(seed)| (strict, dbscan.c:1011);
 *  - expand_cluster keeps `nb` sorted (merge at dbscan.c:854-889) and appends
 *    to the frontier, in ascending order, the members of N(q) that are not
 *    yet in `nb` (dbscan.c:894-920) whenever |N(q)| >= minpts (dbscan.c:847);
 *    points visited before are never queried again (dbscan.c:835-838);
 *  - a frontier point joins the cluster unless an earlier cluster already
 *    holds it (dbscan.c:934-940).
 *
 * The frontier append is the set difference N(q) \ nb that the reference
 * intends.  (The reference reads right_in_left[] one slot past its filled
 * length at dbscan.c:900; when that stale value equals a later member the
 * member is dropped.  The restatement does not reproduce that read.)
 *
 * Output: clusters in id order; members[] holds them back to back in member
 * order, sizes[c] their counts.  Returns the number of clusters.
 */
int orc_dbscan(const uint32_t* D, int n, float eps, int minpts, int* members, int* sizes) {
  return dbscan_core(D, n, eps, minpts, orc_region, members, sizes);
}

static int dbscan_core(const void* D, int n, float eps, int minpts, orc_region_fn region, int* members,
                       int* sizes) {
  /* dbscan.c:980-989 defaults */
  if (eps == -1) eps = 0.015f;
  if (minpts == -1) minpts = 5;
  char* visited = (char*)calloc((size_t)n + 1, 1);
  char* in_cluster = (char*)calloc((size_t)n + 1, 1);
  int* nb = (int*)malloc(sizeof(int) * ((size_t)n + 1));
  int* nbq = (int*)malloc(sizeof(int) * ((size_t)n + 1));
  int* merged = (int*)malloc(sizeof(int) * ((size_t)n + 1));
  int* frontier = (int*)malloc(sizeof(int) * ((size_t)n + 1));
  int n_clusters = 0;
  size_t out_pos = 0;
  for (int i = 0; i < n; i++) {
    if (visited[i]) continue;
    visited[i] = 1;
    int n_nb = region(D, n, i, eps, nb);
    if (!(minpts < n_nb)) continue;
    /* expand_cluster */
    int* cl = members + out_pos;
    int cl_n = 0;
    cl[cl_n++] = i;
    in_cluster[i] = 1;
    int n_front = n_nb;
    memcpy(frontier, nb, sizeof(int) * (size_t)n_nb);
    for (int f = 0; f < n_front; f++) {
      int q = frontier[f];
      if (!visited[q]) {
        visited[q] = 1;
        int n_q = region(D, n, q, eps, nbq);
        if (n_q >= minpts) {
          /* sorted merge of nb and nbq; the members of nbq missing from nb go
             to the frontier in ascending order */
          int a = 0, b = 0, m = 0;
          while (a < n_nb && b < n_q) {
            if (nb[a] < nbq[b]) merged[m++] = nb[a++];
            else if (nbq[b] < nb[a]) {
              frontier[n_front++] = nbq[b];
              merged[m++] = nbq[b++];
            } else {
              merged[m++] = nb[a++];
              b++;
            }
          }
          while (a < n_nb) merged[m++] = nb[a++];
          while (b < n_q) {
            frontier[n_front++] = nbq[b];
            merged[m++] = nbq[b++];
          }
          memcpy(nb, merged, sizeof(int) * (size_t)m);
          n_nb = m;
        }
      }
      if (!in_cluster[q]) {
        cl[cl_n++] = q;
        in_cluster[q] = 1;
      }
    }
    sizes[n_clusters++] = cl_n;
    out_pos += (size_t)cl_n;
  }
  free(visited);
  free(in_cluster);
  free(nb);
  free(nbq);
  free(merged);
  free(frontier);
  return n_clusters;
}

/* ---------------------------------------------------------------------- */
/* FASTA loader, dataset.c:264-344.                                        */
/* ---------------------------------------------------------------------- */

/*
 * Records start at lines whose first byte is '>'.  Every other line
 * contributes its first whitespace-delimited token (sscanf "%s",
 * dataset.c:316), upper-cased (dataset.c:326-328).  A line with no token
 * re-appends the previous token, because the reference's sscanf leaves its
 * line buffer untouched (dataset.c:316-333); before any token was read that
 * buffer is uninitialised in the reference and empty here.  Lines before the
 * first '>' are an error here (the reference writes through index -1).
 *
 * On success *buf holds the sequences back to back, each followed by a NUL,
 * (*lens)[k] their lengths and *n the record count.  Returns 0, or -1 when the
 * file cannot be read, -2 for sequence data before the first header.
 */
int orc_fasta_load(const char* path, char** buf, size_t** lens, int* n) {
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  char* line = NULL;
  size_t cap_line = 0;
  ssize_t got;
  size_t cap = 1024, used = 0;
  char* out = (char*)malloc(cap);
  size_t lcap = 64;
  size_t* L = (size_t*)malloc(sizeof(size_t) * lcap);
  int count = -1;
  char* token = (char*)calloc(1, 1);
  size_t token_len = 0;
  int rc = 0;
  while ((got = getline(&line, &cap_line, f)) != -1) {
    if (line[0] == '>') {
      if (count >= 0) out[used++] = 0;
      count++;
      if ((size_t)count >= lcap) {
        lcap *= 2;
        L = (size_t*)realloc(L, sizeof(size_t) * lcap);
      }
      L[count] = 0;
      continue;
    }
    /* first token, as sscanf("%s") would read it */
    size_t p = 0;
    while (p < (size_t)got && (line[p] == ' ' || line[p] == '\t' || line[p] == '\n' ||
                               line[p] == '\v' || line[p] == '\f' || line[p] == '\r'))
      p++;
    size_t e = p;
    while (e < (size_t)got && !(line[e] == ' ' || line[e] == '\t' || line[e] == '\n' ||
                                line[e] == '\v' || line[e] == '\f' || line[e] == '\r' ||
                                line[e] == 0))
      e++;
    if (e > p) {
      free(token);
      token_len = e - p;
      token = (char*)malloc(token_len + 1);
      for (size_t k = 0; k < token_len; k++) {
        char c = line[p + k];
        token[k] = (c >= 'a' && c <= 'z') ? (char)(c - 'a' + 'A') : c;
      }
      token[token_len] = 0;
    }
    if (count < 0) {
      rc = -2;
      break;
    }
    while (used + token_len + 2 > cap) {
      cap *= 2;
      out = (char*)realloc(out, cap);
    }
    memcpy(out + used, token, token_len);
    used += token_len;
    L[count] += token_len;
  }
  if (rc == 0 && count >= 0) {
    if (used + 1 > cap) out = (char*)realloc(out, used + 1);
    out[used++] = 0;
  }
  free(line);
  free(token);
  fclose(f);
  if (rc != 0) {
    free(out);
    free(L);
    return rc;
  }
  *buf = out;
  *lens = L;
  *n = count + 1;
  return 0;
}

void orc_free(void* p) { free(p); }

/* k-mer counts, kmers.c:157-241 and the index order of kmers.c:26-107: the
   k-mer index has base p of the word in bits 2p..2p+1 (A0 C1 G2 T3); windows
   start at 0..len-k-1 (the last window is never counted); a window with any
   other character matches no k-mer.  out[4^k] receives the counts. */
void orc_kmer_counts(const char* s, size_t len, int k, int16_t* out) {
  size_t nk = (size_t)1 << (2 * k);
  memset(out, 0, sizeof(int16_t) * nk);
  if ((size_t)k > len) return;
  for (size_t i = 0; i + (size_t)k < len; i++) {
    size_t idx = 0;
    int ok = 1;
    for (int p = 0; p < k; p++) {
      int c;
      switch (s[i + (size_t)p]) {
        case 'A': c = 0; break;
        case 'C': c = 1; break;
        case 'G': c = 2; break;
        case 'T': c = 3; break;
        default: c = -1;
      }
      if (c < 0) {
        ok = 0;
        break;
      }
      idx |= (size_t)c << (2 * p);
    }
    if (ok) out[idx]++;
  }
}

/* The frequency row of frequencies_from_dataset (kmers.c:292-371) for one
   NUL-terminated sequence: entry b counts the windows that equal k-mer b in
   frequence_of_kmer_in_sequence (kmers.c:157-241): sequence length is
   strlen(s) (kmers.c:162), windows start at 0 .. len-k-1 (kmers.c:172, 230),
   bytes compare raw.  DNA k-mer b has symbol p = "ACGT"[(b >> 2p) & 3]
   (gen_dna_string_from_binary, kmers.c:26-63); protein k-mer b is the base-20
   number over "ACDEFGHIKLMNPQRSTVWY" with symbol 0 most significant (the
   recursion of kmers.c:109-130, first position outermost).  Counts are kept
   in a short as the reference does (the low 16 bits, kmers.c:171, 211).
   This loops over windows, not over the 4^k / 20^k table entries: the same
   counts, found by decoding each window once.  out[] has 4^k or 20^k
   entries. */
void orc_kmer_frequencies(const char* s, int k, int protein, int16_t* out) {
  static const char dna[] = "ACGT", prot[] = "ACDEFGHIKLMNPQRSTVWY";
  const char* alpha = protein ? prot : dna;
  const int base = protein ? 20 : 4;
  size_t nk = 1;
  for (int i = 0; i < k; i++) nk *= (size_t)base;
  memset(out, 0, sizeof(int16_t) * nk);
  const size_t len = strlen(s);
  if ((size_t)k > len) return;
  for (size_t w = 0; w + (size_t)k < len; w++) {
    size_t idx = 0;
    int ok = 1;
    for (int p = 0; p < k && ok; p++) {
      const char* hit = memchr(alpha, s[w + (size_t)p], (size_t)base);
      if (!hit || s[w + (size_t)p] == 0) {
        ok = 0;
        break;
      }
      const size_t c = (size_t)(hit - alpha);
      if (protein) idx = idx * 20 + c;
      else idx |= c << (2 * p);
    }
    if (ok) out[idx] = (int16_t)(uint16_t)((uint16_t)out[idx] + 1u);
  }
}

/* obtain_projections (kmer2pca.c:141-168): p[j][i] = sum over k of
   data[j][k] * v[i][k], accumulated in the order of k with one fused
   multiply-add per term (the reference's loop as an FMA build compiles it).
   v holds the wanted eigenvectors as rows, largest eigenvalue first. */
void orc_pca_project(const double* data, int64_t n, int64_t nf, const double* v, int64_t dims, double* p) {
  for (int64_t j = 0; j < n; j++)
    for (int64_t i = 0; i < dims; i++) {
      double acc = 0;
      for (int64_t k = 0; k < nf; k++) acc = fma(data[j * nf + k], v[i * nf + k], acc);
      p[j * dims + i] = acc;
    }
}
