/*
 * Test infrastructure only: an all-cores driver around the REFERENCE's own
 * score() (smith-waterman.c:16-80, linked from oracle/_ref/libref.so).
 *
 * It scores rows the way region_query does (dbscan.c:539-556): for query
 * point i, score(seq[k], seq[i], len[k], len[i], work) for every k, with one
 * (max_len+1)^2 work matrix per thread.  Rows are handed out to pthreads one
 * at a time.  Used to produce golden vectors and as the timed CPU baseline.
 * refh_score_block does the same for a list of columns k instead of all of
 * them, and refh_score_pairs for an explicit list of (a, b) pairs, handed out
 * in chunks (sampled pair checks).
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>

unsigned int score(char* A, char* B, size_t len_a, size_t len_b, int* work);

typedef struct {
  char* const* seqs;
  const size_t* lens;
  int n;
  const int* rows;
  int nrows;
  const int* cols;  /* NULL: every sequence */
  int ncols;
  uint32_t* out;
  size_t max_len;
  int next;
  pthread_mutex_t lock;
} job_t;

static void* worker(void* arg) {
  job_t* job = (job_t*)arg;
  int* work = (int*)malloc(sizeof(int) * (job->max_len + 1) * (job->max_len + 1));
  for (;;) {
    pthread_mutex_lock(&job->lock);
    int r = job->next++;
    pthread_mutex_unlock(&job->lock);
    if (r >= job->nrows) break;
    int i = job->rows ? job->rows[r] : r;
    uint32_t* o = job->out + (size_t)r * (size_t)job->ncols;
    for (int c = 0; c < job->ncols; c++) {
      const int k = job->cols ? job->cols[c] : c;
      o[c] = score(job->seqs[k], job->seqs[i], job->lens[k], job->lens[i], work);
    }
  }
  free(work);
  return NULL;
}

static int run_job(job_t job, int n_threads);

int refh_score_rows(char* const* seqs, const size_t* lens, int n, const int* rows, int nrows,
                    uint32_t* out, int n_threads) {
  job_t job;
  job.seqs = seqs;
  job.lens = lens;
  job.n = n;
  job.rows = rows;
  job.nrows = nrows;
  job.cols = NULL;
  job.ncols = n;
  job.out = out;
  return run_job(job, n_threads);
}

/* out[r][c] = score(seq[cols[c]], seq[rows[r]]) */
int refh_score_block(char* const* seqs, const size_t* lens, int n, const int* rows, int nrows,
                     const int* cols, int ncols, uint32_t* out, int n_threads) {
  job_t job;
  job.seqs = seqs;
  job.lens = lens;
  job.n = n;
  job.rows = rows;
  job.nrows = nrows;
  job.cols = cols;
  job.ncols = ncols;
  job.out = out;
  return run_job(job, n_threads);
}

static int run_job(job_t job, int n_threads) {
  job.max_len = 0;
  for (int i = 0; i < job.n; i++)
    if (job.lens[i] > job.max_len) job.max_len = job.lens[i];
  job.next = 0;
  pthread_mutex_init(&job.lock, NULL);
  if (n_threads < 1) n_threads = 1;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
  for (int t = 0; t < n_threads; t++) pthread_create(&th[t], NULL, worker, &job);
  for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&job.lock);
  return 0;
}

/* out[k] = score(seq[a[k]], seq[b[k]]) for k < npairs, chunks of 256 pairs
   handed out to the threads */
typedef struct {
  char* const* seqs;
  const size_t* lens;
  const int* a;
  const int* b;
  long long npairs;
  uint32_t* out;
  size_t max_len;
  long long next;
  pthread_mutex_t lock;
} pair_job_t;

static void* pair_worker(void* arg) {
  pair_job_t* job = (pair_job_t*)arg;
  int* work = (int*)malloc(sizeof(int) * (job->max_len + 1) * (job->max_len + 1));
  for (;;) {
    pthread_mutex_lock(&job->lock);
    long long k0 = job->next;
    job->next += 256;
    pthread_mutex_unlock(&job->lock);
    if (k0 >= job->npairs) break;
    long long k1 = k0 + 256 < job->npairs ? k0 + 256 : job->npairs;
    for (long long k = k0; k < k1; k++) {
      const int x = job->a[k], y = job->b[k];
      job->out[k] = score(job->seqs[x], job->seqs[y], job->lens[x], job->lens[y], work);
    }
  }
  free(work);
  return NULL;
}

int refh_score_pairs(char* const* seqs, const size_t* lens, int n, const int* a, const int* b, long long npairs,
                     uint32_t* out, int n_threads) {
  pair_job_t job;
  job.seqs = seqs;
  job.lens = lens;
  job.a = a;
  job.b = b;
  job.npairs = npairs;
  job.out = out;
  job.max_len = 0;
  for (int i = 0; i < n; i++)
    if (lens[i] > job.max_len) job.max_len = lens[i];
  job.next = 0;
  pthread_mutex_init(&job.lock, NULL);
  if (n_threads < 1) n_threads = 1;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
  for (int t = 0; t < n_threads; t++) pthread_create(&th[t], NULL, pair_worker, &job);
  for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&job.lock);
  return 0;
}
