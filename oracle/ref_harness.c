/*
 * Test infrastructure only: an all-cores driver around the REFERENCE's own
 * score() (smith-waterman.c:16-80, linked from oracle/_ref/libref.so).
 *
 * It scores rows the way region_query does (dbscan.c:539-556): for query
 * point i, score(seq[k], seq[i], len[k], len[i], work) for every k, with one
 * (max_len+1)^2 work matrix per thread.  Rows are handed out to pthreads one
 * at a time.  Used to produce golden vectors and as the timed CPU baseline.
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
    uint32_t* o = job->out + (size_t)r * (size_t)job->n;
    for (int k = 0; k < job->n; k++)
      o[k] = score(job->seqs[k], job->seqs[i], job->lens[k], job->lens[i], work);
  }
  free(work);
  return NULL;
}

int refh_score_rows(char* const* seqs, const size_t* lens, int n, const int* rows, int nrows,
                    uint32_t* out, int n_threads) {
  job_t job;
  job.seqs = seqs;
  job.lens = lens;
  job.n = n;
  job.rows = rows;
  job.nrows = nrows;
  job.out = out;
  job.max_len = 0;
  for (int i = 0; i < n; i++)
    if (lens[i] > job.max_len) job.max_len = lens[i];
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
