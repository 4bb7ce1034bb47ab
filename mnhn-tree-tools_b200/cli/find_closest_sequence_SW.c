/*
 * find_closest_sequence_SW <db.fasta> <query.fasta> <idx> <n_threads> <out.fasta>
 *
 * Drop-in for the reference tool (find_closest_sequence_SW.c:65-153): scores
 * query record idx (1-based) against every database sequence on the GPU and
 * prints "Smith Waterman distance = %i" for the smallest distance (the lowest
 * index wins ties), then writes that database sequence to <out.fasta> as
 * ">sequence_<index>".  As in the reference (find_closest_sequence_SW.c:49-53)
 * the query is scored with the length of the FIRST query record; when that
 * length exceeds the selected record's own length the reference reads past
 * the string, and this tool stops with an error instead.  n_threads is
 * accepted and unused.
 */
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mnhn_dropin.h"
#include "swgpu.h"

int main(int argc, char** argv) {
  FILE *fasta_f, *fasta_q;
  int n_threads = 1;
  dataset ds, query;
  cluster cl;
  char filename[4096];
  unsigned long idx = 0;
  int minimum = INT_MAX, minimal_sequence_index = -1;
  swe_ctx* ctx = NULL;
  swe_status s;
  unsigned* dist;
  const char* dev = getenv("SWGPU_DEVICE");
  swe_opts o = {0};

  if (argc < 6) {
    printf("Arguments are: \n"
           "[file] Fasta file of the database to find the closest sequence in\n"
           "[file] Fasta file containing the query sequence \n"
           " [int] use n_th sequence in fasta query file \n"
           " [int] number of threads to use for this search \n"
           "[file] output fasta containing the closest sequence in the"
           " dataset\n");
    return 1;
  }
  sscanf(argv[3], "%lu", &idx);
  sscanf(argv[4], "%i", &n_threads);
  filename[0] = 0;
  sscanf(argv[5], "%4095s", filename);

  if (NULL == (fasta_f = fopen(argv[1], "r"))) {
    printf("failed to open file %s\n", argv[1]);
    return 1;
  }
  ds = dataset_from_fasta(fasta_f);
  fclose(fasta_f);
  if (NULL == (fasta_q = fopen(argv[2], "r"))) {
    printf("failed to open file %s\n", argv[2]);
    return 1;
  }
  query = dataset_from_fasta(fasta_q);
  fclose(fasta_q);

  if (idx < 1 || idx > (unsigned long)query.n_values) {
    fprintf(stderr, "query index %lu is not a record of %s\n", idx, argv[2]);
    return 1;
  }
  if (query.sequence_lengths[0] > query.sequence_lengths[idx - 1]) {
    fprintf(stderr, "query %lu is shorter than query 1, whose length the reference uses\n", idx);
    return 1;
  }

  o.device = dev ? atoi(dev) : 0;
  s = swe_create(&ctx, &o);
  if (s == SWE_OK) s = swe_upload(ctx, (const char* const*)ds.sequences, ds.sequence_lengths, ds.n_values);
  dist = (unsigned*)malloc(sizeof(unsigned) * (size_t)(ds.n_values > 0 ? ds.n_values : 1));
  if (s == SWE_OK)
    s = swe_score_one_to_many(ctx, query.sequences[idx - 1], query.sequence_lengths[0], dist);
  if (s != SWE_OK) {
    fprintf(stderr, "swgpu: %s (%s)\n", swe_strerror(s), ctx ? swe_last_error(ctx) : "");
    return 1;
  }
  for (int i = 0; i < ds.n_values; ++i) {
    if ((int)dist[i] < minimum) {
      minimum = (int)dist[i];
      minimal_sequence_index = i;
    }
  }
  printf("Smith Waterman distance = %i \n", minimum);
  if (minimal_sequence_index >= 0) {
    cl.members = &minimal_sequence_index;
    cl.n_members = 1;
    cl.id = 0;
    create_single_cluster_file(filename, cl, ds);
  }
  free(dist);
  swe_destroy(ctx);
  free_sequences_from_dataset(ds);
  free_sequences_from_dataset(query);
  return 0;
}
