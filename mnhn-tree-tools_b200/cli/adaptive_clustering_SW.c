/*
 * adaptive_clustering_SW <fasta> <eps_start> <eps_inc> <minpts> <prefix> <n_threads>
 *
 * Drop-in for the reference tool built from adaptive_clustering.c:54-200 with
 * -D_SCAN_SMITH_WATERMAN: the same arguments, "Dataset read!" line, adaptive
 * log on stdout and <prefix>%04d split-set files.  All distances are scored
 * once on the GPU for the whole sweep.  The reference reads argv[5] and
 * argv[6] even when fewer arguments are given; here fewer than six arguments
 * print the usage text.  Exits 1 where the reference calls _exit(1).
 */
#include <stdio.h>
#include <stdlib.h>

#include "mnhn_dropin.h"

static void print_arguments(void) {
  printf("Arguments are: \n"
         "   [file] FASTA file containing sequence dataset \n"
         "   (float) initial epsilon value \n"
         "   (float) epsilon increase between cluster search \n"
         "   (int) minimum numbers of clusters in epsilon neigbourhood \n"
         "   (string) path/andprefix of split_set_files \n"
         "   (int) number of threads to use \n");
}

int main(int argc, char** argv) {
  dataset ds;
  float epsilon_start = 0.f, epsilon_inc = 0.f;
  int minpts = 0, n_threads = 1;
  char split_files_prefix[4096];
  FILE* fasta_f;

  if (argc < 7) {
    print_arguments();
    return 1;
  }
  sscanf(argv[2], "%f", &epsilon_start);
  sscanf(argv[3], "%f", &epsilon_inc);
  sscanf(argv[4], "%i", &minpts);
  split_files_prefix[0] = 0;
  sscanf(argv[5], "%4095s", split_files_prefix);
  sscanf(argv[6], "%i", &n_threads);

  if (NULL == (fasta_f = fopen(argv[1], "r"))) {
    printf("failed to open file %s\n", argv[1]);
    return 1;
  }
  ds = dataset_from_fasta(fasta_f);
  fclose(fasta_f);
  printf("Dataset read!\n");

  adaptive_dbscan(dbscan_SW, ds, epsilon_start, epsilon_inc, minpts, split_files_prefix, n_threads);
  fflush(stdout);
  if (swgpu_last_dropin_status() != 0) return 1;
  free_sequences_from_dataset(ds);
  return 0;
}
