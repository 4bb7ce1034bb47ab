/*
 * cluster_dbscan_SW <fasta> <epsilon> <minpts> <prefix>
 *
 * Drop-in for the reference tool (cluster_dbscan_SW.c:25-71): same arguments,
 * the same "%u clusters obtained" line and, when there are fewer than 500
 * clusters, one FASTA file <prefix>-%03d per cluster.  Distances are scored on
 * the GPU through libswgpu.  Exits 1 on a failed file or GPU error.
 */
#include <stdio.h>
#include <stdlib.h>

#include "mnhn_dropin.h"

int main(int argc, char** argv) {
  dataset ds;
  float epsilon = 0.f;
  int minpts = 0;
  FILE* fasta_f;
  split_set set_of_clusters;

  if (argc < 4) {
    printf("Arguments are: \n"
           " [file] Sequences in FASTA \n"
           " Epsilon \n"
           " minPoints \n"
           " output-files prefix \n");
    return 1;
  }
  sscanf(argv[2], "%f", &epsilon);
  sscanf(argv[3], "%i", &minpts);
  if (NULL == (fasta_f = fopen(argv[1], "r"))) {
    printf("failed to open file %s\n", argv[1]);
    return 1;
  }
  ds = dataset_from_fasta(fasta_f);
  fclose(fasta_f);

  set_of_clusters = dbscan_SW(ds, epsilon, minpts);
  if (swgpu_last_dropin_status() != 0) return 1;

  printf("%u clusters obtained \n", set_of_clusters.n_clusters);
  /* the reference reads argv[4] unconditionally; without it no files are written here */
  if (set_of_clusters.n_clusters < 500 && argc > 4) create_cluster_files(argv[4], set_of_clusters, ds);
  free_sequences_from_dataset(ds);
  free_split_set_and_associated_clusters(set_of_clusters);
  return 0;
}
