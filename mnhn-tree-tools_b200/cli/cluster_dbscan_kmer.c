/*
 * cluster_dbscan_kmerL1 / cluster_dbscan_kmerL2
 *     <fasta> <kmer file> <epsilon> <minpts> <prefix>
 *
 * Drop-in for the reference tools (cluster_dbscan_kmer.c:19-71, built with
 * _CLUSTER_KMER_L1 or _CLUSTER_KMER_L2): DBSCAN over the rows of a fasta2kmer
 * table with the L1 or squared-L2 distance, the "%u clusters obtained" line
 * and, below 500 clusters, one FASTA file <prefix>-%03d per cluster.  This
 * source builds both tools (-DKMER_L1 selects L1).  Exits 1 on a failed file
 * or GPU error.
 */
#define _POSIX_C_SOURCE 200809L /* fdopen */
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <unistd.h>

#include "mnhn_dropin.h"

int main(int argc, char** argv) {
  float epsilon = 0.f;
  int minpts = 0;
  if (argc < 6) {
    printf("Arguments are: \n"
           " [file] Sequences in FASTA \n"
           " [file] Corresponding kmers \n"
           " Epsilon \n"
           " minPoints \n"
           " output-files prefix \n");
    return 1;
  }
  sscanf(argv[3], "%f", &epsilon);
  sscanf(argv[4], "%i", &minpts);
  int kmer_fd = open(argv[2], O_RDONLY);
  if (kmer_fd == -1) {
    printf("failed to open file %s\n", argv[2]);
    return 1;
  }
  data_shape shape = shape_from_kmer_file(kmer_fd);
  FILE* kmer_f = fdopen(kmer_fd, "r");
  dataset ds = load_kmer_from_file_into_dataset(kmer_f, shape);
  fclose(kmer_f);
#ifdef KMER_L1
  split_set set_of_clusters = dbscan_L1(ds, epsilon, minpts);
#else
  split_set set_of_clusters = dbscan_L2(ds, epsilon, minpts);
#endif
  free_values_from_dataset(ds);
  if (swgpu_last_dropin_status() != 0) return 1;
  printf("%u clusters obtained \n", set_of_clusters.n_clusters);

  FILE* fasta_f = fopen(argv[1], "r");
  if (fasta_f == NULL) {
    printf("failed to open file %s\n", argv[1]);
    return 1;
  }
  ds = dataset_from_fasta(fasta_f);
  fclose(fasta_f);
  if (set_of_clusters.n_clusters < 500) create_cluster_files(argv[5], set_of_clusters, ds);
  free_sequences_from_dataset(ds);
  free_split_set_and_associated_clusters(set_of_clusters);
  return 0;
}
