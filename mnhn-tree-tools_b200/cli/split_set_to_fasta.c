/*
 * split_set_to_fasta <fasta> <split_set> <prefix>
 *
 * Drop-in for the reference tool (split_set_to_fasta.c:9-31): one FASTA file
 * <prefix>-%03d per cluster of the split set.  Exits 1 on a bad file.
 */
#include <stdio.h>

#include "mnhn_dropin.h"

int main(int argc, char** argv) {
  if (argc < 4) {
    printf("Arguments are: \n"
           "   1. [file] fasta file of complete dataset\n"
           "   2. [file] file containing the cluster set\n"
           "   3. path prefix where clusters should be stored to\n");
    return 1;
  }
  FILE* f = fopen(argv[1], "r");
  if (f == NULL) {
    printf("failed to open file %s\n", argv[1]);
    return 1;
  }
  split_set s = read_split_set(argv[2]);
  if (swgpu_last_dropin_status() != 0) return 1;
  dataset ds = dataset_from_fasta(f);
  fclose(f);
  create_cluster_files(argv[3], s, ds);
  free_split_set_and_associated_clusters(s);
  free_sequences_from_dataset(ds);
  return 0;
}
