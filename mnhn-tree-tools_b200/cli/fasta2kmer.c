/*
 * fasta2kmer <fasta> <k> <n_threads> <protein 0|1>
 *
 * Drop-in for the reference tool (fasta2kmer.c:8-44): the k-mer frequency
 * table of every sequence, "sequence_<i>" then tab-separated counts, on
 * stdout.  Counting and formatting run on the GPU through libswgpu; n_threads
 * is accepted and ignored.  Exits 1 on a failed file, an unsupported k or a
 * GPU error.
 */
#include <stdio.h>
#include <stdlib.h>

#include "mnhn_dropin.h"

int main(int argc, char** argv) {
  size_t length = 0;
  int n_threads = 1, protein = 0;
  if (argc < 5) {
    printf("Arguments are: \n"
           "  [file] fasta file \n"
           "  [int] kmer length \n"
           "  [int] number of threads \n"
           "  [int] protein ? if yes 1 otherwise 0) \n");
    return 1;
  }
  FILE* in = fopen(argv[1], "r");
  if (in == NULL) {
    printf("Could not open fasta file %s \n", argv[1]);
    return 1;
  }
  sscanf(argv[2], "%zu", &length);
  sscanf(argv[3], "%d", &n_threads);
  sscanf(argv[4], "%i", &protein);
  dataset ds = dataset_from_fasta(in);
  fclose(in);
  kmer_frequencies freq = frequencies_from_dataset(ds, length, n_threads, protein);
  int rc = swgpu_last_dropin_status() != 0;
  if (!rc) {
    write_kmer_base(stdout, freq);
    rc = swgpu_last_dropin_status() != 0;
  }
  free_kmer_frequencies(freq);
  free_sequences_from_dataset(ds);
  return rc;
}
