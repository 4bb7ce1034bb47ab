/*
 * adaptive_clustering_kmer_L1 / adaptive_clustering_kmer_L2
 *     <kmer file> <eps_start> <eps_inc> <minpts> <prefix> <n_threads>
 * adaptive_clustering_PCA
 *     <fasta> <eps_start> <eps_inc> <minpts> <prefix> <n_threads> <dimensions> <projections>
 *
 * Drop-ins for the reference tools built from adaptive_clustering.c:54-200
 * with -D_CLUSTER_KMER_L1, -D_CLUSTER_KMER_L2 or -D_CLUSTER_PCA (this source
 * builds all three: -DPOINTS_KMER_L1, -DPOINTS_KMER_L2 or -DPOINTS_PCA): the
 * same arguments, "Dataset read!" line, adaptive log on stdout and
 * <prefix>%04d split-set files, with every point distance computed once on
 * the GPU for the whole sweep.  Fewer arguments than the reference reads print
 * the usage text.  Exits 1 where the reference calls _exit(1).
 */
#define _POSIX_C_SOURCE 200809L /* fdopen */
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <unistd.h>

#include "mnhn_dropin.h"

static void print_arguments(void) {
  printf("Arguments are: \n"
#ifdef POINTS_PCA
         "   [file] FASTA file containing sequence dataset \n"
#else
         "   [file] kmer file\n"
#endif
         "   (float) initial epsilon value \n"
         "   (float) epsilon increase between cluster search \n"
         "   (int) minimum numbers of clusters in epsilon neigbourhood \n"
         "   (string) path/andprefix of split_set_files \n"
         "   (int) number of threads to use \n"
#ifdef POINTS_PCA
         "   (int) dimensions in projection file (PCA obtained from kmers)\n"
         "   [FILE] PCA projections file obtained i.e. from kers\n"
#endif
  );
}

int main(int argc, char** argv) {
  dataset ds;
  float epsilon_start = 0.f, epsilon_inc = 0.f;
  int minpts = 0, n_threads = 1;
  char split_files_prefix[4096];
#ifdef POINTS_PCA
  const int need = 9;
#else
  const int need = 7;
#endif
  if (argc < need) {
    print_arguments();
    return 1;
  }
  sscanf(argv[2], "%f", &epsilon_start);
  sscanf(argv[3], "%f", &epsilon_inc);
  sscanf(argv[4], "%i", &minpts);
  split_files_prefix[0] = 0;
  sscanf(argv[5], "%4095s", split_files_prefix);
  sscanf(argv[6], "%i", &n_threads);
#ifdef POINTS_PCA
  int dimensions = 0;
  sscanf(argv[7], "%i", &dimensions);
  FILE* fasta_f = fopen(argv[1], "r");
  if (fasta_f == NULL) {
    printf("failed to open file %s\n", argv[1]);
    return 1;
  }
  ds = dataset_from_fasta(fasta_f);
  fclose(fasta_f);
  FILE* projection_f = fopen(argv[8], "r");
  if (projection_f == NULL) {
    printf("failed to open file %s\n", argv[8]);
    return 1;
  }
  load_projections_from_file_into_dataset(projection_f, (size_t)dimensions, &ds);
  fclose(projection_f);
#else
  int kmer_fd = open(argv[1], O_RDONLY);
  if (kmer_fd == -1) {
    printf("failed to open file %s\n", argv[1]);
    return 1;
  }
  data_shape shape = shape_from_kmer_file(kmer_fd);
  FILE* kmer_f = fdopen(kmer_fd, "r");
  ds = load_kmer_from_file_into_dataset(kmer_f, shape);
  fclose(kmer_f);
#endif
  if (swgpu_last_dropin_status() != 0) return 1;
  printf("Dataset read!\n");

#ifdef POINTS_KMER_L1
  adaptive_dbscan(dbscan_L1, ds, epsilon_start, epsilon_inc, minpts, split_files_prefix, n_threads);
#else
  adaptive_dbscan(dbscan_L2, ds, epsilon_start, epsilon_inc, minpts, split_files_prefix, n_threads);
#endif
  fflush(stdout);
  if (swgpu_last_dropin_status() != 0) return 1;
#ifdef POINTS_PCA
  free_dataset(ds);
#else
  free_values_from_dataset(ds);
#endif
  return 0;
}
