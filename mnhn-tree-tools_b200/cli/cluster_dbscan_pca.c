/*
 * cluster_dbscan_pca <fasta> <projections> <dimensions> <epsilon> <minpts>
 *                    <prefix> [values prefix]
 *
 * Drop-in for the reference tool (cluster_dbscan_pca.c:15-77): DBSCAN with the
 * squared-L2 distance over the projections, the "%u clusters obtained" line
 * and, below 500 clusters, one FASTA file <prefix>-%03d per cluster plus, with
 * a seventh argument, the members' projections in <values prefix>-%03d.
 * Exits 1 on a failed file or GPU error.
 */
#include <stdio.h>
#include <stdlib.h>

#include "mnhn_dropin.h"

int main(int argc, char** argv) {
  size_t dimensions = 0;
  float epsilon = 0.f;
  int minpts = 0;
  if (argc < 7) {
    printf("Arguments are: \n"
           " [file] Sequences in FASTA \n"
           " [file] Corresponding PCA from kmers \n"
           " dimensions: dimensions in projections file \n"
           " Epsilon \n"
           " minPoints \n"
           " output-files prefix (FASTA) \n"
           " optional: out-files with values (Projections)\n");
    return 1;
  }
  sscanf(argv[3], "%zu", &dimensions);
  sscanf(argv[4], "%f", &epsilon);
  sscanf(argv[5], "%i", &minpts);
  FILE* fasta_f = fopen(argv[1], "r");
  if (fasta_f == NULL) {
    printf("failed to open file %s\n", argv[1]);
    return 1;
  }
  dataset ds = dataset_from_fasta(fasta_f);
  fclose(fasta_f);
  FILE* projection_f = fopen(argv[2], "r");
  if (projection_f == NULL) {
    printf("failed to open file %s\n", argv[2]);
    return 1;
  }
  load_projections_from_file_into_dataset(projection_f, dimensions, &ds);
  fclose(projection_f);
  if (swgpu_last_dropin_status() != 0) return 1;
  split_set set_of_clusters = dbscan_L2(ds, epsilon, minpts);
  if (swgpu_last_dropin_status() != 0) return 1;
  printf("%u clusters obtained \n", set_of_clusters.n_clusters);
  if (set_of_clusters.n_clusters < 500) {
    create_cluster_files(argv[6], set_of_clusters, ds);
    if (argc == 8) create_cluster_files_with_values(argv[7], set_of_clusters, ds);
  }
  free_split_set_and_associated_clusters(set_of_clusters);
  free_dataset(ds);
  return 0;
}
