/*
 * split_sets_to_newick <min_members> <lengths 0|1|2> [<dimensions> <log> <min_pts>] <split_set...>
 *
 * Drop-in for the reference tool (split_sets_to_newick.c:16-122): the tree of
 * the given layers (lowest eps first) in Newick form on stdout.  With
 * min_members > 0 smaller clusters are dropped first; with lengths 1 or 2 the
 * branch lengths are the differences of min_pts / volume(eps) between layers
 * (hypercube or hypersphere volume in `dimensions`), the eps values read from
 * the adaptive-clustering log.  Exits 1 on a bad file.
 */
#include <stdio.h>
#include <stdlib.h>

#include "mnhn_dropin.h"

int main(int argc, char** argv) {
  int min_members = 0, lengths_mode = 0, dimensions = 0, min_pts = 0;
  if (argc < 4) {
    printf("Arguments are: \n"
           " [int] filter for small clusters 0 = no filter \n"
           "                                 n = minimum of n members in cluster \n"
           " [int] lengths from outputfile 0 = no file \n"
           "                               1 = L1-density (min_pts/hypercube)\n"
           "                               2 = L2-density (min_pts/hypersphere)\n"
           " [int] dimensions for density omitted if lengths = 0 \n"
           " [outfile] clustering run outfile if lengths = (1 or 2) \n"
           " [int] points for density calculations i.e. what min_pts you used\n"
           " [file1 ... filen] split_sets obtainted from adaptive clustering \n"
           "                   calculations in order from lowest to hight\n");
    return 1;
  }
  sscanf(argv[1], "%i", &min_members);
  sscanf(argv[2], "%i", &lengths_mode);
  const int first = lengths_mode ? 6 : 3;
  if (lengths_mode) {
    if (argc < 7) {
      printf("Arguments missing for branch lengths\n");
      return 1;
    }
    sscanf(argv[3], "%i", &dimensions);
    sscanf(argv[5], "%i", &min_pts);
  }
  const int n_sets = argc - first;
  if (n_sets < 1) return 1;
  split_set* s = (split_set*)malloc(sizeof(split_set) * (size_t)n_sets);
  for (int i = 0; i < n_sets; i++) {
    s[i] = read_split_set(argv[first + i]);
    if (swgpu_last_dropin_status() != 0) return 1;
  }
  double* lengths = NULL;
  if (lengths_mode) {
    FILE* out_f = fopen(argv[4], "r");
    if (out_f == NULL) {
      printf("failed to open file %s\n", argv[4]);
      return 1;
    }
    double* eps = get_epsilon_dist_from_adaptive_clustering_output(out_f, n_sets);
    fclose(out_f);
    if (eps == NULL) return 1;
    double* dens = densities_from_epsilons(lengths_mode, dimensions, eps, n_sets, min_pts);
    free(eps);
    if (dens == NULL) return 1;
    lengths = array_deltas(dens, n_sets);
    free(dens);
  }
  if (min_members) {
    for (int i = 0; i < n_sets; i++) {
      split_set f = filtered_split_set_by_min_size(s[i], min_members);
      free_split_set_and_associated_clusters(s[i]);
      s[i] = f;
    }
  }
  cluster_connections** c = (cluster_connections**)malloc(sizeof(cluster_connections*) * (size_t)n_sets);
  for (int i = 1; i < n_sets; i++) c[i - 1] = generate_split_set_relation(s[i - 1], s[i]);
  tree_node* root = generate_tree(n_sets, c, s, lengths);
  print_tree(stdout, root);
  for (int i = 0; i < n_sets; i++) free_split_set_and_associated_clusters(s[i]);
  free(s);
  return 0;
}
