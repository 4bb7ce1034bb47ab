/*
 * tree_pureness <fasta> <target split_set> <split_set...>
 *
 * Drop-in for the reference tool (tree_pureness.c:15-71): for every layer of
 * the tree of the given split sets, "pureness<TAB>cluster factor<TAB>impure
 * fraction" against the target split set.  Exits 1 on a bad file.
 */
#include <stdio.h>
#include <stdlib.h>

#include "mnhn_dropin.h"

int main(int argc, char** argv) {
  if (argc < 4) {
    printf("Arguments are: \n"
           "  [fasta] database of sequences the split sets are refering to \n"
           "  [split-set] target split set for purness evaluation \n"
           "  [split_sets...] cluster files corresponding to a tree \n");
    return 1;
  }
  FILE* fasta_f = fopen(argv[1], "r");
  if (fasta_f == NULL) {
    printf("failed to open file %s\n", argv[1]);
    return 1;
  }
  dataset ds = dataset_from_fasta(fasta_f);
  fclose(fasta_f);
  const int n_sets = argc - 3;
  split_set* s = (split_set*)malloc(sizeof(split_set) * (size_t)n_sets);
  for (int i = 0; i < n_sets; i++) {
    s[i] = read_split_set(argv[3 + i]);
    if (swgpu_last_dropin_status() != 0) return 1;
  }
  split_set target = read_split_set(argv[2]);
  if (swgpu_last_dropin_status() != 0) return 1;
  cluster_connections** c = (cluster_connections**)malloc(sizeof(cluster_connections*) * (size_t)n_sets);
  for (int i = 1; i < n_sets; i++) c[i - 1] = generate_split_set_relation(s[i - 1], s[i]);
  tree_node* root = generate_tree(n_sets, c, s, NULL);
  double* pureness = NULL;
  int* inpure = NULL;
  if (pureness_from_tree(n_sets, root, s, target, &pureness, &inpure) != 0) return 1;
  double* factors = clusters_in_layer_vs_target_clusters(n_sets, s, target);
  double* fraction = inpures_over_total_fraction(n_sets, s, inpure);
  for (int i = 0; i < n_sets; i++) printf("%lf\t%lf\t%lf\n", pureness[i], factors[i], fraction[i]);
  free_sequences_from_dataset(ds);
  return 0;
}
