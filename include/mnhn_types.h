/*
 * Data structures of MNHN-Tree-Tools' Smith-Waterman path, with the field
 * layout of the reference so that reference-style callers link unchanged.
 *
 *   dataset              dataset.h:27-35
 *   cluster              cluster.h:10-15
 *   split_set            cluster.h:20-23
 *   cluster_connections  cluster.h:28-31
 *   neighbors            dbscan.h:5-8
 *   kmer_frequencies     kmers.h:17-21
 *   data_shape           dataset.h:37-40
 *   tree_node            cluster.h:41-48
 *
 * Ownership follows the reference: arrays inside returned structs come from
 * malloc and are released with free() (free_split_set_and_associated_clusters,
 * cluster_io.c:722-729, and free_sequences_from_dataset).
 */
#ifndef MNHN_TYPES_H
#define MNHN_TYPES_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  char** sequences;          /* NUL-terminated, upper-cased sequences */
  size_t* sequence_lengths;  /* strlen of each sequence */
  void** binary_sequences;   /* unused on this path */
  int n_values;              /* number of sequences */
  float** values;            /* values[dimension][point] (k-mer / PCA DBSCAN) */
  int n_dimensions;          /* number of dimensions of values */
  size_t max_sequence_length;
} dataset;

typedef struct {
  int* members;   /* dataset indices, in the order DBSCAN reached them */
  int n_members;
  int id;         /* position of the cluster in its split set */
} cluster;

typedef struct {
  int n_clusters;
  cluster* clusters;
} split_set;

typedef struct {
  int* connections;
  int n_connections;
} cluster_connections;

typedef struct {
  int* members;   /* ascending dataset indices, the query point included */
  int n_members;
} neighbors;

/* dataset.h:37-40: columns and rows of a k-mer table file. */
typedef struct {
  size_t n_features;
  size_t n_samples;
} data_shape;

/* cluster.h:41-48: a node of the layer tree (id "L<layer>C<cluster>N<members>",
   the root "L<layer>C0"; length of the branch to the parent). */
typedef struct tree_node {
  char* id;
  double length;
  int n_members;
  struct tree_node* child;
  struct tree_node* neighbor;
  struct tree_node* parent;
} tree_node;

/* kmers.h:17-21: frequencies[sequence][k-mer index], one malloc'd row per
   sequence (free_kmer_frequencies releases them). */
typedef struct {
  short int** frequencies;
  size_t n_kmers;
  size_t n_seq;
} kmer_frequencies;

#ifdef __cplusplus
}
#endif
#endif /* MNHN_TYPES_H */
