/*
 * Drop-in entry points: the functions of MNHN-Tree-Tools' Smith-Waterman path,
 * with the reference's names and CPU-build signatures, exported by
 * libswgpu.so.  A caller written against the reference (cluster_dbscan_SW.c,
 * adaptive_clustering.c, find_closest_sequence_SW.c, filter.c, comparison.c,
 * fasta2kmer.c) links against libswgpu.so instead of smith_waterman.o,
 * dbscan_SW.o, dataset.o, cluster_io.o and kmers.o.  All distance work runs on the GPU; there is no
 * CPU fallback.  When no usable GPU is present the functions print an error
 * and return the empty result documented below.
 *
 * Each declaration names the reference interface it replaces.
 */
#ifndef MNHN_DROPIN_H
#define MNHN_DROPIN_H

#include <stdio.h>
#include "mnhn_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* smith-waterman.h:1 / smith-waterman.c:16-80.  Distance 4*max(len_a,len_b)
   minus the best linear-gap local alignment score of A[1..len_a] against
   B[1..len_b] (+4 match, -4 mismatch, -3 gap).  A and B must be readable at
   [0..len].  `work` is accepted and ignored.  Returns UINT_MAX on a GPU error. */
unsigned int score(char* A, char* B, size_t len_a, size_t len_b, int* work);

/* dataset.c:264-344.  FASTA records; first token of every sequence line,
   upper-cased; a line without a token repeats the previous token. */
dataset dataset_from_fasta(FILE* in);

/* dataset.c (free_sequences_from_dataset): frees the sequences and lengths. */
void free_sequences_from_dataset(dataset ds);

/* dbscan.h:30 / dbscan.c:950-1047.  DBSCAN over the Smith-Waterman distance
   ((float)d <= epsilon), seed test minpts < |N|, expansion test |N| >= minpts,
   clusters and members in the reference's traversal order.  epsilon == -1
   becomes 0.015 and minpts == -1 becomes 5 (dbscan.c:980-989).  All pair
   distances of a dataset are scored once on the GPU and reused by later calls
   on the same sequences.  Returns {0, NULL} on a GPU error. */
split_set dbscan_SW(dataset ds, float epsilon, int minpts);

/* dbscan.h:28-29 / dbscan.c:563-779, 950-1047.  DBSCAN over ds.values
   (values[dimension][point], n_dimensions x n_values) with the L1 distance
   (neighbours: d <= epsilon) or the squared L2 distance (d <= epsilon*epsilon),
   accumulated in float over the dimensions in order as the reference's
   AVX/FMA build does; same defaults, seed and expansion rules and cluster
   order as dbscan_SW.  The distances of a point set are computed once on the
   GPU and reused by later calls on the same values.  Returns {0, NULL} on a
   GPU error. */
split_set dbscan_L1(dataset ds, float epsilon, int minpts);
split_set dbscan_L2(dataset ds, float epsilon, int minpts);

/* dbscan.h:72-81 / dbscan.c:1117-1380.  Adaptive eps sweep: halving search for
   a start with more than one cluster, eps += inc until one cluster remains,
   layers kept when their cluster count strictly drops, log lines on stdout,
   split sets written to <prefix>%04d.  When `dbscanner` is dbscan_SW,
   dbscan_L1 or dbscan_L2 the distances are computed once for the whole
   sweep.  Layers are produced in eps
   order whatever `n_threads` is.  Where the reference calls _exit(1) this
   function prints the same message and returns; swgpu_last_dropin_status()
   then returns non-zero. */
void adaptive_dbscan(split_set (*dbscanner)(dataset, float, int), dataset ds, float epsilon_start,
                     float epsilon_inc, int minpts, char* split_files_prefix, int n_threads);

/* cluster_io.c:638-669: "SPLIT_SET", int32 n_clusters, then per cluster
   int32 n_members, int32 id, int32 members[]; opened without O_TRUNC. */
void store_split_set(char* filename, split_set s);

/* cluster_io.c:595-636. */
split_set read_split_set(char* filename);

/* cluster_io.c:672-699: records ">sequence_<idx>", 50 characters per line. */
void create_single_cluster_file(char* filename, cluster cl, dataset ds);

/* cluster_io.c:701-720: one file <prefix>-%03d per cluster. */
void create_cluster_files(char* prefix, split_set s, dataset ds);

/* cluster_io.c:564-593: ascending indices that belong to no cluster. */
cluster data_not_in_clusters(split_set s, dataset ds);

/* cluster_io.c:446-501.  The larger cluster (a on ties) is sorted in place
   when it has more than 20 members, as in the reference. */
cluster intersection_of_clusters(cluster a, cluster b);

/* cluster_io.c:407-444: new cluster i is connected to ancient cluster j when
   |j ∩ i| > 0.8 |j|.  Returns new_set.n_clusters entries. */
cluster_connections* generate_split_set_relation(split_set ancient, split_set new_set);

/* cluster_io.c:722-729. */
void free_split_set_and_associated_clusters(split_set s);

/* ---- callers of score() around the path (comparison.h, filter.h, dataset.h) ----
   Two datasets are scored in one pass on the GPU; results equal the
   reference's single-threaded results (n_threads only sets the reference's
   thread count and is ignored here). */

/* comparison.c:84-112: n1 x n2 distances, row i = ds_one[i]; malloc'd. */
unsigned long* smith_waterman_distances_matrix(dataset ds_one, dataset ds_two);
/* comparison.c:156-193: mean distance over ds_one x ds_two. */
double mean_from_smith_waterman_datasets(dataset ds_one, dataset ds_two, size_t n_threads);
/* comparison.c:241-280: sqrt(sum of the integer parts of (d - mean)^2) / (n1 + n2). */
double sigma_from_smith_waterman_datasets(double mean, dataset ds_one, dataset ds_two, size_t n_threads);
/* comparison.c:20-82, 282-323: mean silhouette of ds_one against ds_two. */
double silhouette_from_smith_waterman_datasets(dataset ds_one, dataset ds_two, size_t n_threads);
/* comparison.c:325-350, 388-403: statistics of a caller's matrix (host). */
double mean_from_smith_waterman_distance_matrix(unsigned long* matrix, dataset ds_one, dataset ds_two);
double sigma_from_smith_waterman_distance_matrix(unsigned long* matrix, double mean, dataset ds_one,
                                                 dataset ds_two);
void shortest_longest_distance_in_matrix(unsigned long* matrix, unsigned long* shortest, unsigned long* largest,
                                         dataset ds_one, dataset ds_two);
/* comparison.c:352-386: "i j SW L1 L2" lines for every pair j < i (the L2
   column first, as the reference prints it). */
void print_SW_PCA_L_comparison(FILE* f, dataset ds);
/* filter.c:18-50: sequences with size - minus <= length <= size + plus. */
dataset filter_ds_by_size(dataset in_set, size_t size, size_t plus, size_t minus);
/* filter.c:52-140: sequences within max_distance of target (one query on the GPU). */
dataset filter_by_SW_distance(dataset in_set, char* target, size_t target_length, unsigned int max_distance,
                              int n_threads);
/* dataset.c:85-110: ">sequence_<j>" records, 50 symbols per line. */
void dataset_to_fasta(FILE* f, dataset ds);
/* dataset.c:427-471: `dimensions` floats per sequence into ds->values[dimension][sequence]. */
void load_projections_from_file_into_dataset(FILE* projections, size_t dimensions, dataset* ds);

/* ---- point datasets of the k-mer / PCA DBSCAN tools (dataset.h, cluster.h) ---- */

/* dataset.c:346-381: n_features = tabs in the first line, n_samples =
   newlines from the end of the first line on. */
data_shape shape_from_kmer_file(int infile);
/* dataset.c:384-425: a label then n_features numbers per sample into
   values[feature][sample] (32-byte aligned rows); other fields zeroed. */
dataset load_kmer_from_file_into_dataset(FILE* in_file, data_shape shape);
/* kmer2pca.c:255-268 (data_from_file): the same token stream read as doubles
   ("%lf") into data[sample * n_features + feature], kmer2pca's row-major
   in_data.  Returns 0, or an swe_status when a value is not a number or the
   file ends early (where the reference leaves values unset). */
int swe_read_feature_table(FILE* in_file, data_shape shape, double* data);
/* dataset.c:629-635, 646-649. */
void free_values_from_dataset(dataset ds);
void free_dataset(dataset ds);
/* cluster_io.c:343-379: per member its values, "%f" tab separated, one line
   each; files <prefix>-%03d. */
void create_single_cluster_file_with_values(char* filename, cluster cl, dataset ds);
void create_cluster_files_with_values(char* prefix, split_set s, dataset ds);

/* ---- split-set trees (cluster.h, volumes.h): split_sets_to_newick, tree_pureness ---- */

/* cluster_io.c:124-189: the tree of n_layers split sets linked by the
   relations c[i-1] = generate_split_set_relation(sets[i-1], sets[i]); branch
   lengths tree_lengths[layer] (1 when NULL, 0 for the last layer).  Returns
   the first node of the last layer. */
tree_node* generate_tree(int n_layers, cluster_connections** c, split_set* sets, double* tree_lengths);
/* cluster_io.c:217-235: Newick text to f; the ":length" parts go to stdout,
   as in the reference. */
void print_tree(FILE* f, tree_node* root);
/* cluster_io.c:191-215: clusters with at least min_size members (ids renumbered). */
split_set filtered_split_set_by_min_size(split_set s_in, int min_size);
/* cluster_io.c:14-24: array[i] - array[i+1] (array_length - 1 values, malloc'd). */
double* array_deltas(double* array, int array_length);
/* cluster_io.c:26-93: epsilon_start and the "Epsilon at layer" values of an
   adaptive-clustering log (n_layers values); NULL (with a message) where the
   reference exits. */
double* get_epsilon_dist_from_adaptive_clustering_output(FILE* f, int n_layers);
/* cluster_io.c:95-122: min_points / volume(eps) with the hypercube (type 1)
   or hypersphere (type 2) volume of volumes.c. */
double* densities_from_epsilons(int type, int dimensions, double* epsilons, int n_epsilons, int min_points);
double vol_hypersphere(int dimension, double epsilon);
double vol_hypercube(int dimension, double epsilon);
/* cluster_io.c:237-340: per-layer pureness against a target split set, the
   impure clusters per layer, and the layer/target cluster-count factors. */
int pureness_from_tree(int n_layers, tree_node* root, split_set* s, split_set target, double** pureness_values,
                       int** inpure_clusters);
double* inpures_over_total_fraction(int n_layers, split_set* s, int* inpure_clusters);
double* clusters_in_layer_vs_target_clusters(int n_layers, split_set* s, split_set target);

/* ---- fasta2kmer (kmers.h) ---- */

/* kmers.c:292-371: one row of swe_kmer_count(kmer_length, protein) counts per
   sequence (malloc'd rows), computed on the GPU over strlen(sequence) bytes;
   semantics of swe_kmer_counts.  n_threads is ignored.  kmer_length must be
   1..15 (DNA) or 1..7 (protein); otherwise, or on a GPU error, the result has
   frequencies == NULL and n_seq == 0. */
kmer_frequencies frequencies_from_dataset(dataset ds, size_t kmer_length, int n_threads, int protein);
/* kmers.c:373-385: "sequence_<i>" and the row's counts as "%hi", tab
   separated, one line per sequence; the text is formatted on the GPU. */
void write_kmer_base(FILE* f, kmer_frequencies freq);
/* kmers.c:387-396. */
void free_kmer_frequencies(kmer_frequencies freq);

/* Status of the last drop-in call that can fail without a return code
   (adaptive_dbscan, dbscan_SW, score and the calls above): 0 on success, else
   an swe_status. */
int swgpu_last_dropin_status(void);

#ifdef __cplusplus
}
#endif
#endif /* MNHN_DROPIN_H */
