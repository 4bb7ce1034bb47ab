// The split-set tree consumers of cluster_io.c / volumes.c used by
// split_sets_to_newick.c, tree_pureness.c and filter_split_sets_by_min.c:
// layer trees built from the relations between consecutive layers, their
// Newick text, branch lengths from the densities of the sweep's eps values,
// and the pureness of a tree against a target split set.  Host code: these
// tools read split-set files the GPU sweep wrote.
//
// Output follows the reference, quirks included: print_tree writes the branch
// lengths with printf (to stdout) whatever stream it is given
// (cluster_io.c:229), and the hypersphere volume divides by glibc's gamma(),
// which is the logarithm of the gamma function (volumes.c:7).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "host_internal.h"

extern "C" double gamma(double);  // glibc: log|Gamma(x)|, as the reference links it

namespace {

void fail_status(int s) { swgpu::dropin_set_status(s); }

void print_tree_worker(FILE* f, tree_node* root) {
  if (root->child != nullptr) {
    fprintf(f, "(");
    for (tree_node* n = root->child; n != nullptr; n = n->neighbor) {
      if (n != root->child) fprintf(f, ",");
      print_tree_worker(f, n);
    }
    fprintf(f, ")");
  }
  fprintf(f, "%s", root->id);
  if (root->parent != nullptr) printf(":%f", root->length);
}

// Mismatch share of one cluster against the target clusters (cluster_io.c:237-270).
double pureness_helper(int layer, int this_cluster, int* inpures, split_set* s, split_set target) {
  cluster cur = s[layer].clusters[this_cluster];
  double inpureness = 0;
  int inpure = 0;
  for (int i = 0; i < target.n_clusters; i++) {
    cluster inter = intersection_of_clusters(cur, target.clusters[i]);
    if (inter.members != nullptr) free(inter.members);
    if (cur.n_members != inter.n_members && inter.n_members != 0) {
      inpure = 1;
      const int c = inter.n_members > cur.n_members / 2 ? cur.n_members - inter.n_members : inter.n_members;
      inpureness += (double)c / (double)cur.n_members;
    }
  }
  inpures[layer] += inpure;
  return inpureness;
}

void pureness_worker(double* pureness, int* inpures, tree_node* root, split_set* s, split_set target) {
  for (tree_node* n = root->child; n != nullptr; n = n->neighbor) pureness_worker(pureness, inpures, n, s, target);
  int layer = 0, this_cluster = 0;
  sscanf(root->id, "L%iC%i", &layer, &this_cluster);
  pureness[layer] += pureness_helper(layer, this_cluster, inpures, s, target);
}

}  // namespace

extern "C" {

double vol_hypersphere(int dimension, double epsilon) {
  const double d = (double)dimension;
  return pow(epsilon, d) * (pow(M_PI, d * 0.5) / gamma(d * 0.5 + 1));
}

double vol_hypercube(int dimension, double epsilon) {
  double vol = 1.;
  for (int i = 0; i < dimension; i++) vol *= epsilon;
  return vol;
}

double* array_deltas(double* array, int array_length) {
  double* diffs = (double*)malloc(sizeof(double) * (size_t)(array_length > 1 ? array_length - 1 : 1));
  for (int i = 0; i < array_length - 1; i++) diffs[i] = array[i] - array[i + 1];
  return diffs;
}

double* get_epsilon_dist_from_adaptive_clustering_output(FILE* f, int n_layers) {
  static const char initial_check[] = "epsilon_start:";
  static const char layer_check[] = "  Epsilon at layer";
  double* eps = (double*)malloc(sizeof(double) * (size_t)(n_layers > 0 ? n_layers : 1));
  int count = 0;
  char* line = nullptr;
  size_t cap = 0;
  rewind(f);
  while (getline(&line, &cap, f) != -1) {
    if (count == 0 && strncmp(line, initial_check, 14) == 0) {
      sscanf(line, "%*s %lf", eps);
      count = 1;
    }
    if (strncmp(line, layer_check, 17) != 0) continue;
    if (count < 1) {
      printf("Malformed output file epsilon_start not found before \n   Epsilon at layer: \n");
      free(line);
      free(eps);
      fail_status(SWE_ERR_IO);
      return nullptr;
    }
    if (count == n_layers) break;
    sscanf(line, "  %*s %*s %*s %*s %lf", eps + count);
    count++;
  }
  free(line);
  if (count < n_layers) {
    printf("Not enough layers in output file! \n");
    printf("Counted %i layers, requested %i layers! \n", count, n_layers);
    free(eps);
    fail_status(SWE_ERR_IO);
    return nullptr;
  }
  return eps;
}

double* densities_from_epsilons(int type, int dimensions, double* epsilons, int n_epsilons, int min_points) {
  double (*vol)(int, double) = nullptr;
  if (type == 1) vol = vol_hypercube;
  else if (type == 2) vol = vol_hypersphere;
  else {
    printf("Wrong parameter to densities_from_epsilon (min_points)\n");
    fail_status(SWE_ERR_INVALID);
    return nullptr;
  }
  double* dens = (double*)malloc(sizeof(double) * (size_t)(n_epsilons > 0 ? n_epsilons : 1));
  for (int i = 0; i < n_epsilons; i++) dens[i] = min_points / vol(dimensions, epsilons[i]);
  return dens;
}

tree_node* generate_tree(int n_layers, cluster_connections** c, split_set* sets, double* tree_lengths) {
  if (n_layers < 1 || !sets || sets[n_layers - 1].n_clusters < 1) {  // no root (the reference reads past its arrays)
    fail_status(SWE_ERR_INVALID);
    return nullptr;
  }
  tree_node** nodes = (tree_node**)malloc(sizeof(tree_node*) * (size_t)n_layers);
  for (int i = 0; i < n_layers; i++) {
    nodes[i] = (tree_node*)malloc(sizeof(tree_node) * (size_t)(sets[i].n_clusters > 0 ? sets[i].n_clusters : 1));
    for (int j = 0; j < sets[i].n_clusters; j++) {
      tree_node& t = nodes[i][j];
      t.id = nullptr;
      t.length = i == n_layers - 1 ? 0 : (tree_lengths ? tree_lengths[i] : 1);
      t.n_members = 0;
      t.child = t.neighbor = t.parent = nullptr;
    }
  }
  // children of cluster j of layer i: the clusters of layer i-1 it connects to
  for (int i = n_layers - 1; i > 0; i--) {
    for (int j = 0; j < sets[i].n_clusters; j++) {
      const cluster_connections& cc = c[i - 1][j];
      for (int k = 0; k < cc.n_connections; k++) {
        tree_node* cur = nodes[i - 1] + cc.connections[k];
        cur->parent = nodes[i] + j;
        cur->neighbor = k > 0 ? nodes[i - 1] + cc.connections[k - 1] : nullptr;
        cur->id = (char*)malloc(20);
        cur->n_members = sets[i - 1].clusters[cc.connections[k]].n_members;
        snprintf(cur->id, 20, "L%iC%iN%i", i - 1, cc.connections[k], cur->n_members);
      }
      if (cc.n_connections > 0) nodes[i][j].child = nodes[i - 1] + cc.connections[cc.n_connections - 1];
    }
  }
  tree_node* root = nodes[n_layers - 1];
  root->id = (char*)malloc(20);
  snprintf(root->id, 20, "L%iC%i", n_layers - 1, 0);
  free(nodes);
  return root;
}

split_set filtered_split_set_by_min_size(split_set s_in, int min_size) {
  split_set out;
  out.clusters = (cluster*)malloc(sizeof(cluster) * (size_t)(s_in.n_clusters > 0 ? s_in.n_clusters : 1));
  int count = 0;
  for (int i = 0; i < s_in.n_clusters; i++) {
    const int m = s_in.clusters[i].n_members;
    if (m < min_size) continue;
    cluster& c = out.clusters[count];
    c.n_members = m;
    c.id = count;  // the reference leaves the id unset (it is stored by store_split_set)
    c.members = (int*)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
    memcpy(c.members, s_in.clusters[i].members, sizeof(int) * (size_t)m);
    count++;
  }
  out.n_clusters = count;
  if (count > 0) out.clusters = (cluster*)realloc(out.clusters, sizeof(cluster) * (size_t)count);
  return out;
}

void print_tree(FILE* f, tree_node* root) {
  if (!root) return;
  print_tree_worker(f, root);
  fprintf(f, ";");
}

int pureness_from_tree(int n_layers, tree_node* root, split_set* s, split_set target, double** pureness_values,
                       int** inpure_clusters) {
  if (!root) return 1;
  double* pureness = (double*)calloc((size_t)(n_layers > 0 ? n_layers : 1), sizeof(double));
  int* inpures = (int*)calloc((size_t)(n_layers > 0 ? n_layers : 1), sizeof(int));
  if (!pureness || !inpures) {
    free(pureness);
    free(inpures);
    return 1;
  }
  pureness_worker(pureness, inpures, root, s, target);
  for (int i = 0; i < n_layers; i++) pureness[i] = inpures[i] > 0 ? pureness[i] / (double)inpures[i] : 0;
  *pureness_values = pureness;
  *inpure_clusters = inpures;
  return 0;
}

double* inpures_over_total_fraction(int n_layers, split_set* s, int* inpure_clusters) {
  double* fraction = (double*)malloc(sizeof(double) * (size_t)(n_layers > 0 ? n_layers : 1));
  for (int i = 0; i < n_layers; i++) fraction[i] = (double)inpure_clusters[i] / (double)s[i].n_clusters;
  return fraction;
}

double* clusters_in_layer_vs_target_clusters(int n_layers, split_set* s, split_set target) {
  double* f = (double*)malloc(sizeof(double) * (size_t)(n_layers > 0 ? n_layers : 1));
  for (int i = 0; i < n_layers; i++)
    f[i] = (double)abs(s[i].n_clusters - target.n_clusters) / (double)target.n_clusters;
  return f;
}

}  // extern "C"
