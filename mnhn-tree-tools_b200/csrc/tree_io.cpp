// Split-set trees for split_sets_to_newick.c, tree_pureness.c and
// filter_split_sets_by_min.c (the tree part of cluster_io.c and volumes.c),
// written from their output contracts.  Host code: the tools read split-set
// files the GPU sweep wrote.
//
// The tree.  The kept layers 0 .. n-1 of a sweep are linked by relation
// tables: c[L-1][k] lists the clusters of layer L-1 that cluster k of layer L
// absorbed.  Node (L, k) is the parent of those clusters; its children are
// listed in reverse table order (last connection first).  The root is cluster
// 0 of layer n-1.  A non-root node is labelled L<layer>C<cluster>N<members>
// and the root L<layer>C0; a node of layer L < n-1 carries the branch length
// tree_lengths[L] (1 without lengths), the root 0.
//
// Newick text:  node := [ "(" node { "," node } ")" ] label [ ":" length ],
// then ";".  The length is written "%f" to stdout whatever stream the text
// goes to, as the reference's printer does (cluster_io.c:229); the tool
// prints to stdout, so the text is one stream there.
//
// Pureness of layer L against a target split set: a cluster C of layer L
// that the tree reaches is impure when some target cluster T holds part but
// not all of it; its impurity is the sum over those T, in target order, of
// share(T) / |C| with share(T) = |C n T| when |C n T| <= |C|/2 (integer
// halves) and |C| - |C n T| otherwise.  pureness[L] = (sum of the impurities
// of layer L's impure clusters, added in the order a post-order walk of the
// tree meets them) / (number of impure clusters), 0 when there are none.
//
// The hypersphere volume divides by glibc's gamma(), which returns the
// logarithm of the gamma function (volumes.c:7); the densities keep that.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "host_internal.h"

extern "C" double gamma(double);  // glibc: log|Gamma(x)|, as the reference links it

namespace {

void fail_status(int s) { swgpu::dropin_set_status(s); }

constexpr size_t LABEL_BYTES = 40;

// Nodes of the tree in the order a post-order walk meets them (children in
// list order before their parent), without recursion.
std::vector<const tree_node*> post_order(const tree_node* root) {
  std::vector<const tree_node*> out, pending{root};
  std::vector<const tree_node*> rev;  // reverse post-order: node, then children from the last
  while (!pending.empty()) {
    const tree_node* n = pending.back();
    pending.pop_back();
    rev.push_back(n);
    for (const tree_node* ch = n->child; ch != nullptr; ch = ch->neighbor) pending.push_back(ch);
  }
  out.assign(rev.rbegin(), rev.rend());
  return out;
}

// True when no cluster of s repeats a member and no member sits in two
// clusters; fills owner[point] with the cluster holding it (-1: none).
bool owners_of(const split_set& s, std::vector<int>& owner) {
  int top = -1;
  for (int t = 0; t < s.n_clusters; ++t)
    for (int k = 0; k < s.clusters[t].n_members; ++k) {
      const int m = s.clusters[t].members[k];
      if (m < 0) return false;
      top = std::max(top, m);
    }
  owner.assign((size_t)top + 1, -1);
  for (int t = 0; t < s.n_clusters; ++t)
    for (int k = 0; k < s.clusters[t].n_members; ++k) {
      int& o = owner[(size_t)s.clusters[t].members[k]];
      if (o != -1) return false;
      o = t;
    }
  return true;
}

bool distinct_members(const cluster& c, std::vector<uint8_t>& mark) {
  for (int k = 0; k < c.n_members; ++k)
    if (c.members[k] < 0) return false;
  bool ok = true;
  for (int k = 0; k < c.n_members; ++k) {
    const size_t m = (size_t)c.members[k];
    if (m >= mark.size()) mark.resize(m + 1, 0);
    if (mark[m]) ok = false;
    mark[m] = 1;
  }
  for (int k = 0; k < c.n_members; ++k) mark[(size_t)c.members[k]] = 0;
  return ok;
}

double share_of(int inter, int size) {
  const int part = inter > size / 2 ? size - inter : inter;
  return (double)part / (double)size;
}

}  // namespace

extern "C" {

double vol_hypersphere(int dimension, double epsilon) {
  const double d = (double)dimension;
  const double unit_ball = pow(M_PI, d * 0.5) / gamma(d * 0.5 + 1.0);  // rounded as volumes.c:7 groups it
  return pow(epsilon, d) * unit_ball;
}

double vol_hypercube(int dimension, double epsilon) {
  double v = 1.0;
  for (int d = dimension; d > 0; --d) v *= epsilon;
  return v;
}

double* array_deltas(double* array, int array_length) {
  const int n = array_length > 1 ? array_length - 1 : 0;
  double* d = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int k = 0; k < n; ++k) d[k] = array[k] - array[k + 1];
  return d;
}

// The sweep's log (adaptive_dbscan's stdout): "epsilon_start: <e>" gives the
// first value, each "  Epsilon at layer <k> <..> <e>" line the next one.
double* get_epsilon_dist_from_adaptive_clustering_output(FILE* f, int n_layers) {
  static const char start_tag[] = "epsilon_start:";
  static const char layer_tag[] = "  Epsilon at layer";
  double* eps = (double*)malloc(sizeof(double) * (size_t)(n_layers > 0 ? n_layers : 1));
  int got = 0;
  char* line = nullptr;
  size_t cap = 0;
  rewind(f);
  while (got < n_layers && getline(&line, &cap, f) != -1) {
    if (got == 0 && strncmp(line, start_tag, sizeof(start_tag) - 1) == 0) {
      sscanf(line, "%*s %lf", &eps[0]);
      got = 1;
    }
    if (strncmp(line, layer_tag, sizeof(layer_tag) - 2) != 0) continue;
    if (got == 0) {
      printf("Malformed output file epsilon_start not found before \n   Epsilon at layer: \n");
      free(line);
      free(eps);
      fail_status(SWE_ERR_IO);
      return nullptr;
    }
    if (got < n_layers) sscanf(line, "  %*s %*s %*s %*s %lf", &eps[got++]);
  }
  free(line);
  if (got < n_layers) {
    printf("Not enough layers in output file! \n");
    printf("Counted %i layers, requested %i layers! \n", got, n_layers);
    free(eps);
    fail_status(SWE_ERR_IO);
    return nullptr;
  }
  return eps;
}

double* densities_from_epsilons(int type, int dimensions, double* epsilons, int n_epsilons, int min_points) {
  if (type != 1 && type != 2) {
    printf("Wrong parameter to densities_from_epsilon (min_points)\n");
    fail_status(SWE_ERR_INVALID);
    return nullptr;
  }
  double* dens = (double*)malloc(sizeof(double) * (size_t)(n_epsilons > 0 ? n_epsilons : 1));
  for (int k = 0; k < n_epsilons; ++k) {
    const double v = type == 1 ? vol_hypercube(dimensions, epsilons[k]) : vol_hypersphere(dimensions, epsilons[k]);
    dens[k] = min_points / v;
  }
  return dens;
}

// All nodes of every layer in one block (the reference's callers never free
// a tree), labels in a second block.
tree_node* generate_tree(int n_layers, cluster_connections** c, split_set* sets, double* tree_lengths) {
  if (n_layers < 1 || !sets || sets[n_layers - 1].n_clusters < 1) {  // no root to return
    fail_status(SWE_ERR_INVALID);
    return nullptr;
  }
  std::vector<size_t> first((size_t)n_layers + 1, 0);
  for (int L = 0; L < n_layers; ++L) first[(size_t)L + 1] = first[(size_t)L] + (size_t)std::max(sets[L].n_clusters, 0);
  const size_t total = first[(size_t)n_layers];
  tree_node* node = (tree_node*)calloc(total, sizeof(tree_node));
  char* labels = (char*)calloc(total, LABEL_BYTES);
  if (!node || !labels) {
    free(node);
    free(labels);
    fail_status(SWE_ERR_OOM);
    return nullptr;
  }
  auto at = [&](int L, int k) { return node + first[(size_t)L] + (size_t)k; };
  for (int L = 0; L < n_layers; ++L)
    for (int k = 0; k < sets[L].n_clusters; ++k) {
      tree_node* t = at(L, k);
      t->length = L == n_layers - 1 ? 0.0 : (tree_lengths ? tree_lengths[L] : 1.0);
      t->id = labels + LABEL_BYTES * (size_t)(t - node);
    }
  for (int L = n_layers - 1; L >= 1; --L)
    for (int k = 0; k < sets[L].n_clusters; ++k) {
      const cluster_connections& links = c[L - 1][k];
      tree_node* parent = at(L, k);
      tree_node* next = nullptr;  // sibling list: first connection at the tail
      for (int q = 0; q < links.n_connections; ++q) {
        const int ch = links.connections[q];
        tree_node* t = at(L - 1, ch);
        t->parent = parent;
        t->neighbor = next;
        t->n_members = sets[L - 1].clusters[ch].n_members;
        snprintf(t->id, LABEL_BYTES, "L%iC%iN%i", L - 1, ch, t->n_members);
        next = t;
      }
      if (links.n_connections > 0) parent->child = next;
    }
  tree_node* root = at(n_layers - 1, 0);
  snprintf(root->id, LABEL_BYTES, "L%iC%i", n_layers - 1, 0);
  return root;
}

split_set filtered_split_set_by_min_size(split_set s_in, int min_size) {
  split_set out;
  int keep = 0;
  for (int k = 0; k < s_in.n_clusters; ++k) keep += s_in.clusters[k].n_members >= min_size;
  out.n_clusters = keep;
  out.clusters = (cluster*)malloc(sizeof(cluster) * (size_t)(keep > 0 ? keep : 1));
  int at = 0;
  for (int k = 0; k < s_in.n_clusters; ++k) {
    const cluster& src = s_in.clusters[k];
    if (src.n_members < min_size) continue;
    cluster& dst = out.clusters[at];
    dst.id = at;  // the reference leaves the id unset (store_split_set writes it)
    dst.n_members = src.n_members;
    dst.members = (int*)malloc(sizeof(int) * (size_t)(src.n_members > 0 ? src.n_members : 1));
    if (src.n_members > 0) memcpy(dst.members, src.members, sizeof(int) * (size_t)src.n_members);
    ++at;
  }
  return out;
}

// Newick text with an explicit stack: each frame is a node and the next
// child still to write.
void print_tree(FILE* f, tree_node* root) {
  if (!root) return;
  struct Frame {
    const tree_node* node;
    const tree_node* next;
  };
  std::vector<Frame> stack;
  auto open = [&](const tree_node* n) {
    if (n->child) fputc('(', f);
    stack.push_back({n, n->child});
  };
  open(root);
  while (!stack.empty()) {
    Frame& top = stack.back();
    if (top.next) {
      const tree_node* ch = top.next;
      if (ch != top.node->child) fputc(',', f);
      top.next = ch->neighbor;
      open(ch);
      continue;
    }
    const tree_node* n = top.node;
    stack.pop_back();
    if (n->child) fputc(')', f);
    fputs(n->id, f);
    if (n->parent) printf(":%f", n->length);  // branch lengths on stdout (cluster_io.c:229)
  }
  fputc(';', f);
}

int pureness_from_tree(int n_layers, tree_node* root, split_set* s, split_set target, double** pureness_values,
                       int** inpure_clusters) {
  if (!root) return 1;
  const size_t nl = (size_t)(n_layers > 0 ? n_layers : 1);
  double* sum = (double*)calloc(nl, sizeof(double));
  int* impure = (int*)calloc(nl, sizeof(int));
  if (!sum || !impure) {
    free(sum);
    free(impure);
    return 1;
  }
  std::vector<int> owner;
  const bool target_partition = owners_of(target, owner);
  std::vector<int> count((size_t)std::max(target.n_clusters, 1), 0);
  std::vector<int> touched;
  std::vector<uint8_t> mark;
  for (const tree_node* n : post_order(root)) {
    int L = 0, k = 0;
    sscanf(n->id, "L%iC%i", &L, &k);
    const cluster& cl = s[L].clusters[k];
    double impurity = 0.0;
    bool split = false;
    if (target_partition && distinct_members(cl, mark)) {
      // |C n T| for every T at once from the owner of each member
      touched.clear();
      for (int q = 0; q < cl.n_members; ++q) {
        const int m = cl.members[q];
        const int t = (size_t)m < owner.size() ? owner[(size_t)m] : -1;
        if (t < 0) continue;
        if (count[(size_t)t]++ == 0) touched.push_back(t);
      }
      std::sort(touched.begin(), touched.end());
      for (int t : touched) {
        const int inter = count[(size_t)t];
        count[(size_t)t] = 0;
        if (inter != cl.n_members) {
          split = true;
          impurity += share_of(inter, cl.n_members);
        }
      }
    } else {  // repeated members: the intersection's own counting rule
      for (int t = 0; t < target.n_clusters; ++t) {
        cluster both = intersection_of_clusters(cl, target.clusters[t]);
        free(both.members);
        if (both.n_members != 0 && both.n_members != cl.n_members) {
          split = true;
          impurity += share_of(both.n_members, cl.n_members);
        }
      }
    }
    impure[L] += split ? 1 : 0;
    sum[L] += impurity;
  }
  for (int L = 0; L < n_layers; ++L) sum[L] = impure[L] > 0 ? sum[L] / (double)impure[L] : 0.0;
  *pureness_values = sum;
  *inpure_clusters = impure;
  return 0;
}

double* inpures_over_total_fraction(int n_layers, split_set* s, int* inpure_clusters) {
  double* out = (double*)malloc(sizeof(double) * (size_t)(n_layers > 0 ? n_layers : 1));
  for (int L = 0; L < n_layers; ++L) out[L] = (double)inpure_clusters[L] / (double)s[L].n_clusters;
  return out;
}

double* clusters_in_layer_vs_target_clusters(int n_layers, split_set* s, split_set target) {
  double* out = (double*)malloc(sizeof(double) * (size_t)(n_layers > 0 ? n_layers : 1));
  const double want = (double)target.n_clusters;
  for (int L = 0; L < n_layers; ++L) out[L] = std::fabs((double)s[L].n_clusters - want) / want;
  return out;
}

}  // extern "C"
