// Clustering of the medoid pass: complete linkage over the normalised pair
// distances, the dendrogram cuts, and the per-cluster medoids, as used by
// approximateMedoidIndices (dba.hpp:219-343).
//
// The reference calls hclust-cpp (github.com/cdalitz/hclust-cpp, an
// unvendored submodule with no pinned commit): hclust_fast(...,
// HCLUST_METHOD_COMPLETE, merge, height) (dba.hpp:234), cutree_k (dba.hpp:248)
// and cutree_cdist (dba.hpp:276).  That library wraps Daniel Muellner's
// fastcluster, whose complete linkage is the nearest-neighbour-chain
// algorithm (Muellner, "Modern hierarchical, agglomerative clustering
// algorithms", arXiv:1109.2378, 2011).  This file restates the published
// algorithm and the output conventions the reference relies on:
//   * NN-chain: grow a chain of nearest neighbours from the lowest active
//     index; a node's nearest neighbour is searched with its chain predecessor
//     as the incumbent (ties keep the predecessor; otherwise the lowest index
//     with a strictly smaller distance wins); a reciprocal pair is merged at
//     their distance, the merged cluster keeps the larger index and the
//     smaller one leaves the active set; complete-linkage update
//     d(k, merged) = max(d(k, a), d(k, b)); after a merge the chain backs up
//     one element (or restarts when fewer than two would remain).
//   * Dendrogram in R's hclust convention: merges stably sorted by height;
//     row i holds the two merged nodes, a singleton x as -(x+1) and the
//     cluster made at (sorted) step k as k+1, the smaller node id first
//     (singletons before clusters).
//   * cutree_k: apply the first n-k merges; label clusters 0, 1, ... in order
//     of their lowest member; k < 2 or k > n puts everything in cluster 0.
//     cutree_cdist: k = n - (number of merges with height < cdist).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

#include "odba_internal.h"

namespace odba {

namespace {

inline size_t tri(size_t n, size_t i, size_t j) {  // i < j
  return i * n - i * (i + 1) / 2 + (j - i - 1);
}

struct Merge {
  int a, b;
  double h;
};

}  // namespace

// D: condensed upper-triangle distances (overwritten).  merge: 2(n-1) ints,
// column-major like R's (n-1) x 2 matrix; height: n-1 doubles.
void complete_linkage(int n, double *D, int *merge, double *height) {
  if (n < 2) return;
  const size_t N = size_t(n);
  auto d = [&](int i, int j) -> double & { return i < j ? D[tri(N, i, j)] : D[tri(N, j, i)]; };
  // active indices as a doubly linked list in ascending order
  std::vector<int> succ(n + 1), pred(n + 1);
  for (int i = 0; i <= n; ++i) {
    succ[i] = i + 1;
    pred[i] = i - 1;
  }
  int first = 0;
  auto remove = [&](int i) {
    if (i == first) {
      first = succ[i];
    } else {
      succ[pred[i]] = succ[i];
    }
    if (succ[i] < n) pred[succ[i]] = pred[i];
  };
  std::vector<int> chain(n + 1);
  int tip = 0;  // number of elements on the chain
  std::vector<Merge> found;
  found.reserve(n - 1);
  for (int step = 0; step < n - 1; ++step) {
    int a, b;
    double best;
    if (tip <= 3) {
      // restart from the lowest active node and its nearest neighbour
      a = first;
      chain[0] = a;
      tip = 1;
      b = succ[a];
      best = d(a, b);
      for (int i = succ[b]; i < n; i = succ[i])
        if (d(a, i) < best) {
          best = d(a, i);
          b = i;
        }
    } else {
      // back up: the element below the merged pair, with its predecessor
      tip -= 3;
      a = chain[tip - 1];
      b = chain[tip];
      best = d(a, b);
    }
    for (;;) {
      chain[tip] = b;
      // nearest neighbour of b, the predecessor a as the incumbent
      int c = a;
      for (int i = first; i < n; i = succ[i]) {
        if (i == b) continue;
        const double v = d(i, b);
        if (v < best) {
          best = v;
          c = i;
        }
      }
      a = b;
      b = c;
      ++tip;
      if (b == chain[tip - 2]) break;  // reciprocal nearest neighbours
    }
    found.push_back({a, b, best});
    const int lo = std::min(a, b), hi = std::max(a, b);
    remove(lo);
    for (int i = first; i < n; i = succ[i]) {
      if (i == hi) continue;
      double &t = d(i, hi);
      const double o = d(i, lo);
      if (t < o) t = o;
    }
  }
  // R dendrogram: merges in order of height (stable), nodes relabelled
  std::stable_sort(found.begin(), found.end(), [](const Merge &x, const Merge &y) { return x.h < y.h; });
  std::vector<int> parent(2 * N - 1, -1);
  auto find = [&](int x) {
    int r = x;
    while (parent[r] >= 0) r = parent[r];
    while (parent[x] >= 0) {
      const int up = parent[x];
      parent[x] = r;
      x = up;
    }
    return r;
  };
  for (int i = 0; i < n - 1; ++i) {
    int u = find(found[i].a), v = find(found[i].b);
    parent[u] = parent[v] = n + i;
    if (u > v) std::swap(u, v);
    merge[i] = u < n ? -(u + 1) : u - n + 1;
    merge[i + n - 1] = v < n ? -(v + 1) : v - n + 1;
    height[i] = found[i].h;
  }
}

void cut_tree_k(int n, const int *merge, int k, int *labels) {
  if (k < 2 || k > n) {
    for (int i = 0; i < n; ++i) labels[i] = 0;
    return;
  }
  // union-find over the first n-k merges (R convention node ids)
  std::vector<int> parent(2 * size_t(n) - 1, -1);
  auto node = [&](int m) { return m < 0 ? -m - 1 : n + m - 1; };
  auto find = [&](int x) {
    while (parent[x] >= 0) x = parent[x];
    return x;
  };
  for (int i = 0; i < n - k; ++i) {
    const int u = find(node(merge[i])), v = find(node(merge[i + n - 1]));
    parent[u] = parent[v] = n + i;
  }
  std::vector<int> label_of(2 * size_t(n) - 1, -1);
  int next = 0;
  for (int i = 0; i < n; ++i) {
    const int r = find(i);
    if (label_of[r] < 0) label_of[r] = next++;
    labels[i] = label_of[r];
  }
}

void cut_tree_height(int n, const int *merge, const double *height, double cdist, int *labels) {
  int applied = 0;
  while (applied < n - 1 && height[applied] < cdist) ++applied;
  cut_tree_k(n, merge, n - applied, labels);
}

// Memberships and per-cluster medoids from the T distance triangle, as
// approximateMedoidIndices does after the pair distances (dba.hpp:186-343).
// Returns the number of clusters; medoids must hold n ints.
template <typename T>
int cluster_and_medoids(int n, const T *dists, const uint64_t *lens, double cdist, int *memberships,
                        int *medoids) {
  const size_t npairs = size_t(n) * (n - 1) / 2;
  // sums of squares and the largest distance, in T, in row-major pair order (dba.hpp:186-210)
  std::vector<T> sos(n, T(0));
  T max_distance = T(0);
  for (int s = 0, off = 0; s + 1 < n; off += n - s - 1, ++s)
    for (int j = s + 1; j < n; ++j) {
      T dd = dists[off + (j - s - 1)];
      if (max_distance < dd) max_distance = dd;
      dd *= dd;
      sos[s] += dd;
      sos[j] += dd;
    }
  if (max_distance == 0) max_distance = 1;
  if (cdist == 1) {
    for (int i = 0; i < n; ++i) memberships[i] = 0;
  } else if (n >= 2) {
    std::vector<double> D(npairs);
    for (size_t p = 0; p < npairs; ++p) D[p] = double(dists[p]) / double(max_distance);
    std::vector<int> merge(2 * size_t(n - 1));
    std::vector<double> height(n - 1);
    complete_linkage(n, D.data(), merge.data(), height.data());
    if (cdist > 1) {
      // k clusters, raised until enough of them have several members (dba.hpp:239-265)
      int new_k = int(cdist);
      if (new_k > n) new_k = n;
      int multi = 0;
      do {
        cut_tree_k(n, merge.data(), new_k, memberships);
        std::vector<int> count(new_k, 0);
        for (int i = 0; i < n; ++i) count[memberships[i]]++;
        multi = 0;
        for (int c = 0; c < new_k; ++c)
          if (count[c] > 1) ++multi;
        new_k += int(cdist) - multi;
      } while (multi < int(cdist) && new_k < n);
    } else if (cdist >= 0) {
      cut_tree_height(n, merge.data(), height.data(), cdist, memberships);
    } else {
      // negative thresholds are reserved in the reference (dba.hpp:277-283): one cluster here
      for (int i = 0; i < n; ++i) memberships[i] = 0;
    }
  } else {
    memberships[0] = 0;
  }
  int num_clusters = 1;
  for (int i = 0; i < n; ++i) num_clusters = std::max(num_clusters, memberships[i] + 1);
  // per-cluster medoids (dba.hpp:293-343).  With several clusters the
  // reference accumulates one shared sum-of-squares array across clusters and
  // reads each cluster's distances at its members' positions within the
  // cluster (rows and columns 0..k-1 of the global triangle); kept as is.
  std::vector<T> shared(n, T(0));
  const T *use = num_clusters == 1 ? sos.data() : shared.data();
  for (int c = 0; c < num_clusters; ++c) {
    std::vector<int> idx;
    for (int i = 0; i < n; ++i)
      if (memberships[i] == c) idx.push_back(i);
    const int k = int(idx.size());
    if (num_clusters > 1) {
      for (int i = 0; i + 1 < k; ++i) {
        const size_t off = size_t(i) * n - size_t(i) * (i + 1) / 2;
        for (int j = i + 1; j < k; ++j) {
          const T pd = dists[off + (j - i - 1)];
          shared[i] += pd * pd;
          shared[j] += pd * pd;
        }
      }
    }
    int med = -1;
    if (k > 2) {
      T lowest = std::numeric_limits<T>::max();
      for (int i = 0; i < k; ++i)
        if (use[i] < lowest) {
          med = idx[i];
          lowest = use[i];
        }
    } else if (k == 2) {
      med = lens[idx[0]] > lens[idx[1]] ? idx[0] : idx[1];
    } else if (k == 1) {
      med = idx[0];
    }
    medoids[c] = med;
  }
  return num_clusters;
}

template int cluster_and_medoids<float>(int, const float *, const uint64_t *, double, int *, int *);
template int cluster_and_medoids<double>(int, const double *, const uint64_t *, double, int *, int *);

}  // namespace odba

extern "C" {

int odba_complete_linkage(int n, const double *dists, int *merge, double *height) {
  if (n < 1 || (n >= 2 && (!dists || !merge || !height)))
    return odba::fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or empty input");
  std::vector<double> D(dists, dists + size_t(n) * (n - 1) / 2);
  odba::complete_linkage(n, D.data(), merge, height);
  return ODBA_OK;
}

int odba_cutree_k(int n, const int *merge, int k, int *labels) {
  if (n < 1 || !labels || (n >= 2 && !merge)) return odba::fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer");
  odba::cut_tree_k(n, merge, k, labels);
  return ODBA_OK;
}

int odba_cutree_cdist(int n, const int *merge, const double *height, double cdist, int *labels) {
  if (n < 1 || !labels || (n >= 2 && (!merge || !height)))
    return odba::fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer");
  odba::cut_tree_height(n, merge, height, cdist, labels);
  return ODBA_OK;
}

int odba_cluster_medoids_f32(int n, const float *dists, const uint64_t *lens, double cdist,
                             int *memberships, int *medoids, int *num_clusters) {
  if (n < 1 || !lens || !memberships || !medoids || !num_clusters || (n >= 2 && !dists))
    return odba::fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or empty input");
  *num_clusters = odba::cluster_and_medoids<float>(n, dists, lens, cdist, memberships, medoids);
  return ODBA_OK;
}

int odba_cluster_medoids_f64(int n, const double *dists, const uint64_t *lens, double cdist,
                             int *memberships, int *medoids, int *num_clusters) {
  if (n < 1 || !lens || !memberships || !medoids || !num_clusters || (n >= 2 && !dists))
    return odba::fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or empty input");
  *num_clusters = odba::cluster_and_medoids<double>(n, dists, lens, cdist, memberships, medoids);
  return ODBA_OK;
}

}  // extern "C"
