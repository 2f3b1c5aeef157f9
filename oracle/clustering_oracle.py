"""CPU oracle for the clustering half of the medoid pass.  Test infrastructure.

Independent restatements used to check opendba_b200/csrc/clustering.cpp:

* complete linkage by plain agglomeration (O(n^3)): at every step merge the
  two clusters whose largest member-to-member distance is smallest.  For
  inputs without tied distances the dendrogram is unique, so this checks the
  nearest-neighbour-chain implementation merge for merge.  Output in R's
  hclust convention, as hclust-cpp produces for the reference
  (dba.hpp:234): row i = the two nodes merged at the i-th lowest height,
  singleton x as -(x+1), the cluster made at step k as k+1, smaller node id
  first (singletons before clusters).
* cutree_k / cutree_cdist (dba.hpp:248, 276): first n-k merges applied,
  clusters labelled 0, 1, ... by their lowest member.
* the medoid pass's clustering (dba.hpp:186-343): distance scaling by the
  largest pair distance, the three threshold rules, and the per-cluster
  medoid loop exactly as the reference writes it (one sums-of-squares array
  shared across clusters, cluster-local indices into the global triangle).

Parity against hclust-cpp itself is unpinned: the submodule is not in the
reference tree.
"""
from __future__ import annotations

import numpy as np


def _tri(n, i, j):
    if i > j:
        i, j = j, i
    return i * n - i * (i + 1) // 2 + (j - i - 1)


def complete_linkage(n, dists):
    """(merge (n-1, 2) int array, height (n-1,) float64) in R convention."""
    D = np.asarray(dists, dtype=np.float64)
    clusters = {i: [i] for i in range(n)}        # representative -> members
    node_of = {i: i for i in range(n)}           # representative -> node id
    merges = []
    for step in range(n - 1):
        reps = sorted(clusters)
        best = None
        for ai, a in enumerate(reps):
            for b in reps[ai + 1:]:
                h = max(D[_tri(n, x, y)] for x in clusters[a] for y in clusters[b])
                if best is None or h < best[0]:
                    best = (h, a, b)
        h, a, b = best
        u, v = sorted((node_of[a], node_of[b]))
        merges.append((u, v, h))
        clusters[a] = clusters[a] + clusters.pop(b)
        node_of[a] = n + step
        node_of.pop(b)
    merge = np.zeros((n - 1, 2), dtype=np.int64)
    height = np.zeros(n - 1)
    for i, (u, v, h) in enumerate(merges):
        merge[i] = [-(u + 1) if u < n else u - n + 1, -(v + 1) if v < n else v - n + 1]
        height[i] = h
    return merge, height


def cutree_k(n, merge, k):
    if k < 2 or k > n:
        return np.zeros(n, dtype=np.int64)
    members = {}
    for i in range(n - k):
        parts = []
        for m in merge[i]:
            parts += [int(-m - 1)] if m < 0 else members.pop(int(m))
        members[i + 1] = parts
    group = {x: x for x in range(n)}
    for key, parts in members.items():
        for x in parts:
            group[x] = ("c", key)
    labels, seen = np.zeros(n, dtype=np.int64), {}
    for x in range(n):
        g = group[x]
        if g not in seen:
            seen[g] = len(seen)
        labels[x] = seen[g]
    return labels


def cutree_cdist(n, merge, height, cdist):
    applied = 0
    while applied < n - 1 and height[applied] < cdist:
        applied += 1
    return cutree_k(n, merge, n - applied)


def cluster_and_medoids(dists, lens, cdist):
    """(memberships, medoids per cluster) as approximateMedoidIndices gives them."""
    d = np.asarray(dists)
    T = d.dtype.type
    n = len(lens)
    sos = [T(0)] * n
    max_distance = T(0)
    off = 0
    for s in range(n - 1):
        for j in range(s + 1, n):
            x = d[off + j - s - 1]
            if max_distance < x:
                max_distance = x
            x = T(x * x)
            sos[s] = T(sos[s] + x)
            sos[j] = T(sos[j] + x)
        off += n - s - 1
    if max_distance == 0:
        max_distance = T(1)
    if cdist == 1 or n < 2:
        memb = np.zeros(n, dtype=np.int64)
    else:
        D = d.astype(np.float64) / float(max_distance)
        merge, height = complete_linkage(n, D)
        if cdist > 1:
            new_k = min(int(cdist), n)
            while True:
                memb = cutree_k(n, merge, new_k)
                counts = np.bincount(memb, minlength=new_k)
                multi = int((counts > 1).sum())
                new_k += int(cdist) - multi
                if not (multi < int(cdist) and new_k < n):
                    break
        elif cdist >= 0:
            memb = cutree_cdist(n, merge, height, cdist)
        else:
            memb = np.zeros(n, dtype=np.int64)
    ncl = int(memb.max()) + 1 if n else 1
    shared = [T(0)] * n
    use = sos if ncl == 1 else shared
    medoids = []
    for c in range(ncl):
        idx = [i for i in range(n) if memb[i] == c]
        k = len(idx)
        if ncl > 1:
            for i in range(k - 1):
                off = i * n - i * (i + 1) // 2
                for j in range(i + 1, k):
                    pd = d[off + j - i - 1]
                    shared[i] = T(shared[i] + T(pd * pd))
                    shared[j] = T(shared[j] + T(pd * pd))
        if k > 2:
            lowest, med = np.finfo(d.dtype).max, -1
            for i in range(k):
                if use[i] < lowest:
                    med, lowest = idx[i], use[i]
        elif k == 2:
            med = idx[0] if lens[idx[0]] > lens[idx[1]] else idx[1]
        else:
            med = idx[0]
        medoids.append(med)
    return memb, medoids
