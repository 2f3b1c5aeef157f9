// Test-infrastructure shim, NOT product code.
//
// Definitions of the three hclust-cpp entry points the reference calls
// (dba.hpp:234 hclust_fast, dba.hpp:248 cutree_k, dba.hpp:276 cutree_cdist),
// forwarded to this project's complete linkage and dendrogram cuts
// (opendba_b200/csrc/clustering.cpp).  hclust-cpp itself is an unvendored
// submodule of the reference; with this shim the reference harness runs the
// reference's own clustering code path (threshold logic, distance scaling,
// per-cluster medoids, membership file, per-cluster DBA) around the same
// linkage the B200 library uses, which pins everything in that path except
// the linkage algorithm against hclust-cpp.
#include "submodules/hclust-cpp/fastcluster.h"

#include "odba_internal.h"

namespace odba {
// the library's error slot is not linked into the harness
int fail(int status, const char *) { return status; }
}  // namespace odba

int hclust_fast(int n, double *distmat, int, int *merge, double *height) {
  // the reference's only call site asks for complete linkage (dba.hpp:234)
  odba::complete_linkage(n, distmat, merge, height);
  return 0;
}

void cutree_k(int n, const int *merge, int ncluster, int *labels) {
  odba::cut_tree_k(n, merge, ncluster, labels);
}

void cutree_cdist(int n, const int *merge, double *height, double cdist, int *labels) {
  odba::cut_tree_height(n, merge, height, cdist, labels);
}
