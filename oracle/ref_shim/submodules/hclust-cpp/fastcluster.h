// Test-infrastructure shim, NOT product code.
//
// The reference includes "submodules/hclust-cpp/fastcluster.h" (dba.hpp:26), a
// git submodule that is not vendored in the reference tree.  This header only
// declares the three entry points at the reference's call sites
// (dba.hpp:234 hclust_fast, dba.hpp:248 cutree_k, dba.hpp:276 cutree_cdist)
// so that the reference harness in oracle/ref_harness.cu links.  The matching
// definitions in oracle/ref_hclust_shim.cpp forward to this project's
// complete linkage (opendba_b200/csrc/clustering.cpp).
#ifndef ODBA_REF_SHIM_FASTCLUSTER_H
#define ODBA_REF_SHIM_FASTCLUSTER_H

enum odba_shim_hclust_methods {
  HCLUST_METHOD_SINGLE = 0,
  HCLUST_METHOD_COMPLETE = 1,
  HCLUST_METHOD_AVERAGE = 2,
  HCLUST_METHOD_MEDIAN = 3
};

int hclust_fast(int n, double *distmat, int method, int *merge, double *height);
void cutree_k(int n, const int *merge, int ncluster, int *labels);
void cutree_cdist(int n, const int *merge, double *height, double cdist, int *labels);

#endif
