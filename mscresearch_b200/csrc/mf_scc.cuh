// Strongly connected components and SCC contraction on the device
// (mf_scc.cu).
#pragma once
#include <vector>

#include "mf_common.cuh"

struct SccIn {
    int n;
    i64 arcs;
    const int *row, *col, *rev;  // device: region-ordered paired-arc CSR
    const i64 *cap;              // device: current capacities
    const int *new_id;           // host, n: caller id -> internal id
    const int *old_id;           // host, n: internal id -> caller id
};

struct SccOut {
    int ncomp = 0;
    std::vector<int> comp;  // caller id -> component, numbered by smallest caller id
    std::vector<int> cu, cv;  // contracted arcs in increasing (cu, cv)
    std::vector<i64> cap;     // their summed capacities
};

cudaError_t mf_scc_run(const SccIn &in, cudaStream_t st, SccOut &out);
