// Device partition/reorder entry points (see mf_build.cu).
#pragma once
#include "mf_common.cuh"

struct BuildIn {
    int n;
    int R;
    i64 arcs;
    const int *row;
    const int *col;
    const i64 *cap;
    const int *rev;
    const unsigned char *fwd;  // 1 for the forward arc of an input edge
};

struct BuildOut {
    int *row;           // n+1
    int *col;           // arcs
    i64 *cap;           // arcs
    int *rev;           // arcs
    unsigned char *fwd; // arcs
    int *new_id;        // n: input id -> region-ordered id
    int *old_id;        // n
    int *region_start;  // R+1
    int *region_of;     // n (region-ordered ids)
    double *score;      // n (input ids)
    int *part;          // n (input ids)
};

size_t mf_partition_scratch_bytes(int n, i64 arcs, int R);
cudaError_t mf_partition_reorder(const BuildIn &in, const BuildOut &out, void *scratch,
                                 cudaStream_t st);
void mf_exclusive_scan(int n, const int *in, int *out, int *tmp, cudaStream_t st);
