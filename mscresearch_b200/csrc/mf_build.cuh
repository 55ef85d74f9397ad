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

// Paired-arc CSR in input vertex order (mf_ingest.cu); device arrays.
struct DevCsr {
    int *row = nullptr;  // n+1
    int *col = nullptr;
    i64 *cap = nullptr;
    int *rev = nullptr;
    unsigned char *fwd = nullptr;
    i64 arcs = 0;
};
// Edge triples read from graph.txt bytes on the device (mf_ingest.cu).
struct TextEdges {
    bool header_ok = false;  // the "n m" header scanned
    int n = 0;
    int m_header = 0;
    i64 m = 0;  // triples read: min(m_header, complete triples before the stream ends)
    int *u = nullptr, *v = nullptr;  // 0-based (file ids - 1)
    i64 *c = nullptr;
};
cudaError_t mf_device_csr(int n, i64 m, const int *u, const int *v, const i64 *c, cudaStream_t st,
                          DevCsr &out);
void mf_free_dev_csr(DevCsr &c);
// Stable LSD radix sort (8-bit digits) of N (key, val) pairs by key in
// [0, key_max]; key2 / val2 are scratch of N entries.  The sorted pairs end
// in key / val (the pointers are swapped as the passes require).
cudaError_t mf_radix_sort_pairs(int N, int key_max, int *&key, int *&val, int *&key2, int *&val2,
                                cudaStream_t st);
cudaError_t mf_parse_graph_text(const unsigned char *txt, i64 S, cudaStream_t st, TextEdges &out);
void mf_free_text_edges(TextEdges &t);
