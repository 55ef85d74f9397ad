// The serving kernel: the solver of mf_solver.cu compiled a second time
// with MF_SERVE_TU, which builds only mf_serve_kernel (the request loop of
// the continuous-batching server) and reads capacities through L2, since
// that kernel applies capacity updates to the graphs it reads while it runs.
// Every other launch uses mf_kernel from mf_solver.cu, whose capacity loads
// may use the read-only cache.  The second copy of the solver's functions
// has internal linkage (anonymous namespace); only the two entry points
// below are exported.
#include <climits>
#include <cstring>

#include "mf_solver.cuh"

#define MF_SERVE_TU
namespace {
#include "mf_solver.cu"
}  // namespace

cudaError_t mf_launch_serve_kernel(const KParams &p, int grid, int threads, cudaStream_t st, bool cooperative) {
    return serve_launch_impl(p, grid, threads, st, cooperative);
}

int mf_serve_kernel_max_blocks_per_sm(int threads) { return serve_occupancy_impl(threads); }
