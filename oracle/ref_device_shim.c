/*
 * Device-selection shim for the reference build (test infrastructure only).
 *
 * The reference hard-wires cudaSetDevice(1) (Region_Aware_PR_with_Pruning_
 * BoundaryCore.cu:2573), which fails on a host that shows one GPU; its next
 * cudaGetLastError() check then aborts.  Linking this file into the
 * reference executable (built with the shared CUDA runtime) replaces that
 * one call with cudaSetDevice(MF_REF_DEVICE, default 0) and leaves the
 * reference sources untouched.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stdlib.h>

typedef int (*set_device_fn)(int);

int cudaSetDevice(int device) {
    static set_device_fn real = 0;
    (void)device;
    if (!real) real = (set_device_fn)dlsym(RTLD_NEXT, "cudaSetDevice");
    const char *env = getenv("MF_REF_DEVICE");
    int d = env ? atoi(env) : 0;
    return real ? real(d) : 100; /* 100 = cudaErrorNoDevice */
}
