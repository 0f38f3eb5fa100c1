/*
 * ref_shim.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Lets g++ compile the reference solvers' device functions and grid-stride
 * kernels as ordinary host C++: the CUDA qualifiers vanish and the launch
 * coordinates become thread-local variables.  ref_host.cpp then "launches"
 * a kernel as one call per virtual CUDA block with blockDim = 1 and
 * gridDim = the number of work items, so each call does exactly one
 * iteration of the kernel's grid-stride loop, and splits those calls over
 * OpenMP threads in contiguous chunks.
 */
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <math.h>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline

struct ref_dim3 { unsigned x, y, z; };
extern thread_local ref_dim3 blockIdx, threadIdx, blockDim, gridDim;

/* atomicAdd for kernels that scatter (fv_rec3_2d.cu's compute_rhs and its
 * brutal-fix counter): an OpenMP atomic, so with one thread the additions
 * happen in work-item order */
inline double atomicAdd(double *a, double v)
{
    double old;
#pragma omp atomic capture
    { old = *a; *a += v; }
    return old;
}
inline int atomicAdd(int *a, int v)
{
    int old;
#pragma omp atomic capture
    { old = *a; *a += v; }
    return old;
}
