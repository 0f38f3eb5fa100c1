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
