/*
 * ref_shim.h -- host-side stand-ins for the CUDA built-ins that the
 * reference's device kernels use, so that those kernel sources can be
 * compiled unchanged by g++ and executed on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY. This file is part of the oracle: it lets the
 * test-suite run the reference's own FP64 arithmetic (src/Kernel/** and
 * src/Utils/Neighborhood/**) as a checker. Nothing in the product links it.
 *
 * The reference kernels are plain SIMT code: one thread per item, no shared
 * memory, no barriers, no warp intrinsics (checked by reading every kernel
 * the driver launches). A launch can therefore be emulated by a loop that
 * sets blockIdx/threadIdx and calls the kernel body; the kernels then run
 * with exactly their own floating-point expressions.
 *
 * Force-included (g++ -include) ahead of every reference .cu file.
 */
#ifndef PSB_REF_SHIM_H
#define PSB_REF_SHIM_H

/* Empty qualifiers: with these defined first, CUDA's host_defines.h keeps them. */
#define __host__
#define __device__
#define __global__
#define __shared__
#define __constant__
#define __forceinline__ inline

#include <sys/types.h>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <vector_types.h>
#include <vector_functions.h>

using std::max;
using std::min;

/* Thread/block coordinates of the emulated launch (one set per host thread). */
extern thread_local uint3 blockIdx;
extern thread_local uint3 threadIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

static inline unsigned int __umul24(unsigned int a, unsigned int b) { return a * b; }
static inline int __mul24(int a, int b) { return a * b; }

static inline int __float_as_int(float f) { int i; std::memcpy(&i, &f, 4); return i; }
static inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
static inline long long __double_as_longlong(double d) { long long i; std::memcpy(&i, &d, 8); return i; }
static inline double __longlong_as_double(long long i) { double d; std::memcpy(&d, &i, 8); return d; }

/* Atomics: real host atomics, so that launches emulated on several host
 * threads keep CUDA's atomic semantics. */
static inline int atomicAdd(int* a, int v) { return __atomic_fetch_add(a, v, __ATOMIC_RELAXED); }
static inline unsigned int atomicAdd(unsigned int* a, unsigned int v) { return __atomic_fetch_add(a, v, __ATOMIC_RELAXED); }
static inline int atomicExch(int* a, int v) { return __atomic_exchange_n(a, v, __ATOMIC_RELAXED); }
static inline int atomicCAS(int* a, int cmp, int v) {
    __atomic_compare_exchange_n(a, &cmp, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
    return cmp;
}
static inline unsigned int atomicCAS(unsigned int* a, unsigned int cmp, unsigned int v) {
    __atomic_compare_exchange_n(a, &cmp, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
    return cmp;
}
static inline unsigned long long atomicCAS(unsigned long long* a, unsigned long long cmp, unsigned long long v) {
    __atomic_compare_exchange_n(a, &cmp, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
    return cmp;
}

#endif /* PSB_REF_SHIM_H */
