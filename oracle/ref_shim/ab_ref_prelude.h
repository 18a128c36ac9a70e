// ab_ref_prelude.h -- host-side stand-ins for the CUDA device constructs the
// reference kernels use, so that the reference's own device arithmetic
// (src/aprict/data/cusrc/*.cu, *.h) compiles unchanged with g++ into the
// CPU reference oracle under oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY: nothing in the aprict_b200 package loads this.
#pragma once

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <assert.h>

#include <algorithm>
#include <omp.h>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __shared__ static

// ---- vector types (aggregate, as in CUDA's vector_types.h) ----
struct int2 { int x, y; };
struct int3 { int x, y, z; };
struct uint2 { unsigned int x, y; };
struct uint3 { unsigned int x, y, z; };
struct float2 { float x, y; };
struct ulong2 { unsigned long x, y; };

// ---- thread indices: set by the oracle driver before each "thread" ----
struct ab_dim3 { unsigned int x, y, z; };
extern thread_local ab_dim3 threadIdx, blockIdx, blockDim;
inline void __syncthreads() {}

// ---- min/max with CUDA's overload set: mixed signed/unsigned int pairs
// resolve to the unsigned version, float pairs to fminf/fmaxf. ----
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }
inline unsigned int max(unsigned int a, unsigned int b) { return a > b ? a : b; }
inline unsigned int min(unsigned int a, int b) { return min(a, (unsigned int)b); }
inline unsigned int min(int a, unsigned int b) { return min((unsigned int)a, b); }
inline unsigned int max(unsigned int a, int b) { return max(a, (unsigned int)b); }
inline unsigned int max(int a, unsigned int b) { return max((unsigned int)a, b); }
inline float min(float a, float b) { return fminf(a, b); }
inline float max(float a, float b) { return fmaxf(a, b); }
inline double min(double a, double b) { return fmin(a, b); }
inline double max(double a, double b) { return fmax(a, b); }
inline float norm3d(float a, float b, float c) { return sqrtf(a * a + b * b + c * c); }
using std::abs;

// ---- half precision through the compiler's _Float16 ----
typedef _Float16 half;
inline float __half2float(half h) { return (float)h; }
inline half __float2half(float f) { return (half)f; }
inline half __double2half(double d) { return (half)d; }
inline unsigned short __half_as_ushort(half h) { unsigned short u; memcpy(&u, &h, 2); return u; }
inline half __ushort_as_half(unsigned short u) { half h; memcpy(&h, &u, 2); return h; }

// ---- atomics (the oracle gives every output element to one thread) ----
template <typename T, typename U> inline T atomicAdd(T *p, U v) { T o = *p; *p = (T)(o + v); return o; }

// ---- surfaces: a host descriptor of a 3-D array; x is in bytes ----
typedef unsigned long long cudaSurfaceObject_t;
struct ab_surface {
    unsigned char *base;
    size_t w, h, d;   // extents: x (fastest, elements), y, z
    size_t elem;      // bytes per element
    long long oob;    // out-of-bounds accesses seen
};
template <typename T> inline T surf3Dread(cudaSurfaceObject_t s, int xb, int y, int z) {
    ab_surface *S = reinterpret_cast<ab_surface *>(s);
    T v{};
    if (xb < 0 || y < 0 || z < 0 || (size_t)xb / sizeof(T) >= S->w || (size_t)y >= S->h || (size_t)z >= S->d) {
        __atomic_add_fetch(&S->oob, 1, __ATOMIC_RELAXED);
        return v;
    }
    memcpy(&v, S->base + (((size_t)z * S->h + (size_t)y) * S->w) * sizeof(T) + (size_t)xb, sizeof(T));
    return v;
}
template <typename T> inline void surf3Dwrite(T v, cudaSurfaceObject_t s, int xb, int y, int z) {
    ab_surface *S = reinterpret_cast<ab_surface *>(s);
    if (xb < 0 || y < 0 || z < 0 || (size_t)xb / sizeof(T) >= S->w || (size_t)y >= S->h || (size_t)z >= S->d) {
        __atomic_add_fetch(&S->oob, 1, __ATOMIC_RELAXED);
        return;
    }
    memcpy(S->base + (((size_t)z * S->h + (size_t)y) * S->w) * sizeof(T) + (size_t)xb, &v, sizeof(T));
}
