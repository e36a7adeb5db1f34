/* Host stand-in for the CUDA vocabulary used by the reference's kernel source
 * (src/kernels/meshdata.cu, meshdata.h, eqstate.h), so that those files compile unchanged with
 * g++ and run on the CPU as the pinned parity reference.  Test infrastructure only.
 *
 * A kernel launch becomes a sequential loop over the global thread index (blockDim.x = 1,
 * blockIdx.x = index, threadIdx.x = 0), so every atomic update happens in index order and each
 * run gives the same bits.  The one kernel that needs a whole block at once (minTransportDt,
 * meshdata.cu:6842, shuffles + __syncthreads) is not launched: the driver takes the minimum of the
 * per-element values it reduces.  Every name here is either a plain C++ restatement of the
 * documented CUDA semantics or a no-op where a single host thread makes it one.
 *
 * This header is found before the real <cuda_runtime.h> through the include path of the recipe
 * (oracle/refemu/build.py) and is force-included first.  meshdata.h declares its own
 * `uintptr_t` alias (unsigned long long, the device pointer width), which would clash with the
 * C library's; the macro at the end renames the reference's alias after the standard headers
 * are in.
 */
#ifndef GS_REFEMU_CUDA_RUNTIME_H
#define GS_REFEMU_CUDA_RUNTIME_H

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <assert.h>
#include <stdint.h>
#include <new>
#include <string>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __inline__ inline
#define __noinline__
#define __launch_bounds__(...)
#define __restrict__ __restrict
#define __shared__ static

struct gs_dim3 { unsigned int x, y, z; };
extern thread_local gs_dim3 threadIdx, blockIdx;
extern thread_local gs_dim3 blockDim, gridDim;
constexpr int warpSize = 32;

struct double2 { double x, y; };
struct double3 { double x, y, z; };
struct double4 { double x, y, z, w; };
struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };
inline double2 make_double2(double x, double y) { return double2{x, y}; }
inline double3 make_double3(double x, double y, double z) { return double3{x, y, z}; }
inline double4 make_double4(double x, double y, double z, double w) { return double4{x, y, z, w}; }
inline int2 make_int2(int x, int y) { return int2{x, y}; }

/* CUDA's overloaded min/max (integer and floating forms, mixed int/floating promote) */
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline unsigned min(unsigned a, unsigned b) { return a < b ? a : b; }
inline unsigned max(unsigned a, unsigned b) { return a > b ? a : b; }
inline long long min(long long a, long long b) { return a < b ? a : b; }
inline long long max(long long a, long long b) { return a > b ? a : b; }
inline float min(float a, float b) { return fminf(a, b); }
inline float max(float a, float b) { return fmaxf(a, b); }
inline double min(double a, double b) { return fmin(a, b); }
inline double max(double a, double b) { return fmax(a, b); }
inline double min(double a, int b) { return fmin(a, (double)b); }
inline double max(double a, int b) { return fmax(a, (double)b); }
inline double min(int a, double b) { return fmin((double)a, b); }
inline double max(int a, double b) { return fmax((double)a, b); }
inline double min(double a, float b) { return fmin(a, (double)b); }
inline double max(double a, float b) { return fmax(a, (double)b); }
inline double min(float a, double b) { return fmin((double)a, b); }
inline double max(float a, double b) { return fmax((double)a, b); }

inline int __ffs(int x) { return __builtin_ffs(x); }
inline int __ffs(unsigned x) { return __builtin_ffs((int)x); }
inline long long __double_as_longlong(double d) { long long r; memcpy(&r, &d, 8); return r; }
inline double __longlong_as_double(long long v) { double r; memcpy(&r, &v, 8); return r; }
inline void __threadfence(void) {}
inline void __syncthreads(void) {}
template <class T> inline T __shfl_down_sync(unsigned, T v, int) { return v; }

/* atomics: one host thread, so read-modify-write in program order, returning the old value */
template <class T> inline T atomicAdd(T* a, T v) { T o = *a; *a = o + v; return o; }
template <class T, class A, class B> inline T atomicCAS(T* a, A cmp, B v)
{ T o = *a; if (o == (T)cmp) *a = (T)v; return o; }
template <class T> inline T atomicExch(T* a, T v) { T o = *a; *a = v; return o; }
template <class T> inline T atomicMin(T* a, T v) { T o = *a; if (v < o) *a = v; return o; }
template <class T> inline T atomicMax(T* a, T v) { T o = *a; if (v > o) *a = v; return o; }

#define uintptr_t gs_ref_uintptr_t

#endif
