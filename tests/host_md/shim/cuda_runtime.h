// cuda_runtime.h stand-in for the host test harnesses in tests/host_md: just enough of the CUDA names
// that the library's device headers use, mapped to sequential host code (one thread at a time, so an
// atomic update is a plain update).  Never on the library's include path.
#pragma once
#include <cstring>

typedef struct CUstream_st* cudaStream_t;
struct int4
{
    int x, y, z, w;
};
struct HostDim3
{
    unsigned x = 0, y = 0, z = 0;
};
extern HostDim3 blockIdx, threadIdx, blockDim, gridDim;

#define __host__
#define __device__
#define __global__
#define __shared__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#define __launch_bounds__(...)

template <class T>
inline T __ldg(const T* p)
{
    return *p;
}
template <class T>
inline T __ldcg(const T* p)
{
    return *p;
}
inline double atomicAdd(double* p, double v)
{
    const double o = *p;
    *p = o + v;
    return o;
}
inline float atomicAdd(float* p, float v)
{
    const float o = *p;
    *p = o + v;
    return o;
}
inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v)
{
    const unsigned long long o = *p;
    *p = o + v;
    return o;
}
inline long long __double2ll_rn(double x)
{
    return (long long)__builtin_llrint(x);
}
inline int atomicMax(int* p, int v)
{
    const int o = *p;
    if (v > o) *p = v;
    return o;
}
inline unsigned long long atomicMax(unsigned long long* p, unsigned long long v)
{
    const unsigned long long o = *p;
    if (v > o) *p = v;
    return o;
}
inline long long __double_as_longlong(double d)
{
    long long r;
    std::memcpy(&r, &d, sizeof r);
    return r;
}
inline void __syncthreads() {}
// Warp collectives for a warp of one lane (the host harness runs one thread): the shuffle returns the
// lane's own value and the votes and reductions see that lane alone.  Only the warp-shared J/K kernel uses
// them, and the harness compiles it without running it.
inline double __shfl_xor_sync(unsigned, double v, int) { return v; }
inline int __reduce_max_sync(unsigned, int v) { return v; }
inline int __any_sync(unsigned, int p) { return p != 0; }
