// sphb_common.cuh -- device helpers shared by the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "sphb.h"

#define SPHB_ELEM_TILE 256          // particles per elementwise tile / block
#define SPHB_SCAN_THREADS 1024
#define SPHB_SCAN_ITEMS 4
#define SPHB_SCAN_CHUNK (SPHB_SCAN_THREADS * SPHB_SCAN_ITEMS)
#define SPHB_MAX_STENCIL 2

namespace sphb {

// Records the failure of the last launch for sphb_last_cuda_error.
int launch_status(const char *what);
// Records err for sphb_last_cuda_error.
void record_cuda_error(const char *what, cudaError_t err);

__device__ __forceinline__ void flag(const sphb_engine &e, unsigned bits)
{
    atomicOr(e.work.status, bits);
}

// Programmatic dependent launch.  A kernel launched with launch_pdl may start
// while its predecessor in the stream is still running; pdl_wait() holds it
// until that predecessor has completed and its writes are visible (at once
// when there is none).  pdl_trigger() lets this grid's own dependent launch
// as soon as every block of this grid has started.
__device__ __forceinline__ void pdl_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ void pdl_trigger()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launch with programmatic stream serialization: the kernel must call
// pdl_wait() before it reads anything its predecessor writes.
template <typename... KArgs, typename... Args>
static inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block,
                                     cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Monotone map double -> uint64 so atomicMin/atomicMax order doubles.
__host__ __device__ __forceinline__ unsigned long long enc_double(double v)
{
    unsigned long long b;
#ifdef __CUDA_ARCH__
    b = (unsigned long long)__double_as_longlong(v);
#else
    memcpy(&b, &v, sizeof(b));
#endif
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

__host__ __device__ __forceinline__ double dec_double(unsigned long long e)
{
    unsigned long long b = (e & 0x8000000000000000ull)
                               ? (e & 0x7fffffffffffffffull)
                               : ~e;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double v;
    memcpy(&v, &b, sizeof(v));
    return v;
#endif
}

// Non-negative doubles order like their bit patterns.  Every block of a
// kernel updates the same few maxima, so the atomic is issued only when the
// value can still raise the stored one (a stale read costs one extra atomic,
// never a wrong result).
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *addr,
                                                  double v)
{
    if (!(v >= 0.0)) return;
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    if (b > *(volatile unsigned long long *)addr) atomicMax(addr, b);
}

// atomicMin / atomicMax on order-encoded doubles, skipped when they cannot
// change the stored value.
__device__ __forceinline__ void atomic_min_enc(unsigned long long *addr, unsigned long long v)
{
    if (v < *(volatile unsigned long long *)addr) atomicMin(addr, v);
}

__device__ __forceinline__ void atomic_max_enc(unsigned long long *addr, unsigned long long v)
{
    if (v > *(volatile unsigned long long *)addr) atomicMax(addr, v);
}

// Local cell index -> (cx, cy, cz) within the scene grid.
__device__ __forceinline__ void cell_coords(int c, const int *n, int &cx,
                                            int &cy, int &cz)
{
    cx = c % n[0];
    int r = c / n[0];
    cy = r % n[1];
    cz = r / n[1];
}

// Block-wide reductions (blockDim.x multiple of 32, <= 1024).
template <typename T, typename Op>
__device__ __forceinline__ T block_reduce(T v, Op op, T identity)
{
    __shared__ T red_smem[32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) red_smem[warp] = v;
    __syncthreads();
    const unsigned nw = blockDim.x >> 5;
    v = (threadIdx.x < nw) ? red_smem[threadIdx.x] : identity;
    if (warp == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;  // valid in thread 0
}

template <typename T, typename Op>
__device__ __forceinline__ T warp_reduce(T v, Op op)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;  // valid in every lane
}

struct OpMin {
    __device__ __forceinline__ double operator()(double a, double b) const
    {
        return fmin(a, b);
    }
};
struct OpMax {
    __device__ __forceinline__ double operator()(double a, double b) const
    {
        return fmax(a, b);
    }
};
struct OpSumInt {
    __device__ __forceinline__ int operator()(int a, int b) const { return a + b; }
};
struct OpAddU64 {
    __device__ __forceinline__ unsigned long long
    operator()(unsigned long long a, unsigned long long b) const
    {
        return a + b;
    }
};

// Adds every thread's v into *addr with one global atomic per block.  All
// threads of the block must call it.
__device__ __forceinline__ void block_add_u64(unsigned long long *addr, unsigned long long v)
{
    __shared__ unsigned long long s_acc;
    if (threadIdx.x == 0) s_acc = 0ull;
    __syncthreads();
    v = warp_reduce(v, OpAddU64());
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&s_acc, v);
    __syncthreads();
    if (threadIdx.x == 0 && s_acc) atomicAdd(addr, s_acc);
}

// Kahan-compensated FP32 accumulator: the running value is sum - c.
struct Kahan {
    float sum, c;
    __device__ __forceinline__ Kahan() : sum(0.f), c(0.f) {}
    __device__ __forceinline__ void add(float term)
    {
        float y = term - c;
        float t = sum + y;
        c = (t - sum) - y;
        sum = t;
    }
    // Merge another partial sum (two-sum of the heads, compensations added).
    __device__ __forceinline__ void merge(float osum, float oc)
    {
        float t = sum + osum;
        float bp = t - sum;
        float err = (sum - (t - bp)) + (osum - bp);
        sum = t;
        c = c + oc - err;
    }
    __device__ __forceinline__ double value() const
    {
        return (double)sum - (double)c;
    }
};

// Cubic-spline normalisation at h = 1 (CubicSplineKernel._fac(1.0),
// S/base/kernels.pyx:441-447).
template <int DIM>
__host__ __device__ __forceinline__ double kfac_unit()
{
    return DIM == 2 ? 10.0 / (7.0 * 3.141592653589793)
                    : 1.0 / 3.141592653589793;
}

// x^y of the Tait EOS.  The FP32C path rounds p and cs to float, so an
// integral exponent up to 16 (gamma = 7 gives 7 and 3) is taken by
// repeated squaring in FP64, a few roundings far below the float rounding
// that follows; otherwise, and always on the FP64 path, pow.
template <bool F32>
__device__ __forceinline__ double eos_pow(double x, double y)
{
    if (F32 && rint(y) == y && fabs(y) <= 16.0) {
        int n = (int)fabs(y);
        double b = x, acc = 1.0;
        while (n) {
            if (n & 1) acc *= b;
            b *= b;
            n >>= 1;
        }
        return y < 0.0 ? 1.0 / acc : acc;
    }
    return pow(x, y);
}

}  // namespace sphb
