// sphb_fma_probe.cu -- FP32 and FP64 FMA issue-rate probes (sm_100a), the
// compute denominators of the pair passes' roofline (they are bound by
// instruction issue, not by tensor cores or HBM).  A measurement tool of
// the benchmark, built into its own library (libsphb_probe.so), not part of
// the particle path or of libsphb.so.
//
// Every thread runs 8 independent FMA chains of `iters` steps (enough in
// flight to fill the FMA pipes), and one lane writes a result so the work
// is kept.  2 flops per FMA.

#include <cuda_runtime.h>

namespace sphb_probe {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_probe(T *out, int iters, T a, T b)
{
    T x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = (T)(threadIdx.x + i) * (T)1e-3;
#pragma unroll 1
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
#pragma unroll
            for (int i = 0; i < 8; ++i) x[i] = x[i] * a + b;
        }
    }
    T s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    if (s == (T)-1.2345) out[blockIdx.x] = s;   // never true; keeps the chains
}

}  // namespace sphb_probe

using namespace sphb_probe;

// Flops = blocks * 256 * iters * 16 * 8 * 2.  out: blocks elements of the
// probe's type (float for fp64 == 0, double otherwise).  Returns 0, -1 for
// a bad argument, -3 when the launch failed.
extern "C" __attribute__((visibility("default"))) int sphb_fma_probe(int fp64, void *out,
                                                                     int blocks, int iters,
                                                                     void *stream)
{
    if (!out || blocks <= 0 || iters <= 0) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    if (fp64)
        k_fma_probe<double><<<blocks, 256, 0, st>>>((double *)out, iters, 0.999999, 1e-7);
    else
        k_fma_probe<float><<<blocks, 256, 0, st>>>((float *)out, iters, 0.999999f, 1e-7f);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}
