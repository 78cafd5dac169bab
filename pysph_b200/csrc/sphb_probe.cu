// sphb_probe.cu -- FP32 and FP64 FMA issue-rate probes (sm_100a), the
// compute denominators of the pair passes' roofline (they are bound by
// FP32 issue, not by tensor cores or HBM).
//
// Every thread runs 8 independent FMA chains of `iters` steps (enough in
// flight to fill the FMA pipes), and one lane writes a result so the work
// is kept.  2 flops per FMA.

#include "sphb_common.cuh"

namespace sphb {

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

}  // namespace sphb

using namespace sphb;

// Flops = blocks * 256 * iters * 16 * 8 * 2.  out: blocks elements of the
// probe's type (float for fp64 == 0, double otherwise).
extern "C" int sphb_fma_probe(int fp64, void *out, int blocks, int iters, void *stream)
{
    if (!out || blocks <= 0 || iters <= 0) return SPHB_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (fp64)
        k_fma_probe<double><<<blocks, 256, 0, st>>>((double *)out, iters, 0.999999, 1e-7);
    else
        k_fma_probe<float><<<blocks, 256, 0, st>>>((float *)out, iters, 0.999999f, 1e-7f);
    return launch_status("sphb_fma_probe");
}
