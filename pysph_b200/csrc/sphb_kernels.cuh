// sphb_kernels.cuh -- the smoothing kernels of the pair passes.
//
// Kern<KT> (KT = SPHB_KERNEL_*) gives, for one kernel type:
//   norm<DIM>()             _fac(1.0), the normalisation at h = 1
//   w_bf(q, fac)            W = fac val(q), FP32, branch-free (every piece
//                           computed, one selected) for the list loops
//   gw_bf(q, ir, ih, fac_ih) dW/dr / r in the reference's sign convention,
//                           so grad_a W = (x_a - x_b) gw; FP32
//   w_d<DIM>(r, h), gw_d<DIM>(r, h)  the FP64 forms with the reference's
//                           operations in its order
// with fac = norm<DIM>() / h^DIM, ih = 1 / h, ir = 1 / r, fac_ih = fac ih.
// For r = 0 the FP32 forms see ir = 1/sqrt(1e-30) (finite); every caller
// multiplies gw by r_ab = 0 there.

#pragma once

#include "sphb_common.cuh"

namespace sphb {

template <int KT>
struct Kern;

// CubicSplineKernel (S/base/kernels.pyx:349-454): support 2h,
// val = 1 - 1.5 q^2 (1 - q/2) (q <= 1), (2 - q)^3 / 4 (q <= 2), 0.
template <>
struct Kern<SPHB_KERNEL_CUBIC> {
    template <int DIM>
    __host__ __device__ static double norm() { return kfac_unit<DIM>(); }

    // q < 1: 1 + q^2 (0.75 q - 1.5); else t1^3 / 4 with t1 = max(2 - q, 0)
    __device__ __forceinline__ static float w_bf(float q, float fac)
    {
        const float t1 = fmaxf(2.0f - q, 0.0f);
        const float inner = fmaf(q * q, fmaf(0.75f, q, -1.5f), 1.0f);
        const float outer = 0.25f * (t1 * t1 * t1);
        return fac * (q < 1.0f ? inner : outer);
    }

    // q < 1: (2.25 q - 3) ih; else -0.75 t1^2 / r
    __device__ __forceinline__ static float gw_bf(float q, float ir, float ih, float fac_ih)
    {
        const float t1 = fmaxf(2.0f - q, 0.0f);
        const float inner = (2.25f * q - 3.0f) * ih;
        const float outer = -0.75f * t1 * t1 * ir;
        return fac_ih * (q < 1.0f ? inner : outer);
    }

    template <int DIM>
    __device__ __forceinline__ static double w_d(double rab, double h)
    {
        const double q = rab / h;
        double val;
        const double fac = (DIM == 2 ? 1.0 / (h * h) : 1.0 / (h * h * h)) * kfac_unit<DIM>();
        if (q > 2.0)
            val = 0.0;
        else if (q > 1.0)
            val = 0.25 * (2 - q) * (2 - q) * (2 - q);
        else
            val = 1 - 1.5 * (q * q) * (1 - 0.5 * q);
        return val * fac;
    }

    template <int DIM>
    __device__ __forceinline__ static double gw_d(double rab, double h)
    {
        const double q = rab / h;
        double val = 0.0;
        const double fac = (DIM == 2 ? 1.0 / (h * h) : 1.0 / (h * h * h)) * kfac_unit<DIM>();
        if (q > 2.0) {
        } else if (q >= 1.0) {
            val = -0.75 * (2 - q) * (2 - q) / (h * rab);
        } else if (q > 1e-14) {
            val = 3.0 * (0.75 * q - 1) / (h * h);
        }
        return val * fac;
    }
};

// QuinticSplineKernel (S/base/kernels.pyx:461-560), 2D: support 3h,
// fac = 7 / (478 pi).  Kept as the reference has them: W adds (1 - q)^5 with
// weight 1, and the gradient uses val = 5 t3^4 - 30 t2^4 + 75 t1^4 (the
// opposite sign of dW/dq), t_k = max(k - q, 0).
template <>
struct Kern<SPHB_KERNEL_QUINTIC> {
    template <int DIM>
    __host__ __device__ static double norm()
    {
        return DIM == 2 ? 7. / (478 * 3.141592653589793 * 1.0 * 1.0) : 0.0;
    }

    __device__ __forceinline__ static float p4(float t)
    {
        const float t2 = t * t;
        return t2 * t2;
    }

    __device__ __forceinline__ static float w_bf(float q, float fac)
    {
        const float t3 = fmaxf(3.0f - q, 0.0f);
        const float t2 = fmaxf(2.0f - q, 0.0f);
        const float t1 = fmaxf(1.0f - q, 0.0f);
        return fac * fmaf(p4(t1), t1, fmaf(-6.0f * p4(t2), t2, p4(t3) * t3));
    }

    __device__ __forceinline__ static float gw_bf(float q, float ir, float, float fac_ih)
    {
        const float t3 = fmaxf(3.0f - q, 0.0f);
        const float t2 = fmaxf(2.0f - q, 0.0f);
        const float t1 = fmaxf(1.0f - q, 0.0f);
        return fac_ih * ir * fmaf(75.0f, p4(t1), fmaf(-30.0f, p4(t2), 5.0f * p4(t3)));
    }

    template <int DIM>
    __device__ __forceinline__ static double w_d(double rab, double h)
    {
        const double fac = norm<DIM>() * (1.0 / (h * h));
        const double q = rab / h;
        double val;
        double tmp1 = (3 - q), tmp2 = (2 - q), tmp3 = (1 - q);
        if (q > 3.0) {
            val = 0.0;
        } else {
            tmp1 = __dmul_rn(tmp1, __dmul_rn(__dmul_rn(__dmul_rn(tmp1, tmp1), tmp1), tmp1));
            if (q > 2.0) {
                val = tmp1;
            } else {
                tmp2 = __dmul_rn(tmp2, __dmul_rn(__dmul_rn(__dmul_rn(tmp2, tmp2), tmp2), tmp2));
                val = __dsub_rn(tmp1, __dmul_rn(6.0, tmp2));
                if (!(q > 1.0)) {
                    tmp3 = __dmul_rn(tmp3, __dmul_rn(__dmul_rn(__dmul_rn(tmp3, tmp3), tmp3), tmp3));
                    val = __dadd_rn(val, tmp3);
                }
            }
        }
        return val * fac;
    }

    template <int DIM>
    __device__ __forceinline__ static double gw_d(double rab, double h)
    {
        double fac = norm<DIM>() * (1.0 / (h * h));
        const double q = rab / h;
        double val;
        double tmp1 = (3 - q), tmp2 = (2 - q), tmp3 = (1 - q);
        if (rab < 1e-16) {
            val = 0.0;
        } else {
            fac *= 1. / (h * rab);
            if (q > 3.0) {
                val = 0.0;
            } else {
                tmp1 = __dmul_rn(tmp1, __dmul_rn(__dmul_rn(tmp1, tmp1), tmp1));
                if (q > 2.0) {
                    val = __dmul_rn(5.0, tmp1);
                } else {
                    tmp2 = __dmul_rn(tmp2, __dmul_rn(__dmul_rn(tmp2, tmp2), tmp2));
                    val = __dsub_rn(__dmul_rn(5.0, tmp1), __dmul_rn(30.0, tmp2));
                    if (!(q > 1.0)) {
                        tmp3 = __dmul_rn(tmp3, __dmul_rn(__dmul_rn(tmp3, tmp3), tmp3));
                        val = __dadd_rn(val, __dmul_rn(75.0, tmp3));
                    }
                }
            }
        }
        return val * fac;
    }
};

// WendlandQuinticSplineKernel (S/base/kernels.pyx:562-640), 2D: support 2h,
// val = (1 - q/2)^4 (2q + 1).  Its _fac is written (7./4*PI*h*h), so the
// normalisation is 7 pi / 4 (not 7 / (4 pi)), kept as there.
template <>
struct Kern<SPHB_KERNEL_WENDLAND> {
    template <int DIM>
    __host__ __device__ static double norm()
    {
        return DIM == 2 ? (7. / 4 * 3.141592653589793 * 1.0 * 1.0) : 0.0;
    }

    __device__ __forceinline__ static float w_bf(float q, float fac)
    {
        const float t = fmaxf(fmaf(-0.5f, q, 1.0f), 0.0f);
        const float t2 = t * t;
        return fac * (t2 * t2 * fmaf(2.0f, q, 1.0f));
    }

    // dW/dr / r = -5 q t^3 fac / (h r) = -5 t^3 fac / h^2
    __device__ __forceinline__ static float gw_bf(float q, float, float ih, float fac_ih)
    {
        const float t = fmaxf(fmaf(-0.5f, q, 1.0f), 0.0f);
        return fac_ih * ih * (-5.0f * (t * t * t));
    }

    template <int DIM>
    __device__ __forceinline__ static double w_d(double rab, double h)
    {
        const double fac = norm<DIM>() * (1.0 / (h * h));
        const double q = rab / h;
        double val;
        double tmp = __dsub_rn(1.0, __dmul_rn(0.5, q));
        if (q > 2.0) {
            val = 0.0;
        } else {
            tmp = __dmul_rn(tmp, __dmul_rn(__dmul_rn(tmp, tmp), tmp));
            tmp = __dmul_rn(tmp, __dadd_rn(__dmul_rn(2.0, q), 1.0));
            val = tmp;
        }
        return val * fac;
    }

    template <int DIM>
    __device__ __forceinline__ static double gw_d(double rab, double h)
    {
        double fac = norm<DIM>() * (1.0 / (h * h));
        const double q = rab / h;
        double val;
        double tmp = __dsub_rn(1.0, __dmul_rn(0.5, q));
        if (rab < 1e-16) {
            val = 0.0;
        } else {
            fac *= 1. / (h * rab);
            if (q > 2.0) {
                val = 0;
            } else {
                tmp = __dmul_rn(tmp, __dmul_rn(tmp, tmp));
                val = __dmul_rn(__dmul_rn(tmp, -5.0), q);
            }
        }
        return val * fac;
    }
};

}  // namespace sphb
