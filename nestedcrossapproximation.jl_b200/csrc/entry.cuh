// Device kernel-entry generator: Helmholtz cis(sign k r)/(4 pi r), Laplace 1/(4 pi r), and a
// matrix-backed kernel (AdaptiveCrossApproximation.PointMatrix, test/test_couplingmatrices.jl:15),
// plus the wavenumber derivatives of the point kernels (gradients on frozen skeletons).
//
// The pivots of the batched build are argmax decisions on these values, so every rounding
// step is spelled out with _rn intrinsics (no contraction, no library sin/cos): the host
// reproduces each entry bit for bit.
//
// sin/cos: Cody-Waite reduction x = q pi/2 + y with pi/2 split into three doubles
// (pi/2 to 161 bits: 0x1.921fb54442d18p+0 + 0x1.1a62633145c07p-54 - 0x1.f1976b7ed8fbcp-110),
// then the Taylor series of sin (degree 17) and cos (degree 18) on |y| <= pi/4 in Horner form;
// coefficients are (-1)^k/(2k+1)! and (-1)^k/(2k)! rounded to double. Valid for |x| < 2^20.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace nca {

struct KernelParams {
    int kind;
    int sign;
    double k;
    double rmin;
    const double2 *mat;  // NCA_KERNEL_MATRIX: device copy, column-major
    int64_t ldmat;
    int deriv;           // 1: entries of dK/dk instead of K (Helmholtz and Laplace only)
};

__device__ __forceinline__ void sincos_cw(double x, double *s, double *c) {
    const double PIO2_1 = 0x1.921fb54442d18p+0;
    const double PIO2_2 = 0x1.1a62633145c07p-54;
    const double PIO2_3 = -0x1.f1976b7ed8fbcp-110;
    const double TWO_OVER_PI = 0x1.45f306dc9c883p-1;
    double q = rint(__dmul_rn(x, TWO_OVER_PI));
    double y = __fma_rn(-q, PIO2_1, x);
    y = __fma_rn(-q, PIO2_2, y);
    y = __fma_rn(-q, PIO2_3, y);
    double y2 = __dmul_rn(y, y);
    double ps = 0x1.952c77030ad4ap-49;
    ps = __fma_rn(ps, y2, -0x1.ae7f3e733b81fp-41);
    ps = __fma_rn(ps, y2, 0x1.6124613a86d09p-33);
    ps = __fma_rn(ps, y2, -0x1.ae64567f544e4p-26);
    ps = __fma_rn(ps, y2, 0x1.71de3a556c734p-19);
    ps = __fma_rn(ps, y2, -0x1.a01a01a01a01ap-13);
    ps = __fma_rn(ps, y2, 0x1.1111111111111p-7);
    ps = __fma_rn(ps, y2, -0x1.5555555555555p-3);
    double sn = __fma_rn(__dmul_rn(y, y2), ps, y);
    double pc = -0x1.6827863b97d97p-53;
    pc = __fma_rn(pc, y2, 0x1.ae7f3e733b81fp-45);
    pc = __fma_rn(pc, y2, -0x1.93974a8c07c9dp-37);
    pc = __fma_rn(pc, y2, 0x1.1eed8eff8d898p-29);
    pc = __fma_rn(pc, y2, -0x1.27e4fb7789f5cp-22);
    pc = __fma_rn(pc, y2, 0x1.a01a01a01a01ap-16);
    pc = __fma_rn(pc, y2, -0x1.6c16c16c16c17p-10);
    pc = __fma_rn(pc, y2, 0x1.5555555555555p-5);
    pc = __fma_rn(pc, y2, -0x1.0000000000000p-1);
    double cs = __fma_rn(y2, pc, 1.0);
    long long iq = (long long)q;
    int quadrant = int(((iq % 4) + 4) % 4);
    switch (quadrant) {
    case 0: *s = sn; *c = cs; break;
    case 1: *s = cs; *c = -sn; break;
    case 2: *s = -sn; *c = -cs; break;
    default: *s = -cs; *c = sn; break;
    }
}

// Entry for test point x (global index i) and trial point y (global index j).
__device__ __forceinline__ double2 kernel_entry(const KernelParams &K, double x0, double x1,
                                                double x2, double y0, double y1, double y2,
                                                int64_t i, int64_t j) {
    if (K.kind == 2) return K.mat[i + j * K.ldmat];
    double dx = __dsub_rn(x0, y0), dy = __dsub_rn(x1, y1), dz = __dsub_rn(x2, y2);
    double d2 = __fma_rn(dx, dx, __fma_rn(dy, dy, __dmul_rn(dz, dz)));
    double r = __dsqrt_rn(d2);
    if (r == 0.0 || r < K.rmin) return make_double2(0.0, 0.0);
    const double FOUR_PI = 0x1.921fb54442d18p+3;
    if (K.deriv) {
        // d/dk cis(sign k r) / (4 pi r) = (-sin(k r) + i sign cos(k r)) / (4 pi); Laplace: 0
        if (K.kind == 1) return make_double2(0.0, 0.0);
        double s, c;
        sincos_cw(__dmul_rn(K.k, r), &s, &c);
        const double inv4pi = __ddiv_rn(1.0, FOUR_PI);
        const double re = -__dmul_rn(s, inv4pi), im = __dmul_rn(c, inv4pi);
        return make_double2(re, K.sign < 0 ? -im : im);
    }
    double inv = __ddiv_rn(1.0, __dmul_rn(FOUR_PI, r));
    if (K.kind == 1) return make_double2(inv, 0.0);
    double s, c;
    sincos_cw(__dmul_rn(K.k, r), &s, &c);
    double re = __dmul_rn(c, inv), im = __dmul_rn(s, inv);
    return make_double2(re, K.sign < 0 ? -im : im);
}

// Complex helpers with the fixed rounding sequence of the pivot search.
__device__ __forceinline__ double2 cmul_rn(double2 a, double2 b) {
    return make_double2(__fma_rn(a.x, b.x, -__dmul_rn(a.y, b.y)),
                        __fma_rn(a.x, b.y, __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double cabs2_rn(double2 a) {
    return __fma_rn(a.x, a.x, __dmul_rn(a.y, a.y));
}

}  // namespace nca
