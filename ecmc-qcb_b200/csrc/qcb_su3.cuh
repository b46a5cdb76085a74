// qcb_su3.cuh -- 3x3 complex matrix algebra in registers, templated on the real type.
//
// Device counterparts of the reference's Eigen-based SU(3) helpers
// (src/su3/utils.cpp, src/gauge/GaugeField.cpp).  Matrices are row-major
// (element (i,j) at e[3*i+j]) as in the reference's RowMajor SU3 typedef
// (src/gauge/GaugeField.h:16).
#pragma once
#include <cuda_runtime.h>

#include <cmath>

#define QCB_HD __host__ __device__ __forceinline__

namespace qcb {

template <typename R>
struct Cx {
    R re, im;
};

template <typename R>
QCB_HD Cx<R> mkc(R r, R i) {
    Cx<R> c;
    c.re = r;
    c.im = i;
    return c;
}
template <typename R>
QCB_HD Cx<R> operator+(Cx<R> a, Cx<R> b) { return mkc(a.re + b.re, a.im + b.im); }
template <typename R>
QCB_HD Cx<R> operator-(Cx<R> a, Cx<R> b) { return mkc(a.re - b.re, a.im - b.im); }
template <typename R>
QCB_HD Cx<R> operator*(Cx<R> a, Cx<R> b) { return mkc(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
template <typename R>
QCB_HD Cx<R> scl(R s, Cx<R> a) { return mkc(s * a.re, s * a.im); }
template <typename R>
QCB_HD Cx<R> cconj(Cx<R> a) { return mkc(a.re, -a.im); }
// r += a*b
template <typename R>
QCB_HD void cmac(Cx<R>& r, Cx<R> a, Cx<R> b) {
    r.re = fma(a.re, b.re, fma(-a.im, b.im, r.re));
    r.im = fma(a.re, b.im, fma(a.im, b.re, r.im));
}
// r += a*conj(b)
template <typename R>
QCB_HD void cmac_nc(Cx<R>& r, Cx<R> a, Cx<R> b) {
    r.re = fma(a.re, b.re, fma(a.im, b.im, r.re));
    r.im = fma(a.im, b.re, fma(-a.re, b.im, r.im));
}
// r += conj(a)*b
template <typename R>
QCB_HD void cmac_cn(Cx<R>& r, Cx<R> a, Cx<R> b) {
    r.re = fma(a.re, b.re, fma(a.im, b.im, r.re));
    r.im = fma(a.re, b.im, fma(-a.im, b.re, r.im));
}
// r += conj(a)*conj(b)
template <typename R>
QCB_HD void cmac_cc(Cx<R>& r, Cx<R> a, Cx<R> b) {
    r.re = fma(a.re, b.re, fma(-a.im, b.im, r.re));
    r.im = fma(-a.re, b.im, fma(-a.im, b.re, r.im));
}

template <typename R>
struct M3 {
    Cx<R> e[9];
    QCB_HD Cx<R>& operator()(int i, int j) { return e[i * 3 + j]; }
    QCB_HD const Cx<R>& operator()(int i, int j) const { return e[i * 3 + j]; }
};

template <typename R>
QCB_HD void set_zero(M3<R>& a) {
#pragma unroll
    for (int k = 0; k < 9; k++) a.e[k] = mkc<R>(0, 0);
}
template <typename R>
QCB_HD M3<R> ident() {
    M3<R> a;
    set_zero(a);
    a.e[0] = a.e[4] = a.e[8] = mkc<R>(1, 0);
    return a;
}

template <typename To, typename From>
QCB_HD M3<To> convert(const M3<From>& a) {
    M3<To> r;
#pragma unroll
    for (int k = 0; k < 9; k++) r.e[k] = mkc<To>((To)a.e[k].re, (To)a.e[k].im);
    return r;
}

// r = a*b
template <typename R>
QCB_HD M3<R> mul_nn(const M3<R>& a, const M3<R>& b) {
    M3<R> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s = a(i, 0) * b(0, j);
            cmac(s, a(i, 1), b(1, j));
            cmac(s, a(i, 2), b(2, j));
            r(i, j) = s;
        }
    return r;
}
// r = a*b^dagger
template <typename R>
QCB_HD M3<R> mul_na(const M3<R>& a, const M3<R>& b) {
    M3<R> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s = mkc<R>(0, 0);
            cmac_nc(s, a(i, 0), b(j, 0));
            cmac_nc(s, a(i, 1), b(j, 1));
            cmac_nc(s, a(i, 2), b(j, 2));
            r(i, j) = s;
        }
    return r;
}
// r = a^dagger*b
template <typename R>
QCB_HD M3<R> mul_an(const M3<R>& a, const M3<R>& b) {
    M3<R> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s = mkc<R>(0, 0);
            cmac_cn(s, a(0, i), b(0, j));
            cmac_cn(s, a(1, i), b(1, j));
            cmac_cn(s, a(2, i), b(2, j));
            r(i, j) = s;
        }
    return r;
}
// r += a*b^dagger
template <typename R>
QCB_HD void acc_na(M3<R>& r, const M3<R>& a, const M3<R>& b) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            cmac_nc(r(i, j), a(i, 0), b(j, 0));
            cmac_nc(r(i, j), a(i, 1), b(j, 1));
            cmac_nc(r(i, j), a(i, 2), b(j, 2));
        }
}
// r += a^dagger*b
template <typename R>
QCB_HD void acc_an(M3<R>& r, const M3<R>& a, const M3<R>& b) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            cmac_cn(r(i, j), a(0, i), b(0, j));
            cmac_cn(r(i, j), a(1, i), b(1, j));
            cmac_cn(r(i, j), a(2, i), b(2, j));
        }
}
// r += a*b
template <typename R>
QCB_HD void acc_nn(M3<R>& r, const M3<R>& a, const M3<R>& b) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            cmac(r(i, j), a(i, 0), b(0, j));
            cmac(r(i, j), a(i, 1), b(1, j));
            cmac(r(i, j), a(i, 2), b(2, j));
        }
}
template <typename R>
QCB_HD M3<R> adjoint(const M3<R>& a) {
    M3<R> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r(i, j) = cconj(a(j, i));
    return r;
}

// Re Tr(a * b)
template <typename R>
QCB_HD R re_tr_mul(const M3<R>& a, const M3<R>& b) {
    R s = 0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) s = fma(a(i, k).re, b(k, i).re, fma(-a(i, k).im, b(k, i).im, s));
    return s;
}
// Re Tr(a * b^dagger) = sum_ij Re(a_ij conj(b_ij))
template <typename R>
QCB_HD R re_tr_mul_na(const M3<R>& a, const M3<R>& b) {
    R s = 0;
#pragma unroll
    for (int k = 0; k < 9; k++) s = fma(a.e[k].re, b.e[k].re, fma(a.e[k].im, b.e[k].im, s));
    return s;
}
template <typename R>
QCB_HD R sq_norm(const M3<R>& a) {
    R s = 0;
#pragma unroll
    for (int k = 0; k < 9; k++) s = fma(a.e[k].re, a.e[k].re, fma(a.e[k].im, a.e[k].im, s));
    return s;
}

// proj_lie_su3 (src/su3/utils.cpp:130-134) applied to -a:  B = (A - A^dag)/2, A = B - Tr(B)/3.
// Output is traceless anti-Hermitian with exactly zero real diagonal.
template <typename R>
QCB_HD M3<R> proj_lie(const M3<R>& a) {
    M3<R> b;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            b(i, j).re = R(0.5) * (a(i, j).re - a(j, i).re);
            b(i, j).im = R(0.5) * (a(i, j).im + a(j, i).im);
        }
    R tr3 = (b(0, 0).im + b(1, 1).im + b(2, 2).im) / R(3);
    b(0, 0).im -= tr3;
    b(1, 1).im -= tr3;
    b(2, 2).im -= tr3;
    b(0, 0).re = b(1, 1).re = b(2, 2).re = R(0);
    return b;
}

// 3x3 determinant by cofactor expansion along the first row.
template <typename R>
QCB_HD Cx<R> det3(const M3<R>& m) {
    Cx<R> c0 = m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1);
    Cx<R> c1 = m(1, 0) * m(2, 2) - m(1, 2) * m(2, 0);
    Cx<R> c2 = m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0);
    return (m(0, 0) * c0 - m(0, 1) * c1) + m(0, 2) * c2;
}

// Taylor coefficients 1/n! built by the reference's recurrence c[n] = c[n-1]/n (utils.cpp:163-167).
struct ExpCoeffs {
    double c[19];
    constexpr ExpCoeffs() : c{} {
        c[0] = 1.0;
        for (int n = 1; n <= 18; ++n) c[n] = c[n - 1] / (double)n;
    }
};

// Horner recurrence of exp_su3_luscher (src/su3/utils.cpp:163-186) in double for the invariants
// t = -Re Tr(X^2)/2 and d = Re(i det X): q = (q0, q1, q2) as (re, im) pairs, with
// exp(X) = q0 + q1 X + q2 X^2.  From q_N = c_N: q0' = c_n - i d q2, q1' = q0 - t q2, q2' = q1.
QCB_HD void ch_coeffs(double t, double d, double q[6]) {
    constexpr ExpCoeffs C{};
    double q0r = C.c[18], q0i = 0.0, q1r = 0.0, q1i = 0.0, q2r = 0.0, q2i = 0.0;
#pragma unroll
    for (int n = 17; n >= 0; --n) {
        double n0r = fma(d, q2i, C.c[n]);
        double n0i = -d * q2r;
        double n1r = fma(-t, q2r, q0r);
        double n1i = fma(-t, q2i, q0i);
        q2r = q1r;
        q2i = q1i;
        q0r = n0r;
        q0i = n0i;
        q1r = n1r;
        q1i = n1i;
    }
    q[0] = q0r;
    q[1] = q0i;
    q[2] = q1r;
    q[3] = q1i;
    q[4] = q2r;
    q[5] = q2i;
}

// Invariants t = -Re Tr(X^2)/2 and d = Re(i det X) of an anti-Hermitian X (X_ji = -conj(X_ij),
// zero real diagonal) in double from its independent entries.  With X = iH and a_i = Im X_ii:
//   t = |X01|^2 + |X02|^2 + |X12|^2 + (a0^2 + a1^2 + a2^2)/2,
//   d = det H = a0 a1 a2 + 2 Im(X01 X12 conj(X02)) - a0 |X12|^2 - a1 |X02|^2 - a2 |X01|^2.
// Nine conversions to double instead of eighteen; used for FP32 X, whose force and RK3 forms
// keep the anti-Hermitian symmetry exactly.
template <typename R>
QCB_HD void su3_invariants(const M3<R>& X, double& t, double& d) {
    const double x01r = X(0, 1).re, x01i = X(0, 1).im, x02r = X(0, 2).re, x02i = X(0, 2).im;
    const double x12r = X(1, 2).re, x12i = X(1, 2).im;
    const double a0 = X(0, 0).im, a1 = X(1, 1).im, a2 = X(2, 2).im;
    const double n01 = fma(x01r, x01r, x01i * x01i), n02 = fma(x02r, x02r, x02i * x02i);
    const double n12 = fma(x12r, x12r, x12i * x12i);
    t = (n01 + n02) + n12 + 0.5 * (fma(a0, a0, fma(a1, a1, a2 * a2)));
    const double pr = fma(x01r, x12r, -x01i * x12i), pi = fma(x01r, x12i, x01i * x12r);  // X01 X12
    const double im3 = fma(pi, x02r, -pr * x02i);                                         // Im(p conj(X02))
    d = fma(a0 * a1, a2, fma(2.0, im3, -fma(a0, n12, fma(a1, n02, a2 * n01))));
}

// exp_su3_luscher (src/su3/utils.cpp:145-193): exp(X), X traceless anti-Hermitian, by the
// Cayley-Hamilton form q0 + q1 X + q2 X^2 with the N = 18 Horner recurrence.  The scalar
// invariants and the Horner recurrence run in double for every storage precision R (the
// "Cayley-Hamilton coefficients in FP64" rule); the matrix reconstruction runs in R.
template <typename R>
QCB_HD M3<R> exp_su3(const M3<R>& X) {
    // X^2 is Hermitian: compute the upper triangle and mirror it.
    M3<R> X2;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = i; j < 3; j++) {
            Cx<R> s = X(i, 0) * X(0, j);
            cmac(s, X(i, 1), X(1, j));
            cmac(s, X(i, 2), X(2, j));
            X2(i, j) = s;
        }
    X2(1, 0) = cconj(X2(0, 1));
    X2(2, 0) = cconj(X2(0, 2));
    X2(2, 1) = cconj(X2(1, 2));
    X2(0, 0).im = X2(1, 1).im = X2(2, 2).im = R(0);
    double t, d;
    if constexpr (sizeof(R) == sizeof(double)) {
        const M3<double> Xd = convert<double>(X);
        t = -0.5 * (((double)X2(0, 0).re + (double)X2(1, 1).re) + (double)X2(2, 2).re);
        d = -det3(Xd).im;  // Re(i * det X)
    } else {
        su3_invariants(X, t, d);
    }
    double q[6];
    ch_coeffs(t, d, q);
    Cx<R> q0 = mkc<R>((R)q[0], (R)q[1]), q1 = mkc<R>((R)q[2], (R)q[3]), q2 = mkc<R>((R)q[4], (R)q[5]);
    M3<R> E;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        Cx<R> v = q1 * X.e[k];
        cmac(v, q2, X2.e[k]);
        E.e[k] = v;
    }
    E(0, 0) = E(0, 0) + q0;
    E(1, 1) = E(1, 1) + q0;
    E(2, 2) = E(2, 2) + q0;
    return E;
}

// projection_su3 (src/gauge/GaugeField.cpp:36-58): column Gram-Schmidt, c2 = conj(c0 x c1).
template <typename R>
QCB_HD void project_su3(M3<R>& U) {
    Cx<R> c0[3], c1[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        c0[i] = U(i, 0);
        c1[i] = U(i, 1);
    }
    R n0 = (c0[0].re * c0[0].re + c0[0].im * c0[0].im) + (c0[1].re * c0[1].re + c0[1].im * c0[1].im) +
           (c0[2].re * c0[2].re + c0[2].im * c0[2].im);
    R inv0 = R(1) / sqrt(n0);
#pragma unroll
    for (int i = 0; i < 3; i++) c0[i] = scl(inv0, c0[i]);
    Cx<R> dot = mkc<R>(0, 0);
#pragma unroll
    for (int i = 0; i < 3; i++) cmac_cn(dot, c0[i], c1[i]);
#pragma unroll
    for (int i = 0; i < 3; i++) c1[i] = c1[i] - c0[i] * dot;
    R n1 = (c1[0].re * c1[0].re + c1[0].im * c1[0].im) + (c1[1].re * c1[1].re + c1[1].im * c1[1].im) +
           (c1[2].re * c1[2].re + c1[2].im * c1[2].im);
    R inv1 = R(1) / sqrt(n1);
#pragma unroll
    for (int i = 0; i < 3; i++) c1[i] = scl(inv1, c1[i]);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        U(i, 0) = c0[i];
        U(i, 1) = c1[i];
    }
    U(0, 2) = cconj(c0[1] * c1[2] - c0[2] * c1[1]);
    U(1, 2) = cconj(c0[2] * c1[0] - c0[0] * c1[2]);
    U(2, 2) = cconj(c0[0] * c1[1] - c0[1] * c1[0]);
}

// projection_su3 (src/gauge/GaugeField.cpp:36-58) of an FP32 matrix with the Gram-Schmidt
// arithmetic in double: the first two columns are widened (the third is discarded by the
// projection), each inverse norm is one Newton step y (3 - n y^2) / 2 in double from the FP32
// rsqrtf estimate (relative error ~1e-13, five orders below FP32 rounding), and the result is
// rounded to FP32 once.
QCB_HD void project_su3_f32(M3<float>& U) {
    double c0r[3], c0i[3], c1r[3], c1i[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        c0r[i] = U(i, 0).re;
        c0i[i] = U(i, 0).im;
        c1r[i] = U(i, 1).re;
        c1i[i] = U(i, 1).im;
    }
    auto inv_sqrt = [](double n) {
#ifdef __CUDA_ARCH__
        const double y = (double)rsqrtf((float)n);
#else
        const double y = (double)(1.0f / sqrtf((float)n));
#endif
        return y * fma(-0.5 * n, y * y, 1.5);
    };
    const double n0 = fma(c0r[0], c0r[0], c0i[0] * c0i[0]) + fma(c0r[1], c0r[1], c0i[1] * c0i[1]) +
                      fma(c0r[2], c0r[2], c0i[2] * c0i[2]);
    const double y0 = inv_sqrt(n0);
    double dr = 0.0, di = 0.0;  // conj(c0) . c1
#pragma unroll
    for (int i = 0; i < 3; i++) {
        c0r[i] *= y0;
        c0i[i] *= y0;
        dr = fma(c0r[i], c1r[i], fma(c0i[i], c1i[i], dr));
        di = fma(c0r[i], c1i[i], fma(-c0i[i], c1r[i], di));
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        c1r[i] -= fma(c0r[i], dr, -c0i[i] * di);
        c1i[i] -= fma(c0r[i], di, c0i[i] * dr);
    }
    const double n1 = fma(c1r[0], c1r[0], c1i[0] * c1i[0]) + fma(c1r[1], c1r[1], c1i[1] * c1i[1]) +
                      fma(c1r[2], c1r[2], c1i[2] * c1i[2]);
    const double y1 = inv_sqrt(n1);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        c1r[i] *= y1;
        c1i[i] *= y1;
        U(i, 0) = mkc<float>((float)c0r[i], (float)c0i[i]);
        U(i, 1) = mkc<float>((float)c1r[i], (float)c1i[i]);
    }
    // c2 = conj(c0 x c1)
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int a = (i + 1) % 3, b = (i + 2) % 3;
        const double re = fma(c0r[a], c1r[b], -c0i[a] * c1i[b]) - fma(c0r[b], c1r[a], -c0i[b] * c1i[a]);
        const double im = fma(c0r[a], c1i[b], c0i[a] * c1r[b]) - fma(c0r[b], c1i[a], c0i[b] * c1r[a]);
        U(i, 2) = mkc<float>((float)re, (float)-im);
    }
}

// SU(3) reprojection in double after an FP64 or FP32 update: projection_su3 on double links,
// project_su3_f32 on FP32 links.
template <typename R>
QCB_HD void reproject_fp64(M3<R>& U) {
    if constexpr (sizeof(R) == sizeof(double)) {
        project_su3(U);
    } else {
        project_su3_f32(U);
    }
}

// conj(a b - c d) with a fixed sequence of fused multiply-adds, so that every staple routine that
// rebuilds a third row rounds it identically.
template <typename R>
QCB_HD Cx<R> conj_cross(Cx<R> a, Cx<R> b, Cx<R> c, Cx<R> d) {
    const R re = fma(a.re, b.re, fma(-a.im, b.im, fma(-c.re, d.re, c.im * d.im)));
    const R im = fma(a.re, b.im, fma(a.im, b.re, fma(-c.re, d.im, -(c.im * d.re))));
    return mkc<R>(re, -im);
}

// Third row of an SU(3) matrix from its first two: r2 = conj(r0 x r1).
template <typename R>
QCB_HD void rebuild_row2(M3<R>& U) {
    U(2, 0) = cconj(U(0, 1) * U(1, 2) - U(0, 2) * U(1, 1));
    U(2, 1) = cconj(U(0, 2) * U(1, 0) - U(0, 0) * U(1, 2));
    U(2, 2) = cconj(U(0, 0) * U(1, 1) - U(0, 1) * U(1, 0));
}

}  // namespace qcb
