// su3/utils.h -- host-side SU(3) value type of the C++ compatibility layer.
//
// The reference's SU3 is Eigen::Matrix<std::complex<double>,3,3,RowMajor> (src/su3/utils.h:12);
// Eigen is not used here, so SU3 here is a small row-major 3x3 complex value type with
// the operations host code applies to individual links (element access, products, adjoint,
// trace).  SU3Map is the writable view into a field's host links that GaugeField::view_link
// returns (src/gauge/GaugeField.h:49-56).
#pragma once
#include <complex>

using Complex = std::complex<double>;

struct SU3 {
    Complex m[9];
    Complex& operator()(int i, int j) { return m[3 * i + j]; }
    const Complex& operator()(int i, int j) const { return m[3 * i + j]; }
    static SU3 Zero() {
        SU3 r;
        for (auto& e : r.m) e = Complex(0, 0);
        return r;
    }
    static SU3 Identity() {
        SU3 r = Zero();
        r.m[0] = r.m[4] = r.m[8] = Complex(1, 0);
        return r;
    }
    SU3 adjoint() const {
        SU3 r;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) r(i, j) = std::conj((*this)(j, i));
        return r;
    }
    Complex trace() const { return m[0] + m[4] + m[8]; }
    SU3 operator*(const SU3& b) const {
        SU3 r;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                r(i, j) = (*this)(i, 0) * b(0, j) + (*this)(i, 1) * b(1, j) + (*this)(i, 2) * b(2, j);
        return r;
    }
    SU3 operator+(const SU3& b) const {
        SU3 r;
        for (int k = 0; k < 9; k++) r.m[k] = m[k] + b.m[k];
        return r;
    }
    SU3 operator-(const SU3& b) const {
        SU3 r;
        for (int k = 0; k < 9; k++) r.m[k] = m[k] - b.m[k];
        return r;
    }
    SU3& operator+=(const SU3& b) {
        for (int k = 0; k < 9; k++) m[k] += b.m[k];
        return *this;
    }
    void setZero() { *this = Zero(); }
};

// Writable view of one link inside a host link array.
struct SU3Map {
    Complex* p;
    Complex& operator()(int i, int j) { return p[3 * i + j]; }
    const Complex& operator()(int i, int j) const { return p[3 * i + j]; }
    SU3Map& operator=(const SU3& a) {
        for (int k = 0; k < 9; k++) p[k] = a.m[k];
        return *this;
    }
    operator SU3() const {
        SU3 r;
        for (int k = 0; k < 9; k++) r.m[k] = p[k];
        return r;
    }
    SU3 adjoint() const { return SU3(*this).adjoint(); }
    Complex trace() const { return p[0] + p[4] + p[8]; }
};
struct SU3ConstMap {
    const Complex* p;
    const Complex& operator()(int i, int j) const { return p[3 * i + j]; }
    operator SU3() const {
        SU3 r;
        for (int k = 0; k < 9; k++) r.m[k] = p[k];
        return r;
    }
    SU3 adjoint() const { return SU3(*this).adjoint(); }
    Complex trace() const { return p[0] + p[4] + p[8]; }
};
