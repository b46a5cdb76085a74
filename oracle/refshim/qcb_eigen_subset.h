// qcb_eigen_subset.h -- a small dense-matrix library with the Eigen 3.4 API subset that the
// ECMC-QCB hot-path sources use, so those sources compile unchanged into the reference oracle
// (oracle/_ref).  TEST INFRASTRUCTURE ONLY: nothing in the product includes it.
//
// This is project-written code, not Eigen.  It provides fixed-size Matrix (row- or
// column-major storage), Map over caller memory, products, sums, scalar scaling, adjoint,
// trace, 2x2 and 3x3 determinants, squaredNorm/norm/dot/normalize, block<r,c>, col(j) as an
// lvalue or rvalue, setZero/Zero/Identity, the comma initializer and eval().  Every operation is
// evaluated eagerly into a plain matrix.
//
// Arithmetic order (the results the oracle pins depend on it):
//   * product coefficient (i,j) = (a(i,0) b(0,j) + a(i,1) b(1,j)) + a(i,2) b(2,j), k in index
//     order; chained products associate left to right, as the reference writes them;
//   * trace, sums and dot products add in index order;
//   * complex arithmetic is std::complex's;
//   * a / s divides every coefficient by s (normalize divides by sqrt(squaredNorm)).
// Eigen may vectorise a sum into another association; the difference is a rounding of the
// last bit, far inside the 1e-12 bound the parity tests hold.
//
// Two features the reference's sources name but its hot path never calls are declared and
// refuse to run: HouseholderQR (used only by random_su3, the reference's hot start) and the
// matrix exponential of unsupported/Eigen/MatrixFunctions (used only by exp_analytic).  Either
// prints what was called and aborts.
#ifndef QCB_EIGEN_SUBSET_H
#define QCB_EIGEN_SUBSET_H

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <limits>
#include <string>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace Eigen {

enum StorageOptions { ColMajor = 0, RowMajor = 1 };
typedef std::ptrdiff_t Index;

namespace qcb_detail {
template <class T>
struct is_scalar : std::is_arithmetic<T> {};
template <class R>
struct is_scalar<std::complex<R>> : std::true_type {};

template <class S>
struct real_of {
    typedef S type;
};
template <class R>
struct real_of<std::complex<R>> {
    typedef R type;
};

template <class S>
inline S conj(const S& v) {
    return v;
}
template <class R>
inline std::complex<R> conj(const std::complex<R>& v) {
    return std::complex<R>(v.real(), -v.imag());
}
template <class S>
inline S abs2(const S& v) {
    return v * v;
}
template <class R>
inline R abs2(const std::complex<R>& v) {
    return v.real() * v.real() + v.imag() * v.imag();
}

[[noreturn]] inline void not_provided(const char* what) {
    std::fprintf(stderr, "qcb_eigen_subset: %s is not provided (not on the reference's hot path)\n", what);
    std::abort();
}
}  // namespace qcb_detail

template <class S, int R, int C, int Opt = ((R == 1 && C != 1) ? RowMajor : ColMajor)>
class Matrix;

// Common read interface of every matrix-like object: Derived provides Scalar,
// RowsAtCompileTime, ColsAtCompileTime and coeff(i, j).
template <class Derived>
class MatrixBase {
public:
    const Derived& derived() const { return static_cast<const Derived&>(*this); }
    Derived& derived() { return static_cast<Derived&>(*this); }

    Index rows() const { return Derived::RowsAtCompileTime; }
    Index cols() const { return Derived::ColsAtCompileTime; }
    Index size() const { return Derived::RowsAtCompileTime * Derived::ColsAtCompileTime; }
};

template <class D>
using PlainOf = Matrix<typename D::Scalar, D::RowsAtCompileTime, D::ColsAtCompileTime,
                       ((D::RowsAtCompileTime == 1 && D::ColsAtCompileTime != 1) ? RowMajor : ColMajor)>;

// Operations shared by all matrix-like types, written once over coeff().
template <class Derived>
class DenseOps : public MatrixBase<Derived> {
public:
    using MatrixBase<Derived>::derived;

    auto eval() const { return PlainOf<Derived>(derived()); }

    auto adjoint() const {
        typedef typename Derived::Scalar S;
        Matrix<S, Derived::ColsAtCompileTime, Derived::RowsAtCompileTime> r;
        for (int i = 0; i < Derived::RowsAtCompileTime; i++)
            for (int j = 0; j < Derived::ColsAtCompileTime; j++) r(j, i) = qcb_detail::conj(derived().coeff(i, j));
        return r;
    }
    auto transpose() const {
        typedef typename Derived::Scalar S;
        Matrix<S, Derived::ColsAtCompileTime, Derived::RowsAtCompileTime> r;
        for (int i = 0; i < Derived::RowsAtCompileTime; i++)
            for (int j = 0; j < Derived::ColsAtCompileTime; j++) r(j, i) = derived().coeff(i, j);
        return r;
    }
    auto conjugate() const {
        PlainOf<Derived> r;
        for (int i = 0; i < Derived::RowsAtCompileTime; i++)
            for (int j = 0; j < Derived::ColsAtCompileTime; j++) r(i, j) = qcb_detail::conj(derived().coeff(i, j));
        return r;
    }
    auto trace() const {
        typename Derived::Scalar s = derived().coeff(0, 0);
        const int n = std::min(Derived::RowsAtCompileTime, Derived::ColsAtCompileTime);
        for (int i = 1; i < n; i++) s = s + derived().coeff(i, i);
        return s;
    }
    auto sum() const {
        typename Derived::Scalar s = derived().coeff(0, 0);
        bool first = true;
        for (int i = 0; i < Derived::RowsAtCompileTime; i++)
            for (int j = 0; j < Derived::ColsAtCompileTime; j++) {
                if (first) {
                    first = false;
                    continue;
                }
                s = s + derived().coeff(i, j);
            }
        return s;
    }
    auto determinant() const {
        static_assert(Derived::RowsAtCompileTime == Derived::ColsAtCompileTime, "square only");
        static_assert(Derived::RowsAtCompileTime == 2 || Derived::RowsAtCompileTime == 3, "2x2 or 3x3 only");
        const Derived& m = derived();
        if constexpr (Derived::RowsAtCompileTime == 2) {
            return m.coeff(0, 0) * m.coeff(1, 1) - m.coeff(0, 1) * m.coeff(1, 0);
        } else {
            // cofactor expansion along the first row
            return (m.coeff(0, 0) * (m.coeff(1, 1) * m.coeff(2, 2) - m.coeff(1, 2) * m.coeff(2, 1)) -
                    m.coeff(0, 1) * (m.coeff(1, 0) * m.coeff(2, 2) - m.coeff(1, 2) * m.coeff(2, 0))) +
                   m.coeff(0, 2) * (m.coeff(1, 0) * m.coeff(2, 1) - m.coeff(1, 1) * m.coeff(2, 0));
        }
    }
    auto squaredNorm() const {
        typename qcb_detail::real_of<typename Derived::Scalar>::type s = 0;
        for (int i = 0; i < Derived::RowsAtCompileTime; i++)
            for (int j = 0; j < Derived::ColsAtCompileTime; j++) s += qcb_detail::abs2(derived().coeff(i, j));
        return s;
    }
    auto norm() const { return std::sqrt(squaredNorm()); }

    // <this, other> with this conjugated (vectors).
    template <class O>
    auto dot(const MatrixBase<O>& o) const {
        static_assert(Derived::ColsAtCompileTime == 1 || Derived::RowsAtCompileTime == 1, "vectors only");
        const int n = Derived::RowsAtCompileTime * Derived::ColsAtCompileTime;
        typename Derived::Scalar s = qcb_detail::conj(vcoeff(derived(), 0)) * vcoeff(o.derived(), 0);
        for (int i = 1; i < n; i++) s = s + qcb_detail::conj(vcoeff(derived(), i)) * vcoeff(o.derived(), i);
        return s;
    }

    template <int BR, int BC>
    auto block(Index i0, Index j0) const {
        Matrix<typename Derived::Scalar, BR, BC> r;
        for (int i = 0; i < BR; i++)
            for (int j = 0; j < BC; j++) r(i, j) = derived().coeff((int)i0 + i, (int)j0 + j);
        return r;
    }

    // Matrix exponential of unsupported/Eigen/MatrixFunctions: not provided.
    template <class D = Derived>
    PlainOf<D> exp() const {
        qcb_detail::not_provided("MatrixBase::exp (MatrixFunctions)");
    }

protected:
    template <class T>
    static typename T::Scalar vcoeff(const T& v, int i) {
        return T::ColsAtCompileTime == 1 ? v.coeff(i, 0) : v.coeff(0, i);
    }
};

// A writable column of a matrix (col(j) on an lvalue).
template <class M>
class ColRef : public DenseOps<ColRef<M>> {
public:
    typedef typename M::Scalar Scalar;
    static constexpr int RowsAtCompileTime = M::RowsAtCompileTime, ColsAtCompileTime = 1;
    ColRef(M& m, int j) : m_(m), j_(j) {}
    Scalar coeff(int i, int) const { return m_.coeff(i, j_); }
    template <class O>
    ColRef& operator=(const MatrixBase<O>& v) {
        static_assert(O::RowsAtCompileTime * O::ColsAtCompileTime == RowsAtCompileTime, "size mismatch");
        PlainOf<O> tmp(v.derived());
        for (int i = 0; i < RowsAtCompileTime; i++) m_(i, j_) = tmp(i);
        return *this;
    }
    ColRef& operator=(const ColRef& v) {
        Matrix<Scalar, RowsAtCompileTime, 1> tmp(v);
        for (int i = 0; i < RowsAtCompileTime; i++) m_(i, j_) = tmp(i);
        return *this;
    }

private:
    M& m_;
    int j_;
};

// Row-by-row filling of a matrix: m << a, b, c, ...
template <class M>
class CommaInit {
public:
    CommaInit(M& m, const typename M::Scalar& v) : m_(m), k_(0) { put(v); }
    CommaInit& operator,(const typename M::Scalar& v) {
        put(v);
        return *this;
    }

private:
    void put(const typename M::Scalar& v) {
        const int C = M::ColsAtCompileTime;
        if (k_ >= M::RowsAtCompileTime * C) qcb_detail::not_provided("comma initializer past the end");
        m_.coeffRef(k_ / C, k_ % C) = v;
        k_++;
    }
    M& m_;
    int k_;
};

// Storage and element access shared by Matrix and Map, over a data pointer.
template <class Derived, class S, int R, int C, int Opt>
class DenseStorageOps : public DenseOps<Derived> {
public:
    typedef S Scalar;
    static constexpr int RowsAtCompileTime = R, ColsAtCompileTime = C;
    static constexpr bool IsRowMajor = (Opt & RowMajor) != 0;
    static constexpr int offset(int i, int j) { return IsRowMajor ? i * C + j : j * R + i; }
};

template <class S, int R, int C, int Opt>
class Matrix : public DenseStorageOps<Matrix<S, R, C, Opt>, S, R, C, Opt> {
    typedef DenseStorageOps<Matrix<S, R, C, Opt>, S, R, C, Opt> Base;

public:
    using Base::offset;
    typedef S Scalar;
    static constexpr int RowsAtCompileTime = R, ColsAtCompileTime = C;

    // Eigen leaves a default-constructed matrix uninitialised; zero is one valid value of that.
    Matrix() {
        for (int k = 0; k < R * C; k++) d_[k] = S(0);
    }
    Matrix(const S& x, const S& y, const S& z, const S& w) {
        static_assert(R * C == 4, "four-coefficient constructor is for 4-vectors");
        d_[0] = x;
        d_[1] = y;
        d_[2] = z;
        d_[3] = w;
    }
    Matrix(const Matrix&) = default;
    Matrix& operator=(const Matrix&) = default;
    template <class O>
    Matrix(const MatrixBase<O>& o) {
        assign(o.derived());
    }
    template <class O>
    Matrix& operator=(const MatrixBase<O>& o) {
        Matrix tmp;
        tmp.assign(o.derived());
        *this = tmp;
        return *this;
    }

    Scalar coeff(int i, int j) const { return d_[offset(i, j)]; }
    Scalar& coeffRef(int i, int j) { return d_[offset(i, j)]; }
    Scalar& operator()(Index i, Index j) { return d_[offset((int)i, (int)j)]; }
    const Scalar& operator()(Index i, Index j) const { return d_[offset((int)i, (int)j)]; }
    Scalar& operator()(Index k) { return d_[k]; }
    const Scalar& operator()(Index k) const { return d_[k]; }
    Scalar* data() { return d_; }
    const Scalar* data() const { return d_; }

    static Matrix Zero() { return Matrix(); }
    static Matrix Identity() {
        Matrix m;
        for (int i = 0; i < std::min(R, C); i++) m(i, i) = S(1);
        return m;
    }
    void setZero() {
        for (int k = 0; k < R * C; k++) d_[k] = S(0);
    }
    void normalize() {
        auto z = this->squaredNorm();
        if (z > 0) {
            auto n = std::sqrt(z);
            for (int k = 0; k < R * C; k++) d_[k] = d_[k] / n;
        }
    }

    ColRef<Matrix> col(Index j) { return ColRef<Matrix>(*this, (int)j); }
    Matrix<S, R, 1> col(Index j) const {
        Matrix<S, R, 1> v;
        for (int i = 0; i < R; i++) v(i) = coeff(i, (int)j);
        return v;
    }

    template <class O>
    Matrix& operator+=(const MatrixBase<O>& o) {
        Matrix t(o.derived());
        for (int k = 0; k < R * C; k++) d_[k] = d_[k] + t.d_[k];
        return *this;
    }
    template <class O>
    Matrix& operator-=(const MatrixBase<O>& o) {
        Matrix t(o.derived());
        for (int k = 0; k < R * C; k++) d_[k] = d_[k] - t.d_[k];
        return *this;
    }
    template <class O>
    Matrix& operator*=(const MatrixBase<O>& o);  // product, below
    template <class T, class = std::enable_if_t<qcb_detail::is_scalar<T>::value>>
    Matrix& operator*=(const T& s) {
        for (int k = 0; k < R * C; k++) d_[k] = d_[k] * s;
        return *this;
    }
    template <class T, class = std::enable_if_t<qcb_detail::is_scalar<T>::value>>
    Matrix& operator/=(const T& s) {
        for (int k = 0; k < R * C; k++) d_[k] = d_[k] / s;
        return *this;
    }
    CommaInit<Matrix> operator<<(const Scalar& v) { return CommaInit<Matrix>(*this, v); }

    template <class O>
    void assign(const O& o) {
        static_assert(O::RowsAtCompileTime * O::ColsAtCompileTime == R * C, "size mismatch");
        if constexpr ((O::RowsAtCompileTime == R && O::ColsAtCompileTime == C)) {
            for (int i = 0; i < R; i++)
                for (int j = 0; j < C; j++) d_[offset(i, j)] = o.coeff(i, j);
        } else {  // vector <-> transposed vector
            for (int k = 0; k < R * C; k++)
                d_[k] = O::ColsAtCompileTime == 1 ? o.coeff(k, 0) : o.coeff(0, k);
        }
    }

private:
    S d_[R * C];
};

// View of caller-owned coefficients in PlainT's storage order.  Copying a Map copies the view;
// assigning to a Map copies coefficients into the viewed memory (Eigen's semantics).
template <class PlainT>
class Map : public DenseOps<Map<PlainT>> {
    typedef std::remove_const_t<PlainT> Plain;
    static constexpr bool IsConst = std::is_const<PlainT>::value;

public:
    typedef typename Plain::Scalar Scalar;
    static constexpr int RowsAtCompileTime = Plain::RowsAtCompileTime, ColsAtCompileTime = Plain::ColsAtCompileTime;
    typedef std::conditional_t<IsConst, const Scalar*, Scalar*> Pointer;

    explicit Map(Pointer p) : p_(p) {}
    Map(const Map&) = default;
    Map& operator=(const Map& o) {
        static_assert(!IsConst, "assignment to a read-only Map");
        Plain tmp(o);
        store(tmp);
        return *this;
    }
    template <class O>
    Map& operator=(const MatrixBase<O>& o) {
        static_assert(!IsConst, "assignment to a read-only Map");
        Plain tmp(o.derived());
        store(tmp);
        return *this;
    }

    Scalar coeff(int i, int j) const { return p_[Plain::offset(i, j)]; }
    Scalar& coeffRef(int i, int j) {
        static_assert(!IsConst, "write through a read-only Map");
        return p_[Plain::offset(i, j)];
    }
    Scalar operator()(Index i, Index j) const { return p_[Plain::offset((int)i, (int)j)]; }
    template <bool C = IsConst, std::enable_if_t<!C, int> = 0>
    Scalar& operator()(Index i, Index j) {
        return p_[Plain::offset((int)i, (int)j)];
    }
    Pointer data() const { return p_; }

private:
    void store(const Plain& m) {
        for (int i = 0; i < RowsAtCompileTime; i++)
            for (int j = 0; j < ColsAtCompileTime; j++) p_[Plain::offset(i, j)] = m.coeff(i, j);
    }
    Pointer p_;
};

// ---------------------------------------------------------------- arithmetic
template <class A, class B>
Matrix<typename A::Scalar, A::RowsAtCompileTime, B::ColsAtCompileTime> operator*(const MatrixBase<A>& a,
                                                                                   const MatrixBase<B>& b) {
    static_assert(A::ColsAtCompileTime == B::RowsAtCompileTime, "product size mismatch");
    static_assert(std::is_same<typename A::Scalar, typename B::Scalar>::value, "mixed scalar product");
    const A& x = a.derived();
    const B& y = b.derived();
    Matrix<typename A::Scalar, A::RowsAtCompileTime, B::ColsAtCompileTime> r;
    for (int i = 0; i < A::RowsAtCompileTime; i++)
        for (int j = 0; j < B::ColsAtCompileTime; j++) {
            typename A::Scalar s = x.coeff(i, 0) * y.coeff(0, j);
            for (int k = 1; k < A::ColsAtCompileTime; k++) s = s + x.coeff(i, k) * y.coeff(k, j);
            r(i, j) = s;
        }
    return r;
}

template <class S, int R, int C, int Opt>
template <class O>
Matrix<S, R, C, Opt>& Matrix<S, R, C, Opt>::operator*=(const MatrixBase<O>& o) {
    *this = (*this) * o;
    return *this;
}

template <class A, class B>
PlainOf<A> operator+(const MatrixBase<A>& a, const MatrixBase<B>& b) {
    PlainOf<A> r(a.derived());
    PlainOf<A> t(b.derived());
    for (int i = 0; i < A::RowsAtCompileTime; i++)
        for (int j = 0; j < A::ColsAtCompileTime; j++) r(i, j) = r(i, j) + t(i, j);
    return r;
}
template <class A, class B>
PlainOf<A> operator-(const MatrixBase<A>& a, const MatrixBase<B>& b) {
    PlainOf<A> r(a.derived());
    PlainOf<A> t(b.derived());
    for (int i = 0; i < A::RowsAtCompileTime; i++)
        for (int j = 0; j < A::ColsAtCompileTime; j++) r(i, j) = r(i, j) - t(i, j);
    return r;
}
template <class A>
PlainOf<A> operator-(const MatrixBase<A>& a) {
    PlainOf<A> r(a.derived());
    for (int i = 0; i < A::RowsAtCompileTime; i++)
        for (int j = 0; j < A::ColsAtCompileTime; j++) r(i, j) = -r(i, j);
    return r;
}

template <class T, class A, class = std::enable_if_t<qcb_detail::is_scalar<T>::value>>
auto operator*(const T& s, const MatrixBase<A>& a) {
    typedef decltype(s * std::declval<typename A::Scalar>()) S;
    Matrix<S, A::RowsAtCompileTime, A::ColsAtCompileTime> r;
    for (int i = 0; i < A::RowsAtCompileTime; i++)
        for (int j = 0; j < A::ColsAtCompileTime; j++) r(i, j) = s * a.derived().coeff(i, j);
    return r;
}
template <class T, class A, class = std::enable_if_t<qcb_detail::is_scalar<T>::value>>
auto operator*(const MatrixBase<A>& a, const T& s) {
    typedef decltype(std::declval<typename A::Scalar>() * s) S;
    Matrix<S, A::RowsAtCompileTime, A::ColsAtCompileTime> r;
    for (int i = 0; i < A::RowsAtCompileTime; i++)
        for (int j = 0; j < A::ColsAtCompileTime; j++) r(i, j) = a.derived().coeff(i, j) * s;
    return r;
}
template <class T, class A, class = std::enable_if_t<qcb_detail::is_scalar<T>::value>>
auto operator/(const MatrixBase<A>& a, const T& s) {
    typedef decltype(std::declval<typename A::Scalar>() / s) S;
    Matrix<S, A::RowsAtCompileTime, A::ColsAtCompileTime> r;
    for (int i = 0; i < A::RowsAtCompileTime; i++)
        for (int j = 0; j < A::ColsAtCompileTime; j++) r(i, j) = a.derived().coeff(i, j) / s;
    return r;
}

// ---------------------------------------------------------------- decompositions (not provided)
template <class M>
class HouseholderQR {
public:
    template <class O>
    explicit HouseholderQR(const MatrixBase<O>&) {
        qcb_detail::not_provided("HouseholderQR (the reference's random_su3 hot start)");
    }
    M householderQ() const { qcb_detail::not_provided("HouseholderQR::householderQ"); }
};

// ---------------------------------------------------------------- the typedefs the reference names
typedef Matrix<std::complex<double>, 3, 3> Matrix3cd;
typedef Matrix<std::complex<double>, 2, 2> Matrix2cd;
typedef Matrix<std::complex<double>, 3, 1> Vector3cd;
typedef Matrix<double, 4, 1> Vector4d;
typedef Matrix<double, 3, 3> Matrix3d;

}  // namespace Eigen

#endif
