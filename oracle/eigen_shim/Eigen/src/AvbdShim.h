// Fixed-size, eagerly evaluated linear algebra with the subset of the Eigen 3.4
// API that the SkyePhyX physics sources use (src/physics/*, src/helpers/math.*,
// src/helpers/geometry.*).  TEST INFRASTRUCTURE ONLY: it exists so that the
// reference's own .cpp files compile unmodified into the CPU oracle; nothing in
// the shipped library includes it.
//
// Eigen 3.4.0 (pinned by the reference's CMakeLists.txt:86-91) is not available
// offline, so this header restates the documented behaviour of each entry point
// from the mathematics:
//   * storage is column-major; products, dot products and norms accumulate
//     left to right (k = 0, 1, 2, ...), which is the arithmetic order the CUDA
//     kernels reproduce where bit-exactness is required (narrowphase);
//   * LDLT: symmetric diagonal pivoting (largest remaining |pivot| of the Schur
//     complement), solve uses the pseudo-inverse of D (pivots with
//     |d| <= numeric_limits<S>::min() give a zero component);
//   * JacobiSVD: one-sided (Hestenes) Jacobi, singular values non-negative and
//     sorted in decreasing order, U completed to a full orthonormal basis;
//   * SelfAdjointEigenSolver: cyclic Jacobi, eigenvalues increasing, unit
//     eigenvectors;
//   * Quaternion: coefficients stored (x, y, z, w); Hamilton product; rotation
//     of a vector by v + w*t + u x t with t = 2 (u x v).
// No test of the reference pins results at this boundary, so agreement with
// the genuine Eigen library is unpinned (rounding-level differences only).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <type_traits>

namespace Eigen {

enum DecompositionOptions {
    ComputeFullU = 0x04,
    ComputeThinU = 0x08,
    ComputeFullV = 0x10,
    ComputeThinV = 0x20
};

template <typename S, int R, int C> class Matrix;
template <typename S, int R, int C> class Block;
template <typename S, int N> class DiagonalMatrix;

// ---------------------------------------------------------------------------
// DenseBase: every dense object is (pointer, outer stride), column-major.
// ---------------------------------------------------------------------------
template <typename D, typename S, int R, int C>
class DenseBase {
public:
    typedef S Scalar;
    enum { RowsAtCompileTime = R, ColsAtCompileTime = C, SizeAtCompileTime = R * C };

    const D& derived() const { return *static_cast<const D*>(this); }
    D& derived() { return *static_cast<D*>(this); }

    S* ptr() const { return derived().ptr_(); }
    int ostride() const { return derived().ostride_(); }

    int rows() const { return R; }
    int cols() const { return C; }
    int size() const { return R * C; }

    S& operator()(int i, int j) const { return ptr()[i + j * ostride()]; }
    S& lin(int k) const {
        if (C == 1) return ptr()[k];
        if (R == 1) return ptr()[k * ostride()];
        return ptr()[(k % R) + (k / R) * ostride()];
    }
    S& operator()(int k) const { return lin(k); }
    S& operator[](int k) const { return lin(k); }
    S& x() const { return lin(0); }
    S& y() const { return lin(1); }
    S& z() const { return lin(2); }
    S& w() const { return lin(3); }
    S* data() const { return ptr(); }

    Matrix<S, R, C> eval() const { return Matrix<S, R, C>(*this); }

    // ---- views ----
    template <int N> Block<S, N, 1> head() const { return Block<S, N, 1>(ptr(), ostride()); }
    template <int N> Block<S, N, 1> tail() const { return Block<S, N, 1>(ptr() + (R * C - N), ostride()); }
    template <int N> Block<S, N, 1> segment(int i) const { return Block<S, N, 1>(ptr() + i, ostride()); }
    template <int BR, int BC> Block<S, BR, BC> block(int i, int j) const {
        return Block<S, BR, BC>(ptr() + i + j * ostride(), ostride());
    }
    Block<S, R, 1> col(int j) const { return Block<S, R, 1>(ptr() + j * ostride(), ostride()); }
    Block<S, 1, C> row(int i) const { return Block<S, 1, C>(ptr() + i, ostride()); }

    // ---- writes ----
    D& setZero() { for (int k = 0; k < R * C; ++k) lin(k) = S(0); return derived(); }
    D& setOnes() { for (int k = 0; k < R * C; ++k) lin(k) = S(1); return derived(); }
    D& setConstant(S v) { for (int k = 0; k < R * C; ++k) lin(k) = v; return derived(); }
    D& fill(S v) { return setConstant(v); }
    D& setIdentity() {
        for (int j = 0; j < C; ++j)
            for (int i = 0; i < R; ++i) (*this)(i, j) = (i == j) ? S(1) : S(0);
        return derived();
    }
    D& noalias() { return derived(); }
    void normalize() {
        S n2 = squaredNorm();
        if (n2 > S(0)) {
            S n = std::sqrt(n2);
            for (int k = 0; k < R * C; ++k) lin(k) = lin(k) / n;
        }
    }
    template <typename D2> D& operator+=(const DenseBase<D2, S, R, C>& o) {
        Matrix<S, R, C> t(o);
        for (int k = 0; k < R * C; ++k) lin(k) = lin(k) + t.lin(k);
        return derived();
    }
    template <typename D2> D& operator-=(const DenseBase<D2, S, R, C>& o) {
        Matrix<S, R, C> t(o);
        for (int k = 0; k < R * C; ++k) lin(k) = lin(k) - t.lin(k);
        return derived();
    }
    template <typename T, typename = typename std::enable_if<std::is_arithmetic<T>::value>::type>
    D& operator*=(T s) { for (int k = 0; k < R * C; ++k) lin(k) = lin(k) * S(s); return derived(); }
    template <typename T, typename = typename std::enable_if<std::is_arithmetic<T>::value>::type>
    D& operator/=(T s) { for (int k = 0; k < R * C; ++k) lin(k) = lin(k) / S(s); return derived(); }

    // ---- reductions (left to right) ----
    S sum() const { S s = lin(0); for (int k = 1; k < R * C; ++k) s = s + lin(k); return s; }
    S squaredNorm() const { S s = lin(0) * lin(0); for (int k = 1; k < R * C; ++k) s = s + lin(k) * lin(k); return s; }
    S norm() const { return std::sqrt(squaredNorm()); }
    S trace() const { S s = (*this)(0, 0); for (int i = 1; i < (R < C ? R : C); ++i) s = s + (*this)(i, i); return s; }
    S maxCoeff() const { S m = lin(0); for (int k = 1; k < R * C; ++k) if (lin(k) > m) m = lin(k); return m; }
    S minCoeff() const { S m = lin(0); for (int k = 1; k < R * C; ++k) if (lin(k) < m) m = lin(k); return m; }
    template <typename D2, int R2, int C2> S dot(const DenseBase<D2, S, R2, C2>& o) const {
        static_assert(R * C == R2 * C2, "dot: size mismatch");
        S s = lin(0) * o.lin(0);
        for (int k = 1; k < R * C; ++k) s = s + lin(k) * o.lin(k);
        return s;
    }
    template <typename D2, int R2, int C2> Matrix<S, 3, 1> cross(const DenseBase<D2, S, R2, C2>& o) const {
        static_assert(R * C == 3 && R2 * C2 == 3, "cross: 3-vectors only");
        return Matrix<S, 3, 1>(lin(1) * o.lin(2) - lin(2) * o.lin(1),
                               lin(2) * o.lin(0) - lin(0) * o.lin(2),
                               lin(0) * o.lin(1) - lin(1) * o.lin(0));
    }

    // ---- value-returning operations ----
    Matrix<S, R, C> normalized() const {
        Matrix<S, R, C> r(*this);
        r.normalize();
        return r;
    }
    Matrix<S, C, R> transpose() const {
        Matrix<S, C, R> r;
        for (int j = 0; j < C; ++j)
            for (int i = 0; i < R; ++i) r(j, i) = (*this)(i, j);
        return r;
    }
    Matrix<S, C, R> adjoint() const { return transpose(); }
    Matrix<S, R, C> cwiseAbs() const { Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = std::abs(lin(k)); return r; }
    Matrix<S, R, C> cwiseInverse() const { Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = S(1) / lin(k); return r; }
    template <typename D2> Matrix<S, R, C> cwiseMin(const DenseBase<D2, S, R, C>& o) const {
        Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = std::min(lin(k), o.lin(k)); return r;
    }
    template <typename D2> Matrix<S, R, C> cwiseMax(const DenseBase<D2, S, R, C>& o) const {
        Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = std::max(lin(k), o.lin(k)); return r;
    }
    template <typename D2> Matrix<S, R, C> cwiseProduct(const DenseBase<D2, S, R, C>& o) const {
        Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = lin(k) * o.lin(k); return r;
    }
    DiagonalMatrix<S, R * C> asDiagonal() const { return DiagonalMatrix<S, R * C>(Matrix<S, R * C, 1>(*this)); }

    S determinant() const {
        static_assert(R == C, "determinant: square only");
        const DenseBase& m = *this;
        if (R == 1) return m(0, 0);
        if (R == 2) return m(0, 0) * m(1, 1) - m(0, 1) * m(1, 0);
        if (R == 3) {
            return m(0, 0) * (m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1))
                 - m(1, 0) * (m(0, 1) * m(2, 2) - m(0, 2) * m(2, 1))
                 + m(2, 0) * (m(0, 1) * m(1, 2) - m(0, 2) * m(1, 1));
        }
        // generic: Gaussian elimination with partial pivoting
        Matrix<S, R, C> a(*this);
        S det = S(1);
        for (int k = 0; k < R; ++k) {
            int p = k;
            for (int i = k + 1; i < R; ++i) if (std::abs(a(i, k)) > std::abs(a(p, k))) p = i;
            if (a(p, k) == S(0)) return S(0);
            if (p != k) { for (int j = 0; j < C; ++j) std::swap(a(k, j), a(p, j)); det = -det; }
            det = det * a(k, k);
            for (int i = k + 1; i < R; ++i) {
                S f = a(i, k) / a(k, k);
                for (int j = k; j < C; ++j) a(i, j) = a(i, j) - f * a(k, j);
            }
        }
        return det;
    }
    Matrix<S, R, C> inverse() const;

    class LDLTType;
};

// ---------------------------------------------------------------------------
// Matrix (owning storage)
// ---------------------------------------------------------------------------
template <typename S, int R, int C>
class Matrix : public DenseBase<Matrix<S, R, C>, S, R, C> {
    S m_[R * C];
public:
    typedef DenseBase<Matrix<S, R, C>, S, R, C> Base;
    S* ptr_() const { return const_cast<S*>(m_); }
    int ostride_() const { return R; }

    Matrix() { for (int k = 0; k < R * C; ++k) m_[k] = S(0); }
    Matrix(const Matrix& o) { std::memcpy(m_, o.m_, sizeof(m_)); }
    template <typename D2> Matrix(const DenseBase<D2, S, R, C>& o) {
        for (int j = 0; j < C; ++j)
            for (int i = 0; i < R; ++i) m_[i + j * R] = o(i, j);
    }
    Matrix(const DiagonalMatrix<S, R>& d);
    Matrix(S a, S b) { static_assert(R * C == 2, "2 coefficients"); m_[0] = a; m_[1] = b; }
    Matrix(S a, S b, S c) { static_assert(R * C == 3, "3 coefficients"); m_[0] = a; m_[1] = b; m_[2] = c; }
    Matrix(S a, S b, S c, S d) { static_assert(R * C == 4, "4 coefficients"); m_[0] = a; m_[1] = b; m_[2] = c; m_[3] = d; }
    Matrix(S a, S b, S c, S d, S e, S f) {
        static_assert(R * C == 6, "6 coefficients");
        m_[0] = a; m_[1] = b; m_[2] = c; m_[3] = d; m_[4] = e; m_[5] = f;
    }

    Matrix& operator=(const Matrix& o) { std::memcpy(m_, o.m_, sizeof(m_)); return *this; }
    template <typename D2> Matrix& operator=(const DenseBase<D2, S, R, C>& o) {
        Matrix t(o);
        std::memcpy(m_, t.m_, sizeof(m_));
        return *this;
    }
    Matrix& operator=(const DiagonalMatrix<S, R>& d) { *this = Matrix(d); return *this; }

    static Matrix Zero() { return Matrix(); }
    static Matrix Ones() { Matrix r; r.setOnes(); return r; }
    static Matrix Constant(S v) { Matrix r; r.setConstant(v); return r; }
    static Matrix Identity() { Matrix r; r.setIdentity(); return r; }
    static Matrix Unit(int i) { Matrix r; r.lin(i) = S(1); return r; }
    static Matrix UnitX() { return Unit(0); }
    static Matrix UnitY() { return Unit(1); }
    static Matrix UnitZ() { return Unit(2); }

    // comma initializer (row-major fill order, as documented)
    struct CommaInit {
        Matrix* m; int k;
        CommaInit& operator,(S v) { int i = k / C, j = k % C; (*m)(i, j) = v; ++k; return *this; }
    };
    CommaInit operator<<(S v) { (*this)(0, 0) = v; return CommaInit{this, 1}; }

    typename Base::LDLTType ldlt() const;
};

// ---------------------------------------------------------------------------
// Block / Map (non-owning strided view)
// ---------------------------------------------------------------------------
template <typename S, int R, int C>
class Block : public DenseBase<Block<S, R, C>, S, R, C> {
    S* p_; int s_;
public:
    S* ptr_() const { return p_; }
    int ostride_() const { return s_; }
    Block(S* p, int s) : p_(p), s_(s) {}
    Block(const Block& o) = default;
    Block& operator=(const Block& o) {
        Matrix<S, R, C> t(o);
        for (int j = 0; j < C; ++j) for (int i = 0; i < R; ++i) (*this)(i, j) = t(i, j);
        return *this;
    }
    template <typename D2> Block& operator=(const DenseBase<D2, S, R, C>& o) {
        Matrix<S, R, C> t(o);
        for (int j = 0; j < C; ++j) for (int i = 0; i < R; ++i) (*this)(i, j) = t(i, j);
        return *this;
    }
    Block& operator=(const Matrix<S, R, C>& o) {
        for (int j = 0; j < C; ++j) for (int i = 0; i < R; ++i) (*this)(i, j) = o(i, j);
        return *this;
    }
};

template <typename MatrixType> class Map;
template <typename S, int R, int C>
class Map<Matrix<S, R, C>> : public DenseBase<Map<Matrix<S, R, C>>, S, R, C> {
    S* p_;
public:
    S* ptr_() const { return p_; }
    int ostride_() const { return R; }
    explicit Map(S* p) : p_(p) {}
    explicit Map(const S* p) : p_(const_cast<S*>(p)) {}
    template <typename D2> Map& operator=(const DenseBase<D2, S, R, C>& o) {
        Matrix<S, R, C> t(o);
        for (int k = 0; k < R * C; ++k) p_[k] = t.lin(k);
        return *this;
    }
    Map& operator=(const Map& o) { return operator=(static_cast<const DenseBase<Map, S, R, C>&>(o)); }
};

// ---------------------------------------------------------------------------
// Diagonal matrices
// ---------------------------------------------------------------------------
template <typename S, int N>
class DiagonalMatrix {
public:
    Matrix<S, N, 1> d;
    explicit DiagonalMatrix(const Matrix<S, N, 1>& v) : d(v) {}
    DiagonalMatrix inverse() const { return DiagonalMatrix(d.cwiseInverse()); }
    Matrix<S, N, 1> diagonal() const { return d; }
};

template <typename S, int R, int C>
Matrix<S, R, C>::Matrix(const DiagonalMatrix<S, R>& dm) {
    static_assert(R == C, "diagonal to square matrix");
    for (int j = 0; j < C; ++j)
        for (int i = 0; i < R; ++i) m_[i + j * R] = (i == j) ? dm.d.lin(i) : S(0);
}

template <typename S, int N, typename D2, int C>
Matrix<S, N, C> operator*(const DiagonalMatrix<S, N>& dm, const DenseBase<D2, S, N, C>& m) {
    Matrix<S, N, C> r;
    for (int j = 0; j < C; ++j)
        for (int i = 0; i < N; ++i) r(i, j) = dm.d.lin(i) * m(i, j);
    return r;
}
template <typename S, int N, typename D1, int R>
Matrix<S, R, N> operator*(const DenseBase<D1, S, R, N>& m, const DiagonalMatrix<S, N>& dm) {
    Matrix<S, R, N> r;
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < R; ++i) r(i, j) = m(i, j) * dm.d.lin(j);
    return r;
}

// ---------------------------------------------------------------------------
// Arithmetic operators (eager)
// ---------------------------------------------------------------------------
template <typename D1, typename D2, typename S, int R, int C>
Matrix<S, R, C> operator+(const DenseBase<D1, S, R, C>& a, const DenseBase<D2, S, R, C>& b) {
    Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = a.lin(k) + b.lin(k); return r;
}
template <typename D1, typename D2, typename S, int R, int C>
Matrix<S, R, C> operator-(const DenseBase<D1, S, R, C>& a, const DenseBase<D2, S, R, C>& b) {
    Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = a.lin(k) - b.lin(k); return r;
}
template <typename D1, typename S, int R, int C>
Matrix<S, R, C> operator-(const DenseBase<D1, S, R, C>& a) {
    Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = -a.lin(k); return r;
}
template <typename D1, typename D2, typename S, int R, int K, int C>
Matrix<S, R, C> operator*(const DenseBase<D1, S, R, K>& a, const DenseBase<D2, S, K, C>& b) {
    Matrix<S, R, C> r;
    for (int j = 0; j < C; ++j)
        for (int i = 0; i < R; ++i) {
            S s = a(i, 0) * b(0, j);
            for (int k = 1; k < K; ++k) s = s + a(i, k) * b(k, j);
            r(i, j) = s;
        }
    return r;
}
template <typename D1, typename S, int R, int C, typename T,
          typename = typename std::enable_if<std::is_arithmetic<T>::value>::type>
Matrix<S, R, C> operator*(const DenseBase<D1, S, R, C>& a, T s) {
    Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = a.lin(k) * S(s); return r;
}
template <typename D1, typename S, int R, int C, typename T,
          typename = typename std::enable_if<std::is_arithmetic<T>::value>::type>
Matrix<S, R, C> operator*(T s, const DenseBase<D1, S, R, C>& a) {
    Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = S(s) * a.lin(k); return r;
}
template <typename D1, typename S, int R, int C, typename T,
          typename = typename std::enable_if<std::is_arithmetic<T>::value>::type>
Matrix<S, R, C> operator/(const DenseBase<D1, S, R, C>& a, T s) {
    Matrix<S, R, C> r; for (int k = 0; k < R * C; ++k) r.lin(k) = a.lin(k) / S(s); return r;
}

// inverse via the adjugate (2x2, 3x3) or Gauss-Jordan (larger)
template <typename D, typename S, int R, int C>
Matrix<S, R, C> DenseBase<D, S, R, C>::inverse() const {
    static_assert(R == C, "inverse: square only");
    const DenseBase& m = *this;
    Matrix<S, R, C> r;
    if (R == 1) { r(0, 0) = S(1) / m(0, 0); return r; }
    if (R == 2) {
        S det = m(0, 0) * m(1, 1) - m(0, 1) * m(1, 0);
        S inv = S(1) / det;
        r(0, 0) = m(1, 1) * inv;  r(0, 1) = -m(0, 1) * inv;
        r(1, 0) = -m(1, 0) * inv; r(1, 1) = m(0, 0) * inv;
        return r;
    }
    if (R == 3) {
        S c00 = m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1);
        S c10 = m(0, 2) * m(2, 1) - m(0, 1) * m(2, 2);
        S c20 = m(0, 1) * m(1, 2) - m(0, 2) * m(1, 1);
        S det = m(0, 0) * c00 + m(1, 0) * c10 + m(2, 0) * c20;
        S inv = S(1) / det;
        r(0, 0) = c00 * inv;
        r(0, 1) = c10 * inv;
        r(0, 2) = c20 * inv;
        r(1, 0) = (m(1, 2) * m(2, 0) - m(1, 0) * m(2, 2)) * inv;
        r(1, 1) = (m(0, 0) * m(2, 2) - m(0, 2) * m(2, 0)) * inv;
        r(1, 2) = (m(0, 2) * m(1, 0) - m(0, 0) * m(1, 2)) * inv;
        r(2, 0) = (m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0)) * inv;
        r(2, 1) = (m(0, 1) * m(2, 0) - m(0, 0) * m(2, 1)) * inv;
        r(2, 2) = (m(0, 0) * m(1, 1) - m(0, 1) * m(1, 0)) * inv;
        return r;
    }
    Matrix<S, R, C> a(*this);
    r.setIdentity();
    for (int k = 0; k < R; ++k) {
        int p = k;
        for (int i = k + 1; i < R; ++i) if (std::abs(a(i, k)) > std::abs(a(p, k))) p = i;
        for (int j = 0; j < C; ++j) { std::swap(a(k, j), a(p, j)); std::swap(r(k, j), r(p, j)); }
        S piv = a(k, k);
        for (int j = 0; j < C; ++j) { a(k, j) = a(k, j) / piv; r(k, j) = r(k, j) / piv; }
        for (int i = 0; i < R; ++i) {
            if (i == k) continue;
            S f = a(i, k);
            for (int j = 0; j < C; ++j) { a(i, j) = a(i, j) - f * a(k, j); r(i, j) = r(i, j) - f * r(k, j); }
        }
    }
    return r;
}

// ---------------------------------------------------------------------------
// LDLT: P^T A P = L D L^T with symmetric diagonal pivoting
// ---------------------------------------------------------------------------
template <typename MatrixType> class LDLT;
template <typename S, int N>
class LDLT<Matrix<S, N, N>> {
    Matrix<S, N, N> l_;
    S d_[N];
    int t_[N];
public:
    LDLT() { for (int i = 0; i < N; ++i) { d_[i] = S(0); t_[i] = i; } }
    template <typename D2> explicit LDLT(const DenseBase<D2, S, N, N>& a) { compute(a); }

    template <typename D2> LDLT& compute(const DenseBase<D2, S, N, N>& a_in) {
        Matrix<S, N, N> a(a_in);
        // symmetrise from the lower triangle (the reference only builds symmetric systems)
        for (int j = 0; j < N; ++j)
            for (int i = j + 1; i < N; ++i) a(j, i) = a(i, j);
        for (int k = 0; k < N; ++k) {
            int p = k;
            S best = std::abs(a(k, k));
            for (int i = k + 1; i < N; ++i)
                if (std::abs(a(i, i)) > best) { best = std::abs(a(i, i)); p = i; }
            t_[k] = p;
            if (p != k) {
                for (int j = 0; j < N; ++j) std::swap(a(k, j), a(p, j));
                for (int i = 0; i < N; ++i) std::swap(a(i, k), a(i, p));
            }
            S d = a(k, k);
            d_[k] = d;
            if (d != S(0)) {
                for (int i = k + 1; i < N; ++i) {
                    S lik = a(i, k) / d;
                    for (int j = k + 1; j <= i; ++j) {
                        a(i, j) = a(i, j) - lik * a(j, k);
                    }
                }
                for (int i = k + 1; i < N; ++i) a(i, k) = a(i, k) / d;
                for (int i = k + 1; i < N; ++i)
                    for (int j = i + 1; j < N; ++j) a(i, j) = a(j, i);
            } else {
                for (int i = k + 1; i < N; ++i) a(i, k) = S(0);
            }
        }
        l_ = a;
        return *this;
    }

    template <typename D2> Matrix<S, N, 1> solve(const DenseBase<D2, S, N, 1>& b) const {
        Matrix<S, N, 1> x(b);
        for (int k = 0; k < N; ++k) if (t_[k] != k) std::swap(x.lin(k), x.lin(t_[k]));
        for (int i = 0; i < N; ++i) {            // L y = x
            S s = x.lin(i);
            for (int j = 0; j < i; ++j) s = s - l_(i, j) * x.lin(j);
            x.lin(i) = s;
        }
        const S tiny = std::numeric_limits<S>::min();
        for (int i = 0; i < N; ++i) x.lin(i) = (std::abs(d_[i]) > tiny) ? x.lin(i) / d_[i] : S(0);
        for (int i = N - 1; i >= 0; --i) {       // L^T w = z
            S s = x.lin(i);
            for (int j = i + 1; j < N; ++j) s = s - l_(j, i) * x.lin(j);
            x.lin(i) = s;
        }
        for (int k = N - 1; k >= 0; --k) if (t_[k] != k) std::swap(x.lin(k), x.lin(t_[k]));
        return x;
    }
    Matrix<S, N, 1> vectorD() const { Matrix<S, N, 1> r; for (int i = 0; i < N; ++i) r.lin(i) = d_[i]; return r; }
};

template <typename D, typename S, int R, int C>
class DenseBase<D, S, R, C>::LDLTType : public LDLT<Matrix<S, R, C>> {
public:
    explicit LDLTType(const Matrix<S, R, C>& m) : LDLT<Matrix<S, R, C>>(m) {}
};

template <typename S, int R, int C>
typename Matrix<S, R, C>::Base::LDLTType Matrix<S, R, C>::ldlt() const {
    return typename Base::LDLTType(*this);
}

// ---------------------------------------------------------------------------
// Jacobi rotations used by the SVD and the symmetric eigen-solver
// ---------------------------------------------------------------------------
namespace shim_detail {
template <typename S>
inline void jacobi_rotation(S app, S aqq, S apq, S& c, S& s) {
    // rotation that annihilates apq of the symmetric 2x2 [[app, apq], [apq, aqq]]
    S tau = (aqq - app) / (S(2) * apq);
    S t = (tau >= S(0) ? S(1) : S(-1)) / (std::abs(tau) + std::sqrt(S(1) + tau * tau));
    c = S(1) / std::sqrt(S(1) + t * t);
    s = t * c;
}
}  // namespace shim_detail

// ---------------------------------------------------------------------------
// JacobiSVD (one-sided Hestenes Jacobi), R >= C
// ---------------------------------------------------------------------------
template <typename MatrixType> class JacobiSVD;
template <typename S, int R, int C>
class JacobiSVD<Matrix<S, R, C>> {
    static_assert(R >= C, "JacobiSVD shim: rows >= cols only");
    Matrix<S, R, R> u_;
    Matrix<S, C, C> v_;
    Matrix<S, C, 1> s_;
public:
    template <typename D2> JacobiSVD(const DenseBase<D2, S, R, C>& m, unsigned int = 0) {
        Matrix<S, R, C> a(m);
        Matrix<S, C, C> v = Matrix<S, C, C>::Identity();
        const S eps = std::numeric_limits<S>::epsilon();
        for (int sweep = 0; sweep < 64; ++sweep) {
            bool rotated = false;
            for (int p = 0; p < C - 1; ++p)
                for (int q = p + 1; q < C; ++q) {
                    S alpha = a.col(p).squaredNorm();
                    S beta = a.col(q).squaredNorm();
                    S gamma = a.col(p).dot(a.col(q));
                    if (gamma == S(0) || std::abs(gamma) <= eps * std::sqrt(alpha * beta)) continue;
                    S c, s;
                    shim_detail::jacobi_rotation(alpha, beta, gamma, c, s);
                    for (int i = 0; i < R; ++i) {
                        S ap = a(i, p), aq = a(i, q);
                        a(i, p) = c * ap - s * aq;
                        a(i, q) = s * ap + c * aq;
                    }
                    for (int i = 0; i < C; ++i) {
                        S vp = v(i, p), vq = v(i, q);
                        v(i, p) = c * vp - s * vq;
                        v(i, q) = s * vp + c * vq;
                    }
                    rotated = true;
                }
            if (!rotated) break;
        }
        S sig[C]; int ord[C];
        for (int j = 0; j < C; ++j) { sig[j] = a.col(j).norm(); ord[j] = j; }
        std::stable_sort(ord, ord + C, [&](int x, int y) { return sig[x] > sig[y]; });
        Matrix<S, R, R> u;
        int nu = 0;
        for (int jj = 0; jj < C; ++jj) {
            int j = ord[jj];
            s_.lin(jj) = sig[j];
            v_.col(jj) = v.col(j);
            if (sig[j] > std::numeric_limits<S>::min()) { u.col(jj) = a.col(j) / sig[j]; nu = jj + 1; }
        }
        // complete U to an orthonormal basis (Gram-Schmidt against unit axes)
        for (int jj = nu; jj < R; ++jj) {
            S bestn = S(-1); Matrix<S, R, 1> best;
            for (int e = 0; e < R; ++e) {
                Matrix<S, R, 1> cand = Matrix<S, R, 1>::Unit(e);
                for (int k = 0; k < jj; ++k) cand -= u.col(k) * u.col(k).dot(cand);
                S n = cand.norm();
                if (n > bestn) { bestn = n; best = cand; }
            }
            u.col(jj) = best / bestn;
        }
        u_ = u;
    }
    const Matrix<S, R, R>& matrixU() const { return u_; }
    const Matrix<S, C, C>& matrixV() const { return v_; }
    const Matrix<S, C, 1>& singularValues() const { return s_; }
};

// ---------------------------------------------------------------------------
// SelfAdjointEigenSolver (cyclic Jacobi), eigenvalues increasing
// ---------------------------------------------------------------------------
template <typename MatrixType> class SelfAdjointEigenSolver;
template <typename S, int N>
class SelfAdjointEigenSolver<Matrix<S, N, N>> {
    Matrix<S, N, 1> w_;
    Matrix<S, N, N> v_;
public:
    template <typename D2> explicit SelfAdjointEigenSolver(const DenseBase<D2, S, N, N>& m, int = 0) {
        Matrix<S, N, N> a(m);
        for (int j = 0; j < N; ++j)
            for (int i = j + 1; i < N; ++i) a(j, i) = a(i, j);
        Matrix<S, N, N> v = Matrix<S, N, N>::Identity();
        const S eps = std::numeric_limits<S>::epsilon();
        for (int sweep = 0; sweep < 64; ++sweep) {
            bool rotated = false;
            for (int p = 0; p < N - 1; ++p)
                for (int q = p + 1; q < N; ++q) {
                    S apq = a(p, q);
                    if (apq == S(0)) continue;
                    if (std::abs(apq) <= eps * S(0.5) * std::sqrt(std::abs(a(p, p) * a(q, q)))) { a(p, q) = a(q, p) = S(0); continue; }
                    S c, s;
                    shim_detail::jacobi_rotation(a(p, p), a(q, q), apq, c, s);
                    for (int k = 0; k < N; ++k) {       // A <- A J
                        S akp = a(k, p), akq = a(k, q);
                        a(k, p) = c * akp - s * akq;
                        a(k, q) = s * akp + c * akq;
                    }
                    for (int k = 0; k < N; ++k) {       // A <- J^T A
                        S apk = a(p, k), aqk = a(q, k);
                        a(p, k) = c * apk - s * aqk;
                        a(q, k) = s * apk + c * aqk;
                    }
                    a(p, q) = a(q, p) = S(0);
                    for (int k = 0; k < N; ++k) {
                        S vkp = v(k, p), vkq = v(k, q);
                        v(k, p) = c * vkp - s * vkq;
                        v(k, q) = s * vkp + c * vkq;
                    }
                    rotated = true;
                }
            if (!rotated) break;
        }
        int ord[N]; S ev[N];
        for (int i = 0; i < N; ++i) { ord[i] = i; ev[i] = a(i, i); }
        std::stable_sort(ord, ord + N, [&](int x, int y) { return ev[x] < ev[y]; });
        for (int i = 0; i < N; ++i) { w_.lin(i) = ev[ord[i]]; v_.col(i) = v.col(ord[i]); }
    }
    const Matrix<S, N, 1>& eigenvalues() const { return w_; }
    const Matrix<S, N, N>& eigenvectors() const { return v_; }
};

// ---------------------------------------------------------------------------
// Quaternion / AngleAxis
// ---------------------------------------------------------------------------
template <typename S> class AngleAxis;

template <typename S>
class Quaternion {
    Matrix<S, 4, 1> c_;   // x, y, z, w
public:
    typedef S Scalar;
    Quaternion() {}
    Quaternion(S w, S x, S y, S z) { c_.lin(0) = x; c_.lin(1) = y; c_.lin(2) = z; c_.lin(3) = w; }
    Quaternion(const AngleAxis<S>& aa);
    template <typename D2> explicit Quaternion(const DenseBase<D2, S, 3, 3>& m);

    static Quaternion Identity() { return Quaternion(S(1), S(0), S(0), S(0)); }

    S& w() { return c_.lin(3); }
    S& x() { return c_.lin(0); }
    S& y() { return c_.lin(1); }
    S& z() { return c_.lin(2); }
    S w() const { return c_.lin(3); }
    S x() const { return c_.lin(0); }
    S y() const { return c_.lin(1); }
    S z() const { return c_.lin(2); }

    Block<S, 3, 1> vec() const { return Block<S, 3, 1>(c_.ptr_(), 4); }
    Block<S, 4, 1> coeffs() const { return Block<S, 4, 1>(c_.ptr_(), 4); }

    Quaternion conjugate() const { return Quaternion(w(), -x(), -y(), -z()); }
    Quaternion inverse() const {
        S n2 = squaredNorm();
        Quaternion c = conjugate();
        c.c_ = c.c_ / n2;
        return c;
    }
    S squaredNorm() const { return c_.squaredNorm(); }
    S norm() const { return c_.norm(); }
    void normalize() { c_.normalize(); }
    Quaternion normalized() const { Quaternion r(*this); r.normalize(); return r; }
    S dot(const Quaternion& o) const { return c_.dot(o.c_); }

    Matrix<S, 3, 3> toRotationMatrix() const {
        Matrix<S, 3, 3> r;
        const S tx = S(2) * x(), ty = S(2) * y(), tz = S(2) * z();
        const S twx = tx * w(), twy = ty * w(), twz = tz * w();
        const S txx = tx * x(), txy = ty * x(), txz = tz * x();
        const S tyy = ty * y(), tyz = tz * y(), tzz = tz * z();
        r(0, 0) = S(1) - (tyy + tzz); r(0, 1) = txy - twz;          r(0, 2) = txz + twy;
        r(1, 0) = txy + twz;          r(1, 1) = S(1) - (txx + tzz); r(1, 2) = tyz - twx;
        r(2, 0) = txz - twy;          r(2, 1) = tyz + twx;          r(2, 2) = S(1) - (txx + tyy);
        return r;
    }
    Matrix<S, 3, 3> matrix() const { return toRotationMatrix(); }

    Quaternion operator*(const Quaternion& b) const {
        const Quaternion& a = *this;
        return Quaternion(a.w() * b.w() - a.x() * b.x() - a.y() * b.y() - a.z() * b.z(),
                          a.w() * b.x() + a.x() * b.w() + a.y() * b.z() - a.z() * b.y(),
                          a.w() * b.y() + a.y() * b.w() + a.z() * b.x() - a.x() * b.z(),
                          a.w() * b.z() + a.z() * b.w() + a.x() * b.y() - a.y() * b.x());
    }
    Quaternion& operator*=(const Quaternion& b) { *this = *this * b; return *this; }

    template <typename D2> Matrix<S, 3, 1> operator*(const DenseBase<D2, S, 3, 1>& v_in) const {
        Matrix<S, 3, 1> v(v_in);
        Matrix<S, 3, 1> uv = vec().cross(v);
        uv = uv + uv;
        return v + w() * uv + vec().cross(uv);
    }
};

template <typename S>
class AngleAxis {
public:
    S a; Matrix<S, 3, 1> ax;
    template <typename D2> AngleAxis(S angle, const DenseBase<D2, S, 3, 1>& axis) : a(angle), ax(axis) {}
    Quaternion<S> operator*(const AngleAxis& o) const { return Quaternion<S>(*this) * Quaternion<S>(o); }
    S angle() const { return a; }
    const Matrix<S, 3, 1>& axis() const { return ax; }
};

template <typename S>
Quaternion<S>::Quaternion(const AngleAxis<S>& aa) {
    S ha = S(0.5) * aa.a;
    S sn = std::sin(ha);
    c_.lin(3) = std::cos(ha);
    c_.lin(0) = sn * aa.ax.lin(0);
    c_.lin(1) = sn * aa.ax.lin(1);
    c_.lin(2) = sn * aa.ax.lin(2);
}

template <typename S>
inline Quaternion<S> operator*(const Quaternion<S>& q, const AngleAxis<S>& aa) { return q * Quaternion<S>(aa); }
template <typename S>
inline Quaternion<S> operator*(const AngleAxis<S>& aa, const Quaternion<S>& q) { return Quaternion<S>(aa) * q; }

// ---------------------------------------------------------------------------
// typedefs
// ---------------------------------------------------------------------------
typedef Matrix<float, 2, 1> Vector2f;
typedef Matrix<float, 3, 1> Vector3f;
typedef Matrix<float, 4, 1> Vector4f;
typedef Matrix<float, 2, 2> Matrix2f;
typedef Matrix<float, 3, 3> Matrix3f;
typedef Matrix<float, 4, 4> Matrix4f;
typedef Matrix<double, 2, 1> Vector2d;
typedef Matrix<double, 3, 1> Vector3d;
typedef Matrix<double, 4, 1> Vector4d;
typedef Matrix<double, 2, 2> Matrix2d;
typedef Matrix<double, 3, 3> Matrix3d;
typedef Matrix<double, 4, 4> Matrix4d;
typedef Quaternion<float> Quaternionf;
typedef Quaternion<double> Quaterniond;
typedef AngleAxis<float> AngleAxisf;
typedef AngleAxis<double> AngleAxisd;

}  // namespace Eigen
