// Test infrastructure (oracle only): a small subset of the Eigen 3.4 public API,
// written from Eigen's public documentation so that the reference solver's own
// numerical classes compile in this container, where Eigen is not installed.
// Nothing in the product links this file.
//
// Surface used by the reference (call sites: source/object/Circle.cpp:21,36-39,
// 46,114-115,123-124,193; source/object/ImagePoint.cpp:22-51; every Coord use):
//   Vector2d  - (x,y) and {{x,y}} construction, ()/[]/x()/y(), + - unary-,
//               scalar * and /, compound ops, dot, norm, squaredNorm,
//               normalized, setZero.
//   Vector4d, Matrix4d - coefficient access.
//   Matrix4d::ldlt()   - robust LDL^T with symmetric diagonal pivoting.
//
// Documented semantics reproduced here:
//   * default construction leaves coefficients uninitialised, so a value-
//     initialised owner (make_unique<EulerPhase>()) sees zeros, as with Eigen;
//   * norm() = sqrt(squaredNorm()), squaredNorm() = x*x + y*y;
//   * normalized() returns v / norm() when norm() > 0, else a copy of v;
//   * ldlt() reads the LOWER triangle only and factors A = P^T L D L^T P with
//     the pivot at each step chosen as the largest remaining diagonal entry in
//     absolute value; solve() applies P, L^{-1}, the pseudo-inverse of D
//     (entries treated as zero when |d| is not above the smallest normal
//     double), L^{-T}, P^T.  The elimination order follows the outer-product
//     (right-looking) form of Golub & Van Loan, Matrix Computations, 4.1/4.4,
//     and Higham, Accuracy and Stability of Numerical Algorithms, ch. 10-11.
//     Whether real Eigen rounds identically is not known here: values that go
//     through ldlt() are pinned to this shim, not to Eigen.
#pragma once
// Real Eigen headers pull in these standard headers, and the reference's own
// headers rely on that (e.g. FourthOrderCS.h:16 names std::vector without
// including <vector>).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <functional>
#include <initializer_list>
#include <iostream>
#include <limits>
#include <list>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace Eigen {

enum ComputationInfo { Success = 0, NumericalIssue = 1, NoConvergence = 2, InvalidInput = 3 };

class Vector2d {
public:
    Vector2d() {}
    Vector2d(double x, double y) { m_v[0] = x; m_v[1] = y; }
    template <class A, class B>
    Vector2d(A x, B y) { m_v[0] = static_cast<double>(x); m_v[1] = static_cast<double>(y); }
    Vector2d(std::initializer_list<std::initializer_list<double>> rows) {
        // Eigen 3.4 accepts a single row of N values for a fixed-size vector.
        const double* p = rows.begin()->begin();
        m_v[0] = p[0];
        m_v[1] = p[1];
    }

    double& operator()(std::ptrdiff_t i) { return m_v[i]; }
    const double& operator()(std::ptrdiff_t i) const { return m_v[i]; }
    double& operator[](std::ptrdiff_t i) { return m_v[i]; }
    const double& operator[](std::ptrdiff_t i) const { return m_v[i]; }
    double& x() { return m_v[0]; }
    double& y() { return m_v[1]; }
    const double& x() const { return m_v[0]; }
    const double& y() const { return m_v[1]; }

    Vector2d operator+(const Vector2d& o) const { return Vector2d(m_v[0] + o.m_v[0], m_v[1] + o.m_v[1]); }
    Vector2d operator-(const Vector2d& o) const { return Vector2d(m_v[0] - o.m_v[0], m_v[1] - o.m_v[1]); }
    Vector2d operator-() const { return Vector2d(-m_v[0], -m_v[1]); }
    Vector2d& operator+=(const Vector2d& o) { m_v[0] += o.m_v[0]; m_v[1] += o.m_v[1]; return *this; }
    Vector2d& operator-=(const Vector2d& o) { m_v[0] -= o.m_v[0]; m_v[1] -= o.m_v[1]; return *this; }
    template <class S> Vector2d operator*(S s) const { const double d = static_cast<double>(s); return Vector2d(m_v[0] * d, m_v[1] * d); }
    template <class S> Vector2d operator/(S s) const { const double d = static_cast<double>(s); return Vector2d(m_v[0] / d, m_v[1] / d); }
    template <class S> Vector2d& operator*=(S s) { const double d = static_cast<double>(s); m_v[0] *= d; m_v[1] *= d; return *this; }
    template <class S> Vector2d& operator/=(S s) { const double d = static_cast<double>(s); m_v[0] /= d; m_v[1] /= d; return *this; }

    double dot(const Vector2d& o) const { return m_v[0] * o.m_v[0] + m_v[1] * o.m_v[1]; }
    double squaredNorm() const { return m_v[0] * m_v[0] + m_v[1] * m_v[1]; }
    double norm() const { return std::sqrt(squaredNorm()); }
    Vector2d normalized() const {
        const double z = squaredNorm();
        if (z > 0.0) {
            const double n = std::sqrt(z);
            return Vector2d(m_v[0] / n, m_v[1] / n);
        }
        return *this;
    }
    void setZero() { m_v[0] = 0.0; m_v[1] = 0.0; }

private:
    double m_v[2];
};

template <class S>
inline Vector2d operator*(S s, const Vector2d& v) {
    const double d = static_cast<double>(s);
    return Vector2d(d * v[0], d * v[1]);
}

class Vector4d {
public:
    Vector4d() {}
    double& operator()(std::ptrdiff_t i) { return m_v[i]; }
    const double& operator()(std::ptrdiff_t i) const { return m_v[i]; }
    double& operator[](std::ptrdiff_t i) { return m_v[i]; }
    const double& operator[](std::ptrdiff_t i) const { return m_v[i]; }

private:
    double m_v[4];
};

class LDLT4;

class Matrix4d {
public:
    Matrix4d() {}
    double& operator()(std::ptrdiff_t r, std::ptrdiff_t c) { return m_a[r][c]; }
    const double& operator()(std::ptrdiff_t r, std::ptrdiff_t c) const { return m_a[r][c]; }
    inline LDLT4 ldlt() const;

private:
    double m_a[4][4];
};

// Pivoted LDL^T of the symmetric matrix whose lower triangle is the input's.
class LDLT4 {
public:
    explicit LDLT4(const Matrix4d& a) {
        // Symmetric working copy built from the lower triangle only.
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c)
                m_w[r][c] = (r >= c) ? a(r, c) : a(c, r);
        for (int k = 0; k < 4; ++k) m_perm[k] = k;
        m_info = Success;
        for (int k = 0; k < 4; ++k) {
            // Pivot: largest |diagonal| of the remaining Schur complement
            // (first index wins on ties).
            int p = k;
            double best = std::fabs(m_w[k][k]);
            for (int i = k + 1; i < 4; ++i) {
                const double v = std::fabs(m_w[i][i]);
                if (v > best) { best = v; p = i; }
            }
            if (p != k) {
                for (int c = 0; c < 4; ++c) { double t = m_w[k][c]; m_w[k][c] = m_w[p][c]; m_w[p][c] = t; }
                for (int r = 0; r < 4; ++r) { double t = m_w[r][k]; m_w[r][k] = m_w[r][p]; m_w[r][p] = t; }
                for (int c = 0; c < k; ++c) { double t = m_l[k][c]; m_l[k][c] = m_l[p][c]; m_l[p][c] = t; }
                int t = m_perm[k]; m_perm[k] = m_perm[p]; m_perm[p] = t;
            }
            const double d = m_w[k][k];
            m_d[k] = d;
            const bool usable = std::fabs(d) > (std::numeric_limits<double>::min)();
            for (int i = k + 1; i < 4; ++i) m_l[i][k] = usable ? m_w[i][k] / d : 0.0;
            // Outer-product update of the trailing block.
            for (int i = k + 1; i < 4; ++i)
                for (int j = k + 1; j < 4; ++j)
                    m_w[i][j] = m_w[i][j] - m_l[i][k] * d * m_l[j][k];
        }
    }
    ComputationInfo info() const { return m_info; }

    Vector4d solve(const Vector4d& b) const {
        double y[4];
        for (int k = 0; k < 4; ++k) y[k] = b(m_perm[k]);
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < i; ++k) y[i] -= m_l[i][k] * y[k];
        for (int i = 0; i < 4; ++i)
            y[i] = (std::fabs(m_d[i]) > (std::numeric_limits<double>::min)()) ? y[i] / m_d[i] : 0.0;
        for (int i = 3; i >= 0; --i)
            for (int k = i + 1; k < 4; ++k) y[i] -= m_l[k][i] * y[k];
        Vector4d x;
        for (int k = 0; k < 4; ++k) x(m_perm[k]) = y[k];
        return x;
    }

private:
    double m_w[4][4];
    double m_l[4][4] = {};
    double m_d[4];
    int m_perm[4];
    ComputationInfo m_info;
};

inline LDLT4 Matrix4d::ldlt() const { return LDLT4(*this); }

}  // namespace Eigen
