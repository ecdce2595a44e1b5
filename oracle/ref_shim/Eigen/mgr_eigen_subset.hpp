// mgr_eigen_subset.hpp -- the part of Eigen's API that Magritte's radiation
// path uses, written for this project so the reference's C++ compiles
// without Eigen (TEST INFRASTRUCTURE ONLY: it builds the reference into
// oracle/_ref as a second checker of the C oracle).
//
// Eigen is not vendored by the reference (dependencies/get_dependencies.sh
// pulls an unpinned master of eigen-git-mirror) and is absent here, so the
// arithmetic order below defines what the compiled reference computes:
//   * Vector3d::dot = (x x' + y y') + z z', separately rounded (the order the
//     C oracle and the device tracer restate);
//   * VectorXd::dot = a sequential sum over the elements;
//   * element-wise expressions are evaluated eagerly, one operation at a
//     time, in the order the source writes them (what Eigen's coefficient-
//     wise expression templates also do per element);
//   * SparseLU<.., COLAMDOrdering> is a block solver: analyzePattern splits
//     the matrix into the connected components of its sparsity graph (with
//     n_off_diag = 0 the rate matrix is block diagonal, one nlev x nlev block
//     per cell) and factorize does a dense LU with partial pivoting per block.
//     Pivots and rounding therefore differ from Eigen's supernodal SparseLU.
#pragma once

#include <cassert>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <functional>
#include <iostream>
#include <map>
#include <algorithm>
#include <numeric>
#include <type_traits>
#include <string>
#include <utility>
#include <vector>

namespace Eigen {

enum ComputationInfo { Success = 0, NumericalIssue = 1, NoConvergence = 2, InvalidInput = 3 };

// ---------------------------------------------------------------- Vector3d
class Vector3d {
  public:
    Vector3d() : v_{0.0, 0.0, 0.0} {}
    Vector3d(double x, double y, double z) : v_{x, y, z} {}
    double &operator[](std::size_t i) { return v_[i]; }
    double operator[](std::size_t i) const { return v_[i]; }
    double &operator()(std::size_t i) { return v_[i]; }
    double operator()(std::size_t i) const { return v_[i]; }
    double x() const { return v_[0]; }
    double y() const { return v_[1]; }
    double z() const { return v_[2]; }
    double &x() { return v_[0]; }
    double &y() { return v_[1]; }
    double &z() { return v_[2]; }
    double dot(const Vector3d &o) const {
        const double xx = v_[0] * o.v_[0];
        const double yy = v_[1] * o.v_[1];
        const double zz = v_[2] * o.v_[2];
        const double s = xx + yy;
        return s + zz;
    }
    Vector3d cross(const Vector3d &o) const {
        return Vector3d(v_[1] * o.v_[2] - v_[2] * o.v_[1], v_[2] * o.v_[0] - v_[0] * o.v_[2],
                        v_[0] * o.v_[1] - v_[1] * o.v_[0]);
    }
    double squaredNorm() const { return dot(*this); }
    double norm() const { return std::sqrt(squaredNorm()); }
    Vector3d operator+(const Vector3d &o) const {
        return Vector3d(v_[0] + o.v_[0], v_[1] + o.v_[1], v_[2] + o.v_[2]);
    }
    Vector3d operator-(const Vector3d &o) const {
        return Vector3d(v_[0] - o.v_[0], v_[1] - o.v_[1], v_[2] - o.v_[2]);
    }
    Vector3d operator-() const { return Vector3d(-v_[0], -v_[1], -v_[2]); }
    Vector3d operator*(double s) const { return Vector3d(v_[0] * s, v_[1] * s, v_[2] * s); }
    Vector3d operator/(double s) const { return Vector3d(v_[0] / s, v_[1] / s, v_[2] / s); }
    Vector3d &operator+=(const Vector3d &o) {
        for (int i = 0; i < 3; i++) v_[i] += o.v_[i];
        return *this;
    }
    Vector3d &operator-=(const Vector3d &o) {
        for (int i = 0; i < 3; i++) v_[i] -= o.v_[i];
        return *this;
    }
    static Vector3d Zero() { return Vector3d(); }

  private:
    double v_[3];
};
inline Vector3d operator*(double s, const Vector3d &a) { return Vector3d(s * a[0], s * a[1], s * a[2]); }
inline std::ostream &operator<<(std::ostream &os, const Vector3d &a) {
    return os << a[0] << "\n" << a[1] << "\n" << a[2];
}

// ---------------------------------------------------------------- VectorXd
class VectorXd {
  public:
    VectorXd() = default;
    explicit VectorXd(std::size_t n) : d_(n, 0.0) {}
    template <class I>
    explicit VectorXd(I n, typename std::enable_if<std::is_integral<I>::value>::type * = nullptr)
        : d_((std::size_t)n, 0.0) {}
    void resize(std::size_t n) { d_.resize(n); }
    std::size_t size() const { return d_.size(); }
    double &operator[](std::size_t i) { return d_[i]; }
    double operator[](std::size_t i) const { return d_[i]; }
    double &operator()(std::size_t i) { return d_[i]; }
    double operator()(std::size_t i) const { return d_[i]; }
    double *data() { return d_.data(); }
    const double *data() const { return d_.data(); }
    double dot(const VectorXd &o) const {
        double s = 0.0;
        for (std::size_t i = 0; i < d_.size(); i++) s += d_[i] * o.d_[i];
        return s;
    }
    double sum() const {
        double s = 0.0;
        for (double x : d_) s += x;
        return s;
    }
    double squaredNorm() const { return dot(*this); }
    double norm() const { return std::sqrt(squaredNorm()); }
    void setZero() { std::fill(d_.begin(), d_.end(), 0.0); }
    static VectorXd Zero(std::size_t n) { return VectorXd(n); }
    static VectorXd Constant(std::size_t n, double c) {
        VectorXd r(n);
        std::fill(r.d_.begin(), r.d_.end(), c);
        return r;
    }
    VectorXd &operator+=(const VectorXd &o) {
        for (std::size_t i = 0; i < d_.size(); i++) d_[i] += o.d_[i];
        return *this;
    }
    VectorXd &operator-=(const VectorXd &o) {
        for (std::size_t i = 0; i < d_.size(); i++) d_[i] -= o.d_[i];
        return *this;
    }
    VectorXd &operator*=(double s) {
        for (double &x : d_) x *= s;
        return *this;
    }

  private:
    std::vector<double> d_;
};
inline VectorXd operator+(const VectorXd &a, const VectorXd &b) {
    VectorXd r(a.size());
    for (std::size_t i = 0; i < a.size(); i++) r[i] = a[i] + b[i];
    return r;
}
inline VectorXd operator-(const VectorXd &a, const VectorXd &b) {
    VectorXd r(a.size());
    for (std::size_t i = 0; i < a.size(); i++) r[i] = a[i] - b[i];
    return r;
}
inline VectorXd operator*(double s, const VectorXd &a) {
    VectorXd r(a.size());
    for (std::size_t i = 0; i < a.size(); i++) r[i] = s * a[i];
    return r;
}
inline VectorXd operator*(const VectorXd &a, double s) {
    VectorXd r(a.size());
    for (std::size_t i = 0; i < a.size(); i++) r[i] = a[i] * s;
    return r;
}
inline std::ostream &operator<<(std::ostream &os, const VectorXd &a) {
    for (std::size_t i = 0; i < a.size(); i++) os << a[i] << "\n";
    return os;
}

// ---------------------------------------------------------------- MatrixXd
class MatrixXd {
  public:
    MatrixXd() = default;
    MatrixXd(std::size_t r, std::size_t c) : r_(r), c_(c), d_(r * c, 0.0) {}
    void resize(std::size_t r, std::size_t c) { r_ = r; c_ = c; d_.assign(r * c, 0.0); }
    std::size_t rows() const { return r_; }
    std::size_t cols() const { return c_; }
    double &operator()(std::size_t i, std::size_t j) { return d_[i * c_ + j]; }
    double operator()(std::size_t i, std::size_t j) const { return d_[i * c_ + j]; }
    static MatrixXd Zero(std::size_t r, std::size_t c) { return MatrixXd(r, c); }
    // Gauss-Jordan elimination with partial pivoting (square matrices).
    MatrixXd inverse() const {
        const std::size_t n = r_;
        MatrixXd a(*this), inv(n, n);
        for (std::size_t i = 0; i < n; i++) inv(i, i) = 1.0;
        for (std::size_t c = 0; c < n; c++) {
            std::size_t p = c;
            for (std::size_t r = c + 1; r < n; r++)
                if (std::fabs(a(r, c)) > std::fabs(a(p, c))) p = r;
            for (std::size_t j = 0; j < n; j++) {
                std::swap(a(c, j), a(p, j));
                std::swap(inv(c, j), inv(p, j));
            }
            const double d = a(c, c);
            for (std::size_t j = 0; j < n; j++) { a(c, j) /= d; inv(c, j) /= d; }
            for (std::size_t r = 0; r < n; r++) {
                if (r == c) continue;
                const double f = a(r, c);
                for (std::size_t j = 0; j < n; j++) {
                    a(r, j) -= f * a(c, j);
                    inv(r, j) -= f * inv(c, j);
                }
            }
        }
        return inv;
    }

  private:
    std::size_t r_ = 0, c_ = 0;
    std::vector<double> d_;
};

inline std::ostream &operator<<(std::ostream &os, const MatrixXd &m) {
    for (std::size_t i = 0; i < m.rows(); i++) {
        for (std::size_t j = 0; j < m.cols(); j++) os << (j ? " " : "") << m(i, j);
        os << "\n";
    }
    return os;
}

// ----------------------------------------------------------- sparse matrix
template <class Scalar, class Index = int>
class Triplet {
  public:
    Triplet(Index r = 0, Index c = 0, Scalar v = Scalar(0)) : r_(r), c_(c), v_(v) {}
    Index row() const { return r_; }
    Index col() const { return c_; }
    Scalar value() const { return v_; }

  private:
    Index r_, c_;
    Scalar v_;
};

template <class Scalar, int Options = 0, class Index = int>
class SparseMatrix {
  public:
    SparseMatrix() = default;
    SparseMatrix(long r, long c) { resize(r, c); }
    void resize(long r, long c) {
        rows_ = r;
        cols_ = c;
        row_.assign((std::size_t)r, {});
    }
    long rows() const { return rows_; }
    long cols() const { return cols_; }
    // Sums duplicate entries, in the order the triplets are given.
    template <class It>
    void setFromTriplets(It begin, It end) {
        row_.assign((std::size_t)rows_, {});
        for (It t = begin; t != end; ++t) row_[(std::size_t)t->row()][(long)t->col()] += t->value();
    }
    void makeCompressed() {}
    long nonZeros() const {
        long n = 0;
        for (const auto &r : row_) n += (long)r.size();
        return n;
    }
    double coeff(long i, long j) const {
        auto it = row_[(std::size_t)i].find(j);
        return it == row_[(std::size_t)i].end() ? 0.0 : it->second;
    }
    const std::map<long, Scalar> &row_entries(long i) const { return row_[(std::size_t)i]; }

  private:
    long rows_ = 0, cols_ = 0;
    std::vector<std::map<long, Scalar>> row_;
};
template <class S, int O, class I>
std::ostream &operator<<(std::ostream &os, const SparseMatrix<S, O, I> &m) {
    for (long i = 0; i < m.rows(); i++)
        for (const auto &e : m.row_entries(i)) os << "(" << i << "," << e.first << ") " << e.second << "\n";
    return os;
}

template <class Scalar>
class SparseVector {
  public:
    SparseVector() = default;
    explicit SparseVector(long n) : n_(n) {}

  private:
    long n_ = 0;
};

template <class Index>
struct COLAMDOrdering {};

// Block LU: see the file header.
template <class Matrix, class Ordering = COLAMDOrdering<int>>
class SparseLU {
  public:
    void analyzePattern(const Matrix &A) {
        const long n = A.rows();
        parent_.resize((std::size_t)n);
        std::iota(parent_.begin(), parent_.end(), 0L);
        for (long i = 0; i < n; i++)
            for (const auto &e : A.row_entries(i)) unite(i, e.first);
        std::map<long, long> comp;
        blocks_.clear();
        for (long i = 0; i < n; i++) {
            const long r = find(i);
            auto it = comp.find(r);
            if (it == comp.end()) {
                it = comp.emplace(r, (long)blocks_.size()).first;
                blocks_.emplace_back();
            }
            blocks_[(std::size_t)it->second].idx.push_back(i);
        }
        info_ = Success;
    }
    void factorize(const Matrix &A) {
        info_ = Success;
        msg_.clear();
        for (Block &b : blocks_) {
            const long m = (long)b.idx.size();
            std::map<long, long> local;
            for (long k = 0; k < m; k++) local[b.idx[(std::size_t)k]] = k;
            b.lu.assign((std::size_t)(m * m), 0.0);
            for (long k = 0; k < m; k++)
                for (const auto &e : A.row_entries(b.idx[(std::size_t)k]))
                    b.lu[(std::size_t)(k * m + local[e.first])] = e.second;
            b.piv.resize((std::size_t)m);
            for (long c = 0; c < m; c++) {
                long p = c;
                double best = std::fabs(b.lu[(std::size_t)(c * m + c)]);
                for (long r = c + 1; r < m; r++) {
                    const double v = std::fabs(b.lu[(std::size_t)(r * m + c)]);
                    if (v > best) { best = v; p = r; }
                }
                b.piv[(std::size_t)c] = p;
                if (best == 0.0) {
                    info_ = NumericalIssue;
                    msg_ = "zero pivot";
                    return;
                }
                if (p != c)
                    for (long j = 0; j < m; j++)
                        std::swap(b.lu[(std::size_t)(c * m + j)], b.lu[(std::size_t)(p * m + j)]);
                const double d = b.lu[(std::size_t)(c * m + c)];
                for (long r = c + 1; r < m; r++) {
                    const double f = b.lu[(std::size_t)(r * m + c)] / d;
                    b.lu[(std::size_t)(r * m + c)] = f;
                    for (long j = c + 1; j < m; j++)
                        b.lu[(std::size_t)(r * m + j)] -= f * b.lu[(std::size_t)(c * m + j)];
                }
            }
        }
    }
    VectorXd solve(const VectorXd &y) {
        VectorXd x(y.size());
        for (const Block &b : blocks_) {
            const long m = (long)b.idx.size();
            std::vector<double> z((std::size_t)m);
            for (long k = 0; k < m; k++) z[(std::size_t)k] = y[(std::size_t)b.idx[(std::size_t)k]];
            for (long c = 0; c < m; c++) {
                const long p = b.piv[(std::size_t)c];
                if (p != c) std::swap(z[(std::size_t)c], z[(std::size_t)p]);
                for (long r = c + 1; r < m; r++)
                    z[(std::size_t)r] -= b.lu[(std::size_t)(r * m + c)] * z[(std::size_t)c];
            }
            for (long c = m - 1; c >= 0; c--) {
                double s = z[(std::size_t)c];
                for (long j = c + 1; j < m; j++) s -= b.lu[(std::size_t)(c * m + j)] * z[(std::size_t)j];
                z[(std::size_t)c] = s / b.lu[(std::size_t)(c * m + c)];
            }
            for (long k = 0; k < m; k++) x[(std::size_t)b.idx[(std::size_t)k]] = z[(std::size_t)k];
        }
        return x;
    }
    ComputationInfo info() const { return info_; }
    std::string lastErrorMessage() const { return msg_; }

  private:
    struct Block {
        std::vector<long> idx;
        std::vector<double> lu;
        std::vector<long> piv;
    };
    long find(long i) {
        while (parent_[(std::size_t)i] != i) {
            parent_[(std::size_t)i] = parent_[(std::size_t)parent_[(std::size_t)i]];
            i = parent_[(std::size_t)i];
        }
        return i;
    }
    void unite(long a, long b) {
        a = find(a);
        b = find(b);
        if (a != b) parent_[(std::size_t)std::max(a, b)] = std::min(a, b);
    }
    std::vector<long> parent_;
    std::vector<Block> blocks_;
    ComputationInfo info_ = Success;
    std::string msg_;
};

}  // namespace Eigen
