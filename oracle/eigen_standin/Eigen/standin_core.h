// Dense stand-in for the four Eigen facilities that HI-SLAM2's
// src/droid_kernels.cu uses (TEST INFRASTRUCTURE ONLY: it lets the reference's
// own BA / PGBA / frame_distance sources compile unmodified into oracle/_ref so
// that their outputs pin the numpy oracle).  Written from the documented
// behaviour of the Eigen API, not from Eigen's sources (the eigen submodule of
// the checkout is empty and Eigen is not installed here):
//
//   * Triplet<S>(row, col, value) and SparseMatrix<S>::setFromTriplets: the
//     matrix becomes the sum of all triplets, duplicates added (droid_kernels.cu:1598-1622);
//   * SparseMatrix subtraction and diagonal().array() += expr (:1641-1644, :1664);
//   * VectorX<S> with Zero(n), operator(), subtraction and data() (:1588-1592, :1625-1639);
//   * SimplicialLLT<SparseMatrix<S>>: compute() factors the self-adjoint matrix
//     whose LOWER triangle is given (Eigen's default UpLo = Lower), info() is
//     Success unless a pivot is not positive, solve(b) returns A^-1 b
//     (:1666-1677).  Eigen orders the unknowns with AMD before factoring; this
//     stand-in factors in natural order, which changes rounding only.
//
// Storage is dense (n <= 6 * 300 in every workload here: 26 MB in double).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <vector>

namespace Eigen {

enum ComputationInfo { Success = 0, NumericalIssue = 1, NoConvergence = 2, InvalidInput = 3 };

template <typename S>
class Triplet {
 public:
  Triplet(long r, long c, S v) : r_(r), c_(c), v_(v) {}
  long row() const { return r_; }
  long col() const { return c_; }
  S value() const { return v_; }

 private:
  long r_, c_;
  S v_;
};

// Column vector with the few operations the reference uses.
template <typename S>
class VectorX {
 public:
  VectorX() = default;
  explicit VectorX(long n) : d_(n, S(0)) {}
  static VectorX Zero(long n) { return VectorX(n); }
  long size() const { return (long)d_.size(); }
  S& operator()(long i) { return d_[i]; }
  S operator()(long i) const { return d_[i]; }
  S* data() { return d_.data(); }
  const S* data() const { return d_.data(); }
  VectorX operator-(const VectorX& o) const {
    VectorX r(*this);
    for (size_t i = 0; i < d_.size(); ++i) r.d_[i] -= o.d_[i];
    return r;
  }

 private:
  std::vector<S> d_;
};

using VectorXd = VectorX<double>;

template <typename S>
class SparseMatrix;

// Column-major dense matrix; built from a SparseMatrix (SparseBlock::get_dense).
template <typename S>
class DenseMatrix {
 public:
  explicit DenseMatrix(const SparseMatrix<S>& a) : n_(a.rows()), m_(a.cols()), d_((size_t)n_ * m_) {
    for (long c = 0; c < m_; ++c)
      for (long r = 0; r < n_; ++r) d_[(size_t)c * n_ + r] = a.at(r, c);
  }
  S* data() { return d_.data(); }

 private:
  long n_, m_;
  std::vector<S> d_;
};

using MatrixXd = DenseMatrix<double>;

// diagonal().array() of a SparseMatrix: a reference to the diagonal entries that
// accepts "+=" of an element-wise expression (scalar + scalar * diagonal).
template <typename S>
struct DiagValues {
  std::vector<S> v;
};

template <typename S>
class DiagArray {
 public:
  explicit DiagArray(SparseMatrix<S>* m) : m_(m) {}
  S value(long i) const { return m_->at(i, i); }
  long size() const { return std::min(m_->rows(), m_->cols()); }
  DiagArray& operator+=(const DiagValues<S>& e) {
    for (long i = 0; i < size(); ++i) m_->at(i, i) += e.v[i];
    return *this;
  }

 private:
  SparseMatrix<S>* m_;
};

template <typename S, typename F>
DiagValues<S> operator*(F a, const DiagArray<S>& d) {
  DiagValues<S> r;
  r.v.resize(d.size());
  for (long i = 0; i < d.size(); ++i) r.v[i] = S(a) * d.value(i);
  return r;
}

template <typename S, typename F>
DiagValues<S> operator+(F a, DiagValues<S> e) {
  for (auto& x : e.v) x = S(a) + x;
  return e;
}

template <typename S>
class DiagRef {
 public:
  explicit DiagRef(SparseMatrix<S>* m) : m_(m) {}
  DiagArray<S> array() { return DiagArray<S>(m_); }

 private:
  SparseMatrix<S>* m_;
};

template <typename S>
class SparseMatrix {
 public:
  SparseMatrix() = default;
  SparseMatrix(long rows, long cols) : n_(rows), m_(cols), d_((size_t)rows * cols, S(0)) {}
  long rows() const { return n_; }
  long cols() const { return m_; }
  S& at(long r, long c) { return d_[(size_t)r * m_ + c]; }
  S at(long r, long c) const { return d_[(size_t)r * m_ + c]; }

  template <typename It>
  void setFromTriplets(It begin, It end) {
    std::fill(d_.begin(), d_.end(), S(0));
    for (It t = begin; t != end; ++t) at(t->row(), t->col()) += t->value();
  }

  SparseMatrix operator-(const SparseMatrix& o) const {
    SparseMatrix r(*this);
    for (size_t i = 0; i < d_.size(); ++i) r.d_[i] -= o.d_[i];
    return r;
  }

  DiagRef<S> diagonal() { return DiagRef<S>(this); }

 private:
  long n_ = 0, m_ = 0;
  std::vector<S> d_;
};

// LL^T of the symmetric matrix given by its lower triangle, natural order.
template <typename Mat>
class SimplicialLLT;

template <typename S>
class SimplicialLLT<SparseMatrix<S>> {
 public:
  void compute(const SparseMatrix<S>& a) {
    n_ = a.rows();
    l_.assign((size_t)n_ * n_, S(0));
    info_ = Success;
    for (long j = 0; j < n_; ++j) {
      S d = a.at(j, j);
      for (long k = 0; k < j; ++k) d -= L(j, k) * L(j, k);
      if (!(d > S(0))) {
        info_ = NumericalIssue;
        return;
      }
      const S ljj = std::sqrt(d);
      L(j, j) = ljj;
      for (long i = j + 1; i < n_; ++i) {
        S s = a.at(i, j);
        for (long k = 0; k < j; ++k) s -= L(i, k) * L(j, k);
        L(i, j) = s / ljj;
      }
    }
  }
  ComputationInfo info() const { return info_; }
  VectorX<S> solve(const VectorX<S>& b) const {
    VectorX<S> x(b);
    for (long i = 0; i < n_; ++i) {
      S s = x(i);
      for (long k = 0; k < i; ++k) s -= L(i, k) * x(k);
      x(i) = s / L(i, i);
    }
    for (long i = n_ - 1; i >= 0; --i) {
      S s = x(i);
      for (long k = i + 1; k < n_; ++k) s -= L(k, i) * x(k);
      x(i) = s / L(i, i);
    }
    return x;
  }

 private:
  S& L(long r, long c) { return l_[(size_t)r * n_ + c]; }
  S L(long r, long c) const { return l_[(size_t)r * n_ + c]; }
  long n_ = 0;
  std::vector<S> l_;
  ComputationInfo info_ = InvalidInput;
};

}  // namespace Eigen
