// Minimal stand-ins for the few Eigen names the OccupancyGrid API uses, for
// builds without Eigen (this image has none).  Only what the reference's
// public signatures and its perf test touch: Vector3f / Vector3i with x() y()
// z(), element access, +, -, Zero(), Constant(), squaredNorm(), cwiseAbs(),
// and the column-major Matrix<float, Dynamic, 3> point cloud with rows(),
// resize(), operator()(i, j), col(j).data() and row(i) assignment.  When
// <Eigen/Dense> is available, OccupancyGrid.hpp uses the real Eigen instead.
#pragma once

#include <cstddef>
#include <vector>

namespace Eigen {

using Index = std::ptrdiff_t;
constexpr int Dynamic = -1;

template <typename T, int R, int C>
class Matrix;

template <typename T>
class Matrix<T, 3, 1> {
 public:
  Matrix() : v_{T(0), T(0), T(0)} {}
  Matrix(T x, T y, T z) : v_{x, y, z} {}
  static Matrix Zero() { return Matrix(T(0), T(0), T(0)); }
  static Matrix Ones() { return Matrix(T(1), T(1), T(1)); }
  static Matrix Constant(T c) { return Matrix(c, c, c); }
  T &x() { return v_[0]; }
  T &y() { return v_[1]; }
  T &z() { return v_[2]; }
  T x() const { return v_[0]; }
  T y() const { return v_[1]; }
  T z() const { return v_[2]; }
  T &operator()(Index i) { return v_[i]; }
  T operator()(Index i) const { return v_[i]; }
  T &operator[](Index i) { return v_[i]; }
  T operator[](Index i) const { return v_[i]; }
  T *data() { return v_; }
  const T *data() const { return v_; }
  Matrix operator+(const Matrix &o) const {
    return Matrix(v_[0] + o.v_[0], v_[1] + o.v_[1], v_[2] + o.v_[2]);
  }
  Matrix operator-(const Matrix &o) const {
    return Matrix(v_[0] - o.v_[0], v_[1] - o.v_[1], v_[2] - o.v_[2]);
  }
  bool operator==(const Matrix &o) const {
    return v_[0] == o.v_[0] && v_[1] == o.v_[1] && v_[2] == o.v_[2];
  }
  bool operator!=(const Matrix &o) const { return !(*this == o); }
  T squaredNorm() const {
    const T a = v_[0] * v_[0];
    const T b = v_[1] * v_[1];
    const T c = v_[2] * v_[2];
    return (a + b) + c;
  }
  Matrix cwiseAbs() const {
    return Matrix(v_[0] < 0 ? -v_[0] : v_[0], v_[1] < 0 ? -v_[1] : v_[1],
                  v_[2] < 0 ? -v_[2] : v_[2]);
  }

 private:
  T v_[3];
};

template <typename T>
class Matrix<T, Dynamic, 3> {
 public:
  class ColRef {
   public:
    ColRef(T *p) : p_(p) {}
    T *data() const { return p_; }

   private:
    T *p_;
  };
  class RowRef {
   public:
    RowRef(Matrix *m, Index i) : m_(m), i_(i) {}
    RowRef &operator=(const Matrix<T, 3, 1> &v) {
      for (int j = 0; j < 3; ++j) (*m_)(i_, j) = v(j);
      return *this;
    }

   private:
    Matrix *m_;
    Index i_;
  };
  Matrix() = default;
  Matrix(Index rows, Index cols) { resize(rows, cols); }
  void resize(Index rows, Index /*cols*/) {
    rows_ = rows;
    d_.assign(static_cast<size_t>(rows) * 3, T(0));
  }
  void conservativeResize(Index rows, Index /*cols*/) {
    std::vector<T> n(static_cast<size_t>(rows) * 3, T(0));
    const Index keep = rows < rows_ ? rows : rows_;
    for (int j = 0; j < 3; ++j)
      for (Index i = 0; i < keep; ++i) n[j * rows + i] = d_[j * rows_ + i];
    d_.swap(n);
    rows_ = rows;
  }
  Index rows() const { return rows_; }
  Index cols() const { return 3; }
  T &operator()(Index i, Index j) { return d_[static_cast<size_t>(j) * rows_ + i]; }
  T operator()(Index i, Index j) const { return d_[static_cast<size_t>(j) * rows_ + i]; }
  ColRef col(Index j) { return ColRef(d_.data() + static_cast<size_t>(j) * rows_); }
  const ColRef col(Index j) const {
    return ColRef(const_cast<T *>(d_.data()) + static_cast<size_t>(j) * rows_);
  }
  RowRef row(Index i) { return RowRef(this, i); }
  T *data() { return d_.data(); }
  const T *data() const { return d_.data(); }

 private:
  std::vector<T> d_;
  Index rows_ = 0;
};

using Vector3f = Matrix<float, 3, 1>;
using Vector3i = Matrix<int, 3, 1>;

}  // namespace Eigen
