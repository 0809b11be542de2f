// Host-memory stand-in for the reference's Matrix<T> (include/matrix.hpp),
// used only when the reference's objective headers (examples/gaussian.hpp,
// examples/simulation/fitting/LogLikelihood.h) are compiled for the host.
// It keeps the interface those objectives use (rows/cols ctor, set(ptr, n),
// data()) and stores one host copy; data() returns it, as the reference's
// data() does when compiled for the host.
#pragma once
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <vector>

template <typename T>
class Matrix {
  std::shared_ptr<std::vector<T>> buf_;
  std::size_t rows_ = 0, cols_ = 0;

public:
  Matrix() = default;
  Matrix(std::size_t rows, std::size_t cols)
    : buf_(std::make_shared<std::vector<T>>(rows * cols)), rows_(rows),
      cols_(cols)
  {
    if (!rows || !cols)
      throw std::invalid_argument("Matrix dimensions must be > 0");
  }
  void
  set(const T* host_ptr, std::size_t count)
  {
    if (count != rows_ * cols_)
      throw std::invalid_argument("count must equal rows*cols");
    std::copy(host_ptr, host_ptr + count, buf_->begin());
  }
  const T*
  data() const noexcept
  {
    return buf_ ? buf_->data() : nullptr;
  }
  std::size_t
  rows() const noexcept
  {
    return rows_;
  }
  std::size_t
  cols() const noexcept
  {
    return cols_;
  }
};
