// matrix.hpp -- objective data for device-side objectives, under the
// reference's header name (include/matrix.hpp:20-258): objective headers
// written for the reference (examples/gaussian.hpp:6,
// simulation/fitting/LogLikelihood.h:5) include "matrix.hpp" and hold
// Matrix<T> members that they read through data() in device code.
#pragma once

#include <array>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>

#include <cuda_runtime.h>

// Host and device copies of a dense rows x cols matrix.  data() returns the
// device pointer in device code and the host pointer in host code.  Copies
// share the buffers (reference-counted on the host), so an objective holding
// a Matrix is cheap to copy into kernel parameters; set(...) writes the host
// copy and pushes it to the device, syncHost2Device() pushes the whole host
// copy after direct edits through operator() / hostData().
template <typename T>
class Matrix {
  struct Block {
    T* host = nullptr;
    T* device = nullptr;
    ~Block()
    {
      std::free(host);
      if (device)
        cudaFree(device);
    }
  };
  T* host_data_ = nullptr;
  T* device_data_ = nullptr;
  std::size_t rows_ = 0, cols_ = 0;
  std::shared_ptr<Block>* owner_ = nullptr; // host-side share count

  static void
  check(cudaError_t e)
  {
    if (e != cudaSuccess)
      throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e));
  }
  void
  bounds(std::size_t i, std::size_t j) const
  {
    if (i >= rows_ || j >= cols_)
      throw std::out_of_range("Matrix index out of range");
  }
  void
  release()
  {
    delete owner_;
    owner_ = nullptr;
    host_data_ = device_data_ = nullptr;
  }

public:
  Matrix() noexcept = default;
  Matrix(std::size_t rows, std::size_t cols) : rows_(rows), cols_(cols)
  {
    if (!rows || !cols)
      throw std::invalid_argument("Matrix dimensions must be > 0");
    auto b = std::make_shared<Block>();
    b->host = static_cast<T*>(std::calloc(rows * cols, sizeof(T)));
    if (!b->host)
      throw std::runtime_error("host malloc failed");
    check(cudaMalloc(&b->device, rows * cols * sizeof(T)));
    host_data_ = b->host;
    device_data_ = b->device;
    owner_ = new std::shared_ptr<Block>(std::move(b));
  }
  template <std::size_t N>
  Matrix(std::size_t rows, std::size_t cols, const std::array<T, N>& init)
    : Matrix(rows, cols)
  {
    set(init);
  }
  __host__ __device__ Matrix(const Matrix& o)
    : host_data_(o.host_data_), device_data_(o.device_data_), rows_(o.rows_),
      cols_(o.cols_)
  {
#ifndef __CUDA_ARCH__
    owner_ = o.owner_ ? new std::shared_ptr<Block>(*o.owner_) : nullptr;
#endif
  }
  Matrix&
  operator=(const Matrix& o)
  {
    if (this != &o) {
      release();
      host_data_ = o.host_data_;
      device_data_ = o.device_data_;
      rows_ = o.rows_;
      cols_ = o.cols_;
      owner_ = o.owner_ ? new std::shared_ptr<Block>(*o.owner_) : nullptr;
    }
    return *this;
  }
  __host__ __device__ ~Matrix()
  {
#ifndef __CUDA_ARCH__
    release();
#endif
  }

  void
  set(std::size_t i, std::size_t j, const T& x)
  {
    bounds(i, j);
    host_data_[i * cols_ + j] = x;
    check(cudaMemcpy(device_data_ + i * cols_ + j, &x, sizeof(T),
                     cudaMemcpyHostToDevice));
  }
  template <std::size_t N>
  void
  set(const std::array<T, N>& a)
  {
    set(a.data(), N);
  }
  void
  set(const T* host_ptr, std::size_t count)
  {
    if (count != rows_ * cols_)
      throw std::invalid_argument("count must equal rows*cols");
    std::memcpy(host_data_, host_ptr, count * sizeof(T));
    syncHost2Device();
  }
  void
  syncHost2Device()
  {
    check(cudaMemcpy(device_data_, host_data_, rows_ * cols_ * sizeof(T),
                     cudaMemcpyHostToDevice));
  }
  __host__ __device__ const T*
  data() const noexcept
  {
#ifdef __CUDA_ARCH__
    return device_data_;
#else
    return host_data_;
#endif
  }
  T*
  hostData() noexcept
  {
    return host_data_;
  }
  const T*
  hostData() const noexcept
  {
    return host_data_;
  }
  T*
  deviceData() noexcept
  {
    return device_data_;
  }
  const T*
  deviceData() const noexcept
  {
    return device_data_;
  }
  T&
  operator()(std::size_t i, std::size_t j)
  {
    bounds(i, j);
    return host_data_[i * cols_ + j];
  }
  const T&
  operator()(std::size_t i, std::size_t j) const
  {
    bounds(i, j);
    return host_data_[i * cols_ + j];
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

