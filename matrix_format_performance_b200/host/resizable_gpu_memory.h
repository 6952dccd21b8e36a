// Grow-only device buffer with the interface of the reference's
// resizable_gpu_memory<T> (gpu/resizable_gpu_memory.h:13-44): resize(n)
// reallocates only when n exceeds the capacity (contents are not kept),
// get() returns the device pointer, clear() frees.  Allocation failures throw.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <stdexcept>
#include <string>

template <typename T>
class resizable_gpu_memory {
 public:
  resizable_gpu_memory() = default;
  resizable_gpu_memory(const resizable_gpu_memory &) = delete;
  resizable_gpu_memory &operator=(const resizable_gpu_memory &) = delete;
  ~resizable_gpu_memory() { clear(); }

  void resize(size_t new_size) {
    if (new_size <= size_) return;
    clear();
    if (cudaMalloc(&data_, new_size * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      data_ = nullptr;
      throw std::runtime_error("resizable_gpu_memory: cudaMalloc of " + std::to_string(new_size * sizeof(T)) +
                               " bytes failed");
    }
    size_ = new_size;
  }
  void clear() {
    if (data_) cudaFree(data_);
    data_ = nullptr;
    size_ = 0;
  }
  T *get() { return data_; }
  const T *get() const { return data_; }
  size_t capacity() const { return size_; }

 private:
  T *data_ = nullptr;
  size_t size_ = 0;
};
