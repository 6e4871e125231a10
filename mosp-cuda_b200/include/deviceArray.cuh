#ifndef MOSP_B200_DEVICE_ARRAY_CUH
#define MOSP_B200_DEVICE_ARRAY_CUH

// Owning, move-only device buffer (same interface as the reference's
// DeviceArray, SMShovan/MOSP-CUDA headers/deviceArray.cuh:12-65).

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

template <typename T> class DeviceArray {
public:
  DeviceArray() = default;
  explicit DeviceArray(size_t count) { allocate(count); }
  ~DeviceArray() { reset(); }
  DeviceArray(const DeviceArray &) = delete;
  DeviceArray &operator=(const DeviceArray &) = delete;
  DeviceArray(DeviceArray &&other) noexcept : data_(other.data_), size_(other.size_) {
    other.data_ = nullptr;
    other.size_ = 0;
  }
  DeviceArray &operator=(DeviceArray &&other) noexcept {
    if (this != &other) {
      reset();
      data_ = other.data_;
      size_ = other.size_;
      other.data_ = nullptr;
      other.size_ = 0;
    }
    return *this;
  }

  /// (Re)allocate count elements (storage for at least one); contents
  /// undefined.
  bool allocate(size_t count) {
    reset();
    size_ = count;
    void *p = nullptr;
    if (cudaMalloc(&p, (count > 0 ? count : 1) * sizeof(T)) != cudaSuccess) {
      size_ = 0;
      return false;
    }
    data_ = static_cast<T *>(p);
    return true;
  }
  /// Allocate and copy a host vector.
  bool upload(const std::vector<T> &host) {
    if (!allocate(host.size())) return false;
    return host.empty() || cudaMemcpy(data_, host.data(), host.size() * sizeof(T),
                                      cudaMemcpyHostToDevice) == cudaSuccess;
  }
  /// Copy the whole buffer into a host vector (resized).
  bool download(std::vector<T> &host) const {
    host.resize(size_);
    return size_ == 0 || cudaMemcpy(host.data(), data_, size_ * sizeof(T),
                                    cudaMemcpyDeviceToHost) == cudaSuccess;
  }

  T *data() { return data_; }
  const T *data() const { return data_; }
  size_t size() const { return size_; }

private:
  void reset() {
    if (data_ != nullptr) cudaFree(data_);
    data_ = nullptr;
    size_ = 0;
  }
  T *data_ = nullptr;
  size_t size_ = 0;
};

#endif // MOSP_B200_DEVICE_ARRAY_CUH
