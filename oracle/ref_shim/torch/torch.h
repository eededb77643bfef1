// Shim of the libtorch surface that canoe's src/interface/hydro.hpp and
// src/interface/eos.hpp touch: a strided double tensor view with accessor(),
// narrow() and copy_().  Only accessor() is reached by the compiled
// arithmetic (get_gamma reads the snapy cv / mu ratio tables through it).
#pragma once
#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <vector>

namespace torch {

enum ScalarType { kDouble };
struct TensorOptions {};
inline TensorOptions dtype(ScalarType) { return {}; }

template <typename T, int N>
struct TensorAccessor {
  T *p;
  const int64_t *stride;
  TensorAccessor<T, N - 1> operator[](int64_t i) const {
    return TensorAccessor<T, N - 1>{p + i * stride[0], stride + 1};
  }
};
template <typename T>
struct TensorAccessor<T, 1> {
  T *p;
  const int64_t *stride;
  T &operator[](int64_t i) const { return p[i * stride[0]]; }
};

class Tensor {
 public:
  Tensor() = default;
  Tensor(double *p, std::vector<int64_t> sizes, std::vector<int64_t> strides)
      : p_(p), sizes_(std::move(sizes)), strides_(std::move(strides)) {}
  // an owning 1-D tensor (the harness builds the snapy tables with it)
  static Tensor from_vector(const std::vector<double> &v) {
    Tensor t;
    t.own_ = std::make_shared<std::vector<double>>(v);
    t.p_ = t.own_->data();
    t.sizes_ = {(int64_t)v.size()};
    t.strides_ = {1};
    return t;
  }
  template <typename T, int N>
  TensorAccessor<T, N> accessor() const {
    if ((int)sizes_.size() != N) throw std::runtime_error("accessor rank");
    return TensorAccessor<T, N>{p_, strides_.data()};
  }
  Tensor narrow(int64_t dim, int64_t start, int64_t len) const {
    Tensor t = *this;
    t.p_ = p_ + start * strides_[dim];
    t.sizes_[dim] = len;
    return t;
  }
  Tensor &copy_(const Tensor &) { throw std::runtime_error("copy_ is not part of the pin"); }

 private:
  std::shared_ptr<std::vector<double>> own_;
  double *p_ = nullptr;
  std::vector<int64_t> sizes_, strides_;
};

inline Tensor operator*(double, const Tensor &) {
  throw std::runtime_error("tensor arithmetic is not part of the pin");
}

inline Tensor from_blob(void *p, std::vector<int64_t> sizes, std::vector<int64_t> strides,
                        std::nullptr_t, TensorOptions) {
  return Tensor(static_cast<double *>(p), std::move(sizes), std::move(strides));
}

}  // namespace torch
