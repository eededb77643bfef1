// Shim of Athena++ athena_arrays.hpp: a contiguous array of up to four
// dimensions indexed (n, k, j, i) with i fastest, as Athena++ lays it out.
#pragma once
#include <cstddef>
#include <vector>

template <typename T>
class AthenaArray {
 public:
  AthenaArray() = default;
  AthenaArray(int nx4, int nx3, int nx2, int nx1) { NewAthenaArray(nx4, nx3, nx2, nx1); }
  void NewAthenaArray(int nx1) { NewAthenaArray(1, 1, 1, nx1); }
  void NewAthenaArray(int nx2, int nx1) { NewAthenaArray(1, 1, nx2, nx1); }
  void NewAthenaArray(int nx3, int nx2, int nx1) { NewAthenaArray(1, nx3, nx2, nx1); }
  void NewAthenaArray(int nx4, int nx3, int nx2, int nx1) {
    nx1_ = nx1;
    nx2_ = nx2;
    nx3_ = nx3;
    nx4_ = nx4;
    own_.assign((size_t)nx4 * nx3 * nx2 * nx1, T());
    p_ = own_.data();
  }
  // a view of caller memory (no copy), dimensions as NewAthenaArray
  void InitWithShallowSlice(T *p, int nx4, int nx3, int nx2, int nx1) {
    nx1_ = nx1;
    nx2_ = nx2;
    nx3_ = nx3;
    nx4_ = nx4;
    own_.clear();
    p_ = p;
  }
  T &operator()(int i) { return p_[i]; }
  T operator()(int i) const { return p_[i]; }
  T &operator()(int j, int i) { return p_[i + (size_t)nx1_ * j]; }
  T operator()(int j, int i) const { return p_[i + (size_t)nx1_ * j]; }
  T &operator()(int k, int j, int i) { return p_[i + (size_t)nx1_ * (j + (size_t)nx2_ * k)]; }
  T operator()(int k, int j, int i) const {
    return p_[i + (size_t)nx1_ * (j + (size_t)nx2_ * k)];
  }
  T &operator()(int n, int k, int j, int i) {
    return p_[i + (size_t)nx1_ * (j + (size_t)nx2_ * (k + (size_t)nx3_ * n))];
  }
  T operator()(int n, int k, int j, int i) const {
    return p_[i + (size_t)nx1_ * (j + (size_t)nx2_ * (k + (size_t)nx3_ * n))];
  }
  T *at(int k, int j, int i) { return &(*this)(k, j, i); }
  const T *at(int k, int j, int i) const { return &(*this)(k, j, i); }
  int GetDim1() const { return nx1_; }
  int GetDim2() const { return nx2_; }
  int GetDim3() const { return nx3_; }
  int GetDim4() const { return nx4_; }
  T *data() { return p_; }
  const T *data() const { return p_; }

 private:
  int nx1_ = 0, nx2_ = 0, nx3_ = 0, nx4_ = 0;
  std::vector<T> own_;
  T *p_ = nullptr;
};
