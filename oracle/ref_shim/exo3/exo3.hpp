// Shim of canoe src/exo3/exo3.hpp for a Cartesian block.
//
// The reference's vec_lower returns the three velocity components as a
// std::array<T, 3>, and lmars.cpp:47-53 indexes that result with the
// variable slots ivx, ivy, ivz (IVX = 1 + ny and up), which reads past the
// array.  The intent is the Cartesian identity (lowered velocity = velocity),
// so that the enthalpy carries 1/2 |v|^2.  This shim's vec_lower returns a
// view of the state indexed by variable slot, which is that identity; the
// oracle and the CUDA kernels compute the same 1/2 |v|^2.
#pragma once
#include <athena/athena.hpp>

template <typename T>
struct SlotVector {
  const T *w;
  T operator[](int n) const { return w[n]; }
};

template <typename T, typename M>
SlotVector<T> vec_lower(const T *w, M &&) {
  return SlotVector<T>{w};
}

template <typename T, typename M>
SlotVector<T> vec_raise(const T *w, M &&) {
  return SlotVector<T>{w};
}
