// Ahead-of-time build of the reverse-step kernels for elastic lattices
// (elastoplastic lattices get theirs from the runtime compiler, jit.cpp).
#include "adjoint_kernels.cuh"
#include "engine.hpp"

namespace dl {

template <class T>
AdjKernels aot_adj_kernels() {
  AdjKernels k;
  k.node = reinterpret_cast<const void *>(&k_adj_node<T>);
  k.elem = reinterpret_cast<const void *>(&k_adj_elem<T, AdjElastic>);
  return k;
}

template AdjKernels aot_adj_kernels<float>();
template AdjKernels aot_adj_kernels<double>();

}  // namespace dl
