// Allocation-free internal-force evaluation (see noalloc.cu).
#pragma once

#include <cstddef>

#include "../../include/dynlattice.h"
#include "engine.hpp"

namespace dl {

// Size of the static device scratch array.  A lattice of N nodes and E
// elements needs 2 * r(32 N) + r(12 E sizeof(T)) bytes (r: round up to 256):
// the configuration as positions and rotations, and the end-force slots.  The
// 20^3 BCC lattice (81,261 nodes, 128,000 elements) needs 17.5 MB in FP64.
constexpr size_t kStaticScratchBytes = 24u << 20;

// Device address of the static scratch array on device `dev`, which must be
// current; resolved with cudaGetSymbolAddress on the first call per device.
int static_scratch_address(int dev, void **ptr, const char **why);

// `device`: the device the handle was created on; the call makes it current
// for its duration and restores the caller's device afterwards.
template <class T>
int internal_force_static(const KernelSet &ks, const DevModel<T> &model, int device, const double *X0int,
                          const int32_t *node_old, const double *u, const double *theta, double *fint,
                          cudaStream_t stream, const char **why);

}  // namespace dl
