// Host side of the contact candidate list (see contact.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <stdexcept>
#include <string>

#include "setup.hpp"

namespace dl {

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string &m) : std::runtime_error(m) {}
};
// a feature combination the engine does not cover (DL_ERR_UNSUPPORTED)
struct UnsupportedError : std::runtime_error {
  explicit UnsupportedError(const std::string &m) : std::runtime_error(m) {}
};
// a node without (or with negative) mass (DL_ERR_MASS; ExplicitModule.cpp:450-453)
struct MassError : std::runtime_error {
  explicit MassError(const std::string &m) : std::runtime_error(m) {}
};

// owning device allocation
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  void alloc(size_t n) {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = n;
    if (n) {
      cudaError_t e = cudaMalloc(&p, n);
      if (e != cudaSuccess) {
        p = nullptr;
        bytes = 0;
        cudaGetLastError();
        throw CudaError(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      }
    }
  }
  template <class T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

// The stream-ordered memory pool of the current device that keeps the
// memory freed into it (release threshold: unlimited), created on first use.
cudaMemPool_t retained_pool();
// Give the retained pool's unused memory back to the device.
void trim_retained_pool();

// Owning allocation from retained_pool(): the multi-GB state tapes of the
// adjoint are mapped once per process, and an engine created after another
// one was destroyed reuses them instead of mapping fresh pages.  The owner
// must have synchronised its stream before the destructor runs (the free is
// then ordered on the legacy stream, which has nothing left to wait for).
struct PoolBuf {
  void *p = nullptr;
  size_t bytes = 0;
  PoolBuf() = default;
  PoolBuf(const PoolBuf &) = delete;
  PoolBuf &operator=(const PoolBuf &) = delete;
  ~PoolBuf() {
    if (p) cudaFreeAsync(p, nullptr);
  }
  // replace the allocation by one of n bytes, stream-ordered on s
  void alloc(size_t n, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    bytes = 0;
    if (n) {
      cudaError_t e = cudaMallocFromPoolAsync(&p, n, retained_pool(), s);
      if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        throw CudaError(std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e));
      }
      bytes = n;
    }
  }
  template <class T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

// Node-ordered index of the ends of a pair list, so that every node sums the
// contributions of its pairs in one fixed order: entry v = p * ends + q (end
// q of pair p), sorted by the end's node and, per node, by v.  With the pair
// list itself sorted by its element (or node) indices, the order does not
// depend on the order in which the list build emitted the pairs, and
// repeated runs give the same bits.
struct PairEnds {
  DevBuf key_in, key_out, val_in, val_out, cnt, ptr, tmp;
  size_t cap = 0;
  int64_t launches = 0;
  // ends_node [n_entries]: node of each end (device); N nodes
  void build(const int32_t *ends_node, int n_entries, int N, cudaStream_t s);
};

// Sort a device pair list by its (x, y) key, ascending, through `keys` (two
// buffers of at least n 64-bit words) and `tmp`.
void sort_pairs(int2 *pairs, int n, DevBuf &keys, DevBuf &tmp, cudaStream_t s, int64_t *launches);

struct ContactList {
  cudaStream_t stream = nullptr;
  int N = 0, E = 0;
  double radius = 0.0, margin = 0.0, cell_h = 0.0;
  unsigned n_buckets = 0, capacity = 0;
  int n_pairs = 0, n_blacklist = 0;
  int64_t launches = 0;  // kernels launched (cub's scan counted as its 2 kernels)
  DevBuf nr_ptr, nr, rod, cell, count, start, cursor, items, scalars, scan_tmp, pairs, blacklist, xbuild;
  // per pair of the current list: closed in this step, and its 12 node forces
  // (4 nodes x 3) when closed; the node-ordered index of the pair ends
  DevBuf closed, force, sort_keys, sort_tmp, end_node;
  PairEnds ends;

  void init(const HostLattice &h, cudaStream_t s);
  // candidate pairs within `reach` of each other at positions `pos`
  void build(const double4 *pos, const int2 *conn, double reach);
  // pairs already in contact in the initial configuration (computeBlacklist_)
  void init_blacklist(const double4 *pos, const int2 *conn);
  double max_speed(const double *vel);
};

// Candidate list of the joint contact (JointContactModel): joint pairs within
// 2r + margin of each other at the build positions whose reference distance
// exceeds 2r, as (node A, node B) in internal numbering with A before B in the
// joint list.  Like ContactList it stays valid while no node moves more than
// margin/2.
struct JointList {
  cudaStream_t stream = nullptr;
  int N = 0, J = 0;
  double radius = 0.0, margin = 0.0, cell_h = 0.0;
  unsigned n_buckets = 0, capacity = 0;
  int n_pairs = 0;
  int64_t launches = 0;
  DevBuf node, x0, cell, count, start, cursor, items, scalars, scan_tmp, pairs, xbuild;
  // per pair: closed in this step, its 6 node forces (2 nodes x 3), and the
  // node-ordered index of the pair ends
  DevBuf closed, force, sort_keys, sort_tmp, end_node;
  PairEnds ends;

  void init(const HostLattice &h, cudaStream_t s);
  void build(const double4 *pos);
};

// max_n |v_n| (translations, [6][N] layout) through `scratch` (one word); synchronises `stream`
double node_max_speed(const double *vel, int N, unsigned long long *scratch, cudaStream_t stream);

}  // namespace dl
