// Candidate-pair list of rod--rod contact (B200 broad phase).
//
// The reference searches all rod pairs by bounding boxes and then all element
// pairs of overlapping rods, every step (RodContactModel::findContacts_,
// RodContactModel.cpp:245-446).  A pair can only produce a force when its
// segments are within 2r; this file builds, from the current positions, the
// list of element pairs whose segments are within 2r + margin (uniform hash
// grid of element centres, 27-cell query, exact clamped segment distance),
// excluding what the reference excludes (elements of one rod; an element that
// shares a node with the other rod, :393, :413; pairs closed at INIT, the
// blacklist of computeBlacklist_, :743-936).  Pairs are oriented as the
// reference orients them (A from the rod with the smaller index) because its
// one-sided node-to-segment branch is not symmetric.  The list stays valid
// while no node moves more than margin/2; the engine rebuilds it between
// chunks of steps and the step kernel flags a stale list.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "contact.cuh"
#include "contact_build.hpp"

namespace dl {

namespace {

__device__ __forceinline__ unsigned cell_hash(int ix, int iy, int iz, unsigned mask) {
  return (static_cast<unsigned>(ix) * 73856093u ^ static_cast<unsigned>(iy) * 19349663u ^
          static_cast<unsigned>(iz) * 83492791u) & mask;
}

__global__ void k_cells(const double4 *pos, const int2 *conn, int E, double inv_h, double box_limit, int4 *cell,
                        unsigned *count, unsigned mask, unsigned *flag) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
    const double4 a = pos[conn[e].x], b = pos[conn[e].y];
    const double cx = 0.5 * (a.x + b.x), cy = 0.5 * (a.y + b.y), cz = 0.5 * (a.z + b.z);
    const double ext = fmax(fabs(a.x - b.x), fmax(fabs(a.y - b.y), fabs(a.z - b.z)));
    if (ext > box_limit) atomicOr(flag, 1u);
    const int ix = static_cast<int>(floor(cx * inv_h)), iy = static_cast<int>(floor(cy * inv_h)),
              iz = static_cast<int>(floor(cz * inv_h));
    const unsigned key = cell_hash(ix, iy, iz, mask);
    cell[e] = make_int4(ix, iy, iz, static_cast<int>(key));
    atomicAdd(count + key, 1u);
  }
}

__global__ void k_fill(const int4 *cell, int E, const unsigned *start, unsigned *cursor, int *items) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
    const unsigned key = static_cast<unsigned>(cell[e].w);
    items[start[key] + atomicAdd(cursor + key, 1u)] = e;
  }
}

__device__ __forceinline__ bool node_in_rod(const int32_t *ptr, const int32_t *rods, int node, int rod) {
  for (int i = ptr[node]; i < ptr[node + 1]; ++i)
    if (rods[i] == rod) return true;
  return false;
}

__device__ __forceinline__ bool blacklisted(const unsigned long long *bl, int nbl, int a, int b) {
  const unsigned long long key = (static_cast<unsigned long long>(a) << 32) | static_cast<unsigned>(b);
  int lo = 0, hi = nbl;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (bl[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo < nbl && bl[lo] == key;
}

__global__ void k_pairs(const double4 *pos, const int2 *conn, const int32_t *rod, int E, const int4 *cell,
                        const unsigned *start, const unsigned *count, const int *items, unsigned mask,
                        const int32_t *nr_ptr, const int32_t *nr, const unsigned long long *bl, int nbl,
                        double reach, int2 *pairs, unsigned cap, unsigned *n_pairs) {
  // threads walk the elements in bucket order (items), so neighbouring
  // threads query the same cells
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < E; t += gridDim.x * blockDim.x) {
    const int e = items[t];
    const int4 ce = cell[e];
    const int2 ce2 = conn[e];
    const int re = rod[e];
    PairGeom g;
    const double4 a0 = pos[ce2.x], a1 = pos[ce2.y];
    g.A[0][0] = a0.x; g.A[0][1] = a0.y; g.A[0][2] = a0.z;
    g.A[1][0] = a1.x; g.A[1][1] = a1.y; g.A[1][2] = a1.z;
    const double alo[3] = {fmin(a0.x, a1.x) - reach, fmin(a0.y, a1.y) - reach, fmin(a0.z, a1.z) - reach};
    const double ahi[3] = {fmax(a0.x, a1.x) + reach, fmax(a0.y, a1.y) + reach, fmax(a0.z, a1.z) + reach};
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int ix = ce.x + dx, iy = ce.y + dy, iz = ce.z + dz;
          const unsigned key = cell_hash(ix, iy, iz, mask);
          const unsigned s0 = start[key], n = count[key];
          for (unsigned q = 0; q < n; ++q) {
            const int f = items[s0 + q];
            if (f <= e) continue;
            const int4 cf = cell[f];
            if (cf.x != ix || cf.y != iy || cf.z != iz) continue;  // other cell in the same bucket
            const int rf = rod[f];
            if (rf == re) continue;
            const int2 cf2 = conn[f];
            const double4 b0 = pos[cf2.x], b1 = pos[cf2.y];
            // bounding boxes (inflated by the reach) must overlap
            if (fmax(b0.x, b1.x) < alo[0] || fmin(b0.x, b1.x) > ahi[0] || fmax(b0.y, b1.y) < alo[1] ||
                fmin(b0.y, b1.y) > ahi[1] || fmax(b0.z, b1.z) < alo[2] || fmin(b0.z, b1.z) > ahi[2])
              continue;
            g.B[0][0] = b0.x; g.B[0][1] = b0.y; g.B[0][2] = b0.z;
            g.B[1][0] = b1.x; g.B[1][1] = b1.y; g.B[1][2] = b1.z;
            if (segment_distance(g) > reach) continue;
            if (node_in_rod(nr_ptr, nr, ce2.x, rf) || node_in_rod(nr_ptr, nr, ce2.y, rf) ||
                node_in_rod(nr_ptr, nr, cf2.x, re) || node_in_rod(nr_ptr, nr, cf2.y, re))
              continue;
            // orientation of the reference: A belongs to the rod with the smaller index
            const int pa = (re < rf) ? e : f, pb = (re < rf) ? f : e;
            if (nbl > 0 && blacklisted(bl, nbl, pa, pb)) continue;
            const unsigned slot = atomicAdd(n_pairs, 1u);
            if (slot < cap) pairs[slot] = make_int2(pa, pb);
          }
        }
  }
}

// contact state of each candidate at t = 0 (for the blacklist)
__global__ void k_closed(const double4 *pos, const int2 *conn, const int2 *pairs, int n, double r, unsigned char *closed) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int2 pr = pairs[p];
    PairGeom g;
    const double4 a0 = pos[conn[pr.x].x], a1 = pos[conn[pr.x].y], b0 = pos[conn[pr.y].x], b1 = pos[conn[pr.y].y];
    g.A[0][0] = a0.x; g.A[0][1] = a0.y; g.A[0][2] = a0.z;
    g.A[1][0] = a1.x; g.A[1][1] = a1.y; g.A[1][2] = a1.z;
    g.B[0][0] = b0.x; g.B[0][1] = b0.y; g.B[0][2] = b0.z;
    g.B[1][0] = b1.x; g.B[1][1] = b1.y; g.B[1][2] = b1.z;
    double gap = 0.0, en = 0.0;
    closed[p] = pair_contact(g, r, 1.0, 1.0, nullptr, gap, en) ? 1 : 0;
  }
}

__global__ void k_max_speed(const double *vel, int N, unsigned long long *out) {
  double m = 0.0;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x)
    m = fmax(m, sqrt(vel[n] * vel[n] + vel[N + n] * vel[N + n] + vel[2 * N + n] * vel[2 * N + n]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __double_as_longlong(m));
}

__global__ void k_copy_xyz(const double4 *pos, int N, double *x) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const double4 p = pos[n];
    x[3 * n] = p.x;
    x[3 * n + 1] = p.y;
    x[3 * n + 2] = p.z;
  }
}

// ---- joint contact (JointContactModel): points instead of segments

__global__ void k_jcells(const double4 *pos, const int32_t *node, int J, double inv_h, int4 *cell, unsigned *count,
                         unsigned mask) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < J; j += gridDim.x * blockDim.x) {
    const double4 a = pos[node[j]];
    const int ix = static_cast<int>(floor(a.x * inv_h)), iy = static_cast<int>(floor(a.y * inv_h)),
              iz = static_cast<int>(floor(a.z * inv_h));
    const unsigned key = cell_hash(ix, iy, iz, mask);
    cell[j] = make_int4(ix, iy, iz, static_cast<int>(key));
    atomicAdd(count + key, 1u);
  }
}

// Joint pairs (A, B), A before B in the joint list, within `reach` of each
// other now and more than 2r apart in the reference configuration (the
// reference's second condition, JointContactModel.cpp:262).  Cells are at
// least `reach` wide, so the 27-cell query finds every such pair.
__global__ void k_jpairs(const double4 *pos, const int32_t *node, const double *x0, int J, const int4 *cell,
                         const unsigned *start, const unsigned *count, const int *items, unsigned mask, double reach,
                         double r2, int2 *pairs, unsigned cap, unsigned *n_pairs) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < J; t += gridDim.x * blockDim.x) {
    const int ja = items[t];
    const int4 ca = cell[ja];
    const int na = node[ja];
    const double4 a = pos[na];
    const double Xa = x0[3 * ja], Ya = x0[3 * ja + 1], Za = x0[3 * ja + 2];
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int ix = ca.x + dx, iy = ca.y + dy, iz = ca.z + dz;
          const unsigned key = cell_hash(ix, iy, iz, mask);
          const unsigned s0 = start[key], n = count[key];
          for (unsigned q = 0; q < n; ++q) {
            const int jb = items[s0 + q];
            if (jb <= ja) continue;
            const int4 cb = cell[jb];
            if (cb.x != ix || cb.y != iy || cb.z != iz) continue;  // other cell in the same bucket
            const int nb = node[jb];
            const double4 b = pos[nb];
            const double ex = b.x - a.x, ey = b.y - a.y, ez = b.z - a.z;
            if (ex * ex + ey * ey + ez * ez > reach * reach) continue;
            const double fx = x0[3 * jb] - Xa, fy = x0[3 * jb + 1] - Ya, fz = x0[3 * jb + 2] - Za;
            if (!(sqrt(fx * fx + fy * fy + fz * fz) > r2)) continue;
            const unsigned slot = atomicAdd(n_pairs, 1u);
            if (slot < cap) pairs[slot] = make_int2(na, nb);
          }
        }
  }
}

__global__ void k_pair_keys(const int2 *pairs, int n, unsigned long long *keys) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    keys[p] = (static_cast<unsigned long long>(static_cast<unsigned>(pairs[p].x)) << 32) |
              static_cast<unsigned>(pairs[p].y);
}

__global__ void k_keys_to_pairs(const unsigned long long *keys, int n, int2 *pairs) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    pairs[p] = make_int2(static_cast<int>(keys[p] >> 32), static_cast<int>(keys[p] & 0xffffffffu));
}

// nodes of the four ends of each element pair: A's first, A's second, B's first, B's second
__global__ void k_contact_ends(const int2 *pairs, const int2 *conn, int n, int32_t *ends) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int2 a = conn[pairs[p].x], b = conn[pairs[p].y];
    ends[4 * p] = a.x;
    ends[4 * p + 1] = a.y;
    ends[4 * p + 2] = b.x;
    ends[4 * p + 3] = b.y;
  }
}

// the two ends of each joint pair
__global__ void k_joint_ends(const int2 *pairs, int n, int32_t *ends) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    ends[2 * p] = pairs[p].x;
    ends[2 * p + 1] = pairs[p].y;
  }
}

__global__ void k_end_entries(const int32_t *ends, int n, unsigned *key, int *val, unsigned *cnt) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    key[v] = static_cast<unsigned>(ends[v]);
    val[v] = v;
    atomicAdd(cnt + ends[v], 1u);
  }
}

int blocks_for(int n) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int want = (n + 255) / 256;
  return std::max(1, std::min(want, sms * 8));
}

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

void PairEnds::build(const int32_t *ends_node, int n, int N, cudaStream_t s) {
  const size_t need = static_cast<size_t>(std::max(n, 1));
  if (cap < need || !ptr.p) {
    cap = need + need / 2;
    key_in.alloc(cap * sizeof(unsigned));
    key_out.alloc(cap * sizeof(unsigned));
    val_in.alloc(cap * sizeof(int));
    val_out.alloc(cap * sizeof(int));
    size_t t1 = 0, t2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, static_cast<unsigned *>(nullptr), static_cast<unsigned *>(nullptr),
                                    static_cast<int *>(nullptr), static_cast<int *>(nullptr), static_cast<int>(cap));
    cub::DeviceScan::ExclusiveSum(nullptr, t2, static_cast<unsigned *>(nullptr),
                                  static_cast<unsigned *>(nullptr), N + 1);
    tmp.alloc(std::max<size_t>(std::max(t1, t2), 16));
  }
  if (cnt.bytes < static_cast<size_t>(N + 1) * sizeof(unsigned)) {
    cnt.alloc(static_cast<size_t>(N + 1) * sizeof(unsigned));
    ptr.alloc(static_cast<size_t>(N + 1) * sizeof(unsigned));
  }
  check(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s), "memset");
  if (n > 0) {
    k_end_entries<<<blocks_for(n), 256, 0, s>>>(ends_node, n, key_in.as<unsigned>(), val_in.as<int>(),
                                                 cnt.as<unsigned>());
    ++launches;
    int bits = 1;
    while ((1 << bits) < N) ++bits;
    size_t t = tmp.bytes;
    // LSD radix sort: stable, so the entries of one node keep their order v
    check(cub::DeviceRadixSort::SortPairs(tmp.p, t, key_in.as<unsigned>(), key_out.as<unsigned>(), val_in.as<int>(),
                                          val_out.as<int>(), n, 0, bits, s),
          "sort");
    launches += 2;
  }
  size_t t = tmp.bytes;
  check(cub::DeviceScan::ExclusiveSum(tmp.p, t, cnt.as<unsigned>(), ptr.as<unsigned>(), N + 1, s), "scan");
  launches += 2;
}

void sort_pairs(int2 *pairs, int n, DevBuf &keys, DevBuf &tmp, cudaStream_t s, int64_t *launches) {
  if (n <= 1) return;
  if (keys.bytes < 2 * static_cast<size_t>(n) * sizeof(unsigned long long)) {
    keys.alloc(2 * static_cast<size_t>(n + n / 2) * sizeof(unsigned long long));
    tmp.alloc(0);
  }
  size_t need = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, need, static_cast<unsigned long long *>(nullptr),
                                 static_cast<unsigned long long *>(nullptr), n);
  if (tmp.bytes < need) tmp.alloc(need + need / 2 + 16);
  unsigned long long *k0 = keys.as<unsigned long long>();
  unsigned long long *k1 = k0 + keys.bytes / sizeof(unsigned long long) / 2;
  k_pair_keys<<<blocks_for(n), 256, 0, s>>>(pairs, n, k0);
  size_t t = tmp.bytes;
  check(cub::DeviceRadixSort::SortKeys(tmp.p, t, k0, k1, n, 0, 64, s), "sort");
  k_keys_to_pairs<<<blocks_for(n), 256, 0, s>>>(k1, n, pairs);
  check(cudaGetLastError(), "pair sort");
  *launches += 4;
}

void ContactList::init(const HostLattice &h, cudaStream_t s) {
  stream = s;
  N = h.N;
  E = h.E;
  radius = h.contact.radius;
  margin = h.contact.margin > 0 ? h.contact.margin : 0.5 * radius;
  // node -> rods (internal numbering), for the reference's shared-node exclusion
  std::vector<std::vector<int32_t>> lists(N);
  for (int e = 0; e < E; ++e)
    for (int a = 0; a < 2; ++a) {
      auto &l = lists[h.conn[2 * e + a]];
      if (std::find(l.begin(), l.end(), h.elem_rod[e]) == l.end()) l.push_back(h.elem_rod[e]);
    }
  std::vector<int32_t> ptr(N + 1, 0), rods;
  for (int n = 0; n < N; ++n) {
    ptr[n + 1] = ptr[n] + static_cast<int32_t>(lists[n].size());
    rods.insert(rods.end(), lists[n].begin(), lists[n].end());
  }
  nr_ptr.alloc(ptr.size() * sizeof(int32_t));
  check(cudaMemcpy(nr_ptr.p, ptr.data(), ptr.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
  nr.alloc(std::max<size_t>(1, rods.size()) * sizeof(int32_t));
  if (!rods.empty()) check(cudaMemcpy(nr.p, rods.data(), rods.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
  rod.alloc(static_cast<size_t>(E) * sizeof(int32_t));
  check(cudaMemcpy(rod.p, h.elem_rod.data(), static_cast<size_t>(E) * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
  // cell size: longest element box + 2r + margin, with room for 25 % stretch
  double lmax = 0.0;
  for (int e = 0; e < E; ++e) lmax = std::max(lmax, 1.0 / h.invL0[e]);
  cell_h = 1.25 * lmax + 2.0 * radius + margin;
  unsigned T = 1024;
  while (T < 2u * static_cast<unsigned>(E)) T <<= 1;
  n_buckets = T;
  cell.alloc(static_cast<size_t>(E) * sizeof(int4));
  count.alloc(static_cast<size_t>(T) * sizeof(unsigned));
  start.alloc(static_cast<size_t>(T) * sizeof(unsigned));
  cursor.alloc(static_cast<size_t>(T) * sizeof(unsigned));
  items.alloc(static_cast<size_t>(E) * sizeof(int));
  scalars.alloc(4 * sizeof(unsigned long long));
  xbuild.alloc(static_cast<size_t>(N) * 3 * sizeof(double));
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, static_cast<unsigned *>(nullptr), static_cast<unsigned *>(nullptr),
                                static_cast<int>(T));
  scan_tmp.alloc(std::max<size_t>(tmp, 16));
  capacity = h.contact.max_pairs > 0 ? static_cast<unsigned>(h.contact.max_pairs) : std::max(1024u, 8u * E);
  pairs.alloc(static_cast<size_t>(capacity) * sizeof(int2));
}

void ContactList::build(const double4 *pos, const int2 *conn, double reach) {
  unsigned long long *sc = scalars.as<unsigned long long>();
  for (int attempt = 0; attempt < 8; ++attempt) {
    check(cudaMemsetAsync(count.p, 0, count.bytes, stream), "memset");
    check(cudaMemsetAsync(cursor.p, 0, cursor.bytes, stream), "memset");
    check(cudaMemsetAsync(sc, 0, scalars.bytes, stream), "memset");
    const unsigned mask = n_buckets - 1;
    unsigned *flag = reinterpret_cast<unsigned *>(sc);
    k_cells<<<blocks_for(E), 256, 0, stream>>>(pos, conn, E, 1.0 / cell_h, cell_h - 2.0 * radius - margin,
                                               cell.as<int4>(), count.as<unsigned>(), mask, flag);
    size_t tmp = scan_tmp.bytes;
    check(cub::DeviceScan::ExclusiveSum(scan_tmp.p, tmp, count.as<unsigned>(), start.as<unsigned>(),
                                        static_cast<int>(n_buckets), stream),
          "scan");
    k_fill<<<blocks_for(E), 256, 0, stream>>>(cell.as<int4>(), E, start.as<unsigned>(), cursor.as<unsigned>(),
                                              items.as<int>());
    unsigned *npair = reinterpret_cast<unsigned *>(sc + 1);
    k_pairs<<<blocks_for(E), 256, 0, stream>>>(pos, conn, rod.as<int32_t>(), E, cell.as<int4>(),
                                               start.as<unsigned>(), count.as<unsigned>(), items.as<int>(), mask,
                                               nr_ptr.as<int32_t>(), nr.as<int32_t>(),
                                               blacklist.as<unsigned long long>(), n_blacklist, reach,
                                               pairs.as<int2>(), capacity, npair);
    check(cudaGetLastError(), "contact build");
    launches += 5;
    unsigned host[4] = {0, 0, 0, 0};
    check(cudaMemcpyAsync(host, sc, sizeof host, cudaMemcpyDeviceToHost, stream), "readback");
    check(cudaStreamSynchronize(stream), "sync");
    if (host[0]) {  // an element box outgrew the cell size
      cell_h *= 1.5;
      continue;
    }
    const unsigned np = host[2];
    if (np > capacity) {
      capacity = np + np / 2 + 1024;
      pairs.alloc(static_cast<size_t>(capacity) * sizeof(int2));
      continue;
    }
    n_pairs = static_cast<int>(np);
    // deterministic order: pairs by (A, B), each node's pair ends by pair
    sort_pairs(pairs.as<int2>(), n_pairs, sort_keys, sort_tmp, stream, &launches);
    if (closed.bytes < static_cast<size_t>(capacity)) {
      closed.alloc(static_cast<size_t>(capacity));
      force.alloc(static_cast<size_t>(capacity) * 12 * sizeof(double));
      end_node.alloc(static_cast<size_t>(capacity) * 4 * sizeof(int32_t));
    }
    if (n_pairs > 0) {
      k_contact_ends<<<blocks_for(n_pairs), 256, 0, stream>>>(pairs.as<int2>(), conn, n_pairs,
                                                              end_node.as<int32_t>());
      ++launches;
    }
    ends.build(end_node.as<int32_t>(), 4 * n_pairs, N, stream);
    k_copy_xyz<<<blocks_for(N), 256, 0, stream>>>(pos, N, xbuild.as<double>());
    check(cudaGetLastError(), "contact build");
    ++launches;
    return;
  }
  throw std::runtime_error("contact candidate list could not be built");
}

void ContactList::init_blacklist(const double4 *pos, const int2 *conn) {
  n_blacklist = 0;
  build(pos, conn, 2.0 * radius);
  if (n_pairs == 0) return;
  DevBuf closed;
  closed.alloc(static_cast<size_t>(n_pairs));
  k_closed<<<blocks_for(n_pairs), 256, 0, stream>>>(pos, conn, pairs.as<int2>(), n_pairs, radius,
                                                    closed.as<unsigned char>());
  ++launches;
  std::vector<int2> pr(n_pairs);
  std::vector<unsigned char> cl(n_pairs);
  check(cudaMemcpyAsync(pr.data(), pairs.p, pr.size() * sizeof(int2), cudaMemcpyDeviceToHost, stream), "readback");
  check(cudaMemcpyAsync(cl.data(), closed.p, cl.size(), cudaMemcpyDeviceToHost, stream), "readback");
  check(cudaStreamSynchronize(stream), "sync");
  std::vector<unsigned long long> keys;
  for (int i = 0; i < n_pairs; ++i)
    if (cl[i]) keys.push_back((static_cast<unsigned long long>(pr[i].x) << 32) | static_cast<unsigned>(pr[i].y));
  std::sort(keys.begin(), keys.end());
  n_blacklist = static_cast<int>(keys.size());
  if (n_blacklist) {
    blacklist.alloc(keys.size() * sizeof(unsigned long long));
    check(cudaMemcpy(blacklist.p, keys.data(), keys.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice),
          "upload");
  }
}

double ContactList::max_speed(const double *vel) {
  unsigned long long *sc = scalars.as<unsigned long long>();
  check(cudaMemsetAsync(sc + 3, 0, sizeof(unsigned long long), stream), "memset");
  k_max_speed<<<blocks_for(N), 256, 0, stream>>>(vel, N, sc + 3);
  ++launches;
  unsigned long long bits = 0;
  check(cudaMemcpyAsync(&bits, sc + 3, sizeof bits, cudaMemcpyDeviceToHost, stream), "readback");
  check(cudaStreamSynchronize(stream), "sync");
  double v;
  std::memcpy(&v, &bits, sizeof v);
  return v;
}

void JointList::init(const HostLattice &h, cudaStream_t s) {
  stream = s;
  N = h.N;
  J = static_cast<int>(h.joints.size());
  radius = h.jcontact.radius;
  margin = h.jcontact.margin > 0 ? h.jcontact.margin : 0.5 * radius;
  cell_h = 2.0 * radius + margin;
  unsigned T = 1024;
  while (T < 2u * static_cast<unsigned>(std::max(J, 1))) T <<= 1;
  n_buckets = T;
  const size_t Jn = static_cast<size_t>(std::max(J, 1));
  node.alloc(Jn * sizeof(int32_t));
  x0.alloc(Jn * 3 * sizeof(double));
  if (J > 0) {
    std::vector<double> X(static_cast<size_t>(J) * 3);
    for (int j = 0; j < J; ++j)
      for (int k = 0; k < 3; ++k) X[3 * j + k] = h.X0[static_cast<size_t>(h.node_old[h.joints[j]]) * 3 + k];
    check(cudaMemcpy(node.p, h.joints.data(), static_cast<size_t>(J) * sizeof(int32_t), cudaMemcpyHostToDevice),
          "upload");
    check(cudaMemcpy(x0.p, X.data(), X.size() * sizeof(double), cudaMemcpyHostToDevice), "upload");
  }
  cell.alloc(Jn * sizeof(int4));
  count.alloc(static_cast<size_t>(T) * sizeof(unsigned));
  start.alloc(static_cast<size_t>(T) * sizeof(unsigned));
  cursor.alloc(static_cast<size_t>(T) * sizeof(unsigned));
  items.alloc(Jn * sizeof(int));
  scalars.alloc(4 * sizeof(unsigned long long));
  xbuild.alloc(static_cast<size_t>(N) * 3 * sizeof(double));
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, static_cast<unsigned *>(nullptr), static_cast<unsigned *>(nullptr),
                                static_cast<int>(T));
  scan_tmp.alloc(std::max<size_t>(tmp, 16));
  capacity = std::max(1024u, 4u * static_cast<unsigned>(J));
  pairs.alloc(static_cast<size_t>(capacity) * sizeof(int2));
}

void JointList::build(const double4 *pos) {
  unsigned long long *sc = scalars.as<unsigned long long>();
  const double reach = 2.0 * radius + margin;
  for (int attempt = 0; attempt < 8; ++attempt) {
    n_pairs = 0;
    if (J > 1) {
      check(cudaMemsetAsync(count.p, 0, count.bytes, stream), "memset");
      check(cudaMemsetAsync(cursor.p, 0, cursor.bytes, stream), "memset");
      check(cudaMemsetAsync(sc, 0, scalars.bytes, stream), "memset");
      const unsigned mask = n_buckets - 1;
      k_jcells<<<blocks_for(J), 256, 0, stream>>>(pos, node.as<int32_t>(), J, 1.0 / cell_h, cell.as<int4>(),
                                                  count.as<unsigned>(), mask);
      size_t tmp = scan_tmp.bytes;
      check(cub::DeviceScan::ExclusiveSum(scan_tmp.p, tmp, count.as<unsigned>(), start.as<unsigned>(),
                                          static_cast<int>(n_buckets), stream),
            "scan");
      k_fill<<<blocks_for(J), 256, 0, stream>>>(cell.as<int4>(), J, start.as<unsigned>(), cursor.as<unsigned>(),
                                                items.as<int>());
      unsigned *npair = reinterpret_cast<unsigned *>(sc + 1);
      k_jpairs<<<blocks_for(J), 256, 0, stream>>>(pos, node.as<int32_t>(), x0.as<double>(), J, cell.as<int4>(),
                                                  start.as<unsigned>(), count.as<unsigned>(), items.as<int>(), mask,
                                                  reach, 2.0 * radius, pairs.as<int2>(), capacity, npair);
      check(cudaGetLastError(), "joint contact build");
      launches += 5;
      unsigned host[4] = {0, 0, 0, 0};
      check(cudaMemcpyAsync(host, sc, sizeof host, cudaMemcpyDeviceToHost, stream), "readback");
      check(cudaStreamSynchronize(stream), "sync");
      const unsigned np = host[2];
      if (np > capacity) {
        capacity = np + np / 2 + 1024;
        pairs.alloc(static_cast<size_t>(capacity) * sizeof(int2));
        continue;
      }
      n_pairs = static_cast<int>(np);
    }
    sort_pairs(pairs.as<int2>(), n_pairs, sort_keys, sort_tmp, stream, &launches);
    if (closed.bytes < static_cast<size_t>(capacity)) {
      closed.alloc(static_cast<size_t>(capacity));
      force.alloc(static_cast<size_t>(capacity) * 6 * sizeof(double));
      end_node.alloc(static_cast<size_t>(capacity) * 2 * sizeof(int32_t));
    }
    if (n_pairs > 0) {
      k_joint_ends<<<blocks_for(n_pairs), 256, 0, stream>>>(pairs.as<int2>(), n_pairs, end_node.as<int32_t>());
      ++launches;
    }
    ends.build(end_node.as<int32_t>(), 2 * n_pairs, N, stream);
    k_copy_xyz<<<blocks_for(N), 256, 0, stream>>>(pos, N, xbuild.as<double>());
    check(cudaGetLastError(), "joint contact build");
    ++launches;
    return;
  }
  throw std::runtime_error("joint contact candidate list could not be built");
}

double node_max_speed(const double *vel, int N, unsigned long long *scratch, cudaStream_t stream) {
  check(cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), stream), "memset");
  k_max_speed<<<blocks_for(N), 256, 0, stream>>>(vel, N, scratch);
  unsigned long long bits = 0;
  check(cudaMemcpyAsync(&bits, scratch, sizeof bits, cudaMemcpyDeviceToHost, stream), "readback");
  check(cudaStreamSynchronize(stream), "sync");
  double v;
  std::memcpy(&v, &bits, sizeof v);
  return v;
}

}  // namespace dl
