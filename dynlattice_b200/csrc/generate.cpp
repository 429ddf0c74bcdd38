// Random fibre network generator (engine extension; the reference reads its
// meshes from .geo/.msh files and has no generator of its own).
//
// Straight rods of length L, centres uniform in the cube [0, box]^3,
// directions uniform on the sphere, each split into `elems_per_rod` two-node
// elements.  Rods are inserted one at a time; a rod whose segment comes closer
// than 2r to an accepted rod is rejected and resampled (random sequential
// addition).  Overlap queries use a uniform grid of element midpoints whose
// cell is at least one element plus 2r wide, so the 27 neighbouring cells hold
// every element that can be within 2r of a query element.
//
// The random stream is splitmix64 (Steele, Lea & Flood 2014) and the sampling
// formulas are fixed, so one seed gives one network on every host.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "../../include/dynlattice.h"
#include "contact.cuh"

namespace {

struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  }
  // uniform in [0, 1) with 53 random bits
  double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Grid {
  double lo = 0.0, h = 1.0;
  int n = 1;
  std::vector<std::vector<int>> cells;
  int clampi(int i) const { return i < 0 ? 0 : (i >= n ? n - 1 : i); }
  int index(double x) const { return clampi(static_cast<int>(std::floor((x - lo) / h))); }
};

}  // namespace

extern "C" __attribute__((visibility("default"))) int dl_generate_fibres(int32_t n_rods, double length,
                                                                       int32_t elems_per_rod, double radius,
                                                                       double box, uint64_t seed,
                                                                       int64_t max_tries, double *coords,
                                                                       int32_t *conn, int32_t *elem_rod,
                                                                       int64_t *tries_out) {
  if (n_rods < 0 || elems_per_rod < 1 || !(length > 0.0) || !(radius >= 0.0) || !(box > 0.0) || !coords ||
      !conn || !elem_rod)
    return DL_ERR_INVALID;
  const int epr = elems_per_rod;
  const double le = length / epr, reach = 2.0 * radius;
  Grid g;
  g.lo = -0.5 * length - reach;
  g.h = le + reach;
  g.n = std::max(1, static_cast<int>(std::ceil((box + length + 2.0 * reach) / g.h)));
  if (static_cast<double>(g.n) * g.n * g.n > 5e7) return DL_ERR_UNSUPPORTED;
  g.cells.assign(static_cast<size_t>(g.n) * g.n * g.n, {});
  std::vector<double> seg;  // accepted elements: [e][2][3]
  seg.reserve(static_cast<size_t>(n_rods) * epr * 6);
  SplitMix64 rng{seed};
  int64_t tries = 0;
  const double two_pi = 6.283185307179586476925286766559;
  double cand[64][2][3];
  if (epr > 64) return DL_ERR_UNSUPPORTED;
  for (int r = 0; r < n_rods; ++r) {
    bool placed = false;
    double c[3], d[3];
    while (!placed) {
      if (max_tries > 0 && tries >= max_tries) {
        if (tries_out) *tries_out = tries;
        return DL_ERR_UNSUPPORTED;
      }
      ++tries;
      for (int k = 0; k < 3; ++k) c[k] = box * rng.uniform();
      const double z = 2.0 * rng.uniform() - 1.0, phi = two_pi * rng.uniform();
      const double s = std::sqrt(std::max(0.0, 1.0 - z * z));
      d[0] = s * std::cos(phi);
      d[1] = s * std::sin(phi);
      d[2] = z;
      for (int e = 0; e < epr; ++e)
        for (int a = 0; a < 2; ++a) {
          const double t = (static_cast<double>(e + a) / epr - 0.5) * length;
          for (int k = 0; k < 3; ++k) cand[e][a][k] = c[k] + t * d[k];
        }
      bool clash = false;
      for (int e = 0; e < epr && !clash; ++e) {
        int ci[3];
        for (int k = 0; k < 3; ++k) ci[k] = g.index(0.5 * (cand[e][0][k] + cand[e][1][k]));
        for (int dz = -1; dz <= 1 && !clash; ++dz)
          for (int dy = -1; dy <= 1 && !clash; ++dy)
            for (int dx = -1; dx <= 1 && !clash; ++dx) {
              const int ix = ci[0] + dx, iy = ci[1] + dy, iz = ci[2] + dz;
              if (ix < 0 || iy < 0 || iz < 0 || ix >= g.n || iy >= g.n || iz >= g.n) continue;
              for (int f : g.cells[(static_cast<size_t>(iz) * g.n + iy) * g.n + ix]) {
                dl::PairGeom pg;
                for (int a = 0; a < 2; ++a)
                  for (int k = 0; k < 3; ++k) {
                    pg.A[a][k] = cand[e][a][k];
                    pg.B[a][k] = seg[static_cast<size_t>(f) * 6 + a * 3 + k];
                  }
                if (dl::segment_distance(pg) < reach) {
                  clash = true;
                  break;
                }
              }
            }
      }
      if (clash) continue;
      placed = true;
      for (int e = 0; e < epr; ++e) {
        const int id = static_cast<int>(seg.size() / 6);
        for (int a = 0; a < 2; ++a)
          for (int k = 0; k < 3; ++k) seg.push_back(cand[e][a][k]);
        int ci[3];
        for (int k = 0; k < 3; ++k) ci[k] = g.index(0.5 * (cand[e][0][k] + cand[e][1][k]));
        g.cells[(static_cast<size_t>(ci[2]) * g.n + ci[1]) * g.n + ci[0]].push_back(id);
      }
    }
    // nodes of rod r: (epr + 1) per rod, numbered rod by rod
    const int64_t n0 = static_cast<int64_t>(r) * (epr + 1);
    for (int i = 0; i <= epr; ++i) {
      const double t = (static_cast<double>(i) / epr - 0.5) * length;
      for (int k = 0; k < 3; ++k) coords[(n0 + i) * 3 + k] = c[k] + t * d[k];
    }
    for (int e = 0; e < epr; ++e) {
      const int64_t id = static_cast<int64_t>(r) * epr + e;
      conn[id * 2] = static_cast<int32_t>(n0 + e);
      conn[id * 2 + 1] = static_cast<int32_t>(n0 + e + 1);
      elem_rod[id] = r;
    }
  }
  if (tries_out) *tries_out = tries;
  return DL_OK;
}
