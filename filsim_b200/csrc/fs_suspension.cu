// fs_suspension.cu -- host-side seeded generator of straight-filament
// suspensions (the benchmark inputs). No device code.
//
// Each filament gets one unit quaternion normalised from four N(0,1) draws, as
// Bead::initialBeadRandom does (Bead.hpp:94-98), shared by all its beads; bead
// n sits at C + (n*DL - Nw*DL/2) t, t the quaternion's tangent, as in
// Filament::initialFilamentSetupIsoRandCentred (Filament.cpp:47-66). The centre
// C is uniform in the periodic box. A proposal is rejected while any bead lies
// closer than min_sep (minimum image) to an accepted bead of another filament
// or to a periodic image of the filament's own beads, the test of
// Filament::checkOverlapWithPeriodic (Filament.cpp:126-153) with a separation
// given by the caller. Accepted beads are kept in a cell hash of width
// >= min_sep, so each check looks at 27 cells.
//
// Random numbers: xoshiro256** seeded through splitmix64; normals by the
// Box-Muller transform. The reference's Armadillo RNG is not reproduced.
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <vector>
#include "../../include/filsim_gpu.h"

namespace {

struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) {
      x += 0x9e3779b97f4a7c15ULL;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      s[i] = z ^ (z >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0, 1)
  double normal() {
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925286766559 * u2);
  }
};

struct CellHash {
  int M[3];
  double cw[3];
  std::vector<int> head, next;
  CellHash(const double *L, double min_sep, int cap) {
    for (int d = 0; d < 3; ++d) {
      M[d] = (int)(L[d] / min_sep);
      if (M[d] < 1) M[d] = 1;
      cw[d] = L[d] / M[d];
    }
    head.assign((size_t)M[0] * M[1] * M[2], -1);
    next.assign(cap, -1);
  }
  void coords(const double *L, const double *x, int *c) const {
    for (int d = 0; d < 3; ++d) {
      double w = x[d] - L[d] * floor(x[d] / L[d]);
      int k = (int)(w / cw[d]);
      c[d] = k >= M[d] ? M[d] - 1 : (k < 0 ? 0 : k);
    }
  }
  size_t cell(int x, int y, int z) const {
    x = (x % M[0] + M[0]) % M[0];
    y = (y % M[1] + M[1]) % M[1];
    z = (z % M[2] + M[2]) % M[2];
    return ((size_t)z * M[1] + y) * M[0] + x;
  }
};

inline double min_image(double d, double L) { return d - L * floor(d / L + 0.5); }

}  // namespace

extern "C" fs_status fs_suspension_random(const fs_params *p, int nfil, int nw, unsigned long long seed,
                                          double min_sep, int max_tries, double *X_h, double *q_h) {
  if (!p || nfil < 0 || nw < 1 || !(min_sep > 0) || max_tries < 1 || (nfil > 0 && (!X_h || !q_h)))
    return FS_ERR_INVALID_ARG;
  const double L[3] = {p->npts_x * p->dx, p->npts_y * p->dx, p->npts_z * p->dx};
  const double dl = p->dl, sep2 = min_sep * min_sep;
  CellHash hash(L, min_sep, nfil * nw > 0 ? nfil * nw : 1);
  Rng rng(seed);
  std::vector<double> pos(3 * (size_t)nw);
  int placed = 0;
  for (int f = 0; f < nfil; ++f) {
    bool ok = false;
    double q[4];
    for (int tr = 0; tr < max_tries && !ok; ++tr) {
      double nrm = 0;
      for (int k = 0; k < 4; ++k) {
        q[k] = rng.normal();
        nrm += q[k] * q[k];
      }
      nrm = sqrt(nrm);
      for (int k = 0; k < 4; ++k) q[k] /= nrm;
      double C[3];
      for (int d = 0; d < 3; ++d) C[d] = rng.uniform() * L[d];
      // tangent of q (UnitQuaternion.hpp:341-351)
      const double t[3] = {1 - 2 * q[2] * q[2] - 2 * q[3] * q[3], 2 * (q[1] * q[2] + q[0] * q[3]),
                           2 * (q[1] * q[3] - q[0] * q[2])};
      for (int n = 0; n < nw; ++n)
        for (int d = 0; d < 3; ++d) pos[3 * n + d] = C[d] + (n * dl - nw * dl / 2.0) * t[d];
      ok = true;
      // own periodic images
      for (int i = 0; i < nw && ok; ++i)
        for (int j = i + 1; j < nw && ok; ++j) {
          double r2 = 0, r2d = 0;
          for (int d = 0; d < 3; ++d) {
            double dd = pos[3 * i + d] - pos[3 * j + d];
            double mi = min_image(dd, L[d]);
            r2 += mi * mi;
            r2d += dd * dd;
          }
          if (r2 < sep2 && fabs(r2 - r2d) > 1e-9) ok = false;
        }
      // accepted beads of other filaments
      for (int i = 0; i < nw && ok; ++i) {
        int c[3];
        hash.coords(L, &pos[3 * i], c);
        for (int a = -1; a <= 1 && ok; ++a)
          for (int b = -1; b <= 1 && ok; ++b)
            for (int e = -1; e <= 1 && ok; ++e)
              for (int k = hash.head[hash.cell(c[0] + a, c[1] + b, c[2] + e)]; k >= 0 && ok; k = hash.next[k]) {
                double r2 = 0;
                for (int d = 0; d < 3; ++d) {
                  double mi = min_image(pos[3 * i + d] - X_h[3 * (size_t)k + d], L[d]);
                  r2 += mi * mi;
                }
                if (r2 < sep2) ok = false;
              }
      }
    }
    if (!ok) return FS_ERR_CAPACITY;
    for (int i = 0; i < nw; ++i) {
      const int g = placed + i;
      for (int d = 0; d < 3; ++d) X_h[3 * (size_t)g + d] = pos[3 * i + d];
      for (int k = 0; k < 4; ++k) q_h[4 * (size_t)g + k] = q[k];
      int c[3];
      hash.coords(L, &pos[3 * i], c);
      size_t cc = hash.cell(c[0], c[1], c[2]);
      hash.next[g] = hash.head[cc];
      hash.head[cc] = g;
    }
    placed += nw;
  }
  return FS_OK;
}
