/*
 * or_suspension.c -- CPU restatement of the seeded suspension generator
 * (fs_suspension_random), so that the CPU baseline can build its inputs
 * without loading the GPU library. TEST INFRASTRUCTURE ONLY: bench.py's CPU
 * arms and the tests use it; a CPU test checks that it reproduces the library's
 * generator bit for bit.
 *
 * Placement as Filament::initialFilamentSetupIsoRandCentred (Filament.cpp:47-66):
 * one unit quaternion per filament normalised from four N(0,1) draws
 * (Bead.hpp:94-98), its tangent (UnitQuaternion.hpp:341-351), bead n at
 * C + (n DL - Nw DL / 2) t, centre C uniform in the box; a proposal is
 * rejected while a bead lies closer than min_sep (minimum image) to an
 * accepted bead of another filament or to a periodic image of one of its own
 * beads (Filament::checkOverlapWithPeriodic, Filament.cpp:126-153).
 * Random numbers: splitmix64 seeding of xoshiro256**, Box-Muller normals; the
 * same draw order as the library's generator.
 */
#include "fs_oracle.h"
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct {
  uint64_t s[4];
} or_rng;

static void rng_seed(or_rng *r, uint64_t seed) {
  uint64_t x = seed;
  for (int i = 0; i < 4; ++i) {
    x += 0x9e3779b97f4a7c15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    r->s[i] = z ^ (z >> 31);
  }
}

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t rng_next(or_rng *r) {
  uint64_t *s = r->s;
  const uint64_t out = rotl64(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
  return out;
}

/* 53 random bits in [0, 1) */
static double rng_uniform(or_rng *r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

static double rng_normal(or_rng *r) {
  double u1 = rng_uniform(r), u2 = rng_uniform(r);
  if (u1 < 1e-300) u1 = 1e-300;
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925286766559 * u2);
}

/* accepted beads in a cell hash of width >= min_sep (27 cells per check) */
typedef struct {
  int M[3];
  double cw[3];
  int *head, *next;
} or_hash;

static void hash_coords(const or_hash *h, const double *L, const double *x, int *c) {
  for (int d = 0; d < 3; ++d) {
    const double w = x[d] - L[d] * floor(x[d] / L[d]);
    const int k = (int)(w / h->cw[d]);
    c[d] = k >= h->M[d] ? h->M[d] - 1 : (k < 0 ? 0 : k);
  }
}

static size_t hash_cell(const or_hash *h, int x, int y, int z) {
  x = (x % h->M[0] + h->M[0]) % h->M[0];
  y = (y % h->M[1] + h->M[1]) % h->M[1];
  z = (z % h->M[2] + h->M[2]) % h->M[2];
  return ((size_t)z * h->M[1] + y) * h->M[0] + x;
}

static double min_image(double d, double L) { return d - L * floor(d / L + 0.5); }

int or_suspension_random(const fs_params *p, int nfil, int nw, unsigned long long seed, double min_sep,
                         int max_tries, double *X, double *Q) {
  if (!p || nfil < 0 || nw < 1 || !(min_sep > 0) || max_tries < 1 || (nfil > 0 && (!X || !Q))) return 1;
  const double L[3] = {p->npts_x * p->dx, p->npts_y * p->dx, p->npts_z * p->dx};
  const double dl = p->dl, sep2 = min_sep * min_sep;
  or_hash h;
  size_t ncell = 1;
  for (int d = 0; d < 3; ++d) {
    h.M[d] = (int)(L[d] / min_sep);
    if (h.M[d] < 1) h.M[d] = 1;
    h.cw[d] = L[d] / h.M[d];
    ncell *= (size_t)h.M[d];
  }
  const size_t cap = nfil * (size_t)nw > 0 ? nfil * (size_t)nw : 1;
  h.head = (int *)malloc(sizeof(int) * ncell);
  h.next = (int *)malloc(sizeof(int) * cap);
  double *pos = (double *)malloc(sizeof(double) * 3 * (size_t)nw);
  if (!h.head || !h.next || !pos) {
    free(h.head);
    free(h.next);
    free(pos);
    return 5;
  }
  for (size_t i = 0; i < ncell; ++i) h.head[i] = -1;
  for (size_t i = 0; i < cap; ++i) h.next[i] = -1;
  or_rng rng;
  rng_seed(&rng, seed);
  int placed = 0, status = 0;
  for (int f = 0; f < nfil && status == 0; ++f) {
    int ok = 0;
    double q[4];
    for (int tr = 0; tr < max_tries && !ok; ++tr) {
      double nrm = 0;
      for (int k = 0; k < 4; ++k) {
        q[k] = rng_normal(&rng);
        nrm += q[k] * q[k];
      }
      nrm = sqrt(nrm);
      for (int k = 0; k < 4; ++k) q[k] /= nrm;
      double C[3];
      for (int d = 0; d < 3; ++d) C[d] = rng_uniform(&rng) * L[d];
      const double t[3] = {1 - 2 * q[2] * q[2] - 2 * q[3] * q[3], 2 * (q[1] * q[2] + q[0] * q[3]),
                           2 * (q[1] * q[3] - q[0] * q[2])};
      for (int n = 0; n < nw; ++n)
        for (int d = 0; d < 3; ++d) pos[3 * n + d] = C[d] + (n * dl - nw * dl / 2.0) * t[d];
      ok = 1;
      for (int i = 0; i < nw && ok; ++i)
        for (int j = i + 1; j < nw && ok; ++j) {
          double r2 = 0, r2d = 0;
          for (int d = 0; d < 3; ++d) {
            const double dd = pos[3 * i + d] - pos[3 * j + d];
            const double mi = min_image(dd, L[d]);
            r2 += mi * mi;
            r2d += dd * dd;
          }
          if (r2 < sep2 && fabs(r2 - r2d) > 1e-9) ok = 0;
        }
      for (int i = 0; i < nw && ok; ++i) {
        int c[3];
        hash_coords(&h, L, &pos[3 * i], c);
        for (int a = -1; a <= 1 && ok; ++a)
          for (int b = -1; b <= 1 && ok; ++b)
            for (int e = -1; e <= 1 && ok; ++e)
              for (int k = h.head[hash_cell(&h, c[0] + a, c[1] + b, c[2] + e)]; k >= 0 && ok; k = h.next[k]) {
                double r2 = 0;
                for (int d = 0; d < 3; ++d) {
                  const double mi = min_image(pos[3 * i + d] - X[3 * (size_t)k + d], L[d]);
                  r2 += mi * mi;
                }
                if (r2 < sep2) ok = 0;
              }
      }
    }
    if (!ok) {
      status = 8;
      break;
    }
    for (int i = 0; i < nw; ++i) {
      const int g = placed + i;
      for (int d = 0; d < 3; ++d) X[3 * (size_t)g + d] = pos[3 * i + d];
      for (int k = 0; k < 4; ++k) Q[4 * (size_t)g + k] = q[k];
      int c[3];
      hash_coords(&h, L, &pos[3 * i], c);
      const size_t cc = hash_cell(&h, c[0], c[1], c[2]);
      h.next[g] = h.head[cc];
      h.head[cc] = g;
    }
    placed += nw;
  }
  free(h.head);
  free(h.next);
  free(pos);
  return status;
}
