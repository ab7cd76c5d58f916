/* Forced-include header for compiling the reference's FCM sources
 * (FCMfunctions.cpp, c_array_functions.cpp) as one process, without MPI,
 * FFTW 2.1.5 or Armadillo. It stands in for multi_filament_header.hpp (whose
 * include guard it sets, so that header and the Armadillo-based classes it
 * pulls in are skipped) and provides the same named constants, restated from
 * the reference's definitions (multi_filament_header.hpp:32-60): the grid
 * NPTS_X/Y/Z and the stencil ngd come from the build (-DREF_NPTS=..., -DREF_NGD=...);
 * dx is a / 1.86 (the benchmark configurations) or, with -DREF_DX_SIGMADIP,
 * the reference's sigma_dip / 1.5. Test infrastructure only: the oracle's
 * reference-pinning build (oracle/refshim/Makefile) uses it; nothing in the
 * product does. */
#ifndef REFSHIM_HPP
#define REFSHIM_HPP
#define HEADER_IS_INCLUDED
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>
#include <chrono>
#include "mpi.h"
#include "rfftw_mpi.h"
using namespace std;

#define PROFILING false
#define verbose false
#define PI 3.14159265358979323846264338327950288
#define NPTS_X REF_NPTS_X
#define NPTS_Y REF_NPTS_Y
#define NPTS_Z REF_NPTS_Z
#define ngd REF_NGD
#define a 1.0
#define ah 1.0
#define DL 2.2
#define MU 1.0
#ifdef REF_NSW
#define Nsw REF_NSW
#define max_Nworm REF_MAX_NWORM
#endif
/* barrier parameters, as the benchmark configurations set them (fs_params_default) */
#define Barrier_FS_over_2a (15. * PI)
#define Barrier_distance_cap 2.0
#ifndef REF_INITIAL_FRICTION_STEPS
#define REF_INITIAL_FRICTION_STEPS 0
#endif
#define initialFrictionSteps REF_INITIAL_FRICTION_STEPS
namespace arma {}

#define PI2 (2. * PI)
#define TwoPI (2. * PI)

extern int Np;
const int N = 0;  // the bead count of an older code path, read only by c_array_functions.cpp's unused box()

/* the few Armadillo vector operations FCMStokeslet uses (FCMfunctions.cpp:811-863):
 * a 3-vector filled by <<, element access, +, -, +=, scaling, norm and dot */
struct vec;
struct refshim_filler {
  vec &v;
  int i;
  refshim_filler operator<<(double x);
};
struct vec {
  double d[3] = {0, 0, 0};
  explicit vec(int = 3) {}
  double operator()(int i) const { return d[i]; }
  refshim_filler operator<<(double x) {
    d[0] = x;
    return refshim_filler{*this, 1};
  }
  vec &operator+=(const vec &o) {
    for (int k = 0; k < 3; ++k) d[k] += o.d[k];
    return *this;
  }
};
inline refshim_filler refshim_filler::operator<<(double x) {
  v.d[i] = x;
  return refshim_filler{v, i + 1};
}
inline vec operator+(const vec &p, const vec &q) {
  vec r;
  for (int k = 0; k < 3; ++k) r.d[k] = p.d[k] + q.d[k];
  return r;
}
inline vec operator-(const vec &p, const vec &q) {
  vec r;
  for (int k = 0; k < 3; ++k) r.d[k] = p.d[k] - q.d[k];
  return r;
}
inline vec operator*(double s, const vec &p) {
  vec r;
  for (int k = 0; k < 3; ++k) r.d[k] = s * p.d[k];
  return r;
}
inline vec operator/(const vec &p, double s) {
  vec r;
  for (int k = 0; k < 3; ++k) r.d[k] = p.d[k] / s;
  return r;
}
inline double dot(const vec &p, const vec &q) { return p.d[0] * q.d[0] + p.d[1] * q.d[1] + p.d[2] * q.d[2]; }
inline double norm(const vec &p) { return std::sqrt(dot(p, p)); }
const double mu = MU;
const double sigmadip = a / std::pow(36.0 * PI, 1.0 / 6.0);
#ifdef REF_DX_SIGMADIP
const double dx = sigmadip / 1.5;
#else
const double dx = a / 1.86;
#endif
const double LfcmBox_x = NPTS_X * dx;
const double LfcmBox_y = NPTS_Y * dx;
const double LfcmBox_z = NPTS_Z * dx;
const double sigmadipsq = sigmadip * sigmadip;
const double anormdip = 1.0 / std::sqrt(2.0 * PI * sigmadipsq);
const double anormdip2 = 2.0 * sigmadipsq;
const double sigma = a / std::sqrt(PI);
const double sigmasq = sigma * sigma;
const double anorm = 1.0 / std::sqrt(2.0 * PI * sigmasq);
const double anorm2 = 2.0 * sigmasq;

/* what Fcm::assign_filament_data and the LinkedList read of a filament: its
 * length (also as myNworm) and each bead's Xs, F and TAU by component */
struct refshim_vec3 {
  double v[3];
  double operator()(int i) const { return v[i]; }
};
struct refshim_bead {
  refshim_vec3 Xs, F, TAU;
};
class Filament {
 public:
  std::vector<refshim_bead> beads;
  int myNworm = 0;
  int length() const { return (int)beads.size(); }
};
/* the reference reaches struct Fcm through the headers skipped above */
#include "FCMfunctions.hpp"
#endif
