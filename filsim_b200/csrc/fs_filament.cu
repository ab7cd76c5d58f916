// fs_filament.cu -- filament mechanics, approximate Jacobian and Broyden
// update of the implicit BDF2 step, FP64 on sm_100a.
//
//   k_initial_guess      Filament::initialGuess (Filament.hpp:227-237, Bead.hpp:202-217); with
//                        start order 2 the first bead extrapolated to second order (fs_start.cu)
//   k_unrobot_assign     Filament::unRobotArmify (Filament.hpp:489-505) +
//                        Fcm::assign_filament_data's Y = fmod(Xs, L) (FCMfunctions.cpp:882-918)
//   k_forces             setZeroForcesTorques, applyElasticTorques, applyConstraintForcesTorques,
//                        applyExternalForcesTorques (Filament.hpp:271-402), one thread per bead
//                        adding its links' terms in the reference's order
//   k_jacobian_schur     buildApproximateJacobian with BlockC/D/E/F (Filament.hpp:803-1120) reduced
//                        to the 3Nw x 3Nw Schur complement of its constraint block (one CTA per
//                        filament); k_schur_gj inverts it in shared memory
//   k_error_check        ErrorCheckFCM + dexpinv (MobilityConstraints.cpp:109-143, 447-770)
//   k_schur_apply        filamentJsolver::solve (FilamentJacobianSolver.hpp:49-73): J0^-1 b from
//                        the Schur inverse, then the bad-Broyden history corrections
//   k_broyden_cols       history update of main.cpp:640-663
//   k_update / k_step    Filament::update (Filament.hpp:425-452), Filament::step (:455-478); with
//                        tension order 1 the tensions extrapolated linearly after lambda_extrap_step
#include <algorithm>
#include "fs_internal.cuh"

namespace {

struct Q {
  double s, v[3];
};

__device__ __forceinline__ Q qload(const double *a) {
  Q q;
  q.s = a[0];
  q.v[0] = a[1];
  q.v[1] = a[2];
  q.v[2] = a[3];
  return q;
}
__device__ __forceinline__ void qstore(const Q &q, double *a) {
  a[0] = q.s;
  a[1] = q.v[0];
  a[2] = q.v[1];
  a[3] = q.v[2];
}
__device__ __forceinline__ double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ void cross3(const double *a, const double *b, double *c) {
  double c0 = a[1] * b[2] - a[2] * b[1], c1 = a[2] * b[0] - a[0] * b[2], c2 = a[0] * b[1] - a[1] * b[0];
  c[0] = c0;
  c[1] = c1;
  c[2] = c2;
}
__device__ __forceinline__ double norm3(const double *a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

// expmInPlace (UnitQuaternion.hpp:227-242): q <- (cos(t/2), sin(t/2)/t v) * q
__device__ Q q_expm(Q q, const double *v) {
  double theta = norm3(v);
  if (theta > 1.e-12) {
    double tmp = sin(theta * .5) / theta;
    Q p;
    p.s = cos(theta * .5);
    p.v[0] = tmp * v[0];
    p.v[1] = tmp * v[1];
    p.v[2] = tmp * v[2];
    double scal_tmp = q.s * p.s - dot3(q.v, p.v);
    double t[3];
    cross3(p.v, q.v, t);
    Q r;
    for (int d = 0; d < 3; ++d) r.v[d] = q.s * p.v[d] + p.s * q.v[d] + t[d];
    r.s = scal_tmp;
    return r;
  }
  return q;
}

// tangent / normal / binormal (UnitQuaternion.hpp:341-378)
__device__ __forceinline__ void q_tangent(const Q &q, double *v) {
  double q22 = 2 * q.v[1] * q.v[1], q33 = 2 * q.v[2] * q.v[2];
  v[0] = (1 - q22 - q33);
  v[1] = 2 * (q.v[0] * q.v[1] + q.s * q.v[2]);
  v[2] = 2 * (q.v[0] * q.v[2] - q.s * q.v[1]);
}
__device__ __forceinline__ void q_normal(const Q &q, double *v) {
  double q11 = 2 * q.v[0] * q.v[0], q33 = 2 * q.v[2] * q.v[2];
  v[0] = 2 * (q.v[0] * q.v[1] - q.s * q.v[2]);
  v[1] = (1 - q11 - q33);
  v[2] = 2 * (q.v[1] * q.v[2] + q.s * q.v[0]);
}
__device__ __forceinline__ void q_binormal(const Q &q, double *v) {
  double q11 = 2 * q.v[0] * q.v[0], q22 = 2 * q.v[1] * q.v[1];
  v[0] = 2 * (q.v[0] * q.v[2] + q.s * q.v[1]);
  v[1] = 2 * (q.v[1] * q.v[2] - q.s * q.v[0]);
  v[2] = (1 - q11 - q22);
}
// RotateVector (UnitQuaternion.hpp:323-338)
__device__ void q_rotate(const Q &q, double *v) {
  double vx = v[0], vy = v[1], vz = v[2];
  const double *e = q.v;
  double s = q.s;
  double q11 = 2 * e[0] * e[0], q22 = 2 * e[1] * e[1], q33 = 2 * e[2] * e[2];
  v[0] = (1 - q22 - q33) * vx + 2 * (e[0] * e[1] - s * e[2]) * vy + 2 * (e[0] * e[2] + s * e[1]) * vz;
  v[1] = 2 * (e[0] * e[1] + s * e[2]) * vx + (1 - q11 - q33) * vy + 2 * (e[1] * e[2] - s * e[0]) * vz;
  v[2] = 2 * (e[0] * e[2] - s * e[1]) * vx + 2 * (e[1] * e[2] + s * e[0]) * vy + (1 - q11 - q22) * vz;
}
// assignMidPointOf (UnitQuaternion.hpp:472-489) with quaSquareRootTimInPlace (:411-421)
__device__ Q q_midpoint(const Q &p1, const Q &p2) {
  Q m;
  m.s = p2.s * p1.s + dot3(p2.v, p1.v);
  double cr[3];
  cross3(p2.v, p1.v, cr);
  for (int d = 0; d < 3; ++d) m.v[d] = -p2.s * p1.v[d] + p1.s * p2.v[d] - cr[d];
  if (m.s < -.9999999999999) {
    m.s = 0.;
    m.v[0] = 0.;
    m.v[1] = 0.;
    m.v[2] = 1.;
  } else {
    m.s = sqrt(0.5 * (m.s + 1.));
    for (int d = 0; d < 3; ++d) m.v[d] /= (2. * m.s);
  }
  double scal_tmp = m.s * p1.s - dot3(m.v, p1.v);
  double t[3];
  cross3(m.v, p1.v, t);
  Q o;
  for (int d = 0; d < 3; ++d) o.v[d] = m.s * p1.v[d] + p1.s * m.v[d] + t[d];
  o.s = scal_tmp;
  return o;
}

// dexpinv (MobilityConstraints.cpp:109-143)
__device__ void dexpinv(const double *u, const double *w, double *out) {
  double tmp = norm3(u);
  double cuw[3];
  cross3(u, w, cuw);
  if (tmp >= 1.e-12) {
    double tmp2 = tmp / sin(.5 * tmp);
    tmp2 *= cos(.5 * tmp);
    tmp = .5 * tmp2 - 1.;
    double nu = norm3(u);
    double un[3] = {u[0] / nu, u[1] / nu, u[2] / nu};
    double c1[3], c2[3];
    cross3(un, w, c1);
    cross3(un, c1, c2);
    for (int d = 0; d < 3; ++d) {
      out[d] = w[d] - .5 * cuw[d];
      out[d] -= tmp * c2[d];
    }
  } else {
    tmp = 1. / 12;
    double c2[3];
    cross3(u, cuw, c2);
    for (int d = 0; d < 3; ++d) {
      out[d] = w[d] - .5 * cuw[d];
      out[d] += tmp * c2[d];
    }
  }
}

struct FilConsts {
  double L[3];
  double dt, dl, mu, tol;
  double gravity[3], st[3];
  int impl_euler_steps, lambda_extrap_step;
  // swimming drive: time of the forces (nt dt), per-filament parameters or null
  double tt, swim_curvature;
  int swim_sperm_decay;
  const double *swim;
};

// Strain twist of link i of filament f (nw beads) at time k.tt
// (applyElasticTorques, Filament.hpp:297-326): component 0 is the constant
// STRAINTWISTZ; components 1 and 2 are set on every link by the swimming drive,
// Beta facPref cos(k s - w t + phase) and Alpha facPref sin(...), so they are
// zero for a filament without a drive.
__device__ void link_strain_twist(const FilConsts &k, int f, int nw, int i, double *st) {
  st[0] = k.st[0];
  st[1] = 0.0;
  st[2] = 0.0;
  if (!k.swim) return;
  const double *sw = k.swim + 5 * f;
  const double dL = k.dl, L_filament = (nw - 1) * dL, L_filament_long = nw * dL;
  const double T0 = (k.swim_curvature / L_filament_long);
  const double sarc = dL * i + .5 * dL;
  double facPref;
  if (k.swim_sperm_decay) {
    if (sarc > L_filament / 2.0)
      facPref = T0 * 2.0 * (L_filament - sarc) / L_filament;
    else
      facPref = T0;
  } else {
    facPref = T0 * (L_filament - sarc) / L_filament;
  }
  const double arg = sw[3] * sarc - sw[4] * k.tt + sw[2];
  st[1] = sw[1] * facPref * cos(arg);
  st[2] = sw[0] * facPref * sin(arg);
}

// ---- per-bead / per-filament kernels -----------------------------------------
// order 2 with a history of two steps (*hist_ok == 2): the first bead from
// 3X - 3Xt + Xtt, rounded as written (fs_start.cu); otherwise the reference's 2X - Xt
__global__ void k_initial_guess(int np, const int *__restrict__ seg_id, const double *__restrict__ X,
                                const double *__restrict__ Xt, const double *__restrict__ U,
                                const double *__restrict__ Ut, const double *__restrict__ q, double *__restrict__ Xs,
                                double *__restrict__ Us, double *__restrict__ qs, int order,
                                const double *__restrict__ Xtt, const int *__restrict__ hist_ok) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= np) return;
  if (seg_id[b] == 0) {
    if (order == 2 && *hist_ok >= 2)
      for (int d = 0; d < 3; ++d)
        Xs[3 * b + d] =
            __dadd_rn(__dsub_rn(__dmul_rn(3., X[3 * b + d]), __dmul_rn(3., Xt[3 * b + d])), Xtt[3 * b + d]);
    else
      for (int d = 0; d < 3; ++d) Xs[3 * b + d] = 2. * X[3 * b + d] - Xt[3 * b + d];
  }
  double us[3];
  for (int d = 0; d < 3; ++d) us[d] = 2. * U[3 * b + d] - Ut[3 * b + d];
  for (int d = 0; d < 3; ++d) Us[3 * b + d] = us[d];
  qstore(q_expm(qload(q + 4 * b), us), qs + 4 * b);
}

// One warp per filament, beads in chunks of 32: the lanes form their beads'
// tangents in parallel, then every lane runs the running sum of
// Filament::unRobotArmify (Filament.hpp:489-505) over the chunk in bead order
// (tangents broadcast by shuffles; the same additions in the same order as one
// thread walking the filament) and keeps its own bead's position; the
// fmod(X, L) of assign_filament_data runs per lane.
__global__ void k_unrobot_assign(int nfil, const int *__restrict__ fil_start, const double *__restrict__ qs,
                                 double *__restrict__ Xs, double *__restrict__ Y, FilConsts k) {
  const int f = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (f >= nfil) return;  // warp-uniform
  const int b0 = fil_start[f], b1 = fil_start[f + 1];
  const double half = 0.5 * k.dl;
  double Xsum[3] = {Xs[3 * b0], Xs[3 * b0 + 1], Xs[3 * b0 + 2]};
  double t1[3] = {0.0, 0.0, 0.0};
  for (int c0 = b0; c0 < b1; c0 += 32) {
    const int b = c0 + lane, nb = min(32, b1 - c0);
    double t[3] = {0.0, 0.0, 0.0}, mine[3] = {0.0, 0.0, 0.0};
    if (b < b1) q_tangent(qload(qs + 4 * b), t);
    for (int i = 0; i < nb; ++i) {  // warp-uniform trip count
      double t2[3];
      for (int d = 0; d < 3; ++d) t2[d] = __shfl_sync(0xffffffffu, t[d], i);
      if (c0 + i > b0)
        for (int d = 0; d < 3; ++d) Xsum[d] += (t1[d] + t2[d]) * half;
      for (int d = 0; d < 3; ++d) t1[d] = t2[d];
      if (lane == i)
        for (int d = 0; d < 3; ++d) mine[d] = Xsum[d];
    }
    if (b < b1) {
      for (int d = 0; d < 3; ++d) {
        if (b > b0) Xs[3 * b + d] = mine[d];
        Y[3 * b + d] = fmod(mine[d], k.L[d]);
      }
    }
  }
}

// elastic torque of link (i, i+1) (Filament.hpp:297-340), before the +/- to the beads
__device__ void elastic_link(const double *qi_, const double *qj_, double oneOverDL, double kap, double cmod,
                             const double *st, double *vtmp) {
  Q qi = qload(qi_), qj = qload(qj_);
  Q qm = q_midpoint(qi, qj);
  Q q2 = qj;
  q2.s -= qi.s;
  for (int d = 0; d < 3; ++d) q2.v[d] -= qi.v[d];
  q2.s *= oneOverDL;
  for (int d = 0; d < 3; ++d) q2.v[d] *= oneOverDL;
  double tt[3];
  cross3(q2.v, qm.v, tt);
  double nv[3];
  for (int d = 0; d < 3; ++d) nv[d] = -q2.s * qm.v[d] + qm.s * q2.v[d] + tt[d];
  for (int d = 0; d < 3; ++d) vtmp[d] = 2. * nv[d] - st[d];
  vtmp[0] *= cmod;
  vtmp[1] *= kap;
  vtmp[2] *= kap;
  q_rotate(qm, vtmp);
}

__global__ void k_forces(int np, const int *__restrict__ fil_id, const int *__restrict__ seg_id,
                         const int *__restrict__ fil_start, const double *__restrict__ qs,
                         const double *__restrict__ lam, const double *__restrict__ kap,
                         const double *__restrict__ cmod, double *__restrict__ F, double *__restrict__ TAU,
                         FilConsts k) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= np) return;
  const int f = fil_id[b], i = seg_id[b];
  const int nw = fil_start[f + 1] - fil_start[f];
  const int l0 = fil_start[f] - f;
  const double oneOverDL = 1. / k.dl;
  double tau[3] = {0.0, 0.0, 0.0}, fo[3] = {0.0, 0.0, 0.0}, v[3], st[3];
  // elastic: link i-1 subtracts, link i adds (link order of Filament.hpp:297)
  if (i >= 1) {
    link_strain_twist(k, f, nw, i - 1, st);
    elastic_link(qs + 4 * (b - 1), qs + 4 * b, oneOverDL, kap[f], cmod[f], st, v);
    for (int d = 0; d < 3; ++d) tau[d] -= v[d];
  }
  if (i < nw - 1) {
    link_strain_twist(k, f, nw, i, st);
    elastic_link(qs + 4 * b, qs + 4 * (b + 1), oneOverDL, kap[f], cmod[f], st, v);
    for (int d = 0; d < 3; ++d) tau[d] += v[d];
  }
  // constraint forces and torques (Filament.hpp:351-368)
  const double fac = -.5 * k.dl;
  double t[3], c2[3];
  q_tangent(qload(qs + 4 * b), t);
  if (i >= 1) {
    const double *lm = lam + 3 * (l0 + i - 1);
    for (int d = 0; d < 3; ++d) fo[d] += lm[d];
    cross3(t, lm, c2);
    for (int d = 0; d < 3; ++d) tau[d] += fac * c2[d];
  }
  if (i < nw - 1) {
    const double *lm = lam + 3 * (l0 + i);
    for (int d = 0; d < 3; ++d) fo[d] -= lm[d];
    cross3(t, lm, c2);
    for (int d = 0; d < 3; ++d) tau[d] += fac * c2[d];
  }
  for (int d = 0; d < 3; ++d) {
    F[3 * b + d] = fo[d] + k.gravity[d];
    TAU[3 * b + d] = tau[d];
  }
}

// Spring links (spring_links::apply_spring_link_forces, spring_link_functions.cpp:24-45),
// after the filaments' own forces (main.cpp:354-357): per link, the minimum-image
// displacement of its beads (VecPeriodicX, :139-145) and a Hookean force along it,
// + on the first bead and - on the second. One thread per bead adds its links in
// link order, the order of the reference's sequential loop.
__global__ void k_spring_forces(int np, const int *__restrict__ off, const int *__restrict__ ent,
                                const int *__restrict__ beads, const double *__restrict__ Xs, double ks, double l0,
                                FilConsts k, double *__restrict__ F) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= np) return;
  double f[3] = {F[3 * b], F[3 * b + 1], F[3 * b + 2]};
  for (int e = off[b]; e < off[b + 1]; ++e) {
    const int l = ent[e] >> 1, second = ent[e] & 1;
    const int bn = beads[2 * l], bm = beads[2 * l + 1];
    double disp[3];
    for (int d = 0; d < 3; ++d) {
      disp[d] = Xs[3 * bn + d] - Xs[3 * bm + d];
      disp[d] = disp[d] - k.L[d] * floor(disp[d] / k.L[d] + 0.5);
    }
    const double dist = sqrt(disp[0] * disp[0] + disp[1] * disp[1] + disp[2] * disp[2]);
    const double mag = ks * (dist - l0);
    for (int d = 0; d < 3; ++d) {
      const double sf = -mag * disp[d] / dist;
      if (second)
        f[d] -= sf;
      else
        f[d] += sf;
    }
  }
  for (int d = 0; d < 3; ++d) F[3 * b + d] = f[d];
}

// ---- Jacobian ------------------------------------------------------------------
struct M3 {
  double m[9];
};
__device__ __forceinline__ M3 rcross(const double *x) {
  M3 r;
  r.m[0] = 0.;
  r.m[1] = x[2];
  r.m[2] = -x[1];
  r.m[3] = -x[2];
  r.m[4] = 0.;
  r.m[5] = x[0];
  r.m[6] = x[1];
  r.m[7] = -x[0];
  r.m[8] = 0.;
  return r;
}
__device__ __forceinline__ M3 mt(const M3 &a) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[3 * i + j] = a.m[3 * j + i];
  return r;
}
__device__ M3 mmul(const M3 &a, const M3 &b) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0.0;
      for (int kk = 0; kk < 3; ++kk) acc += a.m[3 * i + kk] * b.m[3 * kk + j];
      r.m[3 * i + j] = acc;
    }
  return r;
}
__device__ __forceinline__ M3 madd(M3 a, const M3 &b) {
  for (int i = 0; i < 9; ++i) a.m[i] += b.m[i];
  return a;
}
__device__ __forceinline__ M3 msub(M3 a, const M3 &b) {
  for (int i = 0; i < 9; ++i) a.m[i] -= b.m[i];
  return a;
}
__device__ __forceinline__ M3 msc(M3 a, double s) {
  for (int i = 0; i < 9; ++i) a.m[i] *= s;
  return a;
}
__device__ __forceinline__ M3 outer(const double *a, const double *b) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[3 * i + j] = a[i] * b[j];
  return r;
}
__device__ M3 blockE_diag(const M3 &dOmega, const M3 &LieMat, const M3 &OmegaMat, const double *Us, double dt) {
  double ov[3];
  for (int i = 0; i < 3; ++i) ov[i] = OmegaMat.m[3 * i] * Us[0] + OmegaMat.m[3 * i + 1] * Us[1] + OmegaMat.m[3 * i + 2] * Us[2];
  M3 inner = msub(dOmega, msc(madd(OmegaMat, mmul(LieMat, dOmega)), 0.5));
  M3 corr = madd(madd(rcross(ov), mmul(LieMat, OmegaMat)), mmul(mmul(LieMat, LieMat), dOmega));
  inner = madd(inner, msc(corr, 1. / 12.));
  return msc(inner, -2 * dt / 3.);
}
__device__ M3 blockE_off(const M3 &dOmega, const M3 &LieMat, double dt) {
  M3 inner = msub(dOmega, msc(mmul(LieMat, dOmega), 0.5));
  inner = madd(inner, msc(mmul(mmul(LieMat, LieMat), dOmega), 1. / 12.));
  return msc(inner, -2 * dt / 3.);
}
__device__ __forceinline__ void frame(const double *qa, double *t, double *n, double *b) {
  Q q = qload(qa);
  q_tangent(q, t);
  q_normal(q, n);
  q_binormal(q, b);
}
// row-major store of a 3x3 block at (r0, c0) of an n-column matrix
__device__ __forceinline__ void put3(double *J, int n, int r0, int c0, const M3 &a) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) J[(size_t)(r0 + i) * n + c0 + j] = a.m[3 * i + j];
}

// the three BlockE blocks of bead row k (Filament.hpp:958-1089), stored into
// the 3nw x 3nw matrix J (row-major, leading dimension n = 3nw)
__device__ void blockE_row(int k, int nw, const double *qs, const double *Us, const double *TAU, const double *lam,
                           double rad_k, double myC, double myKAP, const double *ST, double DL, double dt, double MU,
                           double *J, int n) {
  const double PI = FS_PI;
  const int rE = 0, cE = 0;
  double t[3], nn[3], b[3], tp1[3], np1[3], bp1[3], tm1[3], nm1[3], bm1[3];
  const double Tfac = 1 / (8 * PI * MU * pow(rad_k, 3));
  const M3 LieMat = mt(rcross(Us + 3 * k));
  const double tT[3] = {Tfac * TAU[3 * k], Tfac * TAU[3 * k + 1], Tfac * TAU[3 * k + 2]};
  const M3 OmegaMat = rcross(tT);
  frame(qs + 4 * k, t, nn, b);
  if (k == 0) {
    frame(qs + 4, tp1, np1, bp1);
    M3 ConstraintPart = mmul(msc(rcross(lam), -0.5 * DL), rcross(t));
    double beta = -ST[2] + 0.5 * (np1[0] * b[0] + np1[1] * b[1] + np1[2] * b[2] - nn[0] * bp1[0] - nn[1] * bp1[1] - nn[2] * bp1[2]) / DL;
    double CP[3] = {b[1] * np1[2] - b[2] * np1[1] - nn[1] * bp1[2] + nn[2] * bp1[1],
                    b[2] * np1[0] - b[0] * np1[2] - nn[2] * bp1[0] + nn[0] * bp1[2],
                    b[0] * np1[1] - b[1] * np1[0] - nn[0] * bp1[1] + nn[1] * bp1[0]};
    double ttp[3] = {t[0] + tp1[0], t[1] + tp1[1], t[2] + tp1[2]};
    M3 EP = msc(madd(msc(outer(ttp, CP), 0.5 / DL), msc(rcross(t), beta)), 0.5 * myC);
    EP = madd(EP, msc(msub(msc(mmul(rcross(tp1), rcross(t)), 1. / DL),
                           msc(madd(msc(rcross(nn), ST[0]), msc(rcross(b), ST[1])), 0.5)),
                      0.5 * myKAP));
    M3 dOmega = msc(madd(EP, ConstraintPart), Tfac);
    put3(J, n, rE, cE, blockE_diag(dOmega, LieMat, OmegaMat, Us, dt));
    EP = msc(msub(msc(rcross(tp1), beta), msc(outer(ttp, CP), 0.5 / DL)), 0.5 * myC);
    EP = madd(EP, msc(msub(msc(mmul(mt(rcross(t)), rcross(tp1)), 1. / DL),
                           msc(madd(msc(rcross(np1), ST[0]), msc(rcross(bp1), ST[1])), 0.5)),
                      0.5 * myKAP));
    dOmega = msc(EP, Tfac);
    put3(J, n, rE, cE + 3, blockE_off(dOmega, LieMat, dt));
    return;
  }
  if (k == nw - 1) {
    frame(qs + 4 * (k - 1), tm1, nm1, bm1);
    M3 ConstraintPart = mmul(msc(rcross(lam + 3 * (k - 1)), -0.5 * DL), rcross(t));
    double beta = -ST[2] + 0.5 * (nn[0] * bm1[0] + nn[1] * bm1[1] + nn[2] * bm1[2] - nm1[0] * b[0] - nm1[1] * b[1] - nm1[2] * b[2]) / DL;
    double CPm[3] = {bm1[1] * nn[2] - bm1[2] * nn[1] - nm1[1] * b[2] + nm1[2] * b[1],
                     bm1[2] * nn[0] - bm1[0] * nn[2] - nm1[2] * b[0] + nm1[0] * b[2],
                     bm1[0] * nn[1] - bm1[1] * nn[0] - nm1[0] * b[1] + nm1[1] * b[0]};
    double ttm[3] = {t[0] + tm1[0], t[1] + tm1[1], t[2] + tm1[2]};
    M3 EP = msc(msub(msc(rcross(t), beta), msc(outer(ttm, CPm), 0.5 / DL)), -0.5 * myC);
    EP = msub(EP, msc(msub(msc(mmul(mt(rcross(tm1)), rcross(t)), 1. / DL),
                           msc(madd(msc(rcross(nn), ST[0]), msc(rcross(b), ST[1])), 0.5)),
                      0.5 * myKAP));
    M3 dOmega = msc(madd(EP, ConstraintPart), Tfac);
    put3(J, n, rE + 3 * k, cE + 3 * k, blockE_diag(dOmega, LieMat, OmegaMat, Us + 3 * k, dt));
    EP = msc(msub(msc(rcross(tm1), beta), msc(outer(ttm, CPm), 0.5 / DL)), -0.5 * myC);
    EP = msub(EP, msc(msub(msc(mmul(rcross(t), rcross(tm1)), 1. / DL),
                           msc(madd(msc(rcross(nm1), ST[0]), msc(rcross(bm1), ST[1])), 0.5)),
                      0.5 * myKAP));
    dOmega = msc(EP, Tfac);
    put3(J, n, rE + 3 * k, cE + 3 * k - 3, blockE_off(dOmega, LieMat, dt));
    return;
  }
  frame(qs + 4 * (k - 1), tm1, nm1, bm1);
  frame(qs + 4 * (k + 1), tp1, np1, bp1);
  double lamvec[3] = {lam[3 * (k - 1)] + lam[3 * k], lam[3 * (k - 1) + 1] + lam[3 * k + 1], lam[3 * (k - 1) + 2] + lam[3 * k + 2]};
  M3 ConstraintPart = mmul(msc(rcross(lamvec), -0.5 * DL), rcross(t));
  double beta = -ST[2] + 0.5 * (np1[0] * b[0] + np1[1] * b[1] + np1[2] * b[2] - nn[0] * bp1[0] - nn[1] * bp1[1] - nn[2] * bp1[2]) / DL;
  double CPk[3] = {b[1] * np1[2] - b[2] * np1[1] - nn[1] * bp1[2] + nn[2] * bp1[1],
                   b[2] * np1[0] - b[0] * np1[2] - nn[2] * bp1[0] + nn[0] * bp1[2],
                   b[0] * np1[1] - b[1] * np1[0] - nn[0] * bp1[1] + nn[1] * bp1[0]};
  double tp[3] = {t[0] + tp1[0], t[1] + tp1[1], t[2] + tp1[2]};
  double tm[3] = {t[0] + tm1[0], t[1] + tm1[1], t[2] + tm1[2]};
  M3 EP = msc(madd(msc(outer(tp, CPk), 0.5 / DL), msc(rcross(t), beta)), 0.5 * myC);
  EP = madd(EP, msc(msub(msc(mmul(rcross(tp1), rcross(t)), 1. / DL),
                         msc(madd(msc(rcross(nn), ST[0]), msc(rcross(b), ST[1])), 0.5)),
                    0.5 * myKAP));
  // the k-1 side beta, with the k+1 side CrossPart kept (Filament.hpp:1068-1070)
  beta = -ST[2] + 0.5 * (nn[0] * bm1[0] + nn[1] * bm1[1] + nn[2] * bm1[2] - nm1[0] * b[0] - nm1[1] * b[1] - nm1[2] * b[2]) / DL;
  EP = msub(EP, msc(msub(msc(rcross(t), beta), msc(outer(tm, CPk), 0.5 / DL)), 0.5 * myC));
  EP = msub(EP, msc(msub(msc(mmul(mt(rcross(tm1)), rcross(t)), 1. / DL),
                         msc(madd(msc(rcross(nn), ST[0]), msc(rcross(b), ST[1])), 0.5)),
                    0.5 * myKAP));
  M3 dOmega = msc(madd(ConstraintPart, EP), Tfac);
  put3(J, n, rE + 3 * k, cE + 3 * k, blockE_diag(dOmega, LieMat, OmegaMat, Us + 3 * k, dt));
  EP = msc(msub(msc(rcross(tm1), beta), msc(outer(tm, CPk), 0.5 / DL)), -0.5 * myC);
  EP = msub(EP, msc(msub(msc(mmul(rcross(t), rcross(tm1)), 1. / DL),
                         msc(madd(msc(rcross(nm1), ST[0]), msc(rcross(bm1), ST[1])), 0.5)),
                    0.5 * myKAP));
  dOmega = msc(EP, Tfac);
  put3(J, n, rE + 3 * k, cE + 3 * k - 3, blockE_off(dOmega, LieMat, dt));
  // right block with the k-1 side beta (Filament.hpp:1083)
  EP = msc(msub(msc(rcross(tp1), beta), msc(outer(tp, CPk), 0.5 / DL)), 0.5 * myC);
  EP = madd(EP, msc(msub(msc(mmul(mt(rcross(t)), rcross(tp1)), 1. / DL),
                         msc(madd(msc(rcross(np1), ST[0]), msc(rcross(bp1), ST[1])), 0.5)),
                    0.5 * myKAP));
  dOmega = msc(EP, Tfac);
  put3(J, n, rE + 3 * k, cE + 3 * k + 3, blockE_off(dOmega, LieMat, dt));
}

// ---- approximate Jacobian by the Schur complement of the constraint block --------
//
// With columns [X0 (3) | U (3nw) | lambda (3nw-3)] and rows [first-bead
// position (3) | constraints (3nw-3) | Lie updates (3nw)], the reference's J
// (Filament.hpp:803-867) is
//     J = [ I  0  P  ]    P  = (temp/dt) [I 0 ... 0]
//         [ 0  C  D' ]    C  = BlockC(DL/2), D' = 10 BlockD/dt (block bidiagonal, scalar blocks)
//         [ 0  E  F' ]    E  = BlockE,       F' = BlockF/dt (block bidiagonal)
// Eliminating lambda = D'^-1 (b1 - C u) leaves S u = b2 - F' D'^-1 b1 with
// S = E - F' D'^-1 C (3nw x 3nw). k_jacobian_schur builds S in shared memory and
// stores it; k_schur_gj inverts it (Gauss-Jordan, partial pivoting) in a lean
// kernel with more CTAs per SM; k_schur_apply then applies J^-1 exactly, with the
// reference's 1/dt scaling of the lambda rows (:864).
//
// Per-filament auxiliary data (aux, nw >= 2): d[nw-1], e[nw-1] (D' blocks),
// Fd[nw-1][9] = F'(k,k), Fl[nw-1][9] = F'(k+1,k), t[nw][3] tangents, pcoef.
#define FS_MAX_NW 48

// column cc of rcross(t) (Av = cross(v, t))
__device__ __forceinline__ void rcross_col(const double *t, int cc, double *col) {
  if (cc == 0) { col[0] = 0.; col[1] = -t[2]; col[2] = t[1]; }
  else if (cc == 1) { col[0] = t[2]; col[1] = 0.; col[2] = -t[0]; }
  else { col[0] = -t[1]; col[1] = t[0]; col[2] = 0.; }
}

__global__ void __launch_bounds__(256) k_jacobian_schur(
    const int *__restrict__ fil_start, const double *__restrict__ qs, const double *__restrict__ Us,
    const double *__restrict__ TAU, const double *__restrict__ lam, const double *__restrict__ kap,
    const double *__restrict__ cmod, const long long *__restrict__ soff, const long long *__restrict__ aoff,
    double *__restrict__ Sinv_all, double *__restrict__ aux_all, int nt, FilConsts k, double a, double ah,
    int *__restrict__ flags, const int *__restrict__ keep) {
  extern __shared__ double S[];  // 3nw x 3nw, row-major
  if (keep && *keep) return;  // the previous step's J0 stays (fs_set_broyden_memory)
  const int f = blockIdx.x;
  const int b0 = fil_start[f], nw = fil_start[f + 1] - b0, l0 = b0 - f;
  if (nw < 2) return;  // J0 is the identity
  const int m = 3 * nw, nl = nw - 1;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const double PI = FS_PI, dt = k.dt, DL = k.dl, MU = k.mu;
  const double *q_f = qs + 4 * b0, *Us_f = Us + 3 * b0, *TAU_f = TAU + 3 * b0, *lam_f = lam + 3 * l0;
  double *aux = aux_all + aoff[f];
  double *dd = aux, *ee = aux + nl, *Fd = aux + 2 * nl, *Fl = Fd + 9 * nl, *tt = Fl + 9 * nl, *pcoef = tt + 3 * nw;
#define RAD(kk) ((kk) == 0 ? ah : a)
  for (int e = tid; e < m * m; e += nthr) S[e] = 0.0;
  for (int kk = tid; kk < nw; kk += nthr) {
    double tv[3];
    q_tangent(qload(q_f + 4 * kk), tv);
    for (int d = 0; d < 3; ++d) tt[3 * kk + d] = tv[d];
  }
  const double Jprefac = 10.;
  for (int r = tid; r < nl; r += nthr) {
    // Jprefac * BlockD(nt) / dt (Filament.hpp:912-949)
    double facn = -2. * dt / (18. * PI * MU * RAD(r));
    if (nt <= k.impl_euler_steps) facn *= (3. / 2.);
    dd[r] = Jprefac * facn / dt;
    double facu = 0.0;
    if (r < nw - 2) {
      facu = 2. * dt / (18. * PI * MU * RAD(r + 1));
      if (nt <= k.impl_euler_steps) facu *= (3. / 2.);
      facu = Jprefac * facu / dt;
    }
    ee[r] = facu;
    // BlockF / dt (Filament.hpp:1099-1120)
    double tv[3];
    double fac2 = dt * DL / (24 * PI * MU * pow(RAD(r), 3.));
    q_tangent(qload(q_f + 4 * r), tv);
    M3 tmat = mt(rcross(tv));
    M3 umat = rcross(Us_f + 3 * r);
    M3 blk = msc(madd(msub(tmat, msc(mmul(umat, tmat), 0.5)), msc(mmul(mmul(umat, umat), tmat), 1. / 12.)), fac2 / dt);
    for (int e = 0; e < 9; ++e) Fd[9 * r + e] = blk.m[e];
    fac2 = dt * DL / (24. * PI * MU * pow(RAD(r + 1), 3));
    q_tangent(qload(q_f + 4 * (r + 1)), tv);
    tmat = mt(rcross(tv));
    umat = rcross(Us_f + 3 * (r + 1));
    blk = msc(madd(msub(tmat, msc(mmul(umat, tmat), 0.5)), msc(mmul(mmul(umat, umat), tmat), 1. / 12.)), fac2 / dt);
    for (int e = 0; e < 9; ++e) Fl[9 * r + e] = blk.m[e];
  }
  if (tid == 0) *pcoef = (dt / (9 * PI * MU * RAD(0))) / dt;
  __syncthreads();
  // this->myStrainTwist as applyElasticTorques(nt) left it: its last link (nw >= 2 here)
  double stj[3];
  link_strain_twist(k, f, nw, nw - 2, stj);
  for (int kk = tid; kk < nw; kk += nthr)
    blockE_row(kk, nw, q_f, Us_f, TAU_f, lam_f, RAD(kk), cmod[f], kap[f], stj, DL, dt, MU, S, m);
#undef RAD
  __syncthreads();
  for (int e = tid; e < m; e += nthr) S[e * m + e] += 1.;  // BlockE's identity (Filament.hpp:1092-1094)
  __syncthreads();
  // S -= F' D'^-1 C, one column of C per thread
  const double fac = 0.5 * DL;
  for (int j = tid; j < m; j += nthr) {
    const int mb = j / 3, cc = j % 3;
    double col[3];
    rcross_col(tt + 3 * mb, cc, col);
    double y[3 * (FS_MAX_NW - 1)];
    for (int r = nl - 1; r >= 0; --r) {  // y = D'^-1 C[:, j] (upper bidiagonal back substitution)
      double cf = 0.0;
      if (mb == 0 || mb == r + 1) cf = 1.0;
      else if (mb >= 1 && mb <= r) cf = 2.0;
      for (int d = 0; d < 3; ++d) {
        double cv = (cf == 0.0) ? 0.0 : (cf == 1.0 ? fac * col[d] : fac * col[d] + fac * col[d]);
        double nxt = (r + 1 < nl) ? ee[r] * y[3 * (r + 1) + d] : 0.0;
        y[3 * r + d] = (cv - nxt) / dd[r];
      }
    }
    for (int kb = 0; kb < nw; ++kb) {  // g = F' y, S[:, j] -= g
      double g[3] = {0.0, 0.0, 0.0};
      if (kb < nl)
        for (int i2 = 0; i2 < 3; ++i2)
          g[i2] += Fd[9 * kb + 3 * i2] * y[3 * kb] + Fd[9 * kb + 3 * i2 + 1] * y[3 * kb + 1] +
                   Fd[9 * kb + 3 * i2 + 2] * y[3 * kb + 2];
      if (kb >= 1)
        for (int i2 = 0; i2 < 3; ++i2)
          g[i2] += Fl[9 * (kb - 1) + 3 * i2] * y[3 * (kb - 1)] + Fl[9 * (kb - 1) + 3 * i2 + 1] * y[3 * (kb - 1) + 1] +
                   Fl[9 * (kb - 1) + 3 * i2 + 2] * y[3 * (kb - 1) + 2];
      for (int i2 = 0; i2 < 3; ++i2) S[(3 * kb + i2) * m + j] -= g[i2];
    }
  }
  __syncthreads();
  double *Sout = Sinv_all + soff[f];
  for (int e = tid; e < m * m; e += nthr) Sout[e] = S[e];
}

// Inverse of S (k_jacobian_schur's output, in place) by Gauss-Jordan with partial
// pivoting (the first maximum wins); one CTA per filament with S in shared memory.
__global__ void __launch_bounds__(384) k_schur_gj(const int *__restrict__ fil_start,
                                                  const long long *__restrict__ soff, double *__restrict__ Sinv_all,
                                                  int *__restrict__ flags, const int *__restrict__ keep) {
  extern __shared__ double S[];
  __shared__ int perm[3 * FS_MAX_NW];
  __shared__ double fcol[3 * FS_MAX_NW];
  __shared__ int colsrc[3 * FS_MAX_NW];
  __shared__ int s_piv;
  __shared__ double s_inv, s_diag;
  if (keep && *keep) return;
  const int f = blockIdx.x;
  const int nw = fil_start[f + 1] - fil_start[f];
  if (nw < 2) return;
  const int m = 3 * nw;
  const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5;
  double *Sg = Sinv_all + soff[f];
  for (int e = tid; e < m * m; e += nthr) S[e] = Sg[e];
  __syncthreads();
  // Gauss-Jordan inversion in place with partial pivoting (first maximum wins).
  // Thread (g, c) owns column c for rows g, g + G, ...; per pivot: search (warp 0),
  // swap + scale of the pivot row and a copy of column kc, elimination.
  const int G = nthr / m;
  const bool act = tid < G * m;
  const int cj = tid % m, g0 = tid / m;
  for (int kc = 0; kc < m; ++kc) {
    if (warp == 0) {
      double best = -1.0;
      int bi = kc;
      for (int r = kc + lane; r < m; r += 32) {
        double v = fabs(S[r * m + kc]);
        if (v > best) { best = v; bi = r; }
      }
      for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (lane == 0) {
        s_piv = bi;
        s_inv = 1.0 / S[bi * m + kc];
        s_diag = S[kc * m + kc];
        perm[kc] = bi;
        if (!(best > 0.0)) atomicOr(&flags[FLAG_PIVOT], 1);
      }
    }
    __syncthreads();
    const int p = s_piv;
    const double inv = s_inv;
    if (act && g0 == 0) {
      const double a = S[kc * m + cj], b = S[p * m + cj];
      if (p != kc) S[p * m + cj] = a;
      S[kc * m + cj] = (cj == kc) ? inv : b * inv;  // in place: the pivot column turns into inv
    }
    for (int r = tid; r < m; r += nthr) fcol[r] = (r == p && p != kc) ? s_diag : (r == kc ? 0.0 : S[r * m + kc]);
    __syncthreads();
    if (act) {
      const double prow = S[kc * m + cj];
      for (int r = g0; r < m; r += G) {
        if (r == kc) continue;
        const double base = (cj == kc) ? 0.0 : S[r * m + cj];
        S[r * m + cj] = base - fcol[r] * prow;
      }
    }
    __syncthreads();
  }
  // undo the row interchanges on the columns: column c of the inverse is column colsrc[c]
  if (tid == 0) {
    for (int c = 0; c < m; ++c) colsrc[c] = c;
    for (int kc = m - 1; kc >= 0; --kc) {
      const int p = perm[kc];
      if (p != kc) {
        const int t = colsrc[kc];
        colsrc[kc] = colsrc[p];
        colsrc[p] = t;
      }
    }
  }
  __syncthreads();
  for (int e = tid; e < m * m; e += nthr) {
    const int r = e / m, c = e - r * m;
    Sg[e] = S[r * m + colsrc[c]];
  }
}

// The same inversion with the matrix in registers, for m = 3 nw <= 96: warp
// w = cb RB + rb (RB = ceil(m / 32) row blocks, CB = ceil(m / 24) column blocks)
// holds rows 32 rb .. 32 rb + 31 (one per lane) of columns 24 cb .. 24 cb + 23:
// 12 warps at m = 96, two matrices per SM.
// Per pivot kc (row p and 1 / S[p][kc], found by the previous step):
//   A: the lane holding row p publishes it scaled (prow = row p / v, with
//      1 / v in column kc), the lane holding row kc publishes its old row, the
//      warps holding column kc publish it (fcol);
//   B: row r := r - fcol[r] prow for every r != kc (row p, the old row kc,
//      takes the old (kc, kc) entry as its factor), row kc := prow, column kc
//      of the other rows := -fcol[r] / v; then the warps holding column kc + 1
//      search it over rows > kc (first maximum, by shuffles, per row block).
// Each element sees the operations and roundings of k_schur_gj; two barriers per
// pivot, one register-blocked outer product per thread.
constexpr int GJ_CW = 24;        // columns per warp
constexpr int GJ_MAX_M = 96;     // m handled by the register kernel
__global__ void __launch_bounds__(384, 2) k_schur_gj_reg(const int *__restrict__ fil_start,
                                                      const long long *__restrict__ soff,
                                                      double *__restrict__ Sinv_all, int *__restrict__ flags,
                                                      const int *__restrict__ keep) {
  constexpr int CW = GJ_CW;
  __shared__ double fcol[GJ_MAX_M], rowkc[GJ_MAX_M + CW];
  __shared__ __align__(16) double prow_s[GJ_MAX_M + CW];
  __shared__ double cand_v[3], cand_inv[3];
  __shared__ int cand_r[3];
  __shared__ int perm[GJ_MAX_M], colsrc[GJ_MAX_M], dstcol[GJ_MAX_M];
  if (keep && *keep) return;
  const int f = blockIdx.x;
  const int nw = fil_start[f + 1] - fil_start[f], m = 3 * nw;
  if (nw < 2 || m > GJ_MAX_M) return;  // block-uniform
  const int RB = (m + 31) >> 5, CB = (m + CW - 1) / CW;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool wact = w < RB * CB;  // warp-uniform; spare warps only take the barriers
  const int cb = w / RB, rb = w - cb * RB;
  const int r = 32 * rb + lane, c0 = CW * cb;
  double *Sg = Sinv_all + soff[f];
  double a[CW];
#pragma unroll
  for (int k = 0; k < CW; ++k) a[k] = (wact && r < m && c0 + k < m) ? Sg[(size_t)r * m + c0 + k] : 0.0;
  // first maximum of |a[k]| (k a compile-time slot after unrolling) over rows >
  // after in this row block -> cand[rb]
  auto search = [&](int k, int after) {
    double v = 0.0;
#pragma unroll
    for (int kk = 0; kk < CW; ++kk)
      if (kk == k) v = a[kk];
    double best = (r > after && r < m) ? fabs(v) : -1.0, x = v;
    int bi = r;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      const double ox = __shfl_xor_sync(0xffffffffu, x, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
        x = ox;
      }
    }
    if (lane == 0) {
      cand_v[rb] = best;
      cand_r[rb] = bi;
      cand_inv[rb] = best >= 0.0 ? 1.0 / x : 0.0;
    }
  };
  if (wact && cb == 0) search(0, -1);
  __syncthreads();
  // pivots kc = CW kb + kk: kk unrolled, so column kc is register slot kk of the
  // warps with cb == kb
  for (int kb = 0; kb < CB; ++kb) {
#pragma unroll
    for (int kk = 0; kk < CW; ++kk) {
      const int kc = CW * kb + kk;
      if (kc >= m) break;  // block-uniform
      // phase A
      double best = -1.0, inv = 0.0;
      int p = kc;
#pragma unroll
      for (int q = 0; q < 3; ++q)
        if (q < RB && cand_v[q] > best) {
          best = cand_v[q];
          p = cand_r[q];
          inv = cand_inv[q];
        }
      if (wact) {
        if (r == p) {
#pragma unroll
          for (int k = 0; k < CW; ++k) prow_s[c0 + k] = (cb == kb && k == kk) ? inv : a[k] * inv;
        }
        if (r == kc) {
#pragma unroll
          for (int k = 0; k < CW; ++k) rowkc[c0 + k] = a[k];
        }
        if (cb == kb && r < m) fcol[r] = a[kk];
      }
      if (threadIdx.x == 0) {
        perm[kc] = p;
        if (!(best > 0.0)) atomicOr(&flags[FLAG_PIVOT], 1);
      }
      __syncthreads();
      // phase B
      if (wact) {
        if (r == kc) {
#pragma unroll
          for (int k = 0; k < CW; k += 2) {
            const double2 q = *reinterpret_cast<const double2 *>(&prow_s[c0 + k]);
            a[k] = q.x;
            a[k + 1] = q.y;
          }
        } else {
          const bool rp = (r == p);  // row p: the old row kc, factor = old (kc, kc)
          const double fr = fcol[rp ? kc : (r < m ? r : 0)];
          if (rp) {
#pragma unroll
            for (int k = 0; k < CW; ++k) a[k] = rowkc[c0 + k];
          }
          if (cb == kb) a[kk] = 0.0;
#pragma unroll
          for (int k = 0; k < CW; k += 2) {
            const double2 q = *reinterpret_cast<const double2 *>(&prow_s[c0 + k]);
            a[k] = a[k] - fr * q.x;
            a[k + 1] = a[k + 1] - fr * q.y;
          }
        }
        if (kc + 1 < m) {
          if (kk + 1 < CW) {
            if (cb == kb) search(kk + 1, kc);
          } else if (cb == kb + 1) {
            search(0, kc);
          }
        }
      }
      __syncthreads();
    }
  }
  // undo the row interchanges on the columns: output column c is column colsrc[c]
  if (threadIdx.x == 0) {
    for (int c = 0; c < m; ++c) colsrc[c] = c;
    for (int kc = m - 1; kc >= 0; --kc) {
      const int p = perm[kc];
      if (p != kc) {
        const int t = colsrc[kc];
        colsrc[kc] = colsrc[p];
        colsrc[p] = t;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < m) dstcol[colsrc[threadIdx.x]] = threadIdx.x;
  __syncthreads();
  if (wact && r < m) {
#pragma unroll
    for (int k = 0; k < CW; ++k)
      if (c0 + k < m) Sg[(size_t)r * m + dstcol[c0 + k]] = a[k];
  }
}

// x = J0^-1 b for one filament (shared-memory vectors; 128 threads)
// b: 6nw entries [first-bead position rows | constraint rows | Lie rows]
// x: 6nw entries [X0 | U | lambda/dt]
// aux_g: the filament's D', F', tangents and P coefficient in HBM; aux: shared
// memory for their copy (the serial link recurrences then wait on shared, not
// global, loads)
__device__ void schur_apply_one(int nw, const double *__restrict__ Sinv, const double *__restrict__ aux_g,
                                double *aux, const double *bb, double *x, double *y, double *w, double dt,
                                double fac) {
  const int m = 3 * nw, nl = nw - 1;
  const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = nthr >> 5;
  for (int i = tid; i < 20 * nl + 3 * nw + 1; i += nthr) aux[i] = aux_g[i];
  __syncthreads();
  const double *dd = aux, *ee = aux + nl, *Fd = aux + 2 * nl, *Fl = Fd + 9 * nl, *tt = Fl + 9 * nl;
  const double pcoef = tt[3 * nw];
  const double *b1 = bb + 3, *b2 = bb + m;
  // y = D'^-1 b1
  if (tid < 3) {
    const int d = tid;
    for (int r = nl - 1; r >= 0; --r) {
      double nxt = (r + 1 < nl) ? ee[r] * y[3 * (r + 1) + d] : 0.0;
      y[3 * r + d] = (b1[3 * r + d] - nxt) / dd[r];
    }
  }
  __syncthreads();
  // w = b2 - F' y
  for (int row = tid; row < m; row += nthr) {
    const int kb = row / 3, i2 = row % 3;
    double g = 0.0;
    if (kb < nl) g += Fd[9 * kb + 3 * i2] * y[3 * kb] + Fd[9 * kb + 3 * i2 + 1] * y[3 * kb + 1] + Fd[9 * kb + 3 * i2 + 2] * y[3 * kb + 2];
    if (kb >= 1)
      g += Fl[9 * (kb - 1) + 3 * i2] * y[3 * (kb - 1)] + Fl[9 * (kb - 1) + 3 * i2 + 1] * y[3 * (kb - 1) + 1] +
           Fl[9 * (kb - 1) + 3 * i2 + 2] * y[3 * (kb - 1) + 2];
    w[row] = b2[row] - g;
  }
  __syncthreads();
  // u = S^-1 w: each warp takes eight rows at a time (coalesced row reads, all
  // of their loads in flight together); per row the lane-strided sum and the
  // shuffle tree of a one-row-per-warp product
  double *u = x + 3;
  constexpr int RU = 8;
  for (int row0 = warp * RU; row0 < m; row0 += nwarp * RU) {
    double acc[RU];
#pragma unroll
    for (int q = 0; q < RU; ++q) acc[q] = 0.0;
#pragma unroll 3
    for (int c = lane; c < m; c += 32) {
      const double wc = w[c];
#pragma unroll
      for (int q = 0; q < RU; ++q)
        if (row0 + q < m) acc[q] += Sinv[(size_t)(row0 + q) * m + c] * wc;
    }
#pragma unroll
    for (int q = 0; q < RU; ++q)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < RU; ++q)
        if (row0 + q < m) u[row0 + q] = acc[q];
  }
  __syncthreads();
  // z = b1 - C u, (C u)_r = fac c_0 + 2 fac sum_{1<=q<=r} c_q + fac c_{r+1}, c_q = cross(u_q, t_q)
  // (y is reused for z, then for lambda)
  if (tid < 3) {
    const int d = tid;
    const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
    double c0 = u[d1] * tt[d2] - u[d2] * tt[d1];
    double run = 0.0;
    for (int r = 0; r < nl; ++r) {
      const int q = r + 1;
      double cq = u[3 * q + d1] * tt[3 * q + d2] - u[3 * q + d2] * tt[3 * q + d1];
      double cu = fac * c0 + 2.0 * fac * run + fac * cq;
      y[3 * r + d] = b1[3 * r + d] - cu;
      run += cq;
    }
  }
  __syncthreads();
  // lambda = D'^-1 z (in place), then X0 = b0 - P lambda
  if (tid < 3) {
    const int d = tid;
    for (int r = nl - 1; r >= 0; --r) {
      double nxt = (r + 1 < nl) ? ee[r] * y[3 * (r + 1) + d] : 0.0;
      y[3 * r + d] = (y[3 * r + d] - nxt) / dd[r];
    }
    x[d] = bb[d] - pcoef * y[d];
  }
  __syncthreads();
  for (int i = tid; i < 3 * nl; i += nthr) x[3 + m + i] = y[i] / dt;
  __syncthreads();
}

// x_f = J0_f^-1 b_f, then x += sum_i C_i dots_i (FilamentJacobianSolver.hpp:49-73)
__global__ void __launch_bounds__(128) k_schur_apply(const int *__restrict__ fil_start,
                                                     const long long *__restrict__ soff,
                                                     const long long *__restrict__ aoff,
                                                     const double *__restrict__ Sinv_all,
                                                     const double *__restrict__ aux_all, const double *__restrict__ b,
                                                     double *__restrict__ x, const double *__restrict__ C,
                                                     const double *__restrict__ dots, int iter,
                                                     const int *__restrict__ iter_d,
                                                     const int *__restrict__ off_d, size_t n6, double dt,
                                                     double fac) {
  __shared__ double bb[6 * FS_MAX_NW], xs[6 * FS_MAX_NW], y[3 * FS_MAX_NW], w[3 * FS_MAX_NW];
  __shared__ double auxs[20 * (FS_MAX_NW - 1) + 3 * FS_MAX_NW + 1];
  const int f = blockIdx.x;
  const int b0 = fil_start[f], nw = fil_start[f + 1] - b0, s0 = 6 * b0, n = 6 * nw;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int r = tid; r < n; r += nthr) bb[r] = b[s0 + r];
  __syncthreads();
  if (nw < 2) {
    for (int r = tid; r < n; r += nthr) xs[r] = bb[r];
    __syncthreads();
  } else {
    schur_apply_one(nw, Sinv_all + soff[f], aux_all + aoff[f], auxs, bb, xs, y, w, dt, fac);
  }
  const int ncol = (iter_d ? *iter_d : iter) + (off_d ? *off_d : 0);
  for (int r = tid; r < n; r += nthr) {
    double v = xs[r];
#pragma unroll 4
    for (int i = 0; i < ncol; ++i) v += C[(size_t)i * n6 + s0 + r] * dots[i];
    x[s0 + r] = v;
  }
}

// explicit inverse of filament f's J0 (with the 1/dt rows), one column per CTA (test access)
__global__ void __launch_bounds__(128) k_schur_inverse(int nw, const double *__restrict__ Sinv,
                                                       const double *__restrict__ aux, double dt, double fac,
                                                       double *__restrict__ out) {
  __shared__ double bb[6 * FS_MAX_NW], xs[6 * FS_MAX_NW], y[3 * FS_MAX_NW], w[3 * FS_MAX_NW];
  __shared__ double auxs[20 * (FS_MAX_NW - 1) + 3 * FS_MAX_NW + 1];
  const int n = 6 * nw, e = blockIdx.x, tid = threadIdx.x;
  for (int r = tid; r < n; r += blockDim.x) bb[r] = (r == e) ? 1.0 : 0.0;
  __syncthreads();
  if (nw < 2) {
    for (int r = tid; r < n; r += blockDim.x) xs[r] = bb[r];
    __syncthreads();
  } else {
    schur_apply_one(nw, Sinv, aux, auxs, bb, xs, y, w, dt, fac);
  }
  for (int r = tid; r < n; r += blockDim.x) out[(size_t)r * n + e] = xs[r];
}

// ---- error check ---------------------------------------------------------------
__global__ void k_error_check(int np, const int *__restrict__ fil_id, const int *__restrict__ seg_id,
                              const int *__restrict__ fil_start, const double *__restrict__ Xs,
                              const double *__restrict__ X, const double *__restrict__ Xt,
                              const double *__restrict__ Us, const double *__restrict__ U,
                              const double *__restrict__ V, const double *__restrict__ W, double *__restrict__ err,
                              int nt, FilConsts k, int *__restrict__ flags, unsigned long long *__restrict__ maxbits) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  bool over = false, nonfin = false, expl = false;
  double mx = 0.0;
  if (b < np) {
    const int f = fil_id[b], i = seg_id[b];
    const int b0 = fil_start[f], nw = fil_start[f + 1] - b0;
    const int s0 = 6 * b0;
    double dv[3];
    dexpinv(Us + 3 * b, W + 3 * b, dv);
    const double fourthirds = 4. / 3., onethird = 1. / 3., twothirdsDt = k.dt * 2. / 3.;
    for (int d = 0; d < 3; ++d) {
      double e1, e2;
      if (nt <= k.impl_euler_steps) {
        e1 = Xs[3 * b + d] - X[3 * b + d] - k.dt * V[3 * b + d];
        e2 = Us[3 * b + d] - k.dt * dv[d];
      } else {
        e1 = Xs[3 * b + d] - fourthirds * X[3 * b + d] + onethird * Xt[3 * b + d] - twothirdsDt * V[3 * b + d];
        e2 = Us[3 * b + d] - onethird * U[3 * b + d] - twothirdsDt * dv[d];
      }
      err[s0 + 3 * i + d] = e1;
      err[s0 + 3 * nw + 3 * i + d] = e2;
      over |= (fabs(e1) > k.tol) || (fabs(e2) > k.tol);
      nonfin |= !isfinite(e1) || !isfinite(e2);
      expl |= (fabs(e1) > 1e6) || (fabs(e2) > 1e6);
      mx = fmax(mx, fmax(fabs(e1), fabs(e2)));
    }
  }
  const unsigned full = 0xffffffffu;
  if (__any_sync(full, over) && (threadIdx.x & 31) == 0) atomicOr(&flags[FLAG_CHECK], 1);
  if (__any_sync(full, nonfin) && (threadIdx.x & 31) == 0) atomicOr(&flags[FLAG_NONFINITE], 1);
  if (__any_sync(full, expl) && (threadIdx.x & 31) == 0) atomicOr(&flags[FLAG_EXPLODE], 1);
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(full, mx, o));
  if ((threadIdx.x & 31) == 0 && maxbits) atomicMax(maxbits, fs_dbits(mx));
}

// ---- Broyden ---------------------------------------------------------------------
#define RED_THREADS 256
#define RED_BLOCKS 296

// partial dot products D_i . b for i < iter (iter_d ? *iter_d : iter), plus the
// columns carried from earlier steps (off_d ? *off_d : 0, fs_start.cu): each of the
// RED_BLOCKS blocks sums a fixed strided slice of every column, so the partials
// (and the fixed-order final sums) do not depend on how many columns there are
__global__ void __launch_bounds__(RED_THREADS) k_dots(const double *__restrict__ D, const double *__restrict__ b,
                                                       size_t n6, int iter, const int *__restrict__ iter_d,
                                                       const int *__restrict__ off_d, double *__restrict__ partial) {
  // columns in groups of DOT_COLS: a thread reads b[k] once per group and keeps
  // the group's loads in flight together; each column's sum runs in the same
  // order as one column at a time (k ascending per thread, then the shuffle
  // tree, then the warps in order), so the partials are bitwise those
  constexpr int DOT_COLS = 16;
  __shared__ double sh[DOT_COLS][RED_THREADS / 32];
  const int ncol = (iter_d ? *iter_d : iter) + (off_d ? *off_d : 0);
  for (int i0 = 0; i0 < ncol; i0 += DOT_COLS) {
    double acc[DOT_COLS];
#pragma unroll
    for (int j = 0; j < DOT_COLS; ++j) acc[j] = 0.0;
    for (size_t k = (size_t)blockIdx.x * RED_THREADS + threadIdx.x; k < n6; k += (size_t)gridDim.x * RED_THREADS) {
      const double bk = b[k];
#pragma unroll
      for (int j = 0; j < DOT_COLS; ++j)
        if (i0 + j < ncol) acc[j] += D[(size_t)(i0 + j) * n6 + k] * bk;
    }
#pragma unroll
    for (int j = 0; j < DOT_COLS; ++j) {
      double a = acc[j];
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if ((threadIdx.x & 31) == 0) sh[j][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x < DOT_COLS && i0 + (int)threadIdx.x < ncol) {
      const int j = threadIdx.x;
      double s = 0.0;
      for (int w = 0; w < RED_THREADS / 32; ++w) s += sh[j][w];
      partial[(size_t)(i0 + j) * gridDim.x + blockIdx.x] = s;
    }
    __syncthreads();
  }
}

// fixed-order final sums: one warp per output
__global__ void k_reduce_rows(const double *__restrict__ partial, int nparts, int nrows, double *__restrict__ out,
                              int do_sqrt, const int *__restrict__ nrows_d, const int *__restrict__ off_d) {
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= (nrows_d ? *nrows_d : nrows) + (off_d ? *off_d : 0)) return;
  double acc = 0.0;
  for (int p = lane; p < nparts; p += 32) acc += partial[(size_t)row * nparts + p];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[row] = do_sqrt ? sqrt(acc) : acc;
}

// dE = newerr - err and per-block sums of dE^2
__global__ void __launch_bounds__(RED_THREADS) k_diff_sq(const double *__restrict__ ne, const double *__restrict__ e,
                                                          double *__restrict__ dE, size_t n6,
                                                          double *__restrict__ partial) {
  __shared__ double sh[RED_THREADS / 32];
  double acc = 0.0;
  for (size_t k = (size_t)blockIdx.x * RED_THREADS + threadIdx.x; k < n6; k += (size_t)gridDim.x * RED_THREADS) {
    double d = ne[k] - e[k];
    dE[k] = d;
    acc += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < RED_THREADS / 32; ++w) s += sh[w];
    partial[blockIdx.x] = s;
  }
}

// C_iter = -tmp/|dE| - upd/|dE|, D_iter = dE/|dE| (main.cpp:657-661)
// column iter (iter_d ? *iter_d : iter) of the history, after the columns carried
// from earlier steps (off_d ? *off_d : 0)
__global__ void k_broyden_cols(const double *__restrict__ tmp, const double *__restrict__ upd,
                               const double *__restrict__ dE, const double *__restrict__ nrm, size_t n6,
                               double *__restrict__ Cmat, double *__restrict__ Dmat, int iter,
                               const int *__restrict__ iter_d, const int *__restrict__ off_d) {
  size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n6) return;
  const size_t col = (size_t)((iter_d ? *iter_d : iter) + (off_d ? *off_d : 0)) * n6;
  double *__restrict__ Ccol = Cmat + col;
  double *__restrict__ Dcol = Dmat + col;
  const double n = nrm[0];
  double t = tmp[k] * (-1. / n);
  t -= upd[k] / n;
  Ccol[k] = t;
  Dcol[k] = dE[k] / n;
}

// ---- update / step ----------------------------------------------------------------
__global__ void k_update(int np, const int *__restrict__ fil_id, const int *__restrict__ seg_id,
                         const int *__restrict__ fil_start, const double *__restrict__ u, double *__restrict__ Xs,
                         double *__restrict__ Us, const double *__restrict__ q, double *__restrict__ qs,
                         double *__restrict__ lam) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= np) return;
  const int f = fil_id[b], i = seg_id[b];
  const int b0 = fil_start[f], nw = fil_start[f + 1] - b0, l0 = b0 - f;
  const int s = 6 * b0;
  double us[3];
  if (i == 0) {
    for (int d = 0; d < 3; ++d) {
      Xs[3 * b + d] -= u[s + d];
      us[d] = Us[3 * b + d] - u[s + 3 + d];
    }
  } else {
    for (int d = 0; d < 3; ++d) us[d] = Us[3 * b + d] - u[s + 6 + 3 * (i - 1) + d];
  }
  for (int d = 0; d < 3; ++d) Us[3 * b + d] = us[d];
  qstore(q_expm(qload(q + 4 * b), us), qs + 4 * b);
  if (i < nw - 1)
    for (int d = 0; d < 3; ++d) lam[3 * (l0 + i) + d] -= u[s + 3 * nw + 3 + 3 * i + d];
}

__global__ void k_step(int np, int nlink, double *__restrict__ X, double *__restrict__ Xs, double *__restrict__ Xt,
                       double *__restrict__ U, double *__restrict__ Us, double *__restrict__ Ut,
                       double *__restrict__ q, double *__restrict__ qt, double *__restrict__ lam,
                       double *__restrict__ lam1, double *__restrict__ lam2, int nt, int ex, int tension_order) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < np) {
    const int b = t;
    double uu[3];
    for (int d = 0; d < 3; ++d) {
      Xt[3 * b + d] = X[3 * b + d];
      X[3 * b + d] = Xs[3 * b + d];
      Ut[3 * b + d] = U[3 * b + d];
      uu[d] = Us[3 * b + d];
      U[3 * b + d] = uu[d];
    }
    Q qq = qload(q + 4 * b);
    qstore(qq, qt + 4 * b);
    qstore(q_expm(qq, uu), q + 4 * b);
  }
  if (t < 3 * nlink) {
    const int kk = t;
    if (nt > ex && tension_order == 2) {
      double lamtmp = 3 * lam[kk] - 3 * lam1[kk] + lam2[kk];
      lam2[kk] = lam1[kk];
      lam1[kk] = lam[kk];
      lam[kk] = lamtmp;
    } else if (nt >= ex) {  // the reference: at nt == ex only; tension order 1 from then on
      double lamtmp = 2. * lam[kk] - lam1[kk];
      lam2[kk] = lam1[kk];
      lam1[kk] = lam[kk];
      lam[kk] = lamtmp;
    } else {
      lam1[kk] = lam[kk];
    }
  }
}

FilConsts make_fconsts(const fs_ctx *c) {
  FilConsts k;
  for (int d = 0; d < 3; ++d) {
    k.L[d] = c->L[d];
    k.gravity[d] = c->p.gravity[d];
    k.st[d] = c->p.strain_twist[d];
  }
  k.dt = c->p.dt;
  k.dl = c->p.dl;
  k.mu = c->p.mu;
  k.tol = c->p.tol;
  k.impl_euler_steps = c->p.impl_euler_steps;
  k.lambda_extrap_step = c->p.lambda_extrap_step;
  k.tt = 0.0;
  k.swim_curvature = c->swim_curvature;
  k.swim_sperm_decay = c->swim_sperm_decay;
  k.swim = c->swim;
  return k;
}

}  // namespace

fs_status fil_initial_guess(fs_ctx *c) {
  if (!c->have_state) return FS_ERR_STATE;
  ProfScope ps(c, FS_STAGE_UPDATE);
  const int order = (c->start_order == 2 && c->hist_Xtt) ? 2 : 1;
  k_initial_guess<<<fs_blocks(c->np, 256), 256, 0, c->stream>>>(c->np, c->seg_id, c->X, c->Xt, c->U, c->Ut, c->q,
                                                                 c->Xs, c->Us, c->qs, order, c->hist_Xtt, c->hist_ok);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

fs_status fil_forces(fs_ctx *c, int nt) {
  if (!c->have_state) return FS_ERR_STATE;
  ProfScope ps(c, FS_STAGE_FORCES);
  FilConsts k = make_fconsts(c);
  k.tt = nt * c->p.dt;  // double tt = nt*dt (Filament.hpp:295)
  k_unrobot_assign<<<fs_blocks(c->nfil, 4), 128, 0, c->stream>>>(c->nfil, c->fil_start, c->qs, c->Xs, c->Y, k);
  FS_LAUNCH_CHECK();
  k_forces<<<fs_blocks(c->np, 256), 256, 0, c->stream>>>(c->np, c->fil_id, c->seg_id, c->fil_start, c->qs, c->lam,
                                                          c->kap, c->cc, c->F, c->TAU, k);
  FS_LAUNCH_CHECK();
  if (c->nspring > 0) {
    k_spring_forces<<<fs_blocks(c->np, 256), 256, 0, c->stream>>>(c->np, c->spring_off, c->spring_ent,
                                                                   c->spring_beads, c->Xs, c->spring_k,
                                                                   c->spring_l0, k, c->F);
    FS_LAUNCH_CHECK();
  }
  return FS_OK;
}

// keep (device, or null): nonzero leaves the previous J0 in place
fs_status fil_jacobian_build(fs_ctx *c, int nt, const int *keep) {
  if (!c->have_state) return FS_ERR_STATE;
  ProfScope ps(c, FS_STAGE_JACOBIAN);
  FilConsts k = make_fconsts(c);
  k.tt = nt * c->p.dt;
  const size_t smem = sizeof(double) * 9 * (size_t)c->max_nw * c->max_nw;
  // one thread per Schur column (3 Nw, rounded to warps): three filaments share an SM
  const int jthreads = std::min(256, 32 * ((3 * c->max_nw + 31) / 32));
  k_jacobian_schur<<<c->nfil, jthreads, smem, c->stream>>>(c->fil_start, c->qs, c->Us, c->TAU, c->lam, c->kap, c->cc,
                                                      c->soff, c->aoff, c->Sinv, c->aux, nt, k, c->p.a, c->p.ah,
                                                      c->flags, keep);
  FS_LAUNCH_CHECK();
  // all filaments of at most 32 beads: the register kernel; otherwise the
  // shared-memory kernel for every filament
  if (3 * c->max_nw <= GJ_MAX_M) {
    const int m = 3 * c->max_nw, warps = ((m + 31) / 32) * ((m + GJ_CW - 1) / GJ_CW);
    k_schur_gj_reg<<<c->nfil, 32 * warps, 0, c->stream>>>(c->fil_start, c->soff, c->Sinv, c->flags, keep);
  } else {
    k_schur_gj<<<c->nfil, 384, smem, c->stream>>>(c->fil_start, c->soff, c->Sinv, c->flags, keep);
  }
  FS_LAUNCH_CHECK();
  return FS_OK;
}

fs_status fil_jacobian_prepare(fs_ctx *c) {
  if (c->max_nw > FS_MAX_NW) return FS_ERR_INVALID_ARG;
  const size_t smem = sizeof(double) * 9 * (size_t)c->max_nw * c->max_nw;
  FS_CUDA(cudaFuncSetAttribute(k_jacobian_schur, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  FS_CUDA(cudaFuncSetAttribute(k_schur_gj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return FS_OK;
}

int fil_aux_size(int nw) { return nw < 2 ? 1 : 20 * (nw - 1) + 3 * nw + 1; }

fs_status fil_jacobian_inverse(fs_ctx *c, int f, double *out_d) {
  int fs_h[2];
  long long so, ao;
  FS_CUDA(cudaMemcpyAsync(fs_h, c->fil_start + f, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaMemcpyAsync(&so, c->soff + f, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaMemcpyAsync(&ao, c->aoff + f, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  const int nw = fs_h[1] - fs_h[0], n = 6 * nw;
  k_schur_inverse<<<n, 128, 0, c->stream>>>(nw, c->Sinv + so, c->aux + ao, c->p.dt, 0.5 * c->p.dl, out_d);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

fs_status fil_error_check(fs_ctx *c, const double *V, const double *W, double *err, int nt) {
  if (!c->have_state) return FS_ERR_STATE;
  ProfScope ps(c, FS_STAGE_ERROR_CHECK);
  FilConsts k = make_fconsts(c);
  FS_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(int) * 3, c->stream));  // check, nonfinite, explode
  FS_CUDA(cudaMemsetAsync(c->maxerr_bits, 0, sizeof(unsigned long long), c->stream));
  k_error_check<<<fs_blocks(c->np, 256), 256, 0, c->stream>>>(c->np, c->fil_id, c->seg_id, c->fil_start, c->Xs, c->X,
                                                               c->Xt, c->Us, c->U, V, W, err, nt, k, c->flags,
                                                               c->maxerr_bits);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// iter_d (graph capture): the history length is read on the device; off_d: the
// columns carried from earlier steps before it (fs_set_broyden_memory), or none
fs_status fil_broyden_apply(fs_ctx *c, const double *b, double *x, int iter, const int *iter_d, const int *off_d) {
  if (!c->have_state) return FS_ERR_STATE;
  ProfScope ps(c, FS_STAGE_BROYDEN);
  const size_t n6 = (size_t)6 * c->np;
  if (iter > 0 || iter_d || off_d) {
    // rows launched: a bound on the device count (with the memory on, callers pass
    // iter 0 and no iter_d: the count is the carried and current columns, off_d)
    const int base = iter_d ? c->p.broyden_maxiter : iter;
    const int rows = off_d ? c->p.broyden_maxiter + c->bmem_cols + base : base;
    k_dots<<<RED_BLOCKS, RED_THREADS, 0, c->stream>>>(c->Dmat, b, n6, iter, iter_d, off_d, c->partials);
    FS_LAUNCH_CHECK();
    k_reduce_rows<<<fs_blocks(rows, 8), 256, 0, c->stream>>>(c->partials, RED_BLOCKS, iter, c->dots, 0, iter_d,
                                                             off_d);
    FS_LAUNCH_CHECK();
  }
  k_schur_apply<<<c->nfil, 128, 0, c->stream>>>(c->fil_start, c->soff, c->aoff, c->Sinv, c->aux, b, x, c->Cmat,
                                                 c->dots, iter, iter_d, off_d, n6, c->p.dt, 0.5 * c->p.dl);
  FS_LAUNCH_CHECK();
  return learn_diag_apply(c, b, x);  // learned initial inverse-Jacobian diagonal, when on
}

// main.cpp:641-663 with the current err/newerr/upd: history column `iter`
fs_status fil_broyden_update(fs_ctx *c, int iter, const int *iter_d, const int *off_d) {
  const size_t n6 = (size_t)6 * c->np;
  {
    ProfScope ps(c, FS_STAGE_BROYDEN);
    k_diff_sq<<<RED_BLOCKS, RED_THREADS, 0, c->stream>>>(c->newerr, c->err, c->dE, n6, c->partials);
    FS_LAUNCH_CHECK();
    k_reduce_rows<<<1, 32, 0, c->stream>>>(c->partials, RED_BLOCKS, 1, c->scalars, 1, nullptr, nullptr);
    FS_LAUNCH_CHECK();
  }
  FS_TRY(fil_broyden_apply(c, c->dE, c->tmp, iter, iter_d, off_d));
  ProfScope ps(c, FS_STAGE_BROYDEN);
  k_broyden_cols<<<fs_blocks((long long)n6, 256), 256, 0, c->stream>>>(c->tmp, c->upd, c->dE, c->scalars, n6,
                                                                       c->Cmat, c->Dmat, iter, iter_d, off_d);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

fs_status fil_state_update(fs_ctx *c, const double *upd) {
  if (!c->have_state) return FS_ERR_STATE;
  ProfScope ps(c, FS_STAGE_UPDATE);
  k_update<<<fs_blocks(c->np, 256), 256, 0, c->stream>>>(c->np, c->fil_id, c->seg_id, c->fil_start, upd, c->Xs,
                                                          c->Us, c->q, c->qs, c->lam);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

fs_status fil_step(fs_ctx *c, int nt) {
  if (!c->have_state) return FS_ERR_STATE;
  ProfScope ps(c, FS_STAGE_UPDATE);
  int n = c->np > 3 * c->nlink ? c->np : 3 * c->nlink;
  k_step<<<fs_blocks(n, 256), 256, 0, c->stream>>>(c->np, c->nlink, c->X, c->Xs, c->Xt, c->U, c->Us, c->Ut, c->q,
                                                    c->qt, c->lam, c->lam1, c->lam2, nt, c->p.lambda_extrap_step,
                                                    c->tension_order == 1 ? 1 : 2);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

fs_status fil_max_abs_err(fs_ctx *c, const double *err, double *out_h) {
  (void)err;
  unsigned long long bits;
  FS_CUDA(cudaMemcpyAsync(&bits, c->maxerr_bits, sizeof bits, cudaMemcpyDeviceToHost, c->stream));
  FS_CUDA(cudaStreamSynchronize(c->stream));
  memcpy(out_h, &bits, sizeof bits);
  return FS_OK;
}
