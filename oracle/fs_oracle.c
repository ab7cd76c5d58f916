/*
 * fs_oracle.c -- CPU FP64 restatement of FilSim's FCM mobility solve, collision
 * barrier and implicit BDF2/Broyden step. TEST INFRASTRUCTURE ONLY: the tests,
 * __graft_entry__.smoke() and bench.py's CPU baseline load it to compare results
 * with; nothing in the product links or calls it.
 *
 * Parity unpinned: the reference cannot be built here (it needs MPI, FFTW 2.1.5
 * and Armadillo) and ships no golden vectors. Each function below follows the
 * cited reference lines statement by statement; the FFT is this file's own
 * mixed-radix transform with FFTW's real-to-complex conventions (unnormalised,
 * and a complex-to-real inverse that ignores the imaginary parts of the DC and
 * Nyquist coefficients of the last axis). Known answers in the tests pin it.
 *
 * All citations are file:line in the FilSim sources.
 */
#include "fs_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_PI 3.14159265358979323846264338327950288

/* ------------------------------------------------------------------------ */
/* derived constants: multi_filament_header.hpp:47-60                         */
/* ------------------------------------------------------------------------ */
typedef struct {
  double Lx, Ly, Lz;
  double sigmadipsq, anormdip, anormdip2;
  double sigmasq, anorm, anorm2;
  int ngdh;
} or_consts;

static void or_consts_init(const fs_params *p, or_consts *c) {
  c->Lx = p->npts_x * p->dx;
  c->Ly = p->npts_y * p->dx;
  c->Lz = p->npts_z * p->dx;
  c->sigmadipsq = p->sigma_dip * p->sigma_dip;
  c->anormdip = 1.0 / sqrt(2.0 * OR_PI * c->sigmadipsq);
  c->anormdip2 = 2.0 * c->sigmadipsq;
  c->sigmasq = p->sigma * p->sigma;
  c->anorm = 1.0 / sqrt(2.0 * OR_PI * c->sigmasq);
  c->anorm2 = 2.0 * c->sigmasq;
  c->ngdh = p->ngd / 2;
}

/* ------------------------------------------------------------------------ */
/* FFT: recursive mixed-radix complex transform (stand-in for FFTW 2.1.5)    */
/* ------------------------------------------------------------------------ */
typedef struct {
  int n;
  int nfac;
  int fac[40];
  or_cpx *tw; /* tw[j] = exp(-2 pi i j / n) */
} or_fftplan;

static void or_plan_init(or_fftplan *pl, int n) {
  pl->n = n;
  pl->nfac = 0;
  int m = n;
  while (m % 4 == 0) { pl->fac[pl->nfac++] = 4; m /= 4; }
  while (m % 2 == 0) { pl->fac[pl->nfac++] = 2; m /= 2; }
  for (int f = 3; m > 1; f += 2) {
    while (m % f == 0) { pl->fac[pl->nfac++] = f; m /= f; }
  }
  pl->fac[pl->nfac] = 1;
  pl->tw = (or_cpx *)malloc(sizeof(or_cpx) * (size_t)n);
  for (int j = 0; j < n; ++j) {
    double ang = -2.0 * OR_PI * (double)j / (double)n;
    pl->tw[j].re = cos(ang);
    pl->tw[j].im = sin(ang);
  }
}

static void or_plan_free(or_fftplan *pl) { free(pl->tw); }

/* out[0..n) = DFT of in[0], in[s], ..., in[(n-1)s]; twiddles of the full
 * length N0 = n * ts are tw[j * ts]. sign = -1 forward, +1 backward. */
static void or_fft_rec(const or_cpx *in, or_cpx *out, int n, int s, const or_fftplan *pl, int ts,
                       const int *fac, int sign) {
  if (n == 1) { out[0] = in[0]; return; }
  int p = fac[0];
  int m = n / p;
  for (int r = 0; r < p; ++r) or_fft_rec(in + (size_t)r * s, out + (size_t)r * m, m, s * p, pl, ts * p, fac + 1, sign);
  or_cpx t[64];
  int N0 = pl->n;
  for (int k = 0; k < m; ++k) {
    for (int r = 0; r < p; ++r) {
      or_cpx y = out[(size_t)r * m + k];
      long idx = ((long)r * k % n) * ts % N0;
      or_cpx w = pl->tw[idx];
      if (sign > 0) w.im = -w.im;
      t[r].re = y.re * w.re - y.im * w.im;
      t[r].im = y.re * w.im + y.im * w.re;
    }
    for (int q = 0; q < p; ++q) {
      double sr = 0.0, si = 0.0;
      for (int r = 0; r < p; ++r) {
        long idx = ((long)r * q % p) * (long)m * ts % N0;
        or_cpx w = pl->tw[idx];
        if (sign > 0) w.im = -w.im;
        sr += t[r].re * w.re - t[r].im * w.im;
        si += t[r].re * w.im + t[r].im * w.re;
      }
      out[(size_t)k + (size_t)q * m].re = sr;
      out[(size_t)k + (size_t)q * m].im = si;
    }
  }
}

/* in-place 1-D transform of a strided line (work: n scratch) */
static void or_fft_line(or_cpx *data, size_t stride, const or_fftplan *pl, int sign, or_cpx *work_in, or_cpx *work_out) {
  int n = pl->n;
  for (int i = 0; i < n; ++i) work_in[i] = data[(size_t)i * stride];
  or_fft_rec(work_in, work_out, n, 1, pl, 1, pl->fac, sign);
  for (int i = 0; i < n; ++i) data[(size_t)i * stride] = work_out[i];
}

/* Power-of-two lengths: OR_FB lines at once, interleaved (element e of line b at
 * e * OR_FB + b), by an iterative radix-2 Stockham transform (decimation in
 * frequency, self-sorting), so the inner loops run over the lines and the
 * strided passes read and write OR_FB adjacent values per element. Other
 * lengths use the recursive transform above, one line at a time. */
#define OR_FB 8

static int or_is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* x, y: n * OR_FB values; the result is left in *x (the buffers may swap) */
static void or_fft_block_pow2(or_cpx **x, or_cpx **y, int n, const or_fftplan *pl, int sign) {
  or_cpx *a = *x, *b = *y;
  for (int len = n, s = 1; len > 1; len >>= 1, s <<= 1) {
    const int m = len / 2, ts = n / len;
    for (int pp = 0; pp < m; ++pp) {
      or_cpx w = pl->tw[(size_t)pp * ts];
      if (sign > 0) w.im = -w.im;
      for (int q = 0; q < s; ++q) {
        const or_cpx *a0 = a + ((size_t)q + (size_t)s * pp) * OR_FB;
        const or_cpx *a1 = a + ((size_t)q + (size_t)s * (pp + m)) * OR_FB;
        or_cpx *b0 = b + ((size_t)q + (size_t)s * (2 * pp)) * OR_FB;
        or_cpx *b1 = b + ((size_t)q + (size_t)s * (2 * pp + 1)) * OR_FB;
        for (int l = 0; l < OR_FB; ++l) {
          const double dr = a0[l].re - a1[l].re, di = a0[l].im - a1[l].im;
          b0[l].re = a0[l].re + a1[l].re;
          b0[l].im = a0[l].im + a1[l].im;
          b1[l].re = dr * w.re - di * w.im;
          b1[l].im = dr * w.im + di * w.re;
        }
      }
    }
    or_cpx *t = a;
    a = b;
    b = t;
  }
  *x = a;
  *y = b;
}

/* transforms lines [l0, l0 + nb) (nb <= OR_FB) whose element e sits at
 * base[line * lstride + e * estride] (complex), in place */
static void or_fft_lines(or_cpx *base, long l0, int nb, size_t lstride, size_t estride, const or_fftplan *pl,
                         int sign, or_cpx *wa, or_cpx *wb) {
  const int n = pl->n;
  if (!or_is_pow2(n)) {
    for (int l = 0; l < nb; ++l) or_fft_line(base + (size_t)(l0 + l) * lstride, estride, pl, sign, wa, wb);
    return;
  }
  for (int e = 0; e < n; ++e)
    for (int l = 0; l < OR_FB; ++l)
      wa[(size_t)e * OR_FB + l] = l < nb ? base[(size_t)(l0 + l) * lstride + (size_t)e * estride] : wa[0];
  or_cpx *x = wa, *y = wb;
  or_fft_block_pow2(&x, &y, n, pl, sign);
  for (int e = 0; e < n; ++e)
    for (int l = 0; l < nb; ++l) base[(size_t)(l0 + l) * lstride + (size_t)e * estride] = x[(size_t)e * OR_FB + l];
}

/* Unnormalised 3-D real-to-complex transform; out is [nx][ny][nz/2+1].
 * stride > 1 transforms the first 1/stride of the lines of each pass only (timing samples). */
static void fft_r2c_3d_s(const double *in, or_cpx *out, int nx, int ny, int nz, long stride) {
  int nzh = nz / 2 + 1;
  or_fftplan px, py, pz;
  or_plan_init(&px, nx);
  or_plan_init(&py, ny);
  or_plan_init(&pz, nz);
  int nmax = nx > ny ? nx : ny;
  nmax = nmax > nz ? nmax : nz;
#pragma omp parallel
  {
    or_cpx *wa = (or_cpx *)malloc(sizeof(or_cpx) * (size_t)nmax * OR_FB);
    or_cpx *wb = (or_cpx *)malloc(sizeof(or_cpx) * (size_t)nmax * OR_FB);
    const long nzl = (long)nx * ny;
#pragma omp for schedule(static)
    for (long blk = 0; blk < (nzl + OR_FB - 1) / OR_FB / stride; ++blk) {
      const long l0 = blk * OR_FB;
      const int nb = (int)(nzl - l0 < OR_FB ? nzl - l0 : OR_FB);
      if (or_is_pow2(nz)) {
        for (int e = 0; e < nz; ++e)
          for (int l = 0; l < OR_FB; ++l) {
            wa[(size_t)e * OR_FB + l].re = l < nb ? in[(size_t)(l0 + l) * nz + e] : 0.0;
            wa[(size_t)e * OR_FB + l].im = 0.0;
          }
        or_cpx *x = wa, *y = wb;
        or_fft_block_pow2(&x, &y, nz, &pz, -1);
        for (int l = 0; l < nb; ++l)
          for (int k = 0; k < nzh; ++k) out[(size_t)(l0 + l) * nzh + k] = x[(size_t)k * OR_FB + l];
        continue;
      }
      for (int l = 0; l < nb; ++l) {
        const double *src = in + (size_t)(l0 + l) * nz;
        for (int k = 0; k < nz; ++k) { wa[k].re = src[k]; wa[k].im = 0.0; }
        or_fft_rec(wa, wb, nz, 1, &pz, 1, pz.fac, -1);
        or_cpx *dst = out + (size_t)(l0 + l) * nzh;
        for (int k = 0; k < nzh; ++k) dst[k] = wb[k];
      }
    }
    /* y lines: fixed x, blocks of adjacent kz */
    const long nkb = (nzh + OR_FB - 1) / OR_FB;
#pragma omp for schedule(static)
    for (long blk = 0; blk < (long)nx * nkb / stride; ++blk) {
      const long i = blk / nkb, k0 = (blk % nkb) * OR_FB;
      const int nb = (int)(nzh - k0 < OR_FB ? nzh - k0 : OR_FB);
      or_fft_lines(out + (size_t)i * ny * nzh + k0, 0, nb, 1, nzh, &py, -1, wa, wb);
    }
    /* x lines: blocks of adjacent (y, kz) */
    const long nl = (long)ny * nzh;
#pragma omp for schedule(static)
    for (long blk = 0; blk < (nl + OR_FB - 1) / OR_FB / stride; ++blk) {
      const long l0 = blk * OR_FB;
      const int nb = (int)(nl - l0 < OR_FB ? nl - l0 : OR_FB);
      or_fft_lines(out, l0, nb, 1, (size_t)nl, &px, -1, wa, wb);
    }
    free(wa);
    free(wb);
  }
  or_plan_free(&px);
  or_plan_free(&py);
  or_plan_free(&pz);
}

/* Unnormalised 3-D complex-to-real inverse. Complex transforms along x and y
 * first, then a real inverse along z that, like FFTW's halfcomplex format,
 * uses only the real parts of the k=0 and k=nz/2 coefficients. in is destroyed. */
static void fft_c2r_3d_s(or_cpx *in, double *out, int nx, int ny, int nz, long stride) {
  int nzh = nz / 2 + 1;
  or_fftplan px, py, pz;
  or_plan_init(&px, nx);
  or_plan_init(&py, ny);
  or_plan_init(&pz, nz);
  int nmax = nx > ny ? nx : ny;
  nmax = nmax > nz ? nmax : nz;
#pragma omp parallel
  {
    or_cpx *wa = (or_cpx *)malloc(sizeof(or_cpx) * (size_t)nmax * OR_FB);
    or_cpx *wb = (or_cpx *)malloc(sizeof(or_cpx) * (size_t)nmax * OR_FB);
    const long nl = (long)ny * nzh;
#pragma omp for schedule(static)
    for (long blk = 0; blk < (nl + OR_FB - 1) / OR_FB / stride; ++blk) {
      const long l0 = blk * OR_FB;
      const int nb = (int)(nl - l0 < OR_FB ? nl - l0 : OR_FB);
      or_fft_lines(in, l0, nb, 1, (size_t)nl, &px, +1, wa, wb);
    }
    const long nkb = (nzh + OR_FB - 1) / OR_FB;
#pragma omp for schedule(static)
    for (long blk = 0; blk < (long)nx * nkb / stride; ++blk) {
      const long i = blk / nkb, k0 = (blk % nkb) * OR_FB;
      const int nb = (int)(nzh - k0 < OR_FB ? nzh - k0 : OR_FB);
      or_fft_lines(in + (size_t)i * ny * nzh + k0, 0, nb, 1, nzh, &py, +1, wa, wb);
    }
    const long nzl = (long)nx * ny;
#pragma omp for schedule(static)
    for (long blk = 0; blk < (nzl + OR_FB - 1) / OR_FB / stride; ++blk) {
      const long l0 = blk * OR_FB;
      const int nb = (int)(nzl - l0 < OR_FB ? nzl - l0 : OR_FB);
      if (or_is_pow2(nz)) {
        for (int l = 0; l < OR_FB; ++l) {
          const or_cpx *src = in + (size_t)(l0 + (l < nb ? l : 0)) * nzh;
          wa[l].re = src[0].re;
          wa[l].im = 0.0;
          for (int k = 1; k < nzh; ++k) {
            or_cpx v = src[k];
            if (2 * k == nz) v.im = 0.0;
            else {
              wa[(size_t)(nz - k) * OR_FB + l].re = v.re;
              wa[(size_t)(nz - k) * OR_FB + l].im = -v.im;
            }
            wa[(size_t)k * OR_FB + l] = v;
          }
        }
        or_cpx *x = wa, *y = wb;
        or_fft_block_pow2(&x, &y, nz, &pz, +1);
        for (int l = 0; l < nb; ++l)
          for (int k = 0; k < nz; ++k) out[(size_t)(l0 + l) * nz + k] = x[(size_t)k * OR_FB + l].re;
        continue;
      }
      for (int l = 0; l < nb; ++l) {
        const or_cpx *src = in + (size_t)(l0 + l) * nzh;
        wa[0].re = src[0].re;
        wa[0].im = 0.0;
        for (int k = 1; k < nzh; ++k) {
          wa[k] = src[k];
          if (2 * k == nz) wa[k].im = 0.0;
          else { wa[nz - k].re = src[k].re; wa[nz - k].im = -src[k].im; }
        }
        or_fft_rec(wa, wb, nz, 1, &pz, 1, pz.fac, +1);
        double *dst = out + (size_t)(l0 + l) * nz;
        for (int k = 0; k < nz; ++k) dst[k] = wb[k].re;
      }
    }
    free(wa);
    free(wb);
  }
  or_plan_free(&px);
  or_plan_free(&py);
  or_plan_free(&pz);
}

void or_fft_r2c_3d(const double *in, or_cpx *out, int nx, int ny, int nz) { fft_r2c_3d_s(in, out, nx, ny, nz, 1); }
void or_fft_c2r_3d(or_cpx *in, double *out, int nx, int ny, int nz) { fft_c2r_3d_s(in, out, nx, ny, nz, 1); }

/* ------------------------------------------------------------------------ */
/* FCM: FCMfunctions.cpp                                                    */
/* ------------------------------------------------------------------------ */

/* gaussian_setup for one bead (FCMfunctions.cpp:549-593). */
static void or_gauss_bead(const fs_params *p, const or_consts *c, const double *Yb, double *g, double *gd,
                          double *grad, int *ind) {
  const int N[3] = {p->npts_x, p->npts_y, p->npts_z};
  const double dx = p->dx;
  for (int d = 0; d < 3; ++d) {
    int xc = (int)(Yb[d] / dx);
    for (int i = 0; i < p->ngd; ++i) {
      int xg = xc - c->ngdh + (i + 1);
      ind[d * p->ngd + i] = xg - N[d] * ((int)floor(((double)xg) / ((double)N[d])));
      double xx = ((double)xg) * dx - Yb[d];
      g[d * p->ngd + i] = c->anorm * exp(-xx * xx / c->anorm2);
      gd[d * p->ngd + i] = c->anormdip * exp(-xx * xx / c->anormdip2);
      grad[d * p->ngd + i] = -xx / c->sigmadipsq;
    }
  }
}

/* flow_solve on a real force grid f (3 x nx x ny x nz) into u, with the
 * forward/inverse transforms around it (FCMfunctions.cpp:360-406, 648-736). */
int or_flow_solve(const fs_params *p, const double *f, double *u) {
  const int nx = p->npts_x, ny = p->npts_y, nz = p->npts_z, nzh = nz / 2 + 1;
  const size_t N = (size_t)nx * ny * nz, NH = (size_t)nx * ny * nzh;
  or_cpx *fh = (or_cpx *)malloc(sizeof(or_cpx) * NH * 3);
  if (!fh) return FS_ERR_OOM;
  for (int cpt = 0; cpt < 3; ++cpt) or_fft_r2c_3d(f + cpt * N, fh + cpt * NH, nx, ny, nz);

  /* wavenumbers (FCMfunctions.cpp:129-162) */
  double *qx = (double *)malloc(sizeof(double) * nx), *qy = (double *)malloc(sizeof(double) * ny),
         *qz = (double *)malloc(sizeof(double) * nzh);
  const double TwoPI = 2. * OR_PI;
  const double ffx = TwoPI / (nx * p->dx), ffy = TwoPI / (ny * p->dx), ffz = TwoPI / (nz * p->dx);
  for (int i = 0; i < nx; ++i) qx[i] = (i <= nx / 2) ? i * ffx : (i - nx) * ffx;
  for (int i = 0; i < ny; ++i) qy[i] = (i <= ny / 2) ? i * ffy : (i - ny) * ffy;
  for (int k = 0; k < nzh; ++k) qz[k] = ((double)k) * ffz;

  or_cpx *f1 = fh, *f2 = fh + NH, *f3 = fh + 2 * NH;
  f1[0].re = f1[0].im = 0.0;
  f2[0].re = f2[0].im = 0.0;
  f3[0].re = f3[0].im = 0.0;
  const double totalpts = (double)((long)nx * ny * nz);
  const double smallx = 1e-18;
#pragma omp parallel for schedule(static)
  for (long ij = 0; ij < (long)nx * ny; ++ij) {
    int i = (int)(ij / ny), j = (int)(ij % ny);
    double q1 = qx[i], q2 = qy[j];
    double qq = qy[j] * qy[j] + qx[i] * qx[i] + smallx;
    for (int k = 0; k < nzh; ++k) {
      size_t m = (size_t)ij * nzh + k;
      double q3 = qz[k];
      double norm = 1.0 / (qq + q3 * q3);
      /* real parts, then imaginary parts: the reference applies the same
       * formula to both members of each (re, im) pair (qpad duplicates kz) */
      for (int part = 0; part < 2; ++part) {
        double a1 = part ? f1[m].im : f1[m].re;
        double a2 = part ? f2[m].im : f2[m].re;
        double a3 = part ? f3[m].im : f3[m].re;
        double kdotf = (q1 * a1 + q2 * a2 + q3 * a3) * norm;
        double u1 = norm * (a1 - q1 * (kdotf)) / totalpts;
        double u2 = norm * (a2 - q2 * (kdotf)) / totalpts;
        double u3 = norm * (a3 - q3 * (kdotf)) / totalpts;
        if (part) { f1[m].im = u1; f2[m].im = u2; f3[m].im = u3; }
        else { f1[m].re = u1; f2[m].re = u2; f3[m].re = u3; }
      }
    }
  }
  f1[0].re = f1[0].im = 0.0;
  f2[0].re = f2[0].im = 0.0;
  f3[0].re = f3[0].im = 0.0;
  for (int cpt = 0; cpt < 3; ++cpt) or_fft_c2r_3d(fh + cpt * NH, u + cpt * N, nx, ny, nz);
  free(qx);
  free(qy);
  free(qz);
  free(fh);
  return FS_OK;
}

int or_fcm_mobility(const fs_params *p, int np, const double *Y, const double *F, const double *T, double *V,
                    double *W, double *fgrid, double *ugrid) {
  or_consts c;
  or_consts_init(p, &c);
  const int nx = p->npts_x, ny = p->npts_y, nz = p->npts_z, ngd = p->ngd;
  const size_t N = (size_t)nx * ny * nz;
  double *f = fgrid ? fgrid : (double *)malloc(sizeof(double) * N * 3);
  double *u = ugrid ? ugrid : (double *)malloc(sizeof(double) * N * 3);
  if (!f || !u) return FS_ERR_OOM;
  memset(f, 0, sizeof(double) * N * 3);

  /* gaussian_setup (FCMfunctions.cpp:224-230) and GA_setup (:536-547) */
  double *g = (double *)malloc(sizeof(double) * (size_t)np * 3 * ngd);
  double *gd = (double *)malloc(sizeof(double) * (size_t)np * 3 * ngd);
  double *gr = (double *)malloc(sizeof(double) * (size_t)np * 3 * ngd);
  int *ind = (int *)malloc(sizeof(int) * (size_t)np * 3 * ngd);
  double *GA = (double *)malloc(sizeof(double) * (size_t)np * 6);
#pragma omp parallel for schedule(static)
  for (int b = 0; b < np; ++b) {
    or_gauss_bead(p, &c, Y + 3 * b, g + (size_t)b * 3 * ngd, gd + (size_t)b * 3 * ngd, gr + (size_t)b * 3 * ngd,
                  ind + (size_t)b * 3 * ngd);
    GA[6 * b + 0] = 0.0;
    GA[6 * b + 1] = 0.0;
    GA[6 * b + 2] = 0.0;
    GA[6 * b + 3] = 0.5 * T[3 * b + 2];
    GA[6 * b + 4] = -0.5 * T[3 * b + 1];
    GA[6 * b + 5] = 0.5 * T[3 * b + 0];
  }

  /* mono_and_dipole_force_distribution (FCMfunctions.cpp:596-646). Each
   * thread owns a set of x-planes and walks all beads in order, so every grid
   * point receives its contributions in the reference's bead order. */
  double *fx = f, *fy = f + N, *fz = f + 2 * N;
#pragma omp parallel
  {
    int nth = 1, tid = 0;
#ifdef _OPENMP
    nth = omp_get_num_threads();
    tid = omp_get_thread_num();
#endif
    int x0 = (int)((long)nx * tid / nth), x1 = (int)((long)nx * (tid + 1) / nth);
    for (int b = 0; b < np; ++b) {
      const double *gx = g + (size_t)b * 3 * ngd, *gy = gx + ngd, *gz = gy + ngd;
      const double *dgx = gd + (size_t)b * 3 * ngd, *dgy = dgx + ngd, *dgz = dgy + ngd;
      const double *rx = gr + (size_t)b * 3 * ngd, *ry = rx + ngd, *rz = ry + ngd;
      const int *ix = ind + (size_t)b * 3 * ngd, *iy = ix + ngd, *iz = iy + ngd;
      /* GS = 0 */
      double g11 = 0.0 + GA[6 * b + 0], g22 = 0.0 + GA[6 * b + 1], g33 = 0.0 + GA[6 * b + 2];
      double g12 = 0.0 + GA[6 * b + 3], g21 = 0.0 - GA[6 * b + 3];
      double g13 = 0.0 + GA[6 * b + 4], g31 = 0.0 - GA[6 * b + 4];
      double g23 = 0.0 + GA[6 * b + 5], g32 = 0.0 - GA[6 * b + 5];
      const double F0 = F[3 * b], F1 = F[3 * b + 1], F2 = F[3 * b + 2];
      for (int i = 0; i < ngd; ++i) {
        int ii = ix[i];
        if (ii < x0 || ii >= x1) continue;
        double xx = rx[i];
        for (int j = 0; j < ngd; ++j) {
          int jj = iy[j];
          double yy = ry[j];
          for (int k = 0; k < ngd; ++k) {
            int kk = iz[k];
            double zz = rz[k];
            double temp = gx[i] * gy[j] * gz[k];
            double temp2 = dgx[i] * dgy[j] * dgz[k];
            size_t m = ((size_t)ii * ny + jj) * nz + kk;
            fx[m] = fx[m] + F0 * temp + (g11 * xx + g12 * yy + g13 * zz) * temp2;
            fy[m] = fy[m] + F1 * temp + (g21 * xx + g22 * yy + g23 * zz) * temp2;
            fz[m] = fz[m] + F2 * temp + (g31 * xx + g32 * yy + g33 * zz) * temp2;
          }
        }
      }
    }
  }

  int st = or_flow_solve(p, f, u);
  if (st) return st;

  /* particle_velocities (FCMfunctions.cpp:740-770) and particle_rotations
   * (:774-808) */
  const double *ux = u, *uy = u + N, *uz = u + 2 * N;
  const double norm = p->dx * p->dx * p->dx;
#pragma omp parallel for schedule(static)
  for (int b = 0; b < np; ++b) {
    const double *gx = g + (size_t)b * 3 * ngd, *gy = gx + ngd, *gz = gy + ngd;
    const double *dgx = gd + (size_t)b * 3 * ngd, *dgy = dgx + ngd, *dgz = dgy + ngd;
    const double *rx = gr + (size_t)b * 3 * ngd, *ry = rx + ngd, *rz = ry + ngd;
    const int *ix = ind + (size_t)b * 3 * ngd, *iy = ix + ngd, *iz = iy + ngd;
    double v0 = 0, v1 = 0, v2 = 0;
    for (int i = 0; i < ngd; ++i) {
      int ii = ix[i];
      for (int j = 0; j < ngd; ++j) {
        int jj = iy[j];
        for (int k = 0; k < ngd; ++k) {
          int kk = iz[k];
          size_t m = ((size_t)ii * ny + jj) * nz + kk;
          double temp = gx[i] * gy[j] * gz[k] * norm;
          v0 = v0 + ux[m] * temp;
          v1 = v1 + uy[m] * temp;
          v2 = v2 + uz[m] * temp;
        }
      }
    }
    double w0 = 0, w1 = 0, w2 = 0;
    for (int i = 0; i < ngd; ++i) {
      int ii = ix[i];
      double xx = rx[i];
      for (int j = 0; j < ngd; ++j) {
        int jj = iy[j];
        double yy = ry[j];
        for (int k = 0; k < ngd; ++k) {
          int kk = iz[k];
          double zz = rz[k];
          size_t m = ((size_t)ii * ny + jj) * nz + kk;
          double temp = dgx[i] * dgy[j] * dgz[k] * norm;
          w0 = w0 - 0.5 * (uz[m] * yy - uy[m] * zz) * temp;
          w1 = w1 - 0.5 * (ux[m] * zz - uz[m] * xx) * temp;
          w2 = w2 - 0.5 * (uy[m] * xx - ux[m] * yy) * temp;
        }
      }
    }
    V[3 * b] = v0; V[3 * b + 1] = v1; V[3 * b + 2] = v2;
    W[3 * b] = w0; W[3 * b + 1] = w1; W[3 * b + 2] = w2;
  }
  free(g); free(gd); free(gr); free(ind); free(GA);
  if (!fgrid) free(f);
  if (!ugrid) free(u);
  return FS_OK;
}

/* Fcm::friction_mobility_solve (FCMfunctions.cpp:865-880) */
void or_fcm_friction(const fs_params *p, int np, const double *F, const double *T, double *V, double *W) {
  double a = p->a, mu = p->mu;
  double a1 = 1. / (6 * OR_PI * a * mu);
  double a2 = 1. / (8 * OR_PI * a * a * a * mu);
  for (int b = 0; b < np; ++b) {
    for (int d = 0; d < 3; ++d) {
      V[3 * b + d] = a1 * F[3 * b + d];
      W[3 * b + d] = a2 * T[3 * b + d];
    }
  }
}

/* ------------------------------------------------------------------------ */
/* cells + barrier: CollisionBarrierFilament.cpp                             */
/* ------------------------------------------------------------------------ */

/* LinkedList::initialise cell counts (CollisionBarrierFilament.cpp:277-281) */
void or_cells_dims(const fs_params *p, int *M) {
  double Rref = p->cell_width;
  M[0] = (int)((p->npts_x * p->dx) / Rref);
  M[1] = (int)((p->npts_y * p->dx) / Rref);
  M[2] = (int)((p->npts_z * p->dx) / Rref);
}

/* LinkedList::icell (CollisionBarrierFilament.cpp:307-315) */
static int or_icell(const int *M, int x, int y, int z) {
  double cellix = (double)M[0], celliy = (double)M[1];
  double beta = fmod((double)(x + M[0]), (double)M[0]) + fmod((double)(y + M[1]), (double)M[1]) * cellix +
                fmod((double)(z + M[2]), (double)M[2]) * cellix * celliy;
  return (int)beta;
}

/* LinkedList::bulkmap (CollisionBarrierFilament.cpp:318-343) */
void or_cells_bulkmap(const int *M, int *map) {
  for (int iz = 0; iz < M[2]; iz++)
    for (int iy = 0; iy < M[1]; iy++)
      for (int ix = 0; ix < M[0]; ix++) {
        int imap = or_icell(M, ix, iy, iz) * 13;
        map[imap] = or_icell(M, ix + 1, iy, iz);
        map[imap + 1] = or_icell(M, ix + 1, iy + 1, iz);
        map[imap + 2] = or_icell(M, ix, iy + 1, iz);
        map[imap + 3] = or_icell(M, ix - 1, iy + 1, iz);
        map[imap + 4] = or_icell(M, ix + 1, iy, iz - 1);
        map[imap + 5] = or_icell(M, ix + 1, iy + 1, iz - 1);
        map[imap + 6] = or_icell(M, ix, iy + 1, iz - 1);
        map[imap + 7] = or_icell(M, ix - 1, iy + 1, iz - 1);
        map[imap + 8] = or_icell(M, ix + 1, iy, iz + 1);
        map[imap + 9] = or_icell(M, ix + 1, iy + 1, iz + 1);
        map[imap + 10] = or_icell(M, ix, iy + 1, iz + 1);
        map[imap + 11] = or_icell(M, ix - 1, iy + 1, iz + 1);
        map[imap + 12] = or_icell(M, ix, iy, iz + 1);
      }
}

/* cell index of one unwrapped position (CollisionBarrierFilament.cpp:387-409);
 * the per-axis cell coordinate is clamped into [0, M) where the reference
 * would index out of range for a coordinate that rounds up to the box edge. */
static int or_cell_of(const double *L, const int *M, const double *x) {
  const int large_number = 100000;
  int cidx[3];
  for (int d = 0; d < 3; ++d) {
    double xr = x[d] - L[d] * ((double)((int)(x[d] / L[d] + large_number) - large_number));
    int cc = (int)((xr / L[d]) * (double)M[d]);
    if (cc >= M[d]) cc = M[d] - 1;
    if (cc < 0) cc = 0;
    cidx[d] = cc;
  }
  return cidx[0] + cidx[1] * M[0] + cidx[2] * M[0] * M[1];
}

/* LinkedList::link (CollisionBarrierFilament.cpp:370-433) */
void or_cells_link(const fs_params *p, int np, const double *Xs, int *head, int *list) {
  int M[3];
  or_cells_dims(p, M);
  double L[3] = {p->npts_x * p->dx, p->npts_y * p->dx, p->npts_z * p->dx};
  int ncell = M[0] * M[1] * M[2];
  for (int i = 0; i < ncell; i++) head[i] = -1;
  for (int g = 0; g < np; ++g) {
    int index = or_cell_of(L, M, Xs + 3 * g);
    list[g] = head[index];
    head[index] = g;
  }
}

/* one pair interaction as in CollisionBarrierFilament.cpp:80-149 */
static int or_pair(const fs_params *p, const double *L, const double *Yi, const double *Yj, double *Fx,
                   double *min_dist2) {
  const double Rnm = 2 * p->a;
  const double Rnm2 = Rnm * Rnm;
  const double chiRnm2 = 1.21 * Rnm2;
  const double FS_over_2a = p->barrier_fs_over_2a;
  const double cap = p->barrier_distance_cap, cap2 = cap * cap;
  double xij = Yi[0] - Yj[0], yij = Yi[1] - Yj[1], zij = Yi[2] - Yj[2];
  xij = xij - L[0] * floor(xij / L[0] + 0.5);
  yij = yij - L[1] * floor(yij / L[1] + 0.5);
  zij = zij - L[2] * floor(zij / L[2] + 0.5);
  double rijsq = xij * xij + yij * yij + zij * zij;
  if (rijsq < *min_dist2) *min_dist2 = rijsq;
  if (rijsq < chiRnm2) {
    if (rijsq < cap2) {
      double rij = sqrt(rijsq);
      xij = xij / rij * cap;
      yij = yij / rij * cap;
      zij = zij / rij * cap;
      rijsq = cap2;
    }
    double prefac = chiRnm2 - rijsq;
    prefac /= (chiRnm2 - Rnm2);
    prefac *= prefac;
    prefac *= prefac;
    prefac *= FS_over_2a;
    Fx[0] = prefac * xij;
    Fx[1] = prefac * yij;
    Fx[2] = prefac * zij;
    return 1;
  }
  return 0;
}

/* LinkedList::apply_collision_barrier (CollisionBarrierFilament.cpp:24-271),
 * one rank: F_total = F_on_node, added into F. Returns the pair count; the
 * first max_pairs pairs (i, j) are written to pairs in visiting order. */
/* pair filter of the barrier variants (CollisionBarrierFilament.cpp:57, :474-477, :754) */
static int or_pair_on(int mode, int np, int nt, int ifs, int i, int i_fil, int i_seg, int j, int j_fil, int j_seg) {
  const int base = !(j_fil == i_fil && abs(j_seg - i_seg) == 1) || nt < ifs;
  if (mode == FS_BARRIER_NOT_SWIMMER) return ((i_fil == 0) == (j_fil == 0)) && base;
  if (mode == FS_BARRIER_NOT_TEST_PARTICLES) return base && (i < np - 2 && j < np - 2);
  return base;
}

static int or_collision_barrier_mode(const fs_params *p, int np, const int *fil_id, const int *seg_id,
                                     const double *Y, const int *head, const int *list, const int *map, int nt,
                                     double *F, double *min_dist2_out, int *pairs, int max_pairs, int mode);

int or_collision_barrier(const fs_params *p, int np, const int *fil_id, const int *seg_id, const double *Y,
                         const int *head, const int *list, const int *map, int nt, double *F, double *min_dist2_out,
                         int *pairs, int max_pairs) {
  return or_collision_barrier_mode(p, np, fil_id, seg_id, Y, head, list, map, nt, F, min_dist2_out, pairs,
                                   max_pairs, FS_BARRIER_ALL);
}

static int or_collision_barrier_mode(const fs_params *p, int np, const int *fil_id, const int *seg_id,
                                     const double *Y, const int *head, const int *list, const int *map, int nt,
                                     double *F, double *min_dist2_out, int *pairs, int max_pairs, int mode) {
  int M[3];
  or_cells_dims(p, M);
  int ncell = M[0] * M[1] * M[2];
  double L[3] = {p->npts_x * p->dx, p->npts_y * p->dx, p->npts_z * p->dx};
  double *Fon = (double *)calloc((size_t)np * 3, sizeof(double));
  double min_dist2 = 100000;
  int npairs = 0;
  double Fij[3];
  for (int icell = 0; icell < ncell; icell++) {
    int i = head[icell];
    while (i > -1) {
      int i_fil = fil_id[i], i_seg = seg_id[i];
      double fxi = Fon[3 * i], fyi = Fon[3 * i + 1], fzi = Fon[3 * i + 2];
      for (int nabor = -1; nabor < 13; ++nabor) {
        int j = (nabor < 0) ? list[i] : head[map[13 * icell + nabor]];
        while (j > -1) {
          int j_fil = fil_id[j], j_seg = seg_id[j];
          if (or_pair_on(mode, np, nt, p->initial_friction_steps, i, i_fil, i_seg, j, j_fil, j_seg)) {
            if (or_pair(p, L, Y + 3 * i, Y + 3 * j, Fij, &min_dist2)) {
              fxi += Fij[0];
              fyi += Fij[1];
              fzi += Fij[2];
              Fon[3 * j] -= Fij[0];
              Fon[3 * j + 1] -= Fij[1];
              Fon[3 * j + 2] -= Fij[2];
              if (pairs && npairs < max_pairs) {
                pairs[2 * npairs] = i;
                pairs[2 * npairs + 1] = j;
              }
              npairs++;
            }
          }
          j = list[j];
        }
      }
      Fon[3 * i] = fxi;
      Fon[3 * i + 1] = fyi;
      Fon[3 * i + 2] = fzi;
      i = list[i];
    }
  }
  for (int i = 0; i < 3 * np; ++i) F[i] += Fon[i];
  if (min_dist2_out) *min_dist2_out = min_dist2;
  free(Fon);
  return npairs;
}

/* ------------------------------------------------------------------------ */
/* quaternion helpers: UnitQuaternion.hpp                                   */
/* ------------------------------------------------------------------------ */
typedef struct { double s, v[3]; } or_quat;

static void q_load(or_quat *q, const double *a) { q->s = a[0]; q->v[0] = a[1]; q->v[1] = a[2]; q->v[2] = a[3]; }
static void q_store(const or_quat *q, double *a) { a[0] = q->s; a[1] = q->v[0]; a[2] = q->v[1]; a[3] = q->v[2]; }
static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void cross3(const double *a, const double *b, double *c) {
  double c0 = a[1] * b[2] - a[2] * b[1], c1 = a[2] * b[0] - a[0] * b[2], c2 = a[0] * b[1] - a[1] * b[0];
  c[0] = c0; c[1] = c1; c[2] = c2;
}
static double norm3(const double *a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

/* expmInPlace (UnitQuaternion.hpp:227-242): q <- (cos(t/2), sin(t/2)/t v) * q */
static void q_expm_inplace(or_quat *q, const double *v) {
  double theta = norm3(v);
  if (theta > 1.e-12) {
    double tmp = sin(theta * .5) / theta;
    or_quat p;
    p.s = cos(theta * .5);
    p.v[0] = tmp * v[0]; p.v[1] = tmp * v[1]; p.v[2] = tmp * v[2];
    /* quaproFromLeftInPlace (:141-147): this = p * this */
    double scal_tmp = q->s * p.s - dot3(q->v, p.v);
    double t[3];
    cross3(p.v, q->v, t);
    double nv[3];
    for (int d = 0; d < 3; ++d) nv[d] = q->s * p.v[d] + p.s * q->v[d] + t[d];
    q->v[0] = nv[0]; q->v[1] = nv[1]; q->v[2] = nv[2];
    q->s = scal_tmp;
  }
}

/* assignTangentVec / NormalVec / BinormalVec (UnitQuaternion.hpp:341-378) */
static void q_tangent(const or_quat *q, double *v) {
  double q22 = 2 * q->v[1] * q->v[1], q33 = 2 * q->v[2] * q->v[2];
  v[0] = (1 - q22 - q33);
  v[1] = 2 * (q->v[0] * q->v[1] + q->s * q->v[2]);
  v[2] = 2 * (q->v[0] * q->v[2] - q->s * q->v[1]);
}
static void q_normal(const or_quat *q, double *v) {
  double q11 = 2 * q->v[0] * q->v[0], q33 = 2 * q->v[2] * q->v[2];
  v[0] = 2 * (q->v[0] * q->v[1] - q->s * q->v[2]);
  v[1] = (1 - q11 - q33);
  v[2] = 2 * (q->v[1] * q->v[2] + q->s * q->v[0]);
}
static void q_binormal(const or_quat *q, double *v) {
  double q11 = 2 * q->v[0] * q->v[0], q22 = 2 * q->v[1] * q->v[1];
  v[0] = 2 * (q->v[0] * q->v[2] + q->s * q->v[1]);
  v[1] = 2 * (q->v[1] * q->v[2] - q->s * q->v[0]);
  v[2] = (1 - q11 - q22);
}
/* RotateVector (UnitQuaternion.hpp:323-338) */
static void q_rotate(const or_quat *q, double *v) {
  double vx = v[0], vy = v[1], vz = v[2];
  const double *e = q->v;
  double s = q->s;
  double q11 = 2 * e[0] * e[0], q22 = 2 * e[1] * e[1], q33 = 2 * e[2] * e[2];
  v[0] = (1 - q22 - q33) * vx + 2 * (e[0] * e[1] - s * e[2]) * vy + 2 * (e[0] * e[2] + s * e[1]) * vz;
  v[1] = 2 * (e[0] * e[1] + s * e[2]) * vx + (1 - q11 - q33) * vy + 2 * (e[1] * e[2] - s * e[0]) * vz;
  v[2] = 2 * (e[0] * e[2] - s * e[1]) * vx + 2 * (e[1] * e[2] + s * e[0]) * vy + (1 - q11 - q22) * vz;
}
/* assignMidPointOf (UnitQuaternion.hpp:472-489) with quaSquareRootTimInPlace (:411-421) */
static void q_midpoint(const or_quat *p1, const or_quat *p2, or_quat *out) {
  /* p2.quaproConj(p1) (:108-110) */
  or_quat m;
  m.s = p2->s * p1->s + dot3(p2->v, p1->v);
  double cr[3];
  cross3(p2->v, p1->v, cr);
  for (int d = 0; d < 3; ++d) m.v[d] = -p2->s * p1->v[d] + p1->s * p2->v[d] - cr[d];
  if (m.s < -.9999999999999) {
    m.s = 0.;
    m.v[0] = 0.; m.v[1] = 0.; m.v[2] = 1.;
  } else {
    m.s = sqrt(0.5 * (m.s + 1.));
    for (int d = 0; d < 3; ++d) m.v[d] /= (2. * m.s);
  }
  /* quaproInPlace(p1) (:123-129): m = m * p1 */
  double scal_tmp = m.s * p1->s - dot3(m.v, p1->v);
  double t[3];
  cross3(m.v, p1->v, t);
  for (int d = 0; d < 3; ++d) out->v[d] = m.s * p1->v[d] + p1->s * m.v[d] + t[d];
  out->s = scal_tmp;
}

/* dexpinv (MobilityConstraints.cpp:109-143) */
static void or_dexpinv(const double *u, const double *w, double *out) {
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

/* ------------------------------------------------------------------------ */
/* filament suspension                                                      */
/* ------------------------------------------------------------------------ */
struct or_system {
  fs_params p;
  or_consts c;
  int nfil, np, nlink;
  int *fil_start, *fil_id, *seg_id;
  double *X, *Xs, *Xt, *U, *Us, *Ut, *q, *qs, *qt, *F, *TAU, *lam, *lam1, *lam2, *kap, *cc, *radius;
  double *Y, *V, *W;
  double *Err, *NewErr, *Upd, *tmp, *dE;
  double *Cmat, *Dmat;
  double *Jinv;
  size_t *joff;
  int M[3];
  int *head, *list, *map;
  double min_dist2;
  long long nsolves;
  /* swimming drive: per filament (alpha, beta, phase, wavenumber, angular
   * frequency), or NULL; spring links: bead pairs (global indices) */
  double *swim, swim_curvature;
  int swim_sperm_decay;
  int nspring;
  int *spring_beads;
  double spring_k, spring_l0;
  int barrier_mode;
  /* CPU-baseline workspace (or_stage_costs): grids and Gaussian tables, kept
   * across calls so their pages are touched once */
  double *wf, *wu, *wg, *wgd, *wgr;
  or_cpx *wfh;
  int *wind;
};

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

or_system *or_system_create(const fs_params *p, const fs_host_state *s) {
  or_system *sys = (or_system *)calloc(1, sizeof(or_system));
  sys->p = *p;
  or_consts_init(p, &sys->c);
  sys->nfil = s->nfil;
  sys->np = s->np;
  sys->nlink = s->np - s->nfil;
  int np = s->np, nf = s->nfil;
  sys->fil_start = (int *)malloc(sizeof(int) * (nf + 1));
  memcpy(sys->fil_start, s->fil_start, sizeof(int) * (nf + 1));
  sys->fil_id = (int *)malloc(sizeof(int) * np);
  sys->seg_id = (int *)malloc(sizeof(int) * np);
  sys->radius = dalloc(np);
  for (int f = 0; f < nf; ++f)
    for (int b = sys->fil_start[f]; b < sys->fil_start[f + 1]; ++b) {
      sys->fil_id[b] = f;
      sys->seg_id[b] = b - sys->fil_start[f];
      sys->radius[b] = (b == sys->fil_start[f]) ? p->ah : p->a;
    }
  sys->X = dalloc(3 * np); sys->Xs = dalloc(3 * np); sys->Xt = dalloc(3 * np);
  sys->U = dalloc(3 * np); sys->Us = dalloc(3 * np); sys->Ut = dalloc(3 * np);
  sys->q = dalloc(4 * np); sys->qs = dalloc(4 * np); sys->qt = dalloc(4 * np);
  sys->F = dalloc(3 * np); sys->TAU = dalloc(3 * np);
  sys->lam = dalloc(3 * sys->nlink); sys->lam1 = dalloc(3 * sys->nlink); sys->lam2 = dalloc(3 * sys->nlink);
  sys->kap = dalloc(nf); sys->cc = dalloc(nf);
  sys->Y = dalloc(3 * np); sys->V = dalloc(3 * np); sys->W = dalloc(3 * np);
  sys->Err = dalloc(6 * np); sys->NewErr = dalloc(6 * np); sys->Upd = dalloc(6 * np);
  sys->tmp = dalloc(6 * np); sys->dE = dalloc(6 * np);
  sys->Cmat = dalloc((size_t)6 * np * p->broyden_maxiter);
  sys->Dmat = dalloc((size_t)6 * np * p->broyden_maxiter);
  sys->joff = (size_t *)malloc(sizeof(size_t) * (nf + 1));
  sys->joff[0] = 0;
  for (int f = 0; f < nf; ++f) {
    size_t n = 6 * (size_t)(sys->fil_start[f + 1] - sys->fil_start[f]);
    sys->joff[f + 1] = sys->joff[f] + n * n;
  }
  sys->Jinv = dalloc(sys->joff[nf]);
  or_cells_dims(p, sys->M);
  int ncell = sys->M[0] * sys->M[1] * sys->M[2];
  sys->head = (int *)malloc(sizeof(int) * ncell);
  sys->list = (int *)malloc(sizeof(int) * np);
  sys->map = (int *)malloc(sizeof(int) * 13 * ncell);
  or_cells_bulkmap(sys->M, sys->map);
  sys->min_dist2 = 100000;
  or_system_set(sys, s);
  return sys;
}

void or_system_destroy(or_system *s) {
  if (!s) return;
  void *ptrs[] = {s->fil_start, s->fil_id, s->seg_id, s->radius, s->X, s->Xs, s->Xt, s->U, s->Us, s->Ut,
                  s->q, s->qs, s->qt, s->F, s->TAU, s->lam, s->lam1, s->lam2, s->kap, s->cc, s->Y, s->V,
                  s->W, s->Err, s->NewErr, s->Upd, s->tmp, s->dE, s->Cmat, s->Dmat, s->joff, s->Jinv,
                  s->head, s->list, s->map, s->swim, s->spring_beads, s->wf, s->wu, s->wfh, s->wg, s->wgd,
                  s->wgr, s->wind};
  for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
  free(s);
}

#define OR_COPY(dst, src, n) do { if ((src) && (dst)) memcpy((dst), (src), sizeof(double) * (size_t)(n)); } while (0)

void or_system_set(or_system *sys, const fs_host_state *s) {
  int np = sys->np, nl = sys->nlink, nf = sys->nfil;
  OR_COPY(sys->X, s->X, 3 * np); OR_COPY(sys->Xs, s->Xs, 3 * np); OR_COPY(sys->Xt, s->Xt, 3 * np);
  OR_COPY(sys->U, s->U, 3 * np); OR_COPY(sys->Us, s->Us, 3 * np); OR_COPY(sys->Ut, s->Ut, 3 * np);
  OR_COPY(sys->q, s->q, 4 * np); OR_COPY(sys->qs, s->qs, 4 * np); OR_COPY(sys->qt, s->qt, 4 * np);
  OR_COPY(sys->F, s->F, 3 * np); OR_COPY(sys->TAU, s->TAU, 3 * np);
  OR_COPY(sys->lam, s->lam, 3 * nl); OR_COPY(sys->lam1, s->lam1, 3 * nl); OR_COPY(sys->lam2, s->lam2, 3 * nl);
  OR_COPY(sys->kap, s->kap, nf); OR_COPY(sys->cc, s->c, nf);
}

void or_system_get(or_system *sys, fs_host_state *s) {
  int np = sys->np, nl = sys->nlink, nf = sys->nfil;
  OR_COPY(s->X, sys->X, 3 * np); OR_COPY(s->Xs, sys->Xs, 3 * np); OR_COPY(s->Xt, sys->Xt, 3 * np);
  OR_COPY(s->U, sys->U, 3 * np); OR_COPY(s->Us, sys->Us, 3 * np); OR_COPY(s->Ut, sys->Ut, 3 * np);
  OR_COPY(s->q, sys->q, 4 * np); OR_COPY(s->qs, sys->qs, 4 * np); OR_COPY(s->qt, sys->qt, 4 * np);
  OR_COPY(s->F, sys->F, 3 * np); OR_COPY(s->TAU, sys->TAU, 3 * np);
  OR_COPY(s->lam, sys->lam, 3 * nl); OR_COPY(s->lam1, sys->lam1, 3 * nl); OR_COPY(s->lam2, sys->lam2, 3 * nl);
  OR_COPY(s->kap, sys->kap, nf); OR_COPY(s->c, sys->cc, nf);
}

double *or_system_array(or_system *sys, const char *w) {
  if (!strcmp(w, "Y")) return sys->Y;
  if (!strcmp(w, "V")) return sys->V;
  if (!strcmp(w, "W")) return sys->W;
  if (!strcmp(w, "F")) return sys->F;
  if (!strcmp(w, "TAU")) return sys->TAU;
  if (!strcmp(w, "Xs")) return sys->Xs;
  if (!strcmp(w, "Us")) return sys->Us;
  if (!strcmp(w, "qs")) return sys->qs;
  if (!strcmp(w, "err")) return sys->Err;
  if (!strcmp(w, "update")) return sys->Upd;
  if (!strcmp(w, "lam")) return sys->lam;
  return NULL;
}

/* Filament::initialGuess (Filament.hpp:227-237; Bead.hpp:202-217) */
void or_initial_guess(or_system *s) {
  for (int f = 0; f < s->nfil; ++f) {
    for (int b = s->fil_start[f]; b < s->fil_start[f + 1]; ++b) {
      if (b == s->fil_start[f])
        for (int d = 0; d < 3; ++d) s->Xs[3 * b + d] = 2. * s->X[3 * b + d] - s->Xt[3 * b + d];
      for (int d = 0; d < 3; ++d) s->Us[3 * b + d] = 2. * s->U[3 * b + d] - s->Ut[3 * b + d];
      or_quat q;
      q_load(&q, s->q + 4 * b);
      q_expm_inplace(&q, s->Us + 3 * b);
      q_store(&q, s->qs + 4 * b);
    }
  }
}

void or_set_swimming(or_system *s, const double *swim, double curvature, int sperm_decay) {
  free(s->swim);
  s->swim = NULL;
  if (swim) {
    s->swim = dalloc(5 * (size_t)s->nfil);
    memcpy(s->swim, swim, sizeof(double) * 5 * (size_t)s->nfil);
  }
  s->swim_curvature = curvature;
  s->swim_sperm_decay = sperm_decay;
}

void or_set_spring_links(or_system *s, int nlinks, const int *beads, double k, double l0) {
  free(s->spring_beads);
  s->spring_beads = NULL;
  s->nspring = nlinks > 0 ? nlinks : 0;
  if (s->nspring) {
    s->spring_beads = (int *)malloc(sizeof(int) * 2 * (size_t)nlinks);
    memcpy(s->spring_beads, beads, sizeof(int) * 2 * (size_t)nlinks);
  }
  s->spring_k = k;
  s->spring_l0 = l0;
}

/* Strain twist of link i of filament f at time tt (Filament.hpp:297-326):
 * component 0 is the constant STRAINTWISTZ; components 1 and 2 are set on every
 * link by the swimming drive (zero for a filament without it, since Alpha and
 * Beta are zero). */
static void or_link_strain_twist(const or_system *s, int f, int nw, int i, double tt, double *st) {
  const double dL = s->p.dl;
  st[0] = s->p.strain_twist[0];
  st[1] = 0.0;
  st[2] = 0.0;
  if (!s->swim) return;
  const double *sw = s->swim + 5 * f;
  const double L_filament = (nw - 1) * dL, L_filament_long = nw * dL;
  const double T0 = (s->swim_curvature / L_filament_long);
  const double sarc = dL * i + .5 * dL;
  double facPref;
  if (s->swim_sperm_decay) {
    if (sarc > L_filament / 2.0)
      facPref = T0 * 2.0 * (L_filament - sarc) / L_filament;
    else
      facPref = T0;
  } else {
    facPref = T0 * (L_filament - sarc) / L_filament;
  }
  const double arg = sw[3] * sarc - sw[4] * tt + sw[2];
  st[1] = sw[1] * facPref * cos(arg);
  st[2] = sw[0] * facPref * sin(arg);
}

/* unRobotArmify (Filament.hpp:489-505), setZeroForcesTorques (:271-277),
 * applyElasticTorques (:289-342), applyConstraintForcesTorques (:345-370),
 * applyExternalForcesTorques (:379-402), the spring links
 * (spring_link_functions.cpp:24-45, main.cpp:354-357), then
 * assign_filament_data (FCMfunctions.cpp:882-918). */
void or_filament_forces(or_system *s, int nt) {
  const double tt = nt * s->p.dt;
  const fs_params *p = &s->p;
  const double dL = p->dl, oneOverDL = 1. / p->dl;
  for (int f = 0; f < s->nfil; ++f) {
    int b0 = s->fil_start[f], nw = s->fil_start[f + 1] - b0, l0 = b0 - f;
    /* unRobotArmify */
    double Xsum[3], t1[3], t2[3];
    or_quat q;
    for (int d = 0; d < 3; ++d) Xsum[d] = s->Xs[3 * b0 + d];
    q_load(&q, s->qs + 4 * b0);
    q_tangent(&q, t1);
    for (int i = 1; i < nw; ++i) {
      q_load(&q, s->qs + 4 * (b0 + i));
      q_tangent(&q, t2);
      for (int d = 0; d < 3; ++d) {
        Xsum[d] += (t1[d] + t2[d]) * (0.5 * dL);
        s->Xs[3 * (b0 + i) + d] = Xsum[d];
      }
      for (int d = 0; d < 3; ++d) t1[d] = t2[d];
    }
    /* setZeroForcesTorques */
    for (int i = 0; i < nw; ++i)
      for (int d = 0; d < 3; ++d) { s->F[3 * (b0 + i) + d] = 0.0; s->TAU[3 * (b0 + i) + d] = 0.0; }
    /* applyElasticTorques, with the swimming drive's strain twist per link */
    for (int i = 0; i < nw - 1; ++i) {
      double st[3];
      or_link_strain_twist(s, f, nw, i, tt, st);
      int j = i + 1;
      or_quat qi, qj, qm;
      q_load(&qi, s->qs + 4 * (b0 + i));
      q_load(&qj, s->qs + 4 * (b0 + j));
      q_midpoint(&qi, &qj, &qm);
      or_quat q2 = qj;
      q2.s -= qi.s;
      for (int d = 0; d < 3; ++d) q2.v[d] -= qi.v[d];
      q2.s *= oneOverDL;
      for (int d = 0; d < 3; ++d) q2.v[d] *= oneOverDL;
      /* quaproFromLeftInPlaceConj(q_mid) (:150-157): q2 = conj(qm) * q2 */
      double scal_tmp = q2.s * qm.s + dot3(q2.v, qm.v);
      double tt[3];
      cross3(q2.v, qm.v, tt);
      double nv[3];
      for (int d = 0; d < 3; ++d) nv[d] = -q2.s * qm.v[d] + qm.s * q2.v[d] + tt[d];
      double vtmp[3];
      for (int d = 0; d < 3; ++d) vtmp[d] = 2. * nv[d] - st[d];
      (void)scal_tmp;
      vtmp[0] *= s->cc[f];
      vtmp[1] *= s->kap[f];
      vtmp[2] *= s->kap[f];
      q_rotate(&qm, vtmp);
      for (int d = 0; d < 3; ++d) {
        s->TAU[3 * (b0 + i) + d] += vtmp[d];
        s->TAU[3 * (b0 + j) + d] -= vtmp[d];
      }
    }
    /* applyConstraintForcesTorques */
    const double fac = -.5 * dL;
    for (int i = 0; i < nw - 1; ++i) {
      int j = i + 1;
      const double *lm = s->lam + 3 * (l0 + i);
      for (int d = 0; d < 3; ++d) {
        s->F[3 * (b0 + i) + d] -= lm[d];
        s->F[3 * (b0 + j) + d] += lm[d];
      }
      double tan_tmp[3], c2[3];
      or_quat qq;
      q_load(&qq, s->qs + 4 * (b0 + i));
      q_tangent(&qq, tan_tmp);
      cross3(tan_tmp, lm, c2);
      for (int d = 0; d < 3; ++d) s->TAU[3 * (b0 + i) + d] += fac * c2[d];
      q_load(&qq, s->qs + 4 * (b0 + j));
      q_tangent(&qq, tan_tmp);
      cross3(tan_tmp, lm, c2);
      for (int d = 0; d < 3; ++d) s->TAU[3 * (b0 + j) + d] += fac * c2[d];
    }
    /* applyExternalForcesTorques (gravity per bead) */
    for (int i = 0; i < nw; ++i)
      for (int d = 0; d < 3; ++d) s->F[3 * (b0 + i) + d] += p->gravity[d];
  }
  const double L[3] = {s->c.Lx, s->c.Ly, s->c.Lz};
  /* apply_spring_link_forces, links in order: minimum-image displacement
   * (VecPeriodicX, spring_link_functions.cpp:139-145), Hookean force along it */
  for (int l = 0; l < s->nspring; ++l) {
    const int bn = s->spring_beads[2 * l], bm = s->spring_beads[2 * l + 1];
    double disp[3];
    for (int d = 0; d < 3; ++d) {
      disp[d] = s->Xs[3 * bn + d] - s->Xs[3 * bm + d];
      disp[d] = disp[d] - L[d] * floor(disp[d] / L[d] + 0.5);
    }
    const double dist = sqrt(disp[0] * disp[0] + disp[1] * disp[1] + disp[2] * disp[2]);
    const double spring_mag = s->spring_k * (dist - s->spring_l0);
    for (int d = 0; d < 3; ++d) {
      const double sf = -spring_mag * disp[d] / dist;
      s->F[3 * bn + d] += sf;
      s->F[3 * bm + d] -= sf;
    }
  }
  /* assign_filament_data: Y = fmod(Xs, L) */
  for (int b = 0; b < s->np; ++b)
    for (int d = 0; d < 3; ++d) s->Y[3 * b + d] = fmod(s->Xs[3 * b + d], L[d]);
}

/* ---- 3x3 helpers for the Jacobian blocks (row-major) ---- */
typedef struct { double m[9]; } m3;
static m3 m3_zero(void) { m3 r; memset(r.m, 0, sizeof r.m); return r; }
/* rcross (Filament.hpp:870-881): A v = cross(v, x) */
static m3 rcross(const double *x) {
  m3 r;
  r.m[0] = 0.; r.m[1] = x[2]; r.m[2] = -x[1];
  r.m[3] = -x[2]; r.m[4] = 0.; r.m[5] = x[0];
  r.m[6] = x[1]; r.m[7] = -x[0]; r.m[8] = 0.;
  return r;
}
static m3 m3_t(m3 a) { m3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[3 * i + j] = a.m[3 * j + i]; return r; }
static m3 m3_mul(m3 a, m3 b) {
  m3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc += a.m[3 * i + k] * b.m[3 * k + j];
      r.m[3 * i + j] = acc;
    }
  return r;
}
static m3 m3_add(m3 a, m3 b) { for (int i = 0; i < 9; ++i) a.m[i] += b.m[i]; return a; }
static m3 m3_sub(m3 a, m3 b) { for (int i = 0; i < 9; ++i) a.m[i] -= b.m[i]; return a; }
static m3 m3_scale(m3 a, double s) { for (int i = 0; i < 9; ++i) a.m[i] *= s; return a; }
static void m3_vec(m3 a, const double *v, double *out) {
  for (int i = 0; i < 3; ++i) out[i] = a.m[3 * i] * v[0] + a.m[3 * i + 1] * v[1] + a.m[3 * i + 2] * v[2];
}
static m3 outer(const double *a, const double *b) {
  m3 r;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[3 * i + j] = a[i] * b[j];
  return r;
}

/* diagonal BlockE formula (Filament.hpp:992, 1030-1031, 1072) */
static m3 blockE_diag(m3 dOmega, m3 LieMat, m3 OmegaMat, const double *Us, double dt) {
  double ov[3];
  m3_vec(OmegaMat, Us, ov);
  m3 inner = m3_sub(dOmega, m3_scale(m3_add(OmegaMat, m3_mul(LieMat, dOmega)), 0.5));
  m3 corr = m3_add(m3_add(rcross(ov), m3_mul(LieMat, OmegaMat)), m3_mul(m3_mul(LieMat, LieMat), dOmega));
  inner = m3_add(inner, m3_scale(corr, 1. / 12.));
  return m3_scale(inner, -2 * dt / 3.);
}
/* off-diagonal BlockE formula (Filament.hpp:1000, 1038, 1079, 1086) */
static m3 blockE_off(m3 dOmega, m3 LieMat, double dt) {
  m3 inner = m3_sub(dOmega, m3_scale(m3_mul(LieMat, dOmega), 0.5));
  inner = m3_add(inner, m3_scale(m3_mul(m3_mul(LieMat, LieMat), dOmega), 1. / 12.));
  return m3_scale(inner, -2 * dt / 3.);
}

static void put3(double *J, int n, int r0, int c0, m3 a) {
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) J[(size_t)(r0 + i) * n + c0 + j] = a.m[3 * i + j];
}
static void add3(double *J, int n, int r0, int c0, m3 a) {
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) J[(size_t)(r0 + i) * n + c0 + j] += a.m[3 * i + j];
}

static void frame(const double *qa, double *t, double *nn, double *b) {
  or_quat q;
  q_load(&q, qa);
  q_tangent(&q, t);
  q_normal(&q, nn);
  q_binormal(&q, b);
}

/* Filament::buildApproximateJacobian (Filament.hpp:803-867) with BlockC
 * (:885-909), BlockD (:912-949), BlockE (:952-1096), BlockF (:1099-1120). */
static void or_build_J(or_system *s, int f, int nt, double *J) {
  const fs_params *p = &s->p;
  const double dt = p->dt, DL = p->dl, MU = p->mu, PI = OR_PI;
  const int b0 = s->fil_start[f], nw = s->fil_start[f + 1] - b0, l0 = b0 - f;
  const int n = 6 * nw;
  const double myC = s->cc[f], myKAP = s->kap[f];
  /* this->myStrainTwist as applyElasticTorques(nt) left it: its last link */
  double ST[3];
  if (nw >= 2)
    or_link_strain_twist(s, f, nw, nw - 2, nt * dt, ST);
  else
    for (int d = 0; d < 3; ++d) ST[d] = p->strain_twist[d];
  memset(J, 0, sizeof(double) * (size_t)n * n);
  const double *rad = s->radius + b0;
#define QS(k) (s->qs + 4 * (b0 + (k)))
#define USV(k) (s->Us + 3 * (b0 + (k)))
#define TAUV(k) (s->TAU + 3 * (b0 + (k)))
#define LAM(k) (s->lam + 3 * (l0 + (k)))
  int j = 3 * nw + 3;
  double temp = dt / (9 * PI * MU * rad[0]);
  J[0 * n + 0] = 1; J[1 * n + 1] = 1; J[2 * n + 2] = 1;
  const double Jprefac = 10.;
  J[0 * n + j] = temp / dt;
  J[1 * n + j + 1] = temp / dt;
  J[2 * n + j + 2] = temp / dt;
  if (nw > 1) {
    /* BlockC(0.5*DL) at rows 3.., cols 3.. */
    double fac = 0.5 * DL;
    double tk[3], tkm1[3];
    for (int r = 0; r < nw - 1; ++r) {
      /* row block r built as in BlockC's copy-then-add recursion */
      for (int k = 0; k <= r + 1; ++k) {
        double tv[3];
        or_quat q;
        q_load(&q, QS(k));
        q_tangent(&q, tv);
        m3 blk = m3_scale(rcross(tv), fac);
        if (k == 0 || k == r + 1) put3(J, n, 3 + 3 * r, 3 + 3 * k, blk);
        else { put3(J, n, 3 + 3 * r, 3 + 3 * k, blk); add3(J, n, 3 + 3 * r, 3 + 3 * k, blk); }
      }
    }
    (void)tk; (void)tkm1;
    /* Jprefac * BlockD(nt) / dt at rows 3.., cols 3nw+3.. */
    for (int m = 0; m < nw - 1; ++m) {
      double facn = -2. * dt / (18. * PI * MU * rad[m]);
      if (nt <= p->impl_euler_steps) facn *= (3. / 2.);
      int i = 3 * m;
      for (int d = 0; d < 3; ++d) J[(size_t)(3 + i + d) * n + 3 * nw + 3 + i + d] = Jprefac * facn / dt;
      if (m < nw - 2) {
        facn = 2. * dt / (18. * PI * MU * rad[m + 1]);
        if (nt <= p->impl_euler_steps) facn *= (3. / 2.);
        for (int d = 0; d < 3; ++d) J[(size_t)(3 + i + d) * n + 3 * nw + 3 + i + 3 + d] = Jprefac * facn / dt;
      }
    }
  }
  /* BlockE at rows 3nw.., cols 3.. */
  const int rE = 3 * nw, cE = 3;
  if (nw > 1) {
    double t[3], nn[3], b[3], tp1[3], np1[3], bp1[3], tm1[3], nm1[3], bm1[3];
    /* first bead */
    double Tfac = 1 / (8 * PI * MU * pow(rad[0], 3));
    frame(QS(0), t, nn, b);
    frame(QS(1), tp1, np1, bp1);
    m3 ConstraintPart = m3_mul(m3_scale(rcross(LAM(0)), -0.5 * DL), rcross(t));
    double beta = -ST[2] + 0.5 * (np1[0] * b[0] + np1[1] * b[1] + np1[2] * b[2] - nn[0] * bp1[0] - nn[1] * bp1[1] - nn[2] * bp1[2]) / DL;
    double CP[3] = {b[1] * np1[2] - b[2] * np1[1] - nn[1] * bp1[2] + nn[2] * bp1[1],
                    b[2] * np1[0] - b[0] * np1[2] - nn[2] * bp1[0] + nn[0] * bp1[2],
                    b[0] * np1[1] - b[1] * np1[0] - nn[0] * bp1[1] + nn[1] * bp1[0]};
    double ttp[3] = {t[0] + tp1[0], t[1] + tp1[1], t[2] + tp1[2]};
    m3 EP = m3_scale(m3_add(m3_scale(outer(ttp, CP), 0.5 / DL), m3_scale(rcross(t), beta)), 0.5 * myC);
    EP = m3_add(EP, m3_scale(m3_sub(m3_scale(m3_mul(rcross(tp1), rcross(t)), 1. / DL),
                                    m3_scale(m3_add(m3_scale(rcross(nn), ST[0]), m3_scale(rcross(b), ST[1])), 0.5)),
                             0.5 * myKAP));
    m3 dOmega = m3_scale(m3_add(EP, ConstraintPart), Tfac);
    m3 LieMat = m3_t(rcross(USV(0)));
    double tT[3] = {Tfac * TAUV(0)[0], Tfac * TAUV(0)[1], Tfac * TAUV(0)[2]};
    m3 OmegaMat = rcross(tT);
    put3(J, n, rE + 0, cE + 0, blockE_diag(dOmega, LieMat, OmegaMat, USV(0), dt));
    EP = m3_scale(m3_sub(m3_scale(rcross(tp1), beta), m3_scale(outer(ttp, CP), 0.5 / DL)), 0.5 * myC);
    EP = m3_add(EP, m3_scale(m3_sub(m3_scale(m3_mul(m3_t(rcross(t)), rcross(tp1)), 1. / DL),
                                    m3_scale(m3_add(m3_scale(rcross(np1), ST[0]), m3_scale(rcross(bp1), ST[1])), 0.5)),
                             0.5 * myKAP));
    dOmega = m3_scale(EP, Tfac);
    put3(J, n, rE + 0, cE + 3, blockE_off(dOmega, LieMat, dt));

    /* last bead */
    int N = nw - 1;
    Tfac = 1 / (8 * PI * MU * pow(rad[N], 3));
    frame(QS(N), t, nn, b);
    frame(QS(N - 1), tm1, nm1, bm1);
    ConstraintPart = m3_mul(m3_scale(rcross(LAM(N - 1)), -0.5 * DL), rcross(t));
    beta = -ST[2] + 0.5 * (nn[0] * bm1[0] + nn[1] * bm1[1] + nn[2] * bm1[2] - nm1[0] * b[0] - nm1[1] * b[1] - nm1[2] * b[2]) / DL;
    double CPm[3] = {bm1[1] * nn[2] - bm1[2] * nn[1] - nm1[1] * b[2] + nm1[2] * b[1],
                     bm1[2] * nn[0] - bm1[0] * nn[2] - nm1[2] * b[0] + nm1[0] * b[2],
                     bm1[0] * nn[1] - bm1[1] * nn[0] - nm1[0] * b[1] + nm1[1] * b[0]};
    double ttm[3] = {t[0] + tm1[0], t[1] + tm1[1], t[2] + tm1[2]};
    EP = m3_scale(m3_sub(m3_scale(rcross(t), beta), m3_scale(outer(ttm, CPm), 0.5 / DL)), -0.5 * myC);
    EP = m3_sub(EP, m3_scale(m3_sub(m3_scale(m3_mul(m3_t(rcross(tm1)), rcross(t)), 1. / DL),
                                    m3_scale(m3_add(m3_scale(rcross(nn), ST[0]), m3_scale(rcross(b), ST[1])), 0.5)),
                             0.5 * myKAP));
    dOmega = m3_scale(m3_add(EP, ConstraintPart), Tfac);
    LieMat = m3_t(rcross(USV(N)));
    double tTN[3] = {Tfac * TAUV(N)[0], Tfac * TAUV(N)[1], Tfac * TAUV(N)[2]};
    OmegaMat = rcross(tTN);
    put3(J, n, rE + 3 * N, cE + 3 * N, blockE_diag(dOmega, LieMat, OmegaMat, USV(N), dt));
    EP = m3_scale(m3_sub(m3_scale(rcross(tm1), beta), m3_scale(outer(ttm, CPm), 0.5 / DL)), -0.5 * myC);
    EP = m3_sub(EP, m3_scale(m3_sub(m3_scale(m3_mul(rcross(t), rcross(tm1)), 1. / DL),
                                    m3_scale(m3_add(m3_scale(rcross(nm1), ST[0]), m3_scale(rcross(bm1), ST[1])), 0.5)),
                             0.5 * myKAP));
    dOmega = m3_scale(EP, Tfac);
    put3(J, n, rE + 3 * N, cE + 3 * N - 3, blockE_off(dOmega, LieMat, dt));

    /* interior beads */
    for (int k = 1; k < nw - 1; k++) {
      Tfac = 1 / (8 * PI * MU * pow(rad[k], 3.));
      frame(QS(k - 1), tm1, nm1, bm1);
      frame(QS(k), t, nn, b);
      frame(QS(k + 1), tp1, np1, bp1);
      LieMat = m3_t(rcross(USV(k)));
      double tTk[3] = {Tfac * TAUV(k)[0], Tfac * TAUV(k)[1], Tfac * TAUV(k)[2]};
      OmegaMat = rcross(tTk);
      double lamvec[3] = {LAM(k - 1)[0] + LAM(k)[0], LAM(k - 1)[1] + LAM(k)[1], LAM(k - 1)[2] + LAM(k)[2]};
      ConstraintPart = m3_mul(m3_scale(rcross(lamvec), -0.5 * DL), rcross(t));
      beta = -ST[2] + 0.5 * (np1[0] * b[0] + np1[1] * b[1] + np1[2] * b[2] - nn[0] * bp1[0] - nn[1] * bp1[1] - nn[2] * bp1[2]) / DL;
      double CPk[3] = {b[1] * np1[2] - b[2] * np1[1] - nn[1] * bp1[2] + nn[2] * bp1[1],
                       b[2] * np1[0] - b[0] * np1[2] - nn[2] * bp1[0] + nn[0] * bp1[2],
                       b[0] * np1[1] - b[1] * np1[0] - nn[0] * bp1[1] + nn[1] * bp1[0]};
      double tp[3] = {t[0] + tp1[0], t[1] + tp1[1], t[2] + tp1[2]};
      double tm[3] = {t[0] + tm1[0], t[1] + tm1[1], t[2] + tm1[2]};
      EP = m3_scale(m3_add(m3_scale(outer(tp, CPk), 0.5 / DL), m3_scale(rcross(t), beta)), 0.5 * myC);
      EP = m3_add(EP, m3_scale(m3_sub(m3_scale(m3_mul(rcross(tp1), rcross(t)), 1. / DL),
                                      m3_scale(m3_add(m3_scale(rcross(nn), ST[0]), m3_scale(rcross(b), ST[1])), 0.5)),
                               0.5 * myKAP));
      /* beta recomputed for the k-1 side; the "+1" CrossPart is kept (Filament.hpp:1068-1070) */
      beta = -ST[2] + 0.5 * (nn[0] * bm1[0] + nn[1] * bm1[1] + nn[2] * bm1[2] - nm1[0] * b[0] - nm1[1] * b[1] - nm1[2] * b[2]) / DL;
      EP = m3_sub(EP, m3_scale(m3_sub(m3_scale(rcross(t), beta), m3_scale(outer(tm, CPk), 0.5 / DL)), 0.5 * myC));
      EP = m3_sub(EP, m3_scale(m3_sub(m3_scale(m3_mul(m3_t(rcross(tm1)), rcross(t)), 1. / DL),
                                      m3_scale(m3_add(m3_scale(rcross(nn), ST[0]), m3_scale(rcross(b), ST[1])), 0.5)),
                               0.5 * myKAP));
      dOmega = m3_scale(m3_add(ConstraintPart, EP), Tfac);
      put3(J, n, rE + 3 * k, cE + 3 * k, blockE_diag(dOmega, LieMat, OmegaMat, USV(k), dt));
      /* left off-diagonal */
      EP = m3_scale(m3_sub(m3_scale(rcross(tm1), beta), m3_scale(outer(tm, CPk), 0.5 / DL)), -0.5 * myC);
      EP = m3_sub(EP, m3_scale(m3_sub(m3_scale(m3_mul(rcross(t), rcross(tm1)), 1. / DL),
                                      m3_scale(m3_add(m3_scale(rcross(nm1), ST[0]), m3_scale(rcross(bm1), ST[1])), 0.5)),
                               0.5 * myKAP));
      dOmega = m3_scale(EP, Tfac);
      put3(J, n, rE + 3 * k, cE + 3 * k - 3, blockE_off(dOmega, LieMat, dt));
      /* right off-diagonal (uses the k-1 side beta, Filament.hpp:1083) */
      EP = m3_scale(m3_sub(m3_scale(rcross(tp1), beta), m3_scale(outer(tp, CPk), 0.5 / DL)), 0.5 * myC);
      EP = m3_add(EP, m3_scale(m3_sub(m3_scale(m3_mul(m3_t(rcross(t)), rcross(tp1)), 1. / DL),
                                      m3_scale(m3_add(m3_scale(rcross(np1), ST[0]), m3_scale(rcross(bp1), ST[1])), 0.5)),
                               0.5 * myKAP));
      dOmega = m3_scale(EP, Tfac);
      put3(J, n, rE + 3 * k, cE + 3 * k + 3, blockE_off(dOmega, LieMat, dt));
    }
    for (int k = 0; k < 3 * nw; k++) J[(size_t)(rE + k) * n + cE + k] += 1.;
    /* BlockF / dt at rows 3nw.., cols 3nw+3.. */
    for (int i = 0; i < nw - 1; i++) {
      int jj = 3 * i;
      double tv[3];
      double fac = dt * DL / (24 * PI * MU * pow(rad[i], 3.));
      or_quat q;
      q_load(&q, QS(i));
      q_tangent(&q, tv);
      m3 tmat = m3_t(rcross(tv));
      m3 umat = rcross(USV(i));
      m3 blk = m3_add(m3_sub(tmat, m3_scale(m3_mul(umat, tmat), 0.5)), m3_scale(m3_mul(m3_mul(umat, umat), tmat), 1. / 12.));
      put3(J, n, rE + jj, 3 * nw + 3 + jj, m3_scale(blk, fac / dt));
      fac = dt * DL / (24. * PI * MU * pow(rad[i + 1], 3));
      q_load(&q, QS(i + 1));
      q_tangent(&q, tv);
      tmat = m3_t(rcross(tv));
      umat = rcross(USV(i + 1));
      blk = m3_add(m3_sub(tmat, m3_scale(m3_mul(umat, tmat), 0.5)), m3_scale(m3_mul(m3_mul(umat, umat), tmat), 1. / 12.));
      put3(J, n, rE + jj + 3, 3 * nw + 3 + jj, m3_scale(blk, fac / dt));
    }
  } else {
    for (int d = 0; d < 3; ++d) J[(size_t)(3 + d) * n + 3 + d] = 1;
  }
#undef QS
#undef USV
#undef TAUV
#undef LAM
}

/* explicit inverse by LU with partial pivoting, then solving for the identity
 * columns (the route of LAPACK getrf + getri behind Armadillo's inv()) */
static int or_invert(double *A, int n, double *Ainv) {
  int *piv = (int *)malloc(sizeof(int) * n);
  for (int k = 0; k < n; ++k) {
    int pr = k;
    double best = fabs(A[(size_t)k * n + k]);
    for (int r = k + 1; r < n; ++r) {
      double v = fabs(A[(size_t)r * n + k]);
      if (v > best) { best = v; pr = r; }
    }
    piv[k] = pr;
    if (best == 0.0) { free(piv); return 1; }
    if (pr != k)
      for (int c = 0; c < n; ++c) {
        double t = A[(size_t)k * n + c];
        A[(size_t)k * n + c] = A[(size_t)pr * n + c];
        A[(size_t)pr * n + c] = t;
      }
    double inv = 1.0 / A[(size_t)k * n + k];
    for (int r = k + 1; r < n; ++r) {
      double l = A[(size_t)r * n + k] * inv;
      A[(size_t)r * n + k] = l;
      if (l != 0.0)
        for (int c = k + 1; c < n; ++c) A[(size_t)r * n + c] -= l * A[(size_t)k * n + c];
    }
  }
  double *col = (double *)malloc(sizeof(double) * n);
  for (int e = 0; e < n; ++e) {
    for (int i = 0; i < n; ++i) col[i] = (i == e) ? 1.0 : 0.0;
    for (int k = 0; k < n; ++k)
      if (piv[k] != k) { double t = col[k]; col[k] = col[piv[k]]; col[piv[k]] = t; }
    for (int i = 0; i < n; ++i) {
      double acc = col[i];
      for (int k = 0; k < i; ++k) acc -= A[(size_t)i * n + k] * col[k];
      col[i] = acc;
    }
    for (int i = n - 1; i >= 0; --i) {
      double acc = col[i];
      for (int k = i + 1; k < n; ++k) acc -= A[(size_t)i * n + k] * col[k];
      col[i] = acc / A[(size_t)i * n + i];
    }
    for (int i = 0; i < n; ++i) Ainv[(size_t)i * n + e] = col[i];
  }
  free(col);
  free(piv);
  return 0;
}

/* filamentJsolver::buildJacobian (FilamentJacobianSolver.hpp:36-47) */
void or_build_jacobian(or_system *s, int nt) {
  memset(s->Cmat, 0, sizeof(double) * (size_t)6 * s->np * s->p.broyden_maxiter);
  memset(s->Dmat, 0, sizeof(double) * (size_t)6 * s->np * s->p.broyden_maxiter);
#pragma omp parallel for schedule(dynamic)
  for (int f = 0; f < s->nfil; ++f) {
    int nw = s->fil_start[f + 1] - s->fil_start[f];
    int n = 6 * nw;
    double *J = (double *)malloc(sizeof(double) * (size_t)n * n);
    or_build_J(s, f, nt, J);
    double *Ji = s->Jinv + s->joff[f];
    or_invert(J, n, Ji);
    if (nw > 1)
      for (int r = 3 * nw + 3; r < n; ++r)
        for (int c = 0; c < n; ++c) Ji[(size_t)r * n + c] /= s->p.dt;
    free(J);
  }
}

void or_get_jinv(or_system *s, int f, double *out) {
  int nw = s->fil_start[f + 1] - s->fil_start[f];
  memcpy(out, s->Jinv + s->joff[f], sizeof(double) * (size_t)36 * nw * nw);
}

/* ErrorCheckFCM (MobilityConstraints.cpp:447-770) */
int or_error_check(or_system *s, const double *V, const double *W, double *err, int nt) {
  const double dt = s->p.dt, TOL = s->p.tol;
  int check = 0;
  const double fourthirds = 4. / 3., onethird = 1. / 3., twothirdsDt = dt * 2. / 3.;
  for (int f = 0; f < s->nfil; ++f) {
    int b0 = s->fil_start[f], nw = s->fil_start[f + 1] - b0;
    int s0 = 6 * b0;
    for (int i = 0; i < nw; ++i) {
      int b = b0 + i;
      double e1[3], e2[3], dv[3];
      or_dexpinv(s->Us + 3 * b, W + 3 * b, dv);
      for (int d = 0; d < 3; ++d) {
        if (nt <= s->p.impl_euler_steps) {
          e1[d] = s->Xs[3 * b + d] - s->X[3 * b + d] - dt * V[3 * b + d];
          e2[d] = s->Us[3 * b + d] - dt * dv[d];
        } else {
          e1[d] = s->Xs[3 * b + d] - fourthirds * s->X[3 * b + d] + onethird * s->Xt[3 * b + d] - twothirdsDt * V[3 * b + d];
          e2[d] = s->Us[3 * b + d] - onethird * s->U[3 * b + d] - twothirdsDt * dv[d];
        }
        err[s0 + 3 * i + d] = e1[d];
        err[s0 + 3 * nw + 3 * i + d] = e2[d];
        if (fabs(e1[d]) > TOL || fabs(e2[d]) > TOL) check = 1;
      }
    }
  }
  return check;
}

/* filamentJsolver::solve (FilamentJacobianSolver.hpp:49-73) */
void or_jsolve(or_system *s, const double *b, double *x, int iter) {
#pragma omp parallel for schedule(dynamic)
  for (int f = 0; f < s->nfil; ++f) {
    int b0 = s->fil_start[f], nw = s->fil_start[f + 1] - b0;
    int n = 6 * nw, s0 = 6 * b0;
    const double *Ji = s->Jinv + s->joff[f];
    for (int r = 0; r < n; ++r) {
      double acc = 0.0;
      for (int c = 0; c < n; ++c) acc += Ji[(size_t)r * n + c] * b[s0 + c];
      x[s0 + r] = acc;
    }
  }
  size_t n6 = (size_t)6 * s->np;
  for (int i = 0; i < iter; ++i) {
    const double *dcol = s->Dmat + (size_t)i * n6, *ccol = s->Cmat + (size_t)i * n6;
    double dp = 0.0;
    for (size_t k = 0; k < n6; ++k) dp += dcol[k] * b[k];
    for (size_t k = 0; k < n6; ++k) x[k] += ccol[k] * dp;
  }
}

void or_set_cols(or_system *s, const double *c, const double *d, int iter) {
  size_t n6 = (size_t)6 * s->np;
  if (c) memcpy(s->Cmat + (size_t)iter * n6, c, sizeof(double) * n6);
  if (d) memcpy(s->Dmat + (size_t)iter * n6, d, sizeof(double) * n6);
}

/* Filament::update (Filament.hpp:425-452) with Bead::updateWith /
 * updateWithLie (Bead.hpp:236-256) */
void or_update(or_system *s, const double *u) {
  for (int f = 0; f < s->nfil; ++f) {
    int b0 = s->fil_start[f], nw = s->fil_start[f + 1] - b0, l0 = b0 - f;
    int j = 6 * b0;
    for (int d = 0; d < 3; ++d) {
      s->Xs[3 * b0 + d] -= u[j + d];
      s->Us[3 * b0 + d] -= u[j + 3 + d];
    }
    or_quat q;
    q_load(&q, s->q + 4 * b0);
    q_expm_inplace(&q, s->Us + 3 * b0);
    q_store(&q, s->qs + 4 * b0);
    j = 6 * b0 + 6;
    for (int i = 1; i < nw; ++i) {
      for (int d = 0; d < 3; ++d) s->Us[3 * (b0 + i) + d] -= u[j + d];
      q_load(&q, s->q + 4 * (b0 + i));
      q_expm_inplace(&q, s->Us + 3 * (b0 + i));
      q_store(&q, s->qs + 4 * (b0 + i));
      j += 3;
    }
    for (int i = 0; i < nw - 1; ++i) {
      for (int d = 0; d < 3; ++d) s->lam[3 * (l0 + i) + d] -= u[j + d];
      j += 3;
    }
  }
}

/* Filament::step (Filament.hpp:455-478) with Bead::step (Bead.hpp:266-276) */
void or_step(or_system *s, int nt) {
  for (int b = 0; b < s->np; ++b) {
    for (int d = 0; d < 3; ++d) {
      s->Xt[3 * b + d] = s->X[3 * b + d];
      s->X[3 * b + d] = s->Xs[3 * b + d];
      s->Ut[3 * b + d] = s->U[3 * b + d];
      s->U[3 * b + d] = s->Us[3 * b + d];
    }
    memcpy(s->qt + 4 * b, s->q + 4 * b, sizeof(double) * 4);
    or_quat q;
    q_load(&q, s->q + 4 * b);
    q_expm_inplace(&q, s->U + 3 * b);
    q_store(&q, s->q + 4 * b);
  }
  int ex = s->p.lambda_extrap_step;
  for (int k = 0; k < 3 * s->nlink; ++k) {
    if (nt > ex) {
      double lamtmp = 3 * s->lam[k] - 3 * s->lam1[k] + s->lam2[k];
      s->lam2[k] = s->lam1[k];
      s->lam1[k] = s->lam[k];
      s->lam[k] = lamtmp;
    } else if (nt == ex) {
      double lamtmp = 2. * s->lam[k] - s->lam1[k];
      s->lam2[k] = s->lam1[k];
      s->lam1[k] = s->lam[k];
      s->lam[k] = lamtmp;
    } else {
      s->lam1[k] = s->lam[k];
    }
  }
}

static void or_barrier_and_mobility(or_system *s, int nt) {
  int np = s->np;
  if (s->barrier_mode != FS_BARRIER_OFF)
    or_collision_barrier_mode(&s->p, np, s->fil_id, s->seg_id, s->Y, s->head, s->list, s->map, nt, s->F,
                              &s->min_dist2, NULL, 0, s->barrier_mode);
  if (nt > s->p.initial_friction_steps)
    or_fcm_mobility(&s->p, np, s->Y, s->F, s->TAU, s->V, s->W, NULL, NULL);
  else
    or_fcm_friction(&s->p, np, s->F, s->TAU, s->V, s->W);
  s->nsolves++;
}

void or_set_barrier_mode(or_system *s, int mode) { s->barrier_mode = mode; }

/* one time step: the body of main.cpp:284-754; commit = 0 leaves out
 * Filament::step (the gait-reset driver's trial solves) */
static int or_step_solve(or_system *s, int nt, int *iters_out, int commit);

int or_step_implicit(or_system *s, int nt, int *iters_out) { return or_step_solve(s, nt, iters_out, 1); }

/* main_gaitreset.cpp:302-830: solves without the barrier, without
 * swimmer-network pairs, then with the system's mode, committing the last */
int or_step_gait_reset(or_system *s, int nt, int *iters, double *vwf) {
  const int saved = s->barrier_mode;
  const int modes[3] = {FS_BARRIER_OFF, FS_BARRIER_NOT_SWIMMER, saved};
  const int nw0 = s->nfil > 0 ? s->fil_start[1] - s->fil_start[0] : 0;
  int st = FS_OK;
  for (int pass = 0; pass < 3; ++pass) {
    s->barrier_mode = modes[pass];
    int r = or_step_solve(s, nt, iters ? iters + pass : NULL, pass == 2);
    if (r && !st) st = r;
    if (vwf)
      for (int b = 0; b < nw0; ++b)
        for (int d = 0; d < 3; ++d) {
          vwf[(pass * nw0 + b) * 9 + d] = s->V[3 * b + d];
          vwf[(pass * nw0 + b) * 9 + 3 + d] = s->W[3 * b + d];
          vwf[(pass * nw0 + b) * 9 + 6 + d] = s->F[3 * b + d];
        }
  }
  s->barrier_mode = saved;
  return st;
}

static int or_step_solve(or_system *s, int nt, int *iters_out, int commit) {
  size_t n6 = (size_t)6 * s->np;
  or_initial_guess(s);
  or_filament_forces(s, nt);
  or_build_jacobian(s, nt);
  or_cells_link(&s->p, s->np, s->Xs, s->head, s->list);
  or_barrier_and_mobility(s, nt);
  int check = or_error_check(s, s->V, s->W, s->Err, nt);
  int iter = 0;
  while (check && iter < s->p.broyden_maxiter) {
    or_jsolve(s, s->Err, s->Upd, iter);
    or_update(s, s->Upd);
    or_filament_forces(s, nt);
    or_barrier_and_mobility(s, nt);
    check = or_error_check(s, s->V, s->W, s->NewErr, nt);
    double nrm = 0.0;
    for (size_t k = 0; k < n6; ++k) {
      s->dE[k] = s->NewErr[k] - s->Err[k];
      nrm += s->dE[k] * s->dE[k];
    }
    nrm = sqrt(nrm);
    or_jsolve(s, s->dE, s->tmp, iter);
    for (size_t k = 0; k < n6; ++k) {
      s->tmp[k] *= -1. / nrm;
      s->tmp[k] -= s->Upd[k] / nrm;
    }
    memcpy(s->Cmat + (size_t)iter * n6, s->tmp, sizeof(double) * n6);
    for (size_t k = 0; k < n6; ++k) s->Dmat[(size_t)iter * n6 + k] = s->dE[k] / nrm;
    memcpy(s->Err, s->NewErr, sizeof(double) * n6);
    ++iter;
  }
  if (commit) or_step(s, nt);
  if (iters_out) *iters_out = iter;
  return check ? FS_ERR_NOT_CONVERGED : FS_OK;
}

int or_run_steps(or_system *s, int nt_start, int nsteps, int *iters) {
  int st = FS_OK;
  for (int k = 0; k < nsteps; ++k) {
    int it = 0;
    int r = or_step_implicit(s, nt_start + k, &it);
    if (r && !st) st = r;
    if (iters) iters[k] = it;
  }
  return st;
}

double or_last_min_dist2(or_system *s) { return s->min_dist2; }
long long or_mobility_solves(or_system *s) { return s->nsolves; }

/* ------------------------------------------------------------------------ */
/* CPU-baseline sampling                                                     */
/* ------------------------------------------------------------------------ */
static double or_now(void) {
#ifdef _OPENMP
  return omp_get_wtime();
#else
  return (double)clock() / CLOCKS_PER_SEC;
#endif
}

/* Wall time of the stages of one implicit-step iteration of the current
 * suspension, each run on every stride-th of its independent work units
 * (beads, FFT lines, modes, filaments) and multiplied back by stride:
 * parts[0] spread, [1] forward FFTs, [2] projection, [3] inverse FFTs,
 * [4] interpolation, [5] Jacobian build + inversion (once per step),
 * [6] forces + error check + two J0^-1 applications with 10 history columns
 * (full, not sampled), [7] link + barrier (full). Only the stages whose bit is
 * set in mask run (the others' parts are left as they are); warm = 1 runs them
 * once untimed first. stride = 1 runs every work unit: the full-size stage.
 * The grids live in the system's workspace, allocated and touched on the first
 * call. Returns the thread count, or -1 if the workspace cannot be allocated. */
int or_stage_costs(or_system *s, int stride, unsigned mask, int warm, double *parts) {
  const fs_params *p = &s->p;
  or_consts c;
  or_consts_init(p, &c);
  const int nx = p->npts_x, ny = p->npts_y, nz = p->npts_z, nzh = nz / 2 + 1, ngd = p->ngd, np = s->np;
  const size_t N = (size_t)nx * ny * nz, NH = (size_t)nx * ny * nzh;
  if (!s->wf) {
    s->wf = (double *)malloc(sizeof(double) * 3 * N);
    s->wu = (double *)malloc(sizeof(double) * 3 * N);
    s->wfh = (or_cpx *)malloc(sizeof(or_cpx) * 3 * NH);
    s->wg = dalloc((size_t)np * 3 * ngd);
    s->wgd = dalloc((size_t)np * 3 * ngd);
    s->wgr = dalloc((size_t)np * 3 * ngd);
    s->wind = (int *)calloc((size_t)np * 3 * ngd + 1, sizeof(int));
    if (!s->wf || !s->wu || !s->wfh || !s->wg || !s->wgd || !s->wgr || !s->wind) return -1;
    /* first touch, in parallel, outside any timed region */
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)(3 * N); ++i) s->wf[i] = s->wu[i] = 0.0;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)(3 * NH); ++i) s->wfh[i].re = s->wfh[i].im = 0.0;
  }
  double *f = s->wf, *u = s->wu, *g = s->wg, *gd = s->wgd, *gr = s->wgr;
  or_cpx *fh = s->wfh;
  int *ind = s->wind;
  const double *Y = s->Y, *F = s->F, *T = s->TAU;
  double sink = 0.0;
  for (int rep = warm ? 0 : 1; rep < 2; ++rep) {
  double t0 = or_now();
  if (mask & 1u) {
#pragma omp parallel for schedule(static)
  for (int b = 0; b < np / stride; ++b)
    or_gauss_bead(p, &c, Y + 3 * b, g + (size_t)b * 3 * ngd, gd + (size_t)b * 3 * ngd, gr + (size_t)b * 3 * ngd,
                  ind + (size_t)b * 3 * ngd);
#pragma omp parallel
  {
    int nth = 1, tid = 0;
#ifdef _OPENMP
    nth = omp_get_num_threads();
    tid = omp_get_thread_num();
#endif
    int x0 = (int)((long)nx * tid / nth), x1 = (int)((long)nx * (tid + 1) / nth);
    for (int b = 0; b < np / stride; ++b) {
      const double *gx = g + (size_t)b * 3 * ngd, *gy = gx + ngd, *gz = gy + ngd;
      const double *dgx = gd + (size_t)b * 3 * ngd, *dgy = dgx + ngd, *dgz = dgy + ngd;
      const double *rx = gr + (size_t)b * 3 * ngd, *ry = rx + ngd, *rz = ry + ngd;
      const int *ix = ind + (size_t)b * 3 * ngd, *iy = ix + ngd, *iz = iy + ngd;
      const double g12 = 0.5 * T[3 * b + 2], g13 = -0.5 * T[3 * b + 1], g23 = 0.5 * T[3 * b];
      for (int i = 0; i < ngd; ++i) {
        int ii = ix[i];
        if (ii < x0 || ii >= x1) continue;
        for (int j = 0; j < ngd; ++j)
          for (int k = 0; k < ngd; ++k) {
            size_t m = ((size_t)ii * ny + iy[j]) * nz + iz[k];
            double temp = gx[i] * gy[j] * gz[k], temp2 = dgx[i] * dgy[j] * dgz[k];
            f[m] += F[3 * b] * temp + (g12 * ry[j] + g13 * rz[k]) * temp2;
            f[N + m] += F[3 * b + 1] * temp + (-g12 * rx[i] + g23 * rz[k]) * temp2;
            f[2 * N + m] += F[3 * b + 2] * temp + (-g13 * rx[i] - g23 * ry[j]) * temp2;
          }
      }
    }
  }
  parts[0] = (or_now() - t0) * stride;
  }
  if (mask & 2u) {
  t0 = or_now();
  for (int cpt = 0; cpt < 3; ++cpt) fft_r2c_3d_s(f + cpt * N, fh + cpt * NH, nx, ny, nz, stride);
  parts[1] = (or_now() - t0) * stride;
  }
  if (mask & 4u) {
  t0 = or_now();
  {
    const double TwoPI = 2. * OR_PI;
    const double ffx = TwoPI / (nx * p->dx), ffy = TwoPI / (ny * p->dx), ffz = TwoPI / (nz * p->dx);
    const double totalpts = (double)N;
#pragma omp parallel for schedule(static)
    for (long ij = 0; ij < (long)nx * ny / stride; ++ij) {
      int i = (int)(ij / ny), j = (int)(ij % ny);
      double q1 = (i <= nx / 2 ? i : i - nx) * ffx, q2 = (j <= ny / 2 ? j : j - ny) * ffy;
      double qq = q2 * q2 + q1 * q1 + 1e-18;
      for (int k = 0; k < nzh; ++k) {
        size_t m = (size_t)ij * nzh + k;
        double q3 = k * ffz, norm = 1.0 / (qq + q3 * q3);
        for (int part = 0; part < 2; ++part) {
          double *a1 = part ? &fh[m].im : &fh[m].re, *a2 = part ? &fh[NH + m].im : &fh[NH + m].re,
                 *a3 = part ? &fh[2 * NH + m].im : &fh[2 * NH + m].re;
          double kdotf = (q1 * *a1 + q2 * *a2 + q3 * *a3) * norm;
          *a1 = norm * (*a1 - q1 * kdotf) / totalpts;
          *a2 = norm * (*a2 - q2 * kdotf) / totalpts;
          *a3 = norm * (*a3 - q3 * kdotf) / totalpts;
        }
      }
    }
  }
  parts[2] = (or_now() - t0) * stride;
  }
  if (mask & 8u) {
  t0 = or_now();
  for (int cpt = 0; cpt < 3; ++cpt) fft_c2r_3d_s(fh + cpt * NH, u + cpt * N, nx, ny, nz, stride);
  parts[3] = (or_now() - t0) * stride;
  }
  if (mask & 16u) {
  t0 = or_now();
#pragma omp parallel for schedule(static) reduction(+ : sink)
  for (int b = 0; b < np / stride; ++b) {
    const double *gx = g + (size_t)b * 3 * ngd, *gy = gx + ngd, *gz = gy + ngd;
    const double *dgx = gd + (size_t)b * 3 * ngd, *dgy = dgx + ngd, *dgz = dgy + ngd;
    const double *rx = gr + (size_t)b * 3 * ngd, *ry = rx + ngd, *rz = ry + ngd;
    const int *ix = ind + (size_t)b * 3 * ngd, *iy = ix + ngd, *iz = iy + ngd;
    double v[3] = {0, 0, 0}, w[3] = {0, 0, 0};
    for (int i = 0; i < ngd; ++i)
      for (int j = 0; j < ngd; ++j)
        for (int k = 0; k < ngd; ++k) {
          size_t m = ((size_t)ix[i] * ny + iy[j]) * nz + iz[k];
          double temp = gx[i] * gy[j] * gz[k], tempd = dgx[i] * dgy[j] * dgz[k];
          v[0] += u[m] * temp;
          v[1] += u[N + m] * temp;
          v[2] += u[2 * N + m] * temp;
          w[0] -= 0.5 * (u[2 * N + m] * ry[j] - u[N + m] * rz[k]) * tempd;
          w[1] -= 0.5 * (u[m] * rz[k] - u[2 * N + m] * rx[i]) * tempd;
          w[2] -= 0.5 * (u[N + m] * rx[i] - u[m] * ry[j]) * tempd;
        }
    sink += v[0] + v[1] + v[2] + w[0] + w[1] + w[2];
  }
  parts[4] = (or_now() - t0) * stride;
  }
  if (mask & 32u) {
  t0 = or_now();
#pragma omp parallel for schedule(dynamic)
  for (int fl = 0; fl < s->nfil / stride; ++fl) {
    int nw = s->fil_start[fl + 1] - s->fil_start[fl];
    int n = 6 * nw;
    double *J = (double *)malloc(sizeof(double) * (size_t)n * n);
    or_build_J(s, fl, 2, J);
    or_invert(J, n, s->Jinv + s->joff[fl]);
    free(J);
  }
  parts[5] = (or_now() - t0) * stride;
  }
  if (mask & 64u) {
  t0 = or_now();
  or_filament_forces(s, 2);
  or_error_check(s, s->V, s->W, s->NewErr, 2);
  int hist = p->broyden_maxiter < 10 ? p->broyden_maxiter : 10;
  or_jsolve(s, s->Err, s->Upd, hist);
  or_jsolve(s, s->NewErr, s->tmp, hist);
  parts[6] = or_now() - t0;
  }
  if (mask & 128u) {
  t0 = or_now();
  or_cells_link(p, np, s->Xs, s->head, s->list);
  or_collision_barrier(p, np, s->fil_id, s->seg_id, s->Y, s->head, s->list, s->map, 2, s->F, &s->min_dist2, NULL, 0);
  parts[7] = or_now() - t0;
  }
  }
  parts[8] = sink;
  int nth = 1;
#ifdef _OPENMP
  nth = omp_get_max_threads();
#endif
  return nth;
}

int or_sample_costs(or_system *s, int stride, double *parts) { return or_stage_costs(s, stride, 0xffu, 1, parts); }
