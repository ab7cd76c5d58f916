/* Single-process stand-in for the FFTW 2.1.5 rfftwnd_mpi interface the
 * reference's FCM file calls (FCMfunctions.cpp:16-23, 324-406, 469-470), with
 * FFTW's documented semantics: unnormalised transforms; a real array of
 * nx x ny x nz stored with its last dimension padded to 2 (nz/2 + 1); the
 * real-to-complex result, in place, as complex [y][x][nz/2 + 1] when the
 * transposed order is asked for (one process holds every x and every y); the
 * complex-to-real inverse from that transposed layout, with complex inverse
 * transforms along x and y and then a halfcomplex inverse along z, which has
 * no slots for the imaginary parts of the kz = 0 and kz = nz/2 coefficients.
 * The transforms themselves are this file's own: radix-2 for power-of-two
 * lengths, the direct sum for others. Test infrastructure: only the
 * reference-pinning build uses it. */
#ifndef REFSHIM_RFFTW_MPI_H
#define REFSHIM_RFFTW_MPI_H
#include <complex>
#include <vector>
#include <math.h>
#include <stdlib.h>
#include "mpi.h"

typedef double fftw_real;
typedef struct { fftw_real re, im; } fftw_complex;
typedef enum { FFTW_REAL_TO_COMPLEX = -1, FFTW_COMPLEX_TO_REAL = 1 } fftw_direction;
#define FFTW_MEASURE 1
#define FFTW_ESTIMATE 0
typedef enum { FFTW_NORMAL_ORDER = 0, FFTW_TRANSPOSED_ORDER = 1 } fftwnd_mpi_output_order;

struct refshim_plan {
  int nx, ny, nz;
  fftw_direction dir;
};
typedef refshim_plan *rfftwnd_mpi_plan;

static inline rfftwnd_mpi_plan rfftw3d_mpi_create_plan(MPI_Comm, int nx, int ny, int nz, fftw_direction dir, int) {
  refshim_plan *p = new refshim_plan;
  p->nx = nx;
  p->ny = ny;
  p->nz = nz;
  p->dir = dir;
  return p;
}
static inline void rfftwnd_mpi_destroy_plan(rfftwnd_mpi_plan p) { delete p; }
static inline void rfftwnd_mpi_local_sizes(rfftwnd_mpi_plan p, int *local_nx, int *local_x_start,
                                           int *local_ny_after_transpose, int *local_y_start_after_transpose,
                                           int *total_local_size) {
  *local_nx = p->nx;
  *local_x_start = 0;
  *local_ny_after_transpose = p->ny;
  *local_y_start_after_transpose = 0;
  *total_local_size = p->nx * p->ny * 2 * (p->nz / 2 + 1);
}

/* in-place complex DFT of n points, sign -1 forward, +1 backward: radix-2
 * for n = 2^k, the direct sum otherwise */
static inline void refshim_fft1(std::complex<double> *a, int n, int sign) {
  if (n & (n - 1)) {
    std::vector<std::complex<double>> out((size_t)n);
    for (int k = 0; k < n; ++k) {
      std::complex<double> acc(0.0, 0.0);
      for (int j = 0; j < n; ++j) {
        const double ang = sign * 2.0 * 3.14159265358979323846264338327950288 * (double)((long long)j * k % n) / n;
        acc += a[j] * std::complex<double>(cos(ang), sin(ang));
      }
      out[k] = acc;
    }
    for (int k = 0; k < n; ++k) a[k] = out[k];
    return;
  }
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    for (int i = 0; i < n; i += len)
      for (int k = 0; k < len / 2; ++k) {
        const double ang = sign * 2.0 * 3.14159265358979323846264338327950288 * k / len;
        const std::complex<double> w(cos(ang), sin(ang));
        const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
  }
}

static inline void rfftwnd_mpi(rfftwnd_mpi_plan p, int howmany, fftw_real *data, fftw_real *,
                               fftwnd_mpi_output_order order) {
  const int nx = p->nx, ny = p->ny, nz = p->nz, nzh = nz / 2 + 1, pad = 2 * nzh;
  if (howmany != 1 || order != FFTW_TRANSPOSED_ORDER) abort();
  std::vector<std::complex<double>> c((size_t)nx * ny * nzh), line((size_t)(nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz)));
  // spectrum held as c[(x * ny + y) * nzh + kz] while transforming
  if (p->dir == FFTW_REAL_TO_COMPLEX) {
    for (int x = 0; x < nx; ++x)
      for (int y = 0; y < ny; ++y) {
        const fftw_real *r = data + ((size_t)x * ny + y) * pad;
        for (int z = 0; z < nz; ++z) line[z] = std::complex<double>(r[z], 0.0);
        refshim_fft1(line.data(), nz, -1);
        for (int k = 0; k < nzh; ++k) c[((size_t)x * ny + y) * nzh + k] = line[k];
      }
    for (int x = 0; x < nx; ++x)
      for (int k = 0; k < nzh; ++k) {
        for (int y = 0; y < ny; ++y) line[y] = c[((size_t)x * ny + y) * nzh + k];
        refshim_fft1(line.data(), ny, -1);
        for (int y = 0; y < ny; ++y) c[((size_t)x * ny + y) * nzh + k] = line[y];
      }
    for (int y = 0; y < ny; ++y)
      for (int k = 0; k < nzh; ++k) {
        for (int x = 0; x < nx; ++x) line[x] = c[((size_t)x * ny + y) * nzh + k];
        refshim_fft1(line.data(), nx, -1);
        for (int x = 0; x < nx; ++x) c[((size_t)x * ny + y) * nzh + k] = line[x];
      }
    // transposed order: complex [y][x][kz] over the same storage
    fftw_complex *out = reinterpret_cast<fftw_complex *>(data);
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x)
        for (int k = 0; k < nzh; ++k) {
          const std::complex<double> v = c[((size_t)x * ny + y) * nzh + k];
          out[((size_t)y * nx + x) * nzh + k].re = v.real();
          out[((size_t)y * nx + x) * nzh + k].im = v.imag();
        }
    return;
  }
  const fftw_complex *in = reinterpret_cast<const fftw_complex *>(data);
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x)
      for (int k = 0; k < nzh; ++k)
        c[((size_t)x * ny + y) * nzh + k] =
            std::complex<double>(in[((size_t)y * nx + x) * nzh + k].re, in[((size_t)y * nx + x) * nzh + k].im);
  for (int y = 0; y < ny; ++y)
    for (int k = 0; k < nzh; ++k) {
      for (int x = 0; x < nx; ++x) line[x] = c[((size_t)x * ny + y) * nzh + k];
      refshim_fft1(line.data(), nx, +1);
      for (int x = 0; x < nx; ++x) c[((size_t)x * ny + y) * nzh + k] = line[x];
    }
  for (int x = 0; x < nx; ++x)
    for (int k = 0; k < nzh; ++k) {
      for (int y = 0; y < ny; ++y) line[y] = c[((size_t)x * ny + y) * nzh + k];
      refshim_fft1(line.data(), ny, +1);
      for (int y = 0; y < ny; ++y) c[((size_t)x * ny + y) * nzh + k] = line[y];
    }
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y) {
      const std::complex<double> *h = &c[((size_t)x * ny + y) * nzh];
      line[0] = std::complex<double>(h[0].real(), 0.0);
      for (int k = 1; k < nzh; ++k) {
        if (2 * k == nz) {
          line[k] = std::complex<double>(h[k].real(), 0.0);
        } else {
          line[k] = h[k];
          line[nz - k] = std::conj(h[k]);
        }
      }
      refshim_fft1(line.data(), nz, +1);
      fftw_real *r = data + ((size_t)x * ny + y) * pad;
      for (int z = 0; z < nz; ++z) r[z] = line[z].real();
    }
}
#endif
