// fs_slab.cu -- the pieces of one box's FCM mobility solve split over ranks by
// x slabs, the decomposition the reference makes with FFTW-MPI
// (FCMfunctions.cpp:16-23 plans, :360-406 transforms, :460-461 reductions).
//
// A rank owns planes [x0, x0 + nxs) of the Nx x Ny x Nz box. Its context is a
// WINDOW of nxs + H planes (fs_set_slab gives the window's first plane x0 and
// the box's Nx): the beads whose stencil starts in the rank's planes are
// spread into the window and interpolated from it with the library's own
// kernels (their stencils end inside the window, so its periodic wrap never
// applies), the H halo planes going to / coming from the next rank. The
// transforms here are the FP64 parity arithmetic on cuFFT 1-D plans, in the
// reference's order (z real-to-complex, y, then x after a transpose between
// ranks), with the projection of flow_solve (:648-736) on the transposed
// layout and the reference's inverse semantics: complex inverses along x and
// y, the imaginary parts of the kz = 0 and kz = Nz/2 coefficients dropped,
// then the real inverse along z.
//
// Layouts (complex = double2):
//   f, u      [3][nxs][Ny][Nz] real, the rank's planes
//   spec      [3][nxs][Nz/2+1][Ny]  after fs_slab_forward_yz (y fastest)
//   spec_t    [3][nkz][Ny][Nx]      the rank's kz range, every x (x fastest)
// The exchanges between ranks (halo planes, the transpose) are the caller's
// (NCCL or gloo through torch.distributed in filsim_b200/slab.py).
#include <cufft.h>
#include "fs_internal.cuh"

struct fs_slab_plans {
  int nxs = -1, nkz = -1;                      // shapes the plans were made for
  cufftHandle z_fwd = 0, z_inv = 0, y_fft = 0;  // per plane: z D2Z / Z2D, y Z2Z
  cufftHandle x_fft = 0;                        // per (kz, y) line: x Z2Z
  bool yz_ok = false, x_ok = false;
  double2 *tmp = nullptr;                       // [3][nxs][Ny][Nz/2+1]
  size_t tmp_elems = 0;
};

namespace {

// plane p: a[p][r][q] -> b[p][q][r] (rows x cols = nr x nq), through 32 x 33 tiles;
// drop != 0: zero the imaginary part of the source's first and last rows (kz = 0 and Nz/2)
__global__ void k_plane_transpose(const double2 *__restrict__ a, double2 *__restrict__ b, int nr, int nq,
                                  int drop_rows) {
  __shared__ double2 t[32][33];
  const size_t plane = (size_t)blockIdx.z * nr * nq;
  const int r0 = blockIdx.y * 32, q0 = blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, q = q0 + threadIdx.x;
    if (r < nr && q < nq) {
      double2 v = a[plane + (size_t)r * nq + q];
      if (drop_rows && (r == 0 || r == nr - 1)) v.y = 0.0;
      t[i][threadIdx.x] = v;
    }
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int q = q0 + i, r = r0 + threadIdx.x;
    if (r < nr && q < nq) b[plane + (size_t)q * nr + r] = t[threadIdx.x][i];
  }
}

__device__ __forceinline__ double wavenumber_d(int i, int n, double ff) { return (double)((i <= n / 2) ? i : i - n) * ff; }

// flow_solve (FCMfunctions.cpp:648-736) on spec_t [3][nkz][ny][nx]: one thread per
// mode, the three components together; the k = 0 mode is zeroed
__global__ void k_slab_project(double2 *__restrict__ s, int nkz, int kz0, int ny, int nx, double ffx, double ffy,
                               double ffz, double total) {
  const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t cs = (size_t)nkz * ny * nx;
  if (m >= cs) return;
  const int x = (int)(m % nx), y = (int)((m / nx) % ny), kz = kz0 + (int)(m / ((size_t)nx * ny));
  const double q1 = wavenumber_d(x, nx, ffx), q2 = wavenumber_d(y, ny, ffy), q3 = (double)kz * ffz;
  const double qq = q2 * q2 + q1 * q1 + 1e-18;
  const double norm = 1.0 / (qq + q3 * q3);
  double2 a = s[m], b = s[cs + m], d = s[2 * cs + m];
  if ((x | y | kz) == 0) {
    a = b = d = make_double2(0.0, 0.0);
  } else {
    const double kr = (q1 * a.x + q2 * b.x + q3 * d.x) * norm;
    const double ki = (q1 * a.y + q2 * b.y + q3 * d.y) * norm;
    a = make_double2(norm * (a.x - q1 * kr) / total, norm * (a.y - q1 * ki) / total);
    b = make_double2(norm * (b.x - q2 * kr) / total, norm * (b.y - q2 * ki) / total);
    d = make_double2(norm * (d.x - q3 * kr) / total, norm * (d.y - q3 * ki) / total);
  }
  s[m] = a;
  s[cs + m] = b;
  s[2 * cs + m] = d;
}

fs_status ensure_yz(fs_ctx *c, int nxs) {
  fs_slab_plans *P = c->slab;
  if (P->yz_ok && P->nxs == nxs) return FS_OK;
  if (P->yz_ok) {
    cufftDestroy(P->z_fwd);
    cufftDestroy(P->z_inv);
    cufftDestroy(P->y_fft);
    P->yz_ok = false;
  }
  const int ny = c->ny, nz = c->nz, nzh = nz / 2 + 1;
  const size_t need = (size_t)3 * nxs * ny * nzh;
  if (need > P->tmp_elems) {
    cudaFree(P->tmp);
    P->tmp = nullptr;
    FS_CUDA(cudaMalloc(&P->tmp, sizeof(double2) * need));
    P->tmp_elems = need;
  }
  int n[1];
  n[0] = nz;
  if (cufftPlanMany(&P->z_fwd, 1, n, NULL, 1, nz, NULL, 1, nzh, CUFFT_D2Z, 3 * nxs * ny) != CUFFT_SUCCESS)
    return FS_ERR_CUFFT;
  if (cufftPlanMany(&P->z_inv, 1, n, NULL, 1, nzh, NULL, 1, nz, CUFFT_Z2D, 3 * nxs * ny) != CUFFT_SUCCESS)
    return FS_ERR_CUFFT;
  n[0] = ny;
  if (cufftPlanMany(&P->y_fft, 1, n, NULL, 1, ny, NULL, 1, ny, CUFFT_Z2Z, 3 * nxs * nzh) != CUFFT_SUCCESS)
    return FS_ERR_CUFFT;
  for (cufftHandle h : {P->z_fwd, P->z_inv, P->y_fft})
    if (cufftSetStream(h, c->stream) != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  P->nxs = nxs;
  P->yz_ok = true;
  return FS_OK;
}

fs_status ensure_x(fs_ctx *c, int nkz) {
  fs_slab_plans *P = c->slab;
  if (P->x_ok && P->nkz == nkz) return FS_OK;
  if (P->x_ok) {
    cufftDestroy(P->x_fft);
    P->x_ok = false;
  }
  int n[1] = {c->slab_nx};
  if (cufftPlanMany(&P->x_fft, 1, n, NULL, 1, c->slab_nx, NULL, 1, c->slab_nx, CUFFT_Z2Z, 3 * nkz * c->ny) !=
      CUFFT_SUCCESS)
    return FS_ERR_CUFFT;
  if (cufftSetStream(P->x_fft, c->stream) != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  P->nkz = nkz;
  P->x_ok = true;
  return FS_OK;
}

fs_status slab_check(fs_ctx *c) {
  if (!c) return FS_ERR_INVALID_ARG;
  if (c->slab_nx <= 0) return FS_ERR_STATE;
  if (!c->slab) c->slab = new fs_slab_plans();
  return FS_OK;
}

}  // namespace

void slab_free(fs_ctx *c) {
  fs_slab_plans *P = c->slab;
  if (!P) return;
  if (P->yz_ok) {
    cufftDestroy(P->z_fwd);
    cufftDestroy(P->z_inv);
    cufftDestroy(P->y_fft);
  }
  if (P->x_ok) cufftDestroy(P->x_fft);
  cudaFree(P->tmp);
  delete P;
  c->slab = nullptr;
}

extern "C" {

fs_status fs_set_slab(fs_ctx *c, int x0, int nx_box) {
  // (one rank: the window, its slab plus the halo, is longer than the box)
  if (!c || nx_box < 0 || (nx_box > 0 && (x0 < 0 || x0 >= nx_box))) return FS_ERR_INVALID_ARG;
  c->slab_x0 = nx_box > 0 ? x0 : 0;
  c->slab_nx = nx_box;
  return FS_OK;
}

fs_status fs_fcm_interpolate(fs_ctx *c, const double *u, const double *Y, int np, double *V, double *W) {
  if (!c || np < 0 || np > c->max_beads || (np > 0 && (!u || !Y || !V || !W))) return FS_ERR_INVALID_ARG;
  return fcm_interpolate_only(c, u, Y, np, V, W);
}

fs_status fs_slab_forward_yz(fs_ctx *c, const double *f, int nxs, double *spec) {
  FS_TRY(slab_check(c));
  if (!f || !spec || nxs <= 0 || nxs > c->nx) return FS_ERR_INVALID_ARG;
  FS_TRY(ensure_yz(c, nxs));
  fs_slab_plans *P = c->slab;
  const int ny = c->ny, nzh = c->nz / 2 + 1;
  if (cufftExecD2Z(P->z_fwd, (cufftDoubleReal *)f, (cufftDoubleComplex *)P->tmp) != CUFFT_SUCCESS)
    return FS_ERR_CUFFT;
  dim3 g((nzh + 31) / 32, (ny + 31) / 32, 3 * nxs);
  k_plane_transpose<<<g, dim3(32, 8), 0, c->stream>>>(P->tmp, (double2 *)spec, ny, nzh, 0);
  FS_LAUNCH_CHECK();
  if (cufftExecZ2Z(P->y_fft, (cufftDoubleComplex *)spec, (cufftDoubleComplex *)spec, CUFFT_FORWARD) != CUFFT_SUCCESS)
    return FS_ERR_CUFFT;
  return FS_OK;
}

fs_status fs_slab_solve_x(fs_ctx *c, double *spec_t, int kz0, int nkz) {
  FS_TRY(slab_check(c));
  const int nzh = c->nz / 2 + 1;
  if (!spec_t || kz0 < 0 || nkz < 0 || kz0 + nkz > nzh) return FS_ERR_INVALID_ARG;
  if (nkz == 0) return FS_OK;
  FS_TRY(ensure_x(c, nkz));
  fs_slab_plans *P = c->slab;
  cufftDoubleComplex *s = (cufftDoubleComplex *)spec_t;
  if (cufftExecZ2Z(P->x_fft, s, s, CUFFT_FORWARD) != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  const double TwoPI = 2. * FS_PI;
  const int nx = c->slab_nx, ny = c->ny, nz = c->nz;
  const double total = (double)nx * (double)ny * (double)nz;
  const size_t cs = (size_t)nkz * ny * nx;
  k_slab_project<<<fs_blocks((long long)cs, 256), 256, 0, c->stream>>>(
      (double2 *)spec_t, nkz, kz0, ny, nx, TwoPI / (nx * c->p.dx), TwoPI / (ny * c->p.dx), TwoPI / (nz * c->p.dx),
      total);
  FS_LAUNCH_CHECK();
  if (cufftExecZ2Z(P->x_fft, s, s, CUFFT_INVERSE) != CUFFT_SUCCESS) return FS_ERR_CUFFT;
  return FS_OK;
}

fs_status fs_slab_inverse_yz(fs_ctx *c, double *spec, int nxs, double *u) {
  FS_TRY(slab_check(c));
  if (!spec || !u || nxs <= 0 || nxs > c->nx) return FS_ERR_INVALID_ARG;
  FS_TRY(ensure_yz(c, nxs));
  fs_slab_plans *P = c->slab;
  const int ny = c->ny, nzh = c->nz / 2 + 1;
  if (cufftExecZ2Z(P->y_fft, (cufftDoubleComplex *)spec, (cufftDoubleComplex *)spec, CUFFT_INVERSE) != CUFFT_SUCCESS)
    return FS_ERR_CUFFT;
  dim3 g((ny + 31) / 32, (nzh + 31) / 32, 3 * nxs);
  k_plane_transpose<<<g, dim3(32, 8), 0, c->stream>>>((const double2 *)spec, P->tmp, nzh, ny, 1);
  FS_LAUNCH_CHECK();
  if (cufftExecZ2D(P->z_inv, (cufftDoubleComplex *)P->tmp, (cufftDoubleReal *)u) != CUFFT_SUCCESS)
    return FS_ERR_CUFFT;
  return FS_OK;
}

}  // extern "C"
