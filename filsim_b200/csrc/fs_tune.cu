// fs_tune.cu -- the autotuner: for one context (grid, suspension, precision),
// the fastest combination of the FCM launch variants, timed on the device with
// the context's own beads. No reference counterpart.
//
// Knobs: beads staged per spread pass (32 or 64; the 16^3 tile is fixed by the
// binning), beads per interpolation CTA (4, 8 or 16 warps), on FP32
// power-of-two grids the transform (the five-pass warp FFT of fs_fft.cu or
// cuFFT), and the shape of a warp's column block in the FP32 spread tile
// (x width 2, 4 or 8: 2 x 16 x 8, 4 x 16 x 4 or 8 x 16 x 2 points). A captured
// step graph bakes the launch shapes, so tuning invalidates it.
#include "fs_internal.cuh"

extern "C" {

fs_status fs_set_tuning(fs_ctx *c, const int *choice_h) {
  if (!c || !choice_h) return FS_ERR_INVALID_ARG;
  const int ch = choice_h[0], wpb = choice_h[1], fft = choice_h[2], cx = choice_h[3];
  if ((ch != 32 && ch != 64) || (wpb != 4 && wpb != 8 && wpb != 16) || (fft != 0 && fft != 1) ||
      (cx != 2 && cx != 4 && cx != 8))
    return FS_ERR_INVALID_ARG;
  c->tune_spread_chunk = ch;
  c->tune_spread_cols = cx;
  c->tune_interp_wpb = wpb;
  c->tune_fft32 = fft;
  graph_invalidate(c);
  return FS_OK;
}

fs_status fs_autotune(fs_ctx *c, int reps, int *choice_h, float *best_ms_h) {
  if (!c || reps < 1) return FS_ERR_INVALID_ARG;
  if (!c->have_state) return FS_ERR_STATE;
  FS_TRY(fil_forces(c, c->p.initial_friction_steps + 1));  // Y, F, TAU of the current state
  cudaEvent_t e0, e1;
  FS_CUDA(cudaEventCreate(&e0));
  FS_CUDA(cudaEventCreate(&e1));
  const int ffts = (c->precision == FS_PREC_FP32 && c->fft_tw) ? 2 : 1;
  float best = 1e30f;
  // the column shape only changes the FP32 spread (FP64 keeps the current one)
  const bool f32 = c->precision == FS_PREC_FP32;
  const int cx_lo = f32 ? 2 : c->tune_spread_cols, cx_hi = f32 ? 8 : c->tune_spread_cols;
  int bch = 64, bwpb = 8, bfft = 0, bcx = c->tune_spread_cols;
  fs_status st = FS_OK;
  for (int ch = 32; ch <= 64 && st == FS_OK; ch *= 2)
    for (int wpb = 4; wpb <= 16 && st == FS_OK; wpb *= 2)
      for (int fft = 0; fft < ffts && st == FS_OK; ++fft)
        for (int cx = cx_lo; cx <= cx_hi && st == FS_OK; cx *= 2) {
        c->tune_spread_chunk = ch;
        c->tune_spread_cols = cx;
        c->tune_interp_wpb = wpb;
        c->tune_fft32 = fft;
        st = fcm_set_stream(c, c->stream);
        if (st == FS_OK) st = fcm_mobility(c, c->Y, c->F, c->TAU, c->V, c->W, c->np);  // warm-up
        if (st != FS_OK) break;
        if (cudaEventRecord(e0, c->stream) != cudaSuccess) st = FS_ERR_CUDA;
        for (int r = 0; r < reps && st == FS_OK; ++r) st = fcm_mobility(c, c->Y, c->F, c->TAU, c->V, c->W, c->np);
        float ms = 0.f;
        if (st == FS_OK && (cudaEventRecord(e1, c->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
          st = FS_ERR_CUDA;
        ms /= reps;
        if (st == FS_OK && ms < best) {
          best = ms;
          bch = ch;
          bwpb = wpb;
          bfft = fft;
          bcx = cx;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->tune_spread_chunk = bch;
  c->tune_interp_wpb = bwpb;
  c->tune_fft32 = bfft;
  c->tune_spread_cols = bcx;
  graph_invalidate(c);
  FS_TRY(st);
  FS_TRY(fcm_set_stream(c, c->stream));
  if (choice_h) {
    choice_h[0] = bch;
    choice_h[1] = bwpb;
    choice_h[2] = bfft;
    choice_h[3] = bcx;
  }
  if (best_ms_h) *best_ms_h = best;
  return FS_OK;
}

}  // extern "C"
