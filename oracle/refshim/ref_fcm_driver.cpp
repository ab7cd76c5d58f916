/* C entry points around the reference's own struct Fcm (FCMfunctions.hpp:7-59),
 * compiled from the reference sources by oracle/refshim/Makefile: one FCM
 * mobility solve exactly as the reference runs it (Fcm::initialise,
 * Fcm::mobility_solve, FCMfunctions.cpp:10-464) on one process. Test
 * infrastructure: the oracle's reference pin; nothing in the product calls it. */
#include "FCMfunctions.hpp"

int Np = 0;

extern "C" void ref_fcm_config(int *npts_xyz_ngd, double *dx_out) {
  npts_xyz_ngd[0] = NPTS_X;
  npts_xyz_ngd[1] = NPTS_Y;
  npts_xyz_ngd[2] = NPTS_Z;
  npts_xyz_ngd[3] = ngd;
  *dx_out = dx;
}

/* Y, F, T in, V, W out: np x 3 row-major doubles. The positions are passed
 * as fcm.Y is filled by assign_filament_data (already wrapped by fmod). */
extern "C" int ref_fcm_mobility(int np, const double *Y, const double *F, const double *T, double *V, double *W) {
  Np = np;
  Fcm fcm;
  fcm.initialise(0);
  for (int j = 0; j < np; ++j)
    for (int k = 0; k < 3; ++k) {
      fcm.Y[j][k] = Y[3 * j + k];
      fcm.F[j][k] = F[3 * j + k];
      fcm.T[j][k] = T[3 * j + k];
    }
  fcm.mobility_solve();
  for (int j = 0; j < np; ++j)
    for (int k = 0; k < 3; ++k) {
      V[3 * j + k] = fcm.V[j][k];
      W[3 * j + k] = fcm.W[j][k];
    }
  fcm.free_memory();
  return 0;
}

#ifdef REF_NSW
#include "CollisionBarrierFilament.hpp"

/* LinkedList::initialise, link and apply_collision_barrier
 * (CollisionBarrierFilament.cpp:24-433) as the reference runs them, for nfil
 * filaments (fil_start[nfil + 1] bead prefix, nfil <= Nsw, each at most
 * max_Nworm beads): Xs unwrapped positions (link), Y = fmod(Xs, L) (the
 * barrier), F_inout gains the barrier forces; head (ncell ints), list (np
 * ints) and the minimum squared distance come out. */
extern "C" int ref_barrier(int nfil, const int *fil_start, const double *Xs, const double *Y, double *F_inout, int nt,
                           int *head_out, int *list_out, int *ncell_out, double *min_dist2_out) {
  if (nfil > Nsw) return 1;
  std::vector<Filament> filaments(nfil);
  for (int f = 0; f < nfil; ++f) {
    const int nw = fil_start[f + 1] - fil_start[f];
    if (nw > max_Nworm) return 1;
    filaments[f].myNworm = nw;
    filaments[f].beads.resize(nw);
    for (int i = 0; i < nw; ++i)
      for (int k = 0; k < 3; ++k) filaments[f].beads[i].Xs.v[k] = Xs[3 * (fil_start[f] + i) + k];
  }
  Np = fil_start[nfil];
  Fcm fcm;
  fcm.initialise(0);
  for (int j = 0; j < Np; ++j)
    for (int k = 0; k < 3; ++k) {
      fcm.Y[j][k] = Y[3 * j + k];
      fcm.F[j][k] = F_inout[3 * j + k];
    }
  LinkedList *ll = new LinkedList();
  ll->initialise(0, 1, filaments);
  ll->link(filaments);
  ll->apply_collision_barrier(fcm, nt);
  for (int j = 0; j < Np; ++j)
    for (int k = 0; k < 3; ++k) F_inout[3 * j + k] = fcm.F[j][k];
  *ncell_out = ll->ncell;
  if (head_out) memcpy(head_out, ll->head, sizeof(int) * ll->ncell);
  if (list_out) memcpy(list_out, ll->list, sizeof(int) * Np);
  *min_dist2_out = ll->min_dist2;
  delete ll;
  fcm.free_memory();
  return 0;
}
#endif
