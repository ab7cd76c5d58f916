// fs_runfiles.cu -- the reference's run files (.par, .bak, .dat) as host code,
// so a run of this library resumes the reference's checkpoints (and the
// reference resumes ours) and its outputs feed the reference's plotting
// scripts. Formats follow file_functions.cpp and Filament.hpp:509-748:
//   .bak  nt, then per bead X Xt qs qt U Ut, then per link lam lam1 lam2
//         (std::fixed, precision 16: "%.16f"; every item followed by one space,
//         no newline)
//   .par  a line of column names, a line of values (stream defaults: "%g"),
//         a blank line, "BeadNumbers", the bead counts, a blank line,
//         "BendingModuli are KAP*", the bending factors
//   .dat  a header line "it X Y Z qr qi qj qk ..." and one line per output
//         step: nt, then per bead Xs and qs ("%.16f")
// The readers tokenise on whitespace, which accepts everything the
// reference's getline(..., ' ') readers accept from these writers.
#include <errno.h>
#include <locale.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <string>
#include <vector>
#include "filsim_gpu.h"

namespace {

// The files use the "C" number format whatever the caller's locale: each call
// switches its own thread to the C numeric locale (uselocale, thread-local) and
// restores the previous one on return, as C++ streams with the classic locale do.
struct CNumericLocale {
  locale_t prev = (locale_t)0;
  CNumericLocale() {
    static locale_t c_loc = newlocale(LC_NUMERIC_MASK, "C", (locale_t)0);
    if (c_loc) prev = uselocale(c_loc);
  }
  ~CNumericLocale() {
    if (prev) uselocale(prev);
  }
};

struct File {
  FILE *f = nullptr;
  File(const char *path, const char *mode) { f = fopen(path, mode); }
  ~File() {
    if (f) fclose(f);
  }
  bool close() {
    const bool ok = f && fclose(f) == 0;
    f = nullptr;
    return ok;
  }
};

bool layout_ok(const fs_host_state *s) {
  if (!s || !s->fil_start || s->nfil < 0 || s->np < 0) return false;
  if (s->fil_start[0] != 0 || s->fil_start[s->nfil] != s->np) return false;
  for (int f = 0; f < s->nfil; ++f)
    if (s->fil_start[f + 1] - s->fil_start[f] < 1) return false;
  return true;
}

// "%.16f " for n values (Filament.hpp:651-653 stream settings)
inline void put_fixed(FILE *f, const double *v, int n) {
  for (int i = 0; i < n; ++i) fprintf(f, "%.16f ", v[i]);
}

bool read_all(const char *path, std::string *out) {
  File in(path, "rb");
  if (!in.f) return false;
  char buf[1 << 16];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, in.f)) > 0) out->append(buf, n);
  return !ferror(in.f);
}

// whitespace-separated tokens of text, as views [begin, end)
std::vector<std::pair<const char *, const char *>> tokens(const std::string &text, size_t from = 0) {
  std::vector<std::pair<const char *, const char *>> t;
  const char *p = text.c_str() + from, *e = text.c_str() + text.size();
  while (p < e) {
    while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
    const char *b = p;
    while (p < e && !(*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
    if (p > b) t.emplace_back(b, p);
  }
  return t;
}

bool to_double(const std::pair<const char *, const char *> &tok, double *v) {
  std::string s(tok.first, tok.second);
  char *end = nullptr;
  errno = 0;
  *v = strtod(s.c_str(), &end);
  return end && *end == '\0' && end != s.c_str();
}

bool to_int(const std::pair<const char *, const char *> &tok, int *v) {
  std::string s(tok.first, tok.second);
  char *end = nullptr;
  errno = 0;
  const long x = strtol(s.c_str(), &end, 10);
  if (!end || *end != '\0' || end == s.c_str() || errno || x < -2147483647L || x > 2147483647L) return false;
  *v = (int)x;
  return true;
}

}  // namespace

extern "C" {

fs_status fs_par_write(const char *path, const fs_run_info *info, const fs_host_state *s) {
  CNumericLocale c_numbers;
  if (!path || !info || !layout_ok(s)) return FS_ERR_INVALID_ARG;
  File out(path, "w");
  if (!out.f) return FS_ERR_IO;
  FILE *f = out.f;
  int nworm = 0;
  for (int i = 0; i < s->nfil; ++i) nworm = std::max(nworm, s->fil_start[i + 1] - s->fil_start[i]);
  fprintf(f,
          "SimulationName SimulationTag Nsw Nworm a ah DL Sp4 Kap C MU curvature K0 TimeSteps StepsPerPeriod "
          "TOL gmres_tol broyden_maxiter gmres_maxiter LfcmBox_x plot_steps STRAINTWISTX STRAINTWISTY "
          "STRAINTWISTZ Kap_NetworkFilaments LfcmBox_z LfcmBox_y B StepsPerSettlingTime dt "
          "initialFrictionSteps EnableSpringLinks ConnectedNodesNumSwimmingFilaments ConnectedNodesNumNodes "
          "ConnectedNodesConnectionRadius ConnectedNodesMinNodeSpacing ConnectedNodesSpacingAwayFromNode "
          "NetworkSpringConstant NetworkSpringNaturalLength \n");
  char name[129], tag[129];
  snprintf(name, sizeof name, "%s", info->simulation_name);
  snprintf(tag, sizeof tag, "%s", info->simulation_tag);
  fprintf(f, "%s %s %d %d %g %g %g %g %g %g %g %g %g %g %g %g %d %d %d %g %d %g %g %g %g %g %g %g %g %g %d %d ",
          name, tag, s->nfil, nworm, info->a, info->ah, info->dl, info->sp4, info->kap, info->c, info->mu,
          info->curvature, info->k0, info->time_steps, info->steps_per_period, info->tol, 0, info->broyden_maxiter,
          0, info->box[0], info->plot_steps, info->strain_twist[0], info->strain_twist[1], info->strain_twist[2],
          info->kap_network_filaments, info->box[2], info->box[1], info->bnumber, info->steps_per_settling_time,
          info->dt, info->initial_friction_steps, info->enable_spring_links);
  fprintf(f, "%g %g %g %g %g %g %g \n\n", info->cn_num_swimming_filaments, info->cn_num_nodes,
          info->cn_connection_radius, info->cn_min_node_spacing, info->cn_spacing_away_from_node,
          info->network_spring_constant, info->network_spring_natural_length);
  fprintf(f, "BeadNumbers\n");
  for (int i = 0; i < s->nfil; ++i) fprintf(f, i + 1 < s->nfil ? "%d " : "%d", s->fil_start[i + 1] - s->fil_start[i]);
  fprintf(f, "\n\nBendingModuli are KAP*\n");
  for (int i = 0; i < s->nfil; ++i) {
    const double factor = s->kap ? (info->kap != 0.0 ? s->kap[i] / info->kap : s->kap[i]) : 1.0;
    fprintf(f, i + 1 < s->nfil ? "%g " : "%g", factor);
  }
  fprintf(f, "\n");
  return (ferror(f) || !out.close()) ? FS_ERR_IO : FS_OK;
}

fs_status fs_par_read_layout(const char *path, int *nfil_out, int *np_out, int *fil_start_h, int max_fil) {
  CNumericLocale c_numbers;
  if (!path || !nfil_out || !np_out || !fil_start_h || max_fil < 0) return FS_ERR_INVALID_ARG;
  std::string text;
  if (!read_all(path, &text)) return FS_ERR_IO;
  // line 2, third item: the filament count; line 5 on: the bead numbers
  size_t line_start[5] = {0, 0, 0, 0, 0};
  int line = 0;
  for (size_t i = 0; i < text.size() && line < 4; ++i)
    if (text[i] == '\n') line_start[++line] = i + 1;
  if (line < 4) return FS_ERR_IO;
  const std::string second = text.substr(line_start[1], line_start[2] - line_start[1]);
  auto t2 = tokens(second);
  int nfil = 0;
  if (t2.size() < 3 || !to_int(t2[2], &nfil) || nfil < 0) return FS_ERR_IO;
  if (nfil > max_fil) return FS_ERR_CAPACITY;
  auto tb = tokens(text, line_start[4]);
  if ((int)tb.size() < nfil) return FS_ERR_IO;
  fil_start_h[0] = 0;
  for (int i = 0; i < nfil; ++i) {
    int nb = 0;
    if (!to_int(tb[i], &nb) || nb < 1 || fil_start_h[i] > 2147483647 - nb) return FS_ERR_IO;
    fil_start_h[i + 1] = fil_start_h[i] + nb;
  }
  *nfil_out = nfil;
  *np_out = fil_start_h[nfil];
  return FS_OK;
}

fs_status fs_backup_write(const char *path, const fs_host_state *s, int nt) {
  CNumericLocale c_numbers;
  if (!path || !layout_ok(s) || !s->X || !s->Xt || !s->q || !s->qt || !s->U || !s->Ut)
    return FS_ERR_INVALID_ARG;
  if (s->np > s->nfil && (!s->lam || !s->lam1 || !s->lam2)) return FS_ERR_INVALID_ARG;
  File out(path, "w");
  if (!out.f) return FS_ERR_IO;
  FILE *f = out.f;
  fprintf(f, "%d ", nt);
  for (int fil = 0; fil < s->nfil; ++fil) {
    for (int b = s->fil_start[fil]; b < s->fil_start[fil + 1]; ++b) {
      put_fixed(f, s->X + 3 * b, 3);   // current step
      put_fixed(f, s->Xt + 3 * b, 3);  // previous step
      // Bead::getQuatComponent (Bead.hpp:279-286): qs, scalar first; after
      // Filament::step qs and q hold the same expm(U) q
      put_fixed(f, (s->qs ? s->qs : s->q) + 4 * b, 4);
      put_fixed(f, s->qt + 4 * b, 4);
      put_fixed(f, s->U + 3 * b, 3);
      put_fixed(f, s->Ut + 3 * b, 3);
    }
    const int l0 = s->fil_start[fil] - fil, nl = s->fil_start[fil + 1] - s->fil_start[fil] - 1;
    for (int l = l0; l < l0 + nl; ++l) {
      put_fixed(f, s->lam + 3 * l, 3);
      put_fixed(f, s->lam1 + 3 * l, 3);
      put_fixed(f, s->lam2 + 3 * l, 3);
    }
  }
  return (ferror(f) || !out.close()) ? FS_ERR_IO : FS_OK;
}

fs_status fs_backup_read(const char *path, fs_host_state *s, int *nt_next) {
  CNumericLocale c_numbers;
  if (!path || !nt_next || !layout_ok(s) || !s->X || !s->Xt || !s->q || !s->qt || !s->U || !s->Ut)
    return FS_ERR_INVALID_ARG;
  const int nlink = s->np - s->nfil;
  if (nlink > 0 && (!s->lam || !s->lam1 || !s->lam2)) return FS_ERR_INVALID_ARG;
  std::string text;
  if (!read_all(path, &text)) return FS_ERR_IO;
  auto t = tokens(text);
  const size_t need = 1 + 20 * (size_t)s->np + 9 * (size_t)nlink;
  if (t.size() < need) return FS_ERR_IO;
  int nt = 0;
  if (!to_int(t[0], &nt)) return FS_ERR_IO;
  size_t k = 1;
  auto get = [&](double *dst, int n) {
    for (int i = 0; i < n; ++i)
      if (!to_double(t[k++], dst + i)) return false;
    return true;
  };
  for (int fil = 0; fil < s->nfil; ++fil) {
    for (int b = s->fil_start[fil]; b < s->fil_start[fil + 1]; ++b) {
      if (!get(s->X + 3 * b, 3) || !get(s->Xt + 3 * b, 3) || !get(s->q + 4 * b, 4) || !get(s->qt + 4 * b, 4) ||
          !get(s->U + 3 * b, 3) || !get(s->Ut + 3 * b, 3))
        return FS_ERR_IO;
      // Xs = X, qs = q, Us = U (Filament.hpp:697, 703, 715)
      if (s->Xs) memcpy(s->Xs + 3 * b, s->X + 3 * b, sizeof(double) * 3);
      if (s->qs) memcpy(s->qs + 4 * b, s->q + 4 * b, sizeof(double) * 4);
      if (s->Us) memcpy(s->Us + 3 * b, s->U + 3 * b, sizeof(double) * 3);
    }
    const int l0 = s->fil_start[fil] - fil, nl = s->fil_start[fil + 1] - s->fil_start[fil] - 1;
    for (int l = l0; l < l0 + nl; ++l)
      if (!get(s->lam + 3 * l, 3) || !get(s->lam1 + 3 * l, 3) || !get(s->lam2 + 3 * l, 3)) return FS_ERR_IO;
  }
  *nt_next = nt + 1;  // continue_from_checkpoint returns nt + 1 (file_functions.cpp:317)
  return FS_OK;
}

fs_status fs_data_write_header(const char *path, const fs_host_state *s) {
  CNumericLocale c_numbers;
  if (!path || !layout_ok(s)) return FS_ERR_INVALID_ARG;
  File out(path, "w");
  if (!out.f) return FS_ERR_IO;
  fprintf(out.f, "it ");
  for (int b = 0; b < s->np; ++b) fprintf(out.f, "X Y Z qr qi qj qk ");
  fprintf(out.f, "\n");
  return (ferror(out.f) || !out.close()) ? FS_ERR_IO : FS_OK;
}

fs_status fs_data_append(const char *path, const fs_host_state *s, int nt) {
  CNumericLocale c_numbers;
  if (!path || !layout_ok(s) || !s->Xs || !s->qs) return FS_ERR_INVALID_ARG;
  File out(path, "a");
  if (!out.f) return FS_ERR_IO;
  fprintf(out.f, "%d ", nt);
  for (int b = 0; b < s->np; ++b) {
    put_fixed(out.f, s->Xs + 3 * b, 3);
    put_fixed(out.f, s->qs + 4 * b, 4);
  }
  fprintf(out.f, "\n");
  return (ferror(out.f) || !out.close()) ? FS_ERR_IO : FS_OK;
}

}  // extern "C"
