// C entry points of the CPU oracle for the test suite (ctypes) and the CPU-baseline timing.
// Test infrastructure only.
#include <cstring>
#include <exception>
#include <string>

#include "oracle.hpp"

using streams_oracle::Solver;

namespace {
struct Handle {
  streams_b200::Setup setup;
  Solver* solver = nullptr;
};
thread_local std::string g_err;
}  // namespace

extern "C" {

const char* oracle_error(void) { return g_err.c_str(); }

void* oracle_create(const char* dir, const char* ini_text) {
  try {
    auto* h = new Handle();
    if (ini_text && ini_text[0])
      h->setup = streams_b200::setup_from_ini(streams_b200::IniFile::parse_text(ini_text), dir ? dir : ".");
    else
      h->setup = streams_b200::setup_from_dir(dir ? dir : ".");
    h->solver = new Solver(h->setup);
    return h;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void oracle_destroy(void* hp) {
  auto* h = static_cast<Handle*>(hp);
  if (!h) return;
  delete h->solver;
  delete h;
}

void oracle_init_run(void* hp) { static_cast<Handle*>(hp)->solver->init_run(); }
void oracle_step(void* hp) { static_cast<Handle*>(hp)->solver->step(); }
void oracle_run(void* hp, int n) { static_cast<Handle*>(hp)->solver->run(n); }
void oracle_rk_sync(void* hp) { static_cast<Handle*>(hp)->solver->rk_sync(); }
void oracle_compute_dt(void* hp) {
  auto* s = static_cast<Handle*>(hp)->solver;
  s->compute_aux(1, 0);
  s->compute_dt();
}
// fhat of nface faces (dir, i, j, k) = ijk[4q .. 4q+3] from the current w_aux into out[5q ..]
void oracle_face_flux(void* hp, int nface, const int* ijk, double* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  for (int q = 0; q < nface; ++q) s->face_flux_at(ijk[4 * q], ijk[4 * q + 1], ijk[4 * q + 2], ijk[4 * q + 3], out + 5 * q);
}
// FP64 operations of the face flux at (dir, i, j, k) from the current w_aux, counted through the
// oracle's own code (flops.hpp): out = add/sub, mul, div, sqrt, pow/log, comparisons and max
void oracle_face_flops(void* hp, int dir, int i, int j, int k, long long* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  streams_oracle::flop_tally() = streams_oracle::FlopTally();
  streams_oracle::Counted fh[5];
  s->face_flux_t(dir, i, j, k, fh);
  const auto& t = streams_oracle::flop_tally();
  out[0] = t.add; out[1] = t.mul; out[2] = t.div; out[3] = t.sqrt; out[4] = t.special; out[5] = t.cmp;
}
void oracle_set_dt(void* hp, double dt) { static_cast<Handle*>(hp)->solver->dt = dt; }
void oracle_compute_residual(void* hp) { static_cast<Handle*>(hp)->solver->compute_residual(); }

// sizes[0..3] = nx, ny, nz, ng
void oracle_sizes(void* hp, int* sizes) {
  auto* s = static_cast<Handle*>(hp)->solver;
  sizes[0] = s->nx; sizes[1] = s->ny; sizes[2] = s->nz; sizes[3] = s->ng;
}

void oracle_get_w(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  std::memcpy(out, s->w.data(), s->w.size() * sizeof(double));
}
void oracle_set_w(void* hp, const double* in) {
  auto* s = static_cast<Handle*>(hp)->solver;
  std::memcpy(s->w.data(), in, s->w.size() * sizeof(double));
}
// w_aux(1-ng:..,1:10) Fortran order
void oracle_get_waux(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  std::memcpy(out, s->w_aux.data(), s->w_aux.size() * sizeof(double));
}
void oracle_get_fl(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  std::memcpy(out, s->fl.data(), s->fl.size() * sizeof(double));
}
void oracle_get_fln(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  std::memcpy(out, s->fln.data(), s->fln.size() * sizeof(double));
}
void oracle_get_wallprop(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  std::memcpy(out, s->wallprop.data(), s->wallprop.size() * sizeof(double));
}

// out[0..6] = dt, time, dpdx, rhobulk, ubulk, tbulk, icyc
void oracle_get_scalars(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  out[0] = s->dt; out[1] = s->time; out[2] = s->dpdx; out[3] = s->rhobulk;
  out[4] = s->ubulk; out[5] = s->tbulk; out[6] = s->icyc;
}

// last progress row: 14 columns as in progress.out; returns 0 when no row exists
int oracle_last_progress(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  if (s->rows.empty()) return 0;
  const auto& r = s->rows.back();
  double v[14] = {static_cast<double>(r.icyc), r.dt, r.time, r.residual_rhou, r.dpdx_over_dt, r.rhobulk, r.ubulk,
                  r.tbulk, r.rhomin, r.rhomax, r.tmin, r.tmax, r.pmin, r.pmax};
  std::memcpy(out, v, sizeof(v));
  return 1;
}

// residual row after compute_residual: residual_rhou (raw), rhomin, rhomax, tmin, tmax, pmin, pmax
void oracle_get_residual(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  out[0] = s->residual_rhou; out[1] = s->rhomin; out[2] = s->rhomax; out[3] = s->tmin;
  out[4] = s->tmax; out[5] = s->pmin; out[6] = s->pmax;
}

// running statistics: compute_stats / compute_stats_3d with itav samples already averaged; then
// w_stat(70,nx,ny), w_stat_z(70,nx,ny) or w_stat_3d(14,nx,ny,nz) (which = 0, 1, 2)
void oracle_compute_stats(void* hp, int itav) { static_cast<Handle*>(hp)->solver->compute_stats(itav); }
void oracle_compute_stats_3d(void* hp, int itav) { static_cast<Handle*>(hp)->solver->compute_stats_3d(itav); }
void oracle_set_stats(void* hp, int which, const double* in) {
  auto* s = static_cast<Handle*>(hp)->solver;
  const size_t n2 = static_cast<size_t>(Solver::NV_STAT) * s->nx * s->ny;
  if (which == 0) s->w_stat.assign(in, in + n2);
  if (which == 2) s->w_stat_3d.assign(in, in + static_cast<size_t>(Solver::NV_STAT_3D) * s->nint_());
}
void oracle_get_stats(void* hp, int which, double* out) {
  auto* s = static_cast<Handle*>(hp)->solver;
  const std::vector<double>& v = which == 0 ? s->w_stat : (which == 1 ? s->w_stat_z : s->w_stat_3d);
  std::memcpy(out, v.data(), v.size() * sizeof(double));
}

// case parameters used by the tests: u0, rho0, l0, mu0, volchan, t_bulk_target, num_iter, print_control
void oracle_case_info(void* hp, double* out) {
  const auto& st = static_cast<Handle*>(hp)->setup;
  out[0] = st.u0; out[1] = st.rho0; out[2] = st.l0; out[3] = st.mu0; out[4] = st.volchan;
  out[5] = st.t_bulk_target; out[6] = st.num_iter; out[7] = st.print_control;
}

}  // extern "C"
