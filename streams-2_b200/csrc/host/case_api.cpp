// Host case API and run driver (include/streams_b200_host.h).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>

#include "setup.hpp"
#include "streams_b200_host.h"

struct streams_b200_case {
  streams_b200::Setup s;
};

namespace {
thread_local std::string g_case_err;
}

extern "C" {

const char* streams_b200_case_error(void) { return g_case_err.c_str(); }

int streams_b200_case_load(const char* dir, const char* ini_text, streams_b200_case** out) {
  if (!out) return STREAMS_B200_EINVAL;
  *out = nullptr;
  try {
    auto* c = new streams_b200_case();
    const std::string d = dir ? dir : ".";
    if (ini_text && ini_text[0])
      c->s = streams_b200::setup_from_ini(streams_b200::IniFile::parse_text(ini_text), d);
    else
      c->s = streams_b200::setup_from_dir(d);
    *out = c;
    return STREAMS_B200_OK;
  } catch (const std::exception& e) {
    g_case_err = e.what();
    return STREAMS_B200_EINVAL;
  }
}

int streams_b200_case_free(streams_b200_case* c) {
  delete c;
  return STREAMS_B200_OK;
}

int streams_b200_case_params(const streams_b200_case* c, int precision, streams_b200_params* out) {
  if (!c || !out) return STREAMS_B200_EINVAL;
  c->s.fill_params(out, precision);
  return STREAMS_B200_OK;
}

int streams_b200_case_grid(const streams_b200_case* c, streams_b200_grid* out) {
  if (!c || !out) return STREAMS_B200_EINVAL;
  c->s.fill_grid(out);
  return STREAMS_B200_OK;
}

const double* streams_b200_case_field(const streams_b200_case* c) { return c ? c->s.w.data() : nullptr; }

int streams_b200_case_info(const streams_b200_case* c, double out[12]) {
  if (!c || !out) return STREAMS_B200_EINVAL;
  const auto& s = c->s;
  double v[12] = {s.u0, s.rho0, s.l0, s.mu0, (double)s.num_iter, (double)s.print_control,
                  (double)s.iter_dt_recompute, (double)s.icyc0, s.time0, s.cfl, s.volchan, s.t_bulk_target};
  std::memcpy(out, v, sizeof(v));
  return STREAMS_B200_OK;
}

int streams_b200_case_write_restart(const streams_b200_case* c, const char* dir) {
  if (!c || !dir) return STREAMS_B200_EINVAL;
  try {
    streams_b200::write_restart_inputs(c->s, dir);
  } catch (const std::exception& e) {
    g_case_err = e.what();
    return STREAMS_B200_EINVAL;
  }
  return STREAMS_B200_OK;
}

int streams_b200_case_write_state(const streams_b200_case* c, const double* w, int icyc, double time,
                                  const char* dir) {
  if (!c || !w || !dir) return STREAMS_B200_EINVAL;
  try {
    streams_b200::write_restart_state(c->s, w, icyc, time, dir);
  } catch (const std::exception& e) {
    g_case_err = e.what();
    return STREAMS_B200_EINVAL;
  }
  return STREAMS_B200_OK;
}

int streams_b200_run_case(const streams_b200_case* c, int nsteps, int precision, const char* progress_path,
                          double* last_row, double* w_out) {
  if (!c) return STREAMS_B200_EINVAL;
  const auto& s = c->s;
  streams_b200_params p;
  streams_b200_grid g;
  s.fill_params(&p, precision);
  s.fill_grid(&g);
  streams_b200_ctx* ctx = nullptr;
  int rc = streams_b200_create(&p, &g, &ctx);
  if (rc) {
    g_case_err = streams_b200_global_error();
    return rc;
  }
  FILE* prog = progress_path ? std::fopen(progress_path, "w") : nullptr;
  auto done = [&](int code) {
    if (code) g_case_err = streams_b200_last_error(ctx);
    if (prog) std::fclose(prog);
    streams_b200_destroy(ctx);
    return code;
  };
  if ((rc = streams_b200_copy_from_field(ctx, s.w.data()))) return done(rc);
  if ((rc = streams_b200_set_time(ctx, s.time0))) return done(rc);
  if ((rc = streams_b200_init_run(ctx))) return done(rc);
  const int n = nsteps < 0 ? s.num_iter : nsteps;
  int icyc = s.icyc0;
  while (icyc - s.icyc0 < n) {
    // advance up to the next print step without host synchronisation
    int chunk = s.print_control - ((icyc - s.icyc0) % s.print_control);
    if (icyc - s.icyc0 + chunk > n) chunk = n - (icyc - s.icyc0);
    if ((rc = streams_b200_advance(ctx, chunk, s.iter_dt_recompute, icyc, s.icyc0))) return done(rc);
    icyc += chunk;
    if ((icyc - s.icyc0) % s.print_control == 0) {
      double res[7], sc[7];
      int rr = streams_b200_compute_residual(ctx, res);
      if ((rc = streams_b200_get_scalars(ctx, sc))) return done(rc);
      // print_progress (singleideal_cpu.F90:1695-1732)
      const double resn = res[0] / (s.u0 * s.u0) / s.rho0 * s.l0;
      const double dpn = sc[2] / (s.u0 * s.u0) / s.rho0 * s.l0;
      double row[14] = {(double)icyc, sc[0], sc[1], resn, -dpn / sc[0], sc[3], sc[4], sc[5],
                        res[1], res[2], res[3], res[4], res[5], res[6]};
      if (last_row) std::memcpy(last_row, row, sizeof(row));
      if (prog) {
        std::fprintf(prog, "%10d", icyc);
        for (int q = 1; q < 14; ++q) std::fprintf(prog, "%20.10E", row[q]);
        std::fprintf(prog, "\n");
        std::fflush(prog);
      }
      if (rr == STREAMS_B200_ENAN) return done(rr);
      if (rr) return done(rr);
    }
  }
  if (w_out && (rc = streams_b200_copy_to_field(ctx, w_out))) return done(rc);
  if ((rc = streams_b200_synchronize(ctx))) return done(rc);
  return done(STREAMS_B200_OK);
}

}  // extern "C"
