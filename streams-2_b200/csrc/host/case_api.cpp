// Host case API and run driver (include/streams_b200_host.h).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

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

int streams_b200_case_write_state_stats(const streams_b200_case* c, const double* w, int icyc, double time,
                                        const double* w_stat, const double* w_stat_3d, int itav,
                                        double time_from_last_stat, const char* dir) {
  if (!c || !w || !dir || itav < 0) return STREAMS_B200_EINVAL;
  try {
    streams_b200::StatsOut st;
    st.w_stat = w_stat;
    st.w_stat_3d = w_stat_3d;
    st.itav = itav;
    st.time_from_last_stat = time_from_last_stat;
    streams_b200::write_restart_state(c->s, w, icyc, time, dir, &st);
  } catch (const std::exception& e) {
    g_case_err = e.what();
    return STREAMS_B200_EINVAL;
  }
  return STREAMS_B200_OK;
}

int streams_b200_case_stats_info(const streams_b200_case* c, double out[5]) {
  if (!c || !out) return STREAMS_B200_EINVAL;
  const auto& s = c->s;
  out[0] = s.dtstat; out[1] = s.enable_stat_time; out[2] = s.enable_stat_3d; out[3] = s.itav;
  out[4] = s.time_from_last_stat;
  return STREAMS_B200_OK;
}

int streams_b200_case_stats(const streams_b200_case* c, int which, double* out, long long n) {
  if (!c || !out || (which != 0 && which != 2)) return STREAMS_B200_EINVAL;
  const auto& s = c->s;
  const long long cnt = (long long)(which == 0 ? 70 : 14 * (long long)s.nzmax) * s.nxmax * s.nymax;
  if (n < cnt) return STREAMS_B200_EINVAL;
  const std::vector<double>& v = which == 0 ? s.w_stat : s.w_stat_3d;
  if (v.empty()) std::memset(out, 0, sizeof(double) * (size_t)cnt);
  else std::memcpy(out, v.data(), sizeof(double) * (size_t)cnt);
  return STREAMS_B200_OK;
}

int streams_b200_run_case(const streams_b200_case* c, int nsteps, int precision, const char* progress_path,
                          double* last_row, double* w_out) {
  return streams_b200_run_case_stats(c, nsteps, precision, progress_path, last_row, w_out, nullptr, nullptr,
                                     nullptr, nullptr);
}

int streams_b200_run_case_stats(const streams_b200_case* c, int nsteps, int precision, const char* progress_path,
                                double* last_row, double* w_out, double* w_stat_out, double* w_stat_3d_out,
                                double* stat_clock, const char* output_dir) {
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
  // running statistics (manage_output, singleideal_gpu.F90:2012-2034)
  const bool stat2 = s.dtstat >= 0.0 && s.enable_stat_time > 0;
  const bool stat3 = s.dtstat >= 0.0 && s.enable_stat_3d > 0;
  int itav = s.itav;
  double tfls = s.time_from_last_stat;
  const long long n2 = 70LL * s.nxmax * s.nymax, n3 = 14LL * s.nxmax * s.nymax * s.nzmax;
  if (stat2 && !s.w_stat.empty() && (rc = streams_b200_set_stats(ctx, 0, s.w_stat.data(), n2))) return done(rc);
  if (stat3 && !s.w_stat_3d.empty() && (rc = streams_b200_set_stats(ctx, 2, s.w_stat_3d.data(), n3)))
    return done(rc);
  const int n = nsteps < 0 ? s.num_iter : nsteps;
  int icyc = s.icyc0;
  while (icyc - s.icyc0 < n) {
    // advance up to the next print step without host synchronisation (one step at a time while
    // statistics are sampled: the sampling clock needs every step's dt)
    int chunk = s.print_control - ((icyc - s.icyc0) % s.print_control);
    if (icyc - s.icyc0 + chunk > n) chunk = n - (icyc - s.icyc0);
    if (stat2 || stat3) chunk = 1;
    if ((rc = streams_b200_advance(ctx, chunk, s.iter_dt_recompute, icyc, s.icyc0))) return done(rc);
    icyc += chunk;
    if (stat2 || stat3) {
      double sc[7];
      if ((rc = streams_b200_get_scalars(ctx, sc))) return done(rc);
      tfls = tfls + sc[0];
      if (tfls >= s.dtstat) {
        if (stat2 && (rc = streams_b200_compute_stats(ctx, itav))) return done(rc);
        if (stat3 && (rc = streams_b200_compute_stats_3d(ctx, itav))) return done(rc);
        tfls = 0.0;
        itav = itav + 1;
      }
    }
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
  std::vector<double> wfin, st2, st3;
  double* wdst = w_out;
  if (!wdst && output_dir) {
    wfin.resize(s.w.size());
    wdst = wfin.data();
  }
  if (wdst && (rc = streams_b200_copy_to_field(ctx, wdst))) return done(rc);
  double* s2 = w_stat_out;
  double* s3 = w_stat_3d_out;
  if (output_dir && stat2 && !s2) { st2.resize((size_t)n2); s2 = st2.data(); }
  if (output_dir && stat3 && !s3) { st3.resize((size_t)n3); s3 = st3.data(); }
  if (s2 && (rc = streams_b200_get_stats(ctx, 0, s2, n2))) return done(rc);
  if (s3 && (rc = streams_b200_get_stats(ctx, 2, s3, n3))) return done(rc);
  if (stat_clock) { stat_clock[0] = itav; stat_clock[1] = tfls; }
  double sc[7];
  if ((rc = streams_b200_get_scalars(ctx, sc))) return done(rc);
  if ((rc = streams_b200_synchronize(ctx))) return done(rc);
  if (output_dir) {
    try {
      streams_b200::StatsOut st;
      st.w_stat = stat2 ? s2 : nullptr;
      st.w_stat_3d = stat3 ? s3 : nullptr;
      st.itav = itav;
      st.time_from_last_stat = tfls;
      streams_b200::write_run_output(s, wdst, icyc, sc[1], output_dir, &st);
    } catch (const std::exception& e) {
      g_case_err = e.what();
      streams_b200_destroy(ctx);
      if (prog) std::fclose(prog);
      return STREAMS_B200_EINVAL;
    }
  }
  return done(STREAMS_B200_OK);
}

}  // extern "C"
