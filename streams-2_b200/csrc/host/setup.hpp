// Host-side set-up of a Cartesian STREAmS-2 case: the part of the equation object that runs
// once before the time loop (input parsing, fluid and flow parameters, grid and metrics,
// near-boundary order reduction, initial field).  In the drop-in build this is done by the
// reference's own Fortran equation object (code/src/singleideal/singleideal.F90:284-864) and the
// backend only receives the resulting arrays through the C ABI; this C++ restatement lets the
// backend run stand-alone (driver, tests, bench) from the same singleideal.ini.
//
// Supported here: grid_dim = 1 (Cartesian), grid_type FROMFILE / UNIFORM / CHA, flow_init 0
// (channel), restart_type 0 and 1 (rst.bin), calorically perfect gas, Wray RK3.  Seeded
// random numbers use glibc srand/rand as code/third-party/crandom/crandom.c does; the per-rank
// seeding of an MPI decomposition (seed = rank+1, rank order of MPI_Cart_create with
// reorder=false) is emulated so that multi-rank reference runs are reproduced bit for bit.
#pragma once

#include <string>
#include <vector>

#include "ini.hpp"
#include "streams_b200.h"

namespace streams_b200 {

// Offset arrays: value of index i (Fortran lower bound lo) is at data[i - lo].
struct OffsetArray {
  int lo = 0;
  std::vector<double> data;
  double& operator()(int i) { return data[static_cast<size_t>(i - lo)]; }
  double operator()(int i) const { return data[static_cast<size_t>(i - lo)]; }
  void resize(int lo_, int hi_) {
    lo = lo_;
    data.assign(static_cast<size_t>(hi_ - lo_ + 1), 0.0);
  }
};

struct Setup {
  IniFile ini;
  std::string dir;  // directory holding singleideal.ini and the grid/restart files

  // sizes (single block: nx = nxmax ...)
  int nxmax = 0, nymax = 0, nzmax = 0, ng = 3, ndim = 3;
  int grid_type = 0, metrics_order = 6;
  bool periodic[3] = {false, false, false};
  double domain_size[3] = {0, 0, 0};

  // emulated MPI decomposition (only used to reproduce per-rank random seeding)
  int x_split = 1, y_split = 1, z_split = 1;

  // global grid (grid.F90 naming)
  OffsetArray xg, yg, zg, yn;           // xg(1-ng:nxmax+ng+1), yg(1-ng:nymax+ng), zg(1-ng:nzmax+ng), yn(1:nymax+1+ng)
  OffsetArray dxg, dyg, dzg, d2xg, d2yg, d2zg;
  // local metrics (field.F90 set_local_grid)
  std::vector<double> x, y, z, ynl;     // x(1-ng:nx+ng) ..., ynl = yn(1:ny+1)
  std::vector<double> dcsidx, detady, dzitdz, dcsidxs, detadys, dzitdzs, dcsidx2, detady2, dzitdz2;
  double coeff_deriv1[4][4] = {};       // [lmax-1][l-1]
  double coeff_deriv2[4][5] = {};
  std::vector<int> ep_ord[3];           // ep_ord_change per direction, 0..n

  // flow/fluid parameters
  int flow_init = 0, visc_model = 1, calorically_perfect = 1, indx_cp_l = 0, indx_cp_r = 0, rfac_type = 0;
  double gam = 1.4, gm = 2.5, gm1 = 0.4, prandtl = 0.72, rfac = 0, powerlaw_vtexp = 0.76,
         sutherland_s = 110.4, t_ref_dim = 220;
  std::vector<double> cp_coeff, cv_coeff;  // indices indx_cp_l..indx_cp_r+1 stored from 0
  double l0 = 1, t0 = 1, rho0 = 1, rgas0 = 1;
  double mach = 0, reynolds = 0, reynolds_friction = 0, theta_wall = 0, aoa = 0;
  double t_recovery = 0, t_wall = 0, t_bulk_target = 0;
  double p0 = 0, c0 = 0, u0 = 0, mu0 = 0, s0 = 0, ttot0 = 0, ptot0 = 0;
  double winf[5] = {0, 0, 0, 0, 0};
  double volchan = 0;
  bool channel_case = false;

  // numerics
  int ep_order = 6, nkeep = 0, visc_order = 6, conservative_viscous = 1, weno_scheme = 3,
      weno_version = 0, flux_splitting = 0, rk_type = 1, rand_type = 2, correct_bound_ord = 0;
  double sensor_threshold = 0;
  int nrk = 3;
  double rhork[3] = {0, 0, 0}, gamrk[3] = {0, 0, 0};

  // boundary conditions
  int bctags[6] = {0, 0, 0, 0, 0, 0}, bctags_nr[6] = {0, 0, 0, 0, 0, 0}, force_zero_flux[6] = {0, 0, 0, 0, 0, 0};
  int eul_imin = 1, eul_imax = 1, eul_jmin = 1, eul_jmax = 1, eul_kmin = 1, eul_kmax = 1;
  bool is_y_staggered = false;

  // controls
  int restart_type = 0, num_iter = 0, iter_dt_recompute = 1, print_control = 1, icyc0 = 0;
  double cfl = 0, time0 = 0;

  // boundary layer (flow_init = 1): recycling-rescaling inflow (recyc_prepare,
  // singleideal.F90:1512-1588) and the mean profile it rescales
  bool recyc = false;
  double x_recyc = 0, betarecyc = 1, glund1 = 1;
  int i_recyc = 0, jbl_inflow = 1;
  std::vector<double> deltavec, deltavvec;  // BL thickness / viscous length at xg(1-ng .. nxmax+ng+1)
  std::vector<double> wmean;                // wmean(1-ng:nx+ng+1, 1:ny, 4), Fortran order
  std::vector<double> yplus_inflow, eta_inflow, yplus_recyc, eta_recyc, eta_recyc_blend;  // (1-ng:ny+ng)
  std::vector<int> map_j_inn, map_j_out, map_j_out_blend;  // (1:ny)
  std::vector<double> weta_inflow;          // (1:ny)
  std::vector<double> wmean_inflow;         // wmean(1-i, j, m), i = 1..ng: [m][j][i-1] (C order)
  // state of the crandom sequence after the set-up (seed and draws taken): the solver draws the
  // recycling plane's random perturbations from it at every stage
  unsigned rng_seed = 1;
  long long rng_draws = 0;
  // impinging oblique shock (bc ymax = 7, set_oblique_shock singleideal.F90:2953-3016)
  double xshock_imp = 0, shock_angle = 0, tanhfacs = 1;
  double winf_past_shock[5] = {0, 0, 0, 0, 0};

  // running statistics ([output] dtstat, enable_stat_time, enable_stat_3d): the averaging clock
  // and, on a restart with restart_type = 2, the averages read from stat.bin / stat3d.bin in the
  // reference's layouts w_stat(70, nx, ny), w_stat_3d(14, nx, ny, nz) (empty: start from zero)
  double dtstat = -1.0;  // < 0: the key is absent and the stand-alone run loop samples nothing
  int enable_stat_time = 1, enable_stat_3d = 0;
  int itav = 0;
  double time_from_last_stat = 0.0;
  std::vector<double> w_stat, w_stat_3d;

  // initial conserved field w(1-ng:nx+ng,1-ng:ny+ng,1-ng:nz+ng,5), Fortran order
  std::vector<double> w;

  size_t ncells_ghost() const {
    return static_cast<size_t>(nxmax + 2 * ng) * (nymax + 2 * ng) * (nzmax + 2 * ng);
  }
  size_t widx(int i, int j, int k, int m) const {
    const size_t sx = nxmax + 2 * ng, sy = nymax + 2 * ng, sz = nzmax + 2 * ng;
    return (((static_cast<size_t>(m) * sz + (k + ng - 1)) * sy + (j + ng - 1)) * sx + (i + ng - 1));
  }

  // Fill the C-ABI structs; the grid struct points into this object.
  void fill_params(streams_b200_params* p, int precision) const;
  void fill_grid(streams_b200_grid* g) const;
};

// Build a case from <dir>/singleideal.ini (and grid / restart files in <dir> when used).
Setup setup_from_dir(const std::string& dir);
// Build a case from an already parsed input (files are looked up in dir).
Setup setup_from_ini(const IniFile& ini, const std::string& dir);

// get_reynolds_cha (singleideal.F90:3052-3172): bulk Reynolds number of a channel with
// friction Reynolds number retau.  yn has ny+1 entries (half channel).
double get_reynolds_cha(double retau, double rm, double trat, double s2tinf, double vtexp, bool visc_exp,
                        double gam, double rfac, int ny, const double* yn);

// Write the files with which the reference itself starts the same case:
// x.dat, y.dat, z.dat, yn.dat (with ghosts), rst.bin and field_info0.dat.
void write_restart_inputs(const Setup& s, const std::string& dir);
// Running statistics to write with a restart (null arrays are not written).
struct StatsOut {
  const double* w_stat = nullptr;     // (70, nx, ny)
  const double* w_stat_3d = nullptr;  // (14, nx, ny, nz)
  int itav = 0;
  double time_from_last_stat = 0.0;
};
// The same from a conserved field w (ghosted, Fortran order) at step icyc and time, plus a
// singleideal.ini of the case with restart_type = 1 (2 with statistics): a run resumes from dir.
void write_restart_state(const Setup& s, const double* w, int icyc, double time, const std::string& dir,
                         const StatsOut* st = nullptr);
// The files the end of run() writes (singleideal_gpu.F90:1660-1683): rst.bin, stat.bin and
// stat3d.bin when given, field_info0.dat.
void write_run_output(const Setup& s, const double* w, int icyc, double time, const std::string& dir,
                      const StatsOut* st);

}  // namespace streams_b200
