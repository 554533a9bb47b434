// CPU oracle (test infrastructure, not product code).
//
// A C++ restatement of STREAmS-2's pure-MPI CPU backend for the Cartesian per-Runge-Kutta-stage
// right-hand side and update, on one block (the MPI halo exchange becomes a periodic copy):
//   control flow : code/src/singleideal/singleideal_cpu.F90 (run, rk_sync, force_rhs, force_var,
//                  update_ghost, compute_dt, compute_residual, print_progress, visflx, compute_aux)
//   arithmetic   : code/src/singleideal/kernels_cpu.F90 (each routine below cites its lines)
//   ghost fills  : code/src/base_cpu.F90 bcswap / bcswap_var (face halos only, no corners)
// The case set-up (grid, parameters, initial field) comes from the package's host set-up code
// (streams-2_b200/csrc/host/setup.cpp); the golden progress row of the reference's own
// regression suite (tests/tests.ini, subsonic_channel) pins set-up and time advance together.
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg use this code, as the checker.
#pragma once

#include <string>
#include <vector>

#include "flops.hpp"
#include "glibc_rand.hpp"
#include "setup.hpp"

namespace streams_oracle {

using streams_b200::Setup;

struct ProgressRow {
  int icyc;
  double dt, time, residual_rhou, dpdx_over_dt, rhobulk, ubulk, tbulk, rhomin, rhomax, tmin, tmax, pmin, pmax;
};

class Solver {
 public:
  explicit Solver(const Setup& s);

  // run() preamble (singleideal_cpu.F90:1542-1557 and the first compute_dt)
  void init_run();
  // one iteration of the integration loop (singleideal_cpu.F90:1576-1637, cfl > 0 path)
  void step();
  // integration loop for n steps; appends a progress row at every print_control step
  void run(int nsteps);

  void compute_aux(int central, int ghost);
  void compute_dt();
  void rk_sync();
  void compute_residual();
  ProgressRow progress_row() const;
  // hybrid convective flux at face (i,j,k) of direction dir (0 x, 1 y, 2 z) from the current
  // w_aux (fhat of euler_{x,y,z}_*hybrid_kernel); the test suite checks it face by face against
  // an independent restatement
  void face_flux_at(int dir, int i, int j, int k, double fh[5]) const { face_flux(dir, i, j, k, fh); }

  // running statistics, as manage_output calls them after a step (itav samples already averaged):
  // compute_stats (singleideal.F90:2003-2179) and compute_stats_3d (:2513-2543)
  static constexpr int NV_STAT = 70, NV_STAT_3D = 14;
  void compute_stats(int itav);
  void compute_stats_3d(int itav);
  std::vector<double> w_stat, w_stat_z;  // (nv_stat, nx, ny), statistic index fastest
  std::vector<double> w_stat_3d;         // (nv_stat_3d, nx, ny, nz)

  // state (Fortran layouts)
  const Setup& s;
  int nx, ny, nz, ng, sx, sy, sz;
  std::vector<double> w;      // w(1-ng:nx+ng,1-ng:ny+ng,1-ng:nz+ng,5)
  std::vector<double> w_aux;  // w_aux(...,10)
  std::vector<double> fl, fln;  // (nx,ny,nz,5)
  std::vector<double> fhat;   // (1-ng:..., 5)
  std::vector<double> wallprop;  // (1-ng:nx+ng,1-ng:nz+ng,2:4)
  double dt = 0, time = 0, dpdx = 0, rhobulk = 0, ubulk = 0, tbulk = 0;
  double residual_rhou = 0, rhomin = 0, rhomax = 0, tmin = 0, tmax = 0, pmin = 0, pmax = 0;
  int icyc = 0;
  std::vector<ProgressRow> rows;
  // recycling inflow: the random plane inflow_random_plane(1:ny,1:nz,1:3) and the crandom
  // sequence it is drawn from (continued from the set-up's draws)
  std::vector<double> random_plane;
  streams_b200::GlibcRand rng{1};

  size_t gi(int i, int j, int k) const {
    return (static_cast<size_t>(k + ng - 1) * sy + (j + ng - 1)) * sx + (i + ng - 1);
  }
  size_t ncg() const { return static_cast<size_t>(sx) * sy * sz; }
  double& W(int i, int j, int k, int m) { return w[m * ncg() + gi(i, j, k)]; }
  double& A(int i, int j, int k, int m) { return w_aux[(m - 1) * ncg() + gi(i, j, k)]; }
  double A(int i, int j, int k, int m) const { return w_aux[(m - 1) * ncg() + gi(i, j, k)]; }
  double& FH(int i, int j, int k, int m) { return fhat[(m - 1) * ncg() + gi(i, j, k)]; }
  size_t ii(int i, int j, int k) const { return (static_cast<size_t>(k - 1) * ny + (j - 1)) * nx + (i - 1); }
  size_t nint_() const { return static_cast<size_t>(nx) * ny * nz; }
  double& FL(int i, int j, int k, int m) { return fl[(m - 1) * nint_() + ii(i, j, k)]; }
  double& FLN(int i, int j, int k, int m) { return fln[(m - 1) * nint_() + ii(i, j, k)]; }

  // grid accessors (1-based, ghosts included)
  double X(int i) const { return s.x[i + ng - 1]; }
  double Y(int j) const { return s.y[j + ng - 1]; }
  double Z(int k) const { return s.z[k + ng - 1]; }

 private:
  void bcswap();
  void bcswap_var(int m);
  void update_ghost(int do_swap);
  void eval_aux(int i0, int i1, int j0, int j1, int k0, int k1);
  void euler(int dir);
  void visflx_reduced_ord2(int update_sensor);
  void visflx_faces();
  void sensor();
  void bcextr_var(int m);
  void visflx_div_ord2();
  void visflx_nosensor();
  void sensor_visc_order();
  void visflx_div();
  void force_rhs();
  void force_var();
  void face_flux(int dir, int i, int j, int k, double fh[5]) const;
 public:
  // the same face flux in any scalar type (Counted of flops.hpp tallies its operations)
  template <class T>
  void face_flux_t(int dir, int i, int j, int k, T fh[5]) const;

 private:
  void bcextr(int ilat);
  void bcwall(int ilat);
  void bcwall_staggered(int ilat);
  void bcrecyc();
  void bcshock();
  void draw_random_plane();
  void bc_nr();
  // thermodynamics (kernels_cpu.F90:7096-7176): get_temperature_from_e_dev (Newton from t_start
  // for a thermally perfect gas), get_e_from_temperature_dev, get_gamloc_dev, cp(T)
  double temp_from_e(double ee, double t_start) const;
  double e_from_temp(double tt) const;
  double cploc_at(double tt) const;
  double gamloc_at(double tt) const;
  double cp(int l) const { return s.cp_coeff[static_cast<size_t>(l - s.indx_cp_l)]; }
  double cv(int l) const { return s.cv_coeff[static_cast<size_t>(l - s.indx_cp_l)]; }
};

}  // namespace streams_oracle
