// Command-line driver of the CPU oracle: runs <dir>/singleideal.ini for num_iter steps (or the
// count given) and prints the progress rows in the reference's progress.out format
// (singleideal_cpu.F90:1695-1732, format '(1i10,20es20.10)').  Test infrastructure only.
#include <cstdio>
#include <cstdlib>
#include <exception>

#include "oracle.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <case dir> [nsteps]\n", argv[0]);
    return 2;
  }
  try {
    streams_b200::Setup s = streams_b200::setup_from_dir(argv[1]);
    streams_oracle::Solver sol(s);
    int n = argc > 2 ? std::atoi(argv[2]) : s.num_iter;
    sol.init_run();
    sol.run(n);
    for (const auto& r : sol.rows)
      std::printf("%10d%20.10E%20.10E%20.10E%20.10E%20.10E%20.10E%20.10E%20.10E%20.10E%20.10E%20.10E%20.10E%20.10E\n",
                  r.icyc, r.dt, r.time, r.residual_rhou, r.dpdx_over_dt, r.rhobulk, r.ubulk, r.tbulk, r.rhomin,
                  r.rhomax, r.tmin, r.tmax, r.pmin, r.pmax);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
