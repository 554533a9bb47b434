// Stand-alone driver: the counterpart of main_<backend>.F90 (code/src/singleideal/main_cpu.F90:1-18)
// for the B200 backend.  Runs <dir>/singleideal.ini on the current GPU, writes <dir>/progress.out
// and, at the end, the restart files of the reference's run() into <dir>.
//   streams_b200_run <dir> [nsteps] [precision]
#include <cstdio>
#include <cstdlib>
#include <string>

#include "streams_b200_host.h"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <case dir> [nsteps] [precision 0|1]\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  const int nsteps = argc > 2 ? std::atoi(argv[2]) : -1;
  const int prec = argc > 3 ? std::atoi(argv[3]) : 0;
  streams_b200_case* c = nullptr;
  if (streams_b200_case_load(dir.c_str(), nullptr, &c)) {
    std::fprintf(stderr, "input error: %s\n", streams_b200_case_error());
    return 1;
  }
  double row[14];
  const std::string prog = dir + "/progress.out";
  // as run() ends: rst.bin, stat.bin / stat3d.bin (when [output] dtstat is set) and field_info0.dat
  int rc = streams_b200_run_case_stats(c, nsteps, prec, prog.c_str(), row, nullptr, nullptr, nullptr, nullptr,
                                       dir.c_str());
  if (rc) {
    std::fprintf(stderr, "run failed (%d): %s\n", rc, streams_b200_case_error());
    streams_b200_case_free(c);
    return rc == STREAMS_B200_ENAN ? 99 : 1;
  }
  std::printf("%10d", (int)row[0]);
  for (int q = 1; q < 14; ++q) std::printf("%20.10E", row[q]);
  std::printf("\n");
  streams_b200_case_free(c);
  return 0;
}
