// main.cpp -- command-line solver, the operator surface of the reference's
// magmaHC-main (GPU-HC/cmd/magmaHC-main.cpp:30-115):
//
//   ghc-main -p <problem> [--root <problems dir>] [--precision fp64|fp32|mixed]
//            [--polish <iters>] [--out <dir>]
//
// Loads <root>/<problem>/gpuhc_settings.yaml and its data files, solves the
// shipped target parameters on the GPU, writes the converged endpoints to
// <out>/GPU_Converged_HC_tracks.txt in the reference's format
// (Evaluations::Write_Converged_Sols, GPU-HC/magmaHC/Evaluations.cpp:66-86)
// and prints the reference's counts (GPU_HC_Solver.cpp:366-383).
// Unlike the reference, failures exit non-zero.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unistd.h>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "../../include/ghc.h"

static void usage() {
  std::printf(
      "Usage: ghc-main -p <problem> [options]\n\n"
      "options:\n"
      "  -p, --problem     problem folder name (e.g. P3P)\n"
      "  -r, --root        directory holding the problem folders (default: problems/ next to this binary)\n"
      "  --precision       fp64 (default) | fp32 | mixed\n"
      "  --polish          Newton iterations at t = 1 after tracking (default 0 = reference behaviour)\n"
      "  -o, --out         directory for GPU_Converged_HC_tracks.txt (default: current directory)\n"
      "  -h, --help        show this help message and exit\n");
}

static std::string exe_dir(const char* argv0) {
  char buf[4096];
  const ssize_t n = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
  std::string p = n > 0 ? std::string(buf, n) : std::string(argv0);
  const size_t s = p.rfind('/');
  return s == std::string::npos ? std::string(".") : p.substr(0, s);
}

int main(int argc, char** argv) {
  std::string problem, root = exe_dir(argv[0]) + "/problems", out = ".", prec = "fp64";
  int polish = 0;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto next = [&](std::string& dst) {
      if (i + 1 >= argc) {
        usage();
        std::exit(2);
      }
      dst = argv[++i];
    };
    if (a == "-p" || a == "--problem") next(problem);
    else if (a == "-r" || a == "--root") next(root);
    else if (a == "-o" || a == "--out") next(out);
    else if (a == "--precision") next(prec);
    else if (a == "--polish") {
      std::string v;
      next(v);
      polish = std::atoi(v.c_str());
    } else if (a == "-h" || a == "--help") {
      usage();
      return 0;
    } else {
      std::fprintf(stderr, "[ERROR] unknown argument %s\n", a.c_str());
      usage();
      return 2;
    }
  }
  if (problem.empty()) {
    usage();
    return 2;
  }
  const int precision = prec == "fp32" ? GHC_PREC_FP32 : prec == "mixed" ? GHC_PREC_MIXED : GHC_PREC_FP64;
  if (prec != "fp64" && prec != "fp32" && prec != "mixed") {
    std::fprintf(stderr, "[ERROR] --precision must be fp64, fp32 or mixed\n");
    return 2;
  }
  ghc_problem* pb = nullptr;
  int rc = ghc_problem_load(root.c_str(), problem.c_str(), &pb);
  if (rc) {
    std::fprintf(stderr, "[DATA LOAD ERROR] %s\n", ghc_last_error());
    return 1;
  }
  ghc_problem_info info;
  ghc_problem_get_info(pb, &info);
  const long n = info.paths;
  std::vector<double> ep(2 * (size_t)n * info.N);
  std::vector<uint8_t> status(n), conv(n), inf(n);
  std::vector<int32_t> steps(n);
  double ms[3] = {0, 0, 0};
  rc = ghc_solve_host(pb, precision, 1, nullptr, 1.0, polish, ep.data(), status.data(), conv.data(), inf.data(),
                      steps.data(), ms);
  if (rc) {
    std::fprintf(stderr, "[ERROR] %s\n", ghc_last_error());
    ghc_problem_free(pb);
    return 1;
  }
  const std::string path = out + "/GPU_Converged_HC_tracks.txt";
  std::ofstream f(path);
  if (!f) {
    std::fprintf(stderr, "[ERROR] File %s not writable\n", path.c_str());
  } else {
    f << "-------------------- RANSAC Iteration 1 --------------------\n\n";
    for (long bs = 0; bs < n; ++bs) {
      if (!conv[bs]) continue;
      for (int v = 0; v < info.N; ++v)
        f << std::setprecision(20) << ep[2 * ((size_t)bs * info.N + v)] << "\t" << std::setprecision(20)
          << ep[2 * ((size_t)bs * info.N + v) + 1] << "\n";
      f << "\n";
    }
    f << "\n";
  }
  ghc_counts c;
  // the reference's tolerances (GPU-HC/magmaHC/definitions.hpp:24-25): 1e-4 for the imaginary parts and duplicates
  ghc_count_results(info.N, (int)n, ep.data(), conv.data(), inf.data(), 1e-4, 1e-4, &c);
  std::printf("---------------------------------------------------------------------------------\n");
  std::printf("## Solving %s (%s)\n", info.name, prec.c_str());
  std::printf("## Timings:\n");
  std::printf(" - GPU Computation Time = %7.2f (ms)\n", ms[1]);
  std::printf(" - H2D Transfer Time    = %7.2f (ms)\n", ms[0]);
  std::printf(" - D2H Transfer Time    = %7.2f (ms)\n", ms[2]);
  std::printf("## Evaluation of GPU-HC Solutions: \n");
  std::printf(" - Number of Converged Solutions:       %d\n", c.converged);
  std::printf(" - Number of Real Solutions:            %d\n", c.real);
  std::printf(" - Number of Infinity Failed Solutions: %d\n", c.infinity);
  std::printf(" - Number of Unique Solutions:          %d\n", c.unique);
  ghc_problem_free(pb);
  return 0;
}
