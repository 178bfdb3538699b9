// krans_nullspace on the B200 engine: the reference CLI
// (apps/krans_nullspace.cpp) for its iterative solvers, with the same flags,
// defaults, outputs (N.csv, report.json, N_left.csv) and exit codes, running
// on the device through the C++ drop-in adapters. The reference's direct
// dense solvers (svd, qrcp, cod, fullpivlu) and the optional third-party
// solvers are not part of the device engine and are reported as unknown.
#include <algorithm>
#include <chrono>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "krans/Solvers/CyclicLanczosSolver.hpp"
#include "krans/Solvers/LOBPCGSolver.hpp"
#include "krans/adapters/cuda/CudaCsrMatrixAdapter.hpp"
#include "krans/adapters/cuda/CudaVectorFactory.hpp"

namespace {

using Basis = std::vector<std::unique_ptr<krans::VectorInterface>>;

std::string lower(std::string s) {
  for (auto &c : s)
    c = (char)std::tolower((unsigned char)c);
  return s;
}

void usage(const char *argv0) {
  std::cerr << "KraNS Nullspace CLI (B200 engine)\n"
            << "Usage:\n"
            << "  " << argv0 << " --solver [cyclic|lobpcg] --input <matrix.(mtx|ija)>\n"
            << "           [--out N.csv] [--report report.json] [--seed <int>] [--device cuda]\n"
            << "           [--precision fp64|mixed] [--gpu <index>]\n"
            << "Cyclic options: --k --ncv --max-restarts --tol-abs --tol-rel --proj-passes --cg-maxit\n"
            << "                --cg-rel --prescreen --stagnation --verbose --left\n"
            << "LOBPCG options: --k --lobpcg-block --lobpcg-max-it --lobpcg-restart --lobpcg-soft-lock\n"
            << "                --tol-abs --tol-rel --verbose\n";
}

// write_csv_basis (include/krans/Utils/ExportIO.hpp): one row per entry, one
// column per vector, fixed notation with 17 digits, no header
bool write_csv(const std::string &path, const Basis &B) {
  std::ofstream out(path);
  if (!out)
    return false;
  out.setf(std::ios::fixed, std::ios::floatfield);
  out << std::setprecision(17);
  if (B.empty())
    return true;
  std::vector<const double *> cols;
  for (const auto &v : B)
    cols.push_back(v->data());
  const std::size_t rows = B.front()->size();
  for (std::size_t i = 0; i < rows; ++i) {
    for (std::size_t j = 0; j < cols.size(); ++j) {
      out << cols[j][i];
      if (j + 1 < cols.size())
        out << ',';
    }
    out << '\n';
  }
  return (bool)out;
}

} // namespace

int main(int argc, char **argv) {
  std::string solver = "cyclic", input, out_csv = "N.csv", report = "report.json", device = "cuda";
  std::string precision = "fp64";
  int gpu = 0;
  int k = 1, ncv = 48, max_restarts = 80, proj_passes = 1, cg_maxit = 80, stagnation = 30;
  double tol_abs = 1e-12, tol_rel = 1e-10, cg_rel = 1e-10, prescreen = 0.8;
  bool verbose = false, left = false;
  unsigned seed = 1;
  int lob_block = 0, lob_max_it = 1000, lob_soft = 1;
  double lob_restart = 0.9;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&]() -> const char * {
      if (i + 1 >= argc) {
        usage(argv[0]);
        std::exit(2);
      }
      return argv[++i];
    };
    try {
      if (a == "--solver")
        solver = lower(val());
      else if (a == "--input")
        input = val();
      else if (a == "--out")
        out_csv = val();
      else if (a == "--report")
        report = val();
      else if (a == "--device")
        device = lower(val());
      else if (a == "--precision")
        precision = lower(val());
      else if (a == "--gpu")
        gpu = std::stoi(val());
      else if (a == "--tol")
        (void)val(); // direct solvers only
      else if (a == "--k")
        k = std::stoi(val());
      else if (a == "--tol-abs")
        tol_abs = std::stod(val());
      else if (a == "--tol-rel")
        tol_rel = std::stod(val());
      else if (a == "--verbose")
        verbose = true;
      else if (a == "--ncv")
        ncv = std::stoi(val());
      else if (a == "--max-restarts")
        max_restarts = std::stoi(val());
      else if (a == "--proj-passes")
        proj_passes = std::stoi(val());
      else if (a == "--cg-maxit")
        cg_maxit = std::stoi(val());
      else if (a == "--cg-rel")
        cg_rel = std::stod(val());
      else if (a == "--prescreen")
        prescreen = std::stod(val());
      else if (a == "--stagnation")
        stagnation = std::stoi(val());
      else if (a == "--seed")
        seed = (unsigned)std::stoul(val());
      else if (a == "--left")
        left = true;
      else if (a == "--lobpcg-block")
        lob_block = std::stoi(val());
      else if (a == "--lobpcg-max-it")
        lob_max_it = std::stoi(val());
      else if (a == "--lobpcg-restart")
        lob_restart = std::stod(val());
      else if (a == "--lobpcg-soft-lock")
        lob_soft = std::stoi(val());
      else if (a == "--help" || a == "-h") {
        usage(argv[0]);
        return 0;
      } else {
        std::cerr << "Unknown argument: " << a << "\n";
        usage(argv[0]);
        return 2;
      }
    } catch (const std::exception &) {
      std::cerr << "Bad value for " << a << "\n";
      return 2;
    }
  }
  if (input.empty()) {
    std::cerr << "Error: --input is required.\n";
    usage(argv[0]);
    return 2;
  }
  if (device != "cuda") {
    std::cerr << "Unsupported device: " << device << " (this engine runs on cuda)\n";
    return 2;
  }
  if (solver != "cyclic" && solver != "lobpcg") {
    std::cerr << "Unknown solver: " << solver << " (the device engine provides cyclic and lobpcg)\n";
    usage(argv[0]);
    return 2;
  }
  const bool mixed = precision == "mixed";
  krans_ctx *ctx = nullptr;
  if (krans_ctx_create(gpu, 0, &ctx) != KRANS_OK) {
    std::cerr << "CUDA context: " << krans_last_error() << "\n";
    return 2;
  }
  int rc = 0;
  {
    using clk = std::chrono::steady_clock;
    auto t0 = clk::now();
    std::unique_ptr<krans::cuda::CudaCsrMatrixAdapter> A;
    try {
      A = krans::cuda::CudaCsrMatrixAdapter::load(ctx, input, mixed);
    } catch (const std::exception &e) {
      std::cerr << "Matrix load error: " << e.what() << "\n";
      krans_ctx_destroy(ctx);
      return 2;
    }
    const double t_load = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
    const std::size_t m = A->rows(), n = A->cols();
    krans::cuda::CudaVectorFactory vf(ctx, n, seed);
    Basis right, left_basis;
    double rel_for_report = tol_rel;
    t0 = clk::now();
    try {
      if (solver == "cyclic") {
        krans::solvers::CyclicLanczosOptions opt;
        opt.k = k > 0 ? (std::size_t)k : 1;
        opt.ncv = ncv > 0 ? (std::size_t)ncv : 48;
        opt.max_restarts = max_restarts >= 0 ? (std::size_t)max_restarts : 80;
        opt.tol_abs = tol_abs;
        opt.tol_rel = tol_rel;
        opt.projector_passes = std::max(1, proj_passes);
        opt.cg_maxit = cg_maxit >= 0 ? (std::size_t)cg_maxit : 80;
        opt.cg_rel_tol = cg_rel;
        opt.prescreen_factor = prescreen;
        opt.stagnation_restarts = (std::size_t)std::max(0, stagnation);
        opt.return_left_space = left;
        opt.verbose = verbose;
        opt.precision = mixed ? KRANS_PREC_MIXED : KRANS_PREC_FP64;
        auto R = krans::solvers::find_nullspace_cyclic_lanczos_ex(*A, vf, opt);
        right = std::move(R.right_null);
        left_basis = std::move(R.left_null);
      } else {
        krans::solvers::LOBPCGOptions opt;
        opt.nev = k > 0 ? (std::size_t)k : 1;
        opt.block_size = lob_block > 0 ? (std::size_t)lob_block : 0;
        opt.max_iters = lob_max_it > 0 ? (std::size_t)lob_max_it : 1000;
        opt.restart = (lob_restart > 0.1 && lob_restart <= 1.0) ? lob_restart : 0.9;
        opt.soft_locking = lob_soft != 0;
        opt.tol_abs = tol_abs;
        opt.tol_rel = tol_rel;
        opt.gs_tol = 1e-14;
        opt.gs_reorth = true;
        opt.frob_samples = 4;
        opt.verbose = verbose;
        right = krans::solvers::find_nullspace_lobpcg(*A, vf, opt);
      }
    } catch (const std::exception &e) {
      std::cerr << "Solver error: " << e.what() << "\n";
      rc = 1;
    }
    const double t_solve = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
    if (rc == 0) {
      const std::size_t nullity = right.size(), rank = n >= nullity ? n - nullity : 0;
      if (!write_csv(out_csv, right)) {
        std::cerr << "Failed to write " << out_csv << "\n";
        rc = 3;
      }
      bool wrote_left = false;
      if (rc == 0 && left && !left_basis.empty())
        wrote_left = write_csv("N_left.csv", left_basis);
      // diagnostics (diagnose_basis, ExportIO.hpp): ||A u|| per vector and
      // the largest |<u_i, u_j>|, i != j
      std::vector<double> res;
      double maxdot = 0.0;
      if (rc == 0) {
        auto y = vf.create_zero_of_size(m);
        for (const auto &u : right) {
          A->multiply(*u, *y);
          res.push_back(y->norm());
        }
        for (std::size_t i = 0; i < right.size(); ++i)
          for (std::size_t j = i + 1; j < right.size(); ++j)
            maxdot = std::max(maxdot, std::fabs(right[i]->dot(*right[j])));
        std::ofstream out(report);
        out << std::setprecision(17);
        out << "{\n  \"solver\": \"" << solver << "\",\n  \"rows\": " << m << ",\n  \"cols\": " << n
            << ",\n  \"rank\": " << rank << ",\n  \"nullity\": " << nullity << ",\n  \"tol_rel\": "
            << rel_for_report << ",\n  \"timings_ms\": { \"load\": " << t_load << ", \"solve\": " << t_solve
            << " },\n  \"residuals\": [";
        for (std::size_t i = 0; i < res.size(); ++i)
          out << (i ? ", " : "") << res[i];
        out << "],\n  \"max_offdiag_abs_dot\": " << maxdot << "\n}\n";
        if (!out) {
          std::cerr << "Failed to write " << report << "\n";
          rc = 4;
        }
      }
      if (rc == 0)
        std::cout << "OK [" << solver << "]  m=" << m << " n=" << n << " rank~" << rank << " nullity=" << nullity
                  << " | load=" << t_load << " ms, solve=" << t_solve << " ms\n"
                  << "Wrote: " << out_csv << " and " << report << (wrote_left ? " (plus N_left.csv)" : "") << "\n";
    }
  }
  krans_ctx_destroy(ctx);
  return rc;
}
