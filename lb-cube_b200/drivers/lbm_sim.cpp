// lbm_sim on the engine: the D3Q19 periodic-box driver of LB-Cube
// (src/main.cpp) ported to the C ABI.
//
// Same command line (-nx -ny -nz -steps -out_freq -init rest|tgv -gpu),
// relaxation time 0.8, BGK, double populations, the same initial states, and
// the same outputs in the working directory: diagnostics.csv (step,
// total_mass, total_kinetic_energy, max_velocity_magnitude every -out_freq
// steps and at step 0) and the legacy VTK file lbm_<step, 6 digits>.vtk at the
// same steps. What changes is where the work happens:
// * the diagnostics are reduced on the device (lbm_fluid_diagnostics_async);
//   only five doubles reach the host per output, where the reference copies
//   all 19 population planes back (main.cpp:595-606);
// * the VTK file is written from the device's macroscopic fields (five values
//   per cell copied instead of 19) by the engine's writer, byte for byte the
//   reference's write_vtk;
// * the MLUPS figure is also reported for the stepping kernels alone (CUDA
//   events around the step launches), next to the reference's wall-clock
//   figure, which includes the output (main.cpp:570-629).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <format>
#include <fstream>
#include <iostream>
#include <numbers>
#include <string>
#include <vector>

#include "driver_common.hpp"

namespace {

using namespace lbport;

enum class Init { Rest, TaylorGreen };

struct Config {
  std::size_t nx{64}, ny{64}, nz{64};
  int steps{1000};
  int output_frequency{100};
  Init init{Init::TaylorGreen};
};

Config parse_arguments(int argc, char** argv) {
  std::vector<std::string> args(argv + 1, argv + argc);
  Config c;
  for (std::size_t i = 0; i < args.size(); ++i) {
    const std::string& arg = args[i];
    if (arg == "-nx") {
      c.nx = parse_size_arg(args, i);
    } else if (arg == "-ny") {
      c.ny = parse_size_arg(args, i);
    } else if (arg == "-nz") {
      c.nz = parse_size_arg(args, i);
    } else if (arg == "-steps") {
      c.steps = parse_int_arg(args, i);
    } else if (arg == "-out_freq") {
      c.output_frequency = parse_int_arg(args, i);
    } else if (arg == "-init") {
      if (i + 1 >= args.size()) throw std::invalid_argument("missing value for " + arg);
      const std::string v = args[++i];
      if (v == "rest") c.init = Init::Rest;
      else if (v == "tgv") c.init = Init::TaylorGreen;
      else throw std::invalid_argument("-init must be either 'rest' or 'tgv'");
    } else if (arg == "-cpu") {
      reject_cpu();
    } else if (arg == "-gpu") {
    } else {
      throw std::invalid_argument("unknown argument: " + arg);
    }
  }
  if (c.steps < 0) throw std::invalid_argument("-steps must be non-negative");
  if (c.output_frequency <= 0) throw std::invalid_argument("-out_freq must be greater than zero");
  return c;
}

// Density and velocity of the initial state, as the reference initialisers
// compute them in double (main.cpp:294-310 rest; :323-403 the 3-D Taylor-Green
// vortex with u0 = 0.01 and its pressure perturbation); the engine then forms
// the equilibrium populations on the device (lbm_init_equilibrium_async, the
// same expression as compute_equilibrium).
void initial_fields(const Config& c, std::vector<double>& rho, std::vector<double>& u) {
  const std::size_t n = c.nx * c.ny * c.nz;
  rho.assign(n, 1.0);
  u.assign(3 * n, 0.0);
  if (c.init == Init::Rest) return;
  constexpr double cs2 = 1.0 / 3.0;
  constexpr double u0 = 0.01;
  const double kx = 2.0 * std::numbers::pi_v<double> / static_cast<double>(c.nx);
  const double ky = 2.0 * std::numbers::pi_v<double> / static_cast<double>(c.ny);
  const double kz = 2.0 * std::numbers::pi_v<double> / static_cast<double>(c.nz);
  for (std::size_t z = 0; z < c.nz; ++z) {
    const double pz = kz * static_cast<double>(z);
    for (std::size_t y = 0; y < c.ny; ++y) {
      const double py = ky * static_cast<double>(y);
      for (std::size_t x = 0; x < c.nx; ++x) {
        const double px = kx * static_cast<double>(x);
        const double dp = (u0 * u0) / (16.0 * cs2) * (std::cos(2.0 * px) + std::cos(2.0 * py)) *
                          (std::cos(2.0 * pz) + 2.0);
        const std::size_t cell = (z * c.ny + y) * c.nx + x;
        rho[cell] = 1.0 + dp;
        u[cell] = u0 * std::sin(px) * std::cos(py) * std::cos(pz);
        u[n + cell] = -u0 * std::cos(px) * std::sin(py) * std::cos(pz);
      }
    }
  }
}

}  // namespace

int main(int argc, char** argv) {
  try {
    constexpr double relaxation_time = 0.8;
    constexpr double omega = 1.0 / relaxation_time;
    const Config c = parse_arguments(argc, argv);
    const std::size_t n = c.nx * c.ny * c.nz;

    std::ofstream diagnostics{"diagnostics.csv"};
    if (!diagnostics) throw std::runtime_error("failed to open diagnostics.csv");
    diagnostics << "step,total_mass,total_kinetic_energy,max_velocity_magnitude\n";
    std::cout << "LB-Cube D3Q19 simulation\n"
              << "Grid: " << c.nx << " x " << c.ny << " x " << c.nz << '\n'
              << "Steps: " << c.steps << '\n'
              << "Output frequency: " << c.output_frequency << '\n'
              << "Initial condition: " << (c.init == Init::Rest ? "rest" : "tgv") << '\n'
              << "Backend: GPU\n"
              << "Omega: " << omega << '\n'
              << std::flush;

    cudaStream_t stream;
    check_cuda(cudaStreamCreate(&stream), "cudaStreamCreate");
    DeviceArray<double> f0(19 * n), f1(19 * n), rho(n), vel(3 * n), speed(n);
    const std::size_t pb = lbm_diagnostics_partials_bytes(LBM_D3Q19, c.nx, c.ny, c.nz);
    DeviceArray<unsigned char> partials(pb);
    DeviceArray<double> diag(5);
    {
      std::vector<double> hr, hu;
      initial_fields(c, hr, hu);
      rho.upload(hr);
      vel.upload(hu);
    }
    check_engine(lbm_init_equilibrium_async(LBM_D3Q19, LBM_DOUBLE, rho.get(), vel.get(), f0.get(), c.nx,
                                            c.ny, c.nz, stream),
                 "init_equilibrium");
    double* cur = f0.get();
    double* nxt = f1.get();

    auto output = [&](int step) {
      check_engine(lbm_fluid_diagnostics_async(LBM_D3Q19, LBM_DOUBLE, cur, c.nx, c.ny, c.nz, HUGE_VAL,
                                               reinterpret_cast<double*>(partials.get()), pb, diag.get(),
                                               stream),
                   "fluid diagnostics");
      check_engine(lbm_macro_fields_async(LBM_D3Q19, LBM_DOUBLE, cur, c.nx, c.ny, c.nz, rho.get(),
                                          vel.get(), speed.get(), stream),
                   "macro fields");
      check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
      const std::vector<double> d = diag.download(5);
      diagnostics << std::format("{},{:.17g},{:.17g},{:.17g}\n", step, d[0], d[1], d[2]);
      const std::vector<double> hr = rho.download(n), hu = vel.download(3 * n), hs = speed.download(n);
      const std::string path = std::format("lbm_{:06}.vtk", step);
      if (lbm_write_vtk_legacy(path.c_str(), 3, c.nx, c.ny, c.nz, static_cast<std::size_t>(step),
                               LBM_DOUBLE, hr.data(), hu.data(), hs.data()) != 0)
        throw std::runtime_error("failed to write " + path);
    };

    KernelTimer timer(stream);
    const auto start = std::chrono::high_resolution_clock::now();
    output(0);
    timer.begin();
    for (int step = 1; step <= c.steps; ++step) {
      check_engine(lbm_step_async(LBM_D3Q19, LBM_DOUBLE, LBM_BGK, cur, nxt, c.nx, c.ny, c.nz, omega, stream),
                   "step");
      std::swap(cur, nxt);
      if (step % c.output_frequency == 0) {
        timer.end();
        output(step);
        std::cout << "Step " << step << " / " << c.steps << " complete\n" << std::flush;
        timer.begin();
      }
    }
    timer.end();
    check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    const auto stop = std::chrono::high_resolution_clock::now();
    const double elapsed = std::chrono::duration<double>(stop - start).count();
    const double updates = static_cast<double>(n) * static_cast<double>(c.steps);
    std::cout << "Elapsed time: " << elapsed << " s\n"
              << "Performance: " << updates / elapsed / 1.0e6 << " MLUPS\n"
              << "Kernel time: " << timer.seconds() << " s\n"
              << "Kernel performance: " << (timer.seconds() > 0 ? updates / timer.seconds() / 1.0e6 : 0.0)
              << " MLUPS\n"
              << std::flush;
    cudaStreamDestroy(stream);
    return EXIT_SUCCESS;
  } catch (const std::exception& error) {
    std::cerr << "Error: " << error.what() << '\n';
    return EXIT_FAILURE;
  }
}
