// lbm_reaction_sim on the engine: LB-Cube's 2-D reactive-mixing driver
// (src/simulate_reaction.cpp) ported to the C ABI.
//
// Same command line (-nx -ny -steps -out_freq -u0 -tau -tau_c -k_react -gpu),
// D2Q9 BGK fluid and two D2Q5 species in double, the same initial state
// (Taylor-Green fluid, A = 1 in the left half, B = 1 in the right half) and
// the same outputs: reaction_diagnostics.csv (the eight ReactiveDiagnostics
// fields at step 0 and every -out_freq steps) and reaction_<step>.vtk. What
// changes:
// * each step is one fused launch (lbm_fluid_reaction_ab_async: the fluid
//   step, then the reaction advected by the post-step fluid, as the driver
//   sequences its two launches, simulate_reaction.cpp:518-543);
// * at an output step that launch also writes the statistics partials and
//   the diagnostics are formed on the device, so eight doubles reach the host
//   where the reference copies the fluid and both species back to run
//   compute_reactive_stats (:557-580);
// * the VTK file is written from device-computed concentrations and velocity
//   (four values per cell copied instead of 19);
// * the MLUPS figure is also reported for the stepping kernels alone.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
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

struct Config {
  std::size_t nx{256}, ny{256};
  int steps{5000};
  int output_frequency{250};
  double fluid_relaxation_time{0.6};
  double scalar_relaxation_time{0.8};
  double initial_velocity{0.04};
  double reaction_rate{0.05};
};

Config parse_arguments(int argc, char** argv) {
  std::vector<std::string> args(argv + 1, argv + argc);
  Config c;
  for (std::size_t i = 0; i < args.size(); ++i) {
    const std::string& arg = args[i];
    if (arg == "-nx") c.nx = parse_size_arg(args, i);
    else if (arg == "-ny") c.ny = parse_size_arg(args, i);
    else if (arg == "-steps") c.steps = parse_int_arg(args, i);
    else if (arg == "-out_freq") c.output_frequency = parse_int_arg(args, i);
    else if (arg == "-u0") c.initial_velocity = parse_real_arg(args, i);
    else if (arg == "-tau") c.fluid_relaxation_time = parse_real_arg(args, i);
    else if (arg == "-tau_c") c.scalar_relaxation_time = parse_real_arg(args, i);
    else if (arg == "-k_react") c.reaction_rate = parse_real_arg(args, i);
    else if (arg == "-cpu") reject_cpu();
    else if (arg == "-gpu") {
    } else throw std::invalid_argument("unknown argument: " + arg);
  }
  if (c.steps < 0) throw std::invalid_argument("-steps must be non-negative");
  if (c.output_frequency <= 0) throw std::invalid_argument("-out_freq must be greater than zero");
  if (c.fluid_relaxation_time <= 0.5 || c.scalar_relaxation_time <= 0.5)
    throw std::invalid_argument("relaxation times must be greater than 0.5");
  if (c.reaction_rate < 0.0) throw std::invalid_argument("-k_react must be non-negative");
  return c;
}

// Density, velocity and the two concentrations of the initial state, as the
// reference driver computes them in double (simulate_reaction.cpp:168-216:
// taylor_green_macro and initialize_fields); the engine forms the equilibrium
// populations on the device.
void initial_fields(const Config& c, std::vector<double>& rho, std::vector<double>& u,
                    std::vector<double>& ca, std::vector<double>& cb) {
  const std::size_t n = c.nx * c.ny;
  rho.assign(n, 0.0);
  u.assign(2 * n, 0.0);
  ca.assign(n, 0.0);
  cb.assign(n, 0.0);
  constexpr double cs2 = 1.0 / 3.0;
  const double u0 = c.initial_velocity;
  const double kx = 2.0 * std::numbers::pi_v<double> / static_cast<double>(c.nx);
  const double ky = 2.0 * std::numbers::pi_v<double> / static_cast<double>(c.ny);
  for (std::size_t y = 0; y < c.ny; ++y) {
    for (std::size_t x = 0; x < c.nx; ++x) {
      const double px = kx * static_cast<double>(x);
      const double py = ky * static_cast<double>(y);
      const double dp = (u0 * u0) / (4.0 * cs2) * (std::cos(2.0 * px) + std::cos(2.0 * py));
      const std::size_t cell = y * c.nx + x;
      rho[cell] = 1.0 - dp;
      u[cell] = -u0 * std::cos(px) * std::sin(py);
      u[n + cell] = u0 * std::sin(px) * std::cos(py);
      ca[cell] = x < c.nx / 2 ? 1.0 : 0.0;
      cb[cell] = x < c.nx / 2 ? 0.0 : 1.0;
    }
  }
}

// The reference driver's reaction_<step>.vtk (simulate_reaction.cpp:240-301):
// C_A, C_B, k C_A C_B and the fluid velocity, 17 significant digits.
void write_reaction_vtk(std::size_t nx, std::size_t ny, std::size_t step, double k,
                        const std::vector<double>& ca, const std::vector<double>& cb,
                        const std::vector<double>& u) {
  const std::string filename = std::format("reaction_{:06}.vtk", step);
  std::ofstream vtk{filename};
  if (!vtk) throw std::runtime_error("failed to open " + filename);
  const std::size_t n = nx * ny;
  std::string text;
  text.reserve(n * 110 + 512);
  text += "# vtk DataFile Version 3.0\n";
  text += std::format("LB-Cube reactive mixing step {}\n", step);
  text += "ASCII\nDATASET STRUCTURED_POINTS\n";
  text += std::format("DIMENSIONS {} {} 1\n", nx, ny);
  text += "ORIGIN 0 0 0\nSPACING 1 1 1\n";
  text += std::format("POINT_DATA {}\n", n);
  text += "SCALARS C_A double 1\nLOOKUP_TABLE default\n";
  for (std::size_t i = 0; i < n; ++i) text += std::format("{:.17g}\n", ca[i]);
  text += "SCALARS C_B double 1\nLOOKUP_TABLE default\n";
  for (std::size_t i = 0; i < n; ++i) text += std::format("{:.17g}\n", cb[i]);
  text += "SCALARS reaction_rate double 1\nLOOKUP_TABLE default\n";
  for (std::size_t i = 0; i < n; ++i) text += std::format("{:.17g}\n", k * ca[i] * cb[i]);
  text += "VECTORS velocity double\n";
  for (std::size_t i = 0; i < n; ++i) text += std::format("{:.17g} {:.17g} 0\n", u[i], u[n + i]);
  vtk << text;
  if (!vtk) throw std::runtime_error("failed to write " + filename);
}

}  // namespace

int main(int argc, char** argv) {
  try {
    const Config c = parse_arguments(argc, argv);
    const double omega = 1.0 / c.fluid_relaxation_time;
    const double omega_c = 1.0 / c.scalar_relaxation_time;
    const std::size_t n = c.nx * c.ny;

    std::ofstream diagnostics{"reaction_diagnostics.csv"};
    if (!diagnostics) throw std::runtime_error("failed to open reaction_diagnostics.csv");
    diagnostics << "step,mean_A,mean_B,var_A,var_B,covariance,"
                << "segregation_intensity,true_reaction_rate,mixed_reaction_rate\n";
    std::cout << "LB-Cube D2Q9/D2Q5 reactive mixing\n"
              << "Grid: " << c.nx << " x " << c.ny << '\n'
              << "Steps: " << c.steps << '\n'
              << "Output frequency: " << c.output_frequency << '\n'
              << "Backend: GPU\n"
              << "Fluid omega: " << omega << '\n'
              << "Scalar omega: " << omega_c << '\n'
              << "Reaction rate: " << c.reaction_rate << '\n'
              << std::flush;

    cudaStream_t stream;
    check_cuda(cudaStreamCreate(&stream), "cudaStreamCreate");
    DeviceArray<double> f0(9 * n), f1(9 * n), a0(5 * n), a1(5 * n), b0(5 * n), b1(5 * n);
    DeviceArray<double> rho(n), vel(2 * n), ca(n), cb(n), diag(8);
    const std::size_t pb = lbm_stats_partials_bytes(LBM_D2Q9, c.nx, c.ny, 1);
    DeviceArray<double> partials(pb / sizeof(double));
    {
      std::vector<double> hr, hu, ha, hb;
      initial_fields(c, hr, hu, ha, hb);
      rho.upload(hr);
      vel.upload(hu);
      ca.upload(ha);
      cb.upload(hb);
    }
    check_engine(lbm_init_equilibrium_async(LBM_D2Q9, LBM_DOUBLE, rho.get(), vel.get(), f0.get(), c.nx, c.ny,
                                            1, stream), "fluid init");
    check_engine(lbm_init_equilibrium_async(LBM_D2Q5, LBM_DOUBLE, ca.get(), vel.get(), a0.get(), c.nx, c.ny,
                                            1, stream), "species A init");
    check_engine(lbm_init_equilibrium_async(LBM_D2Q5, LBM_DOUBLE, cb.get(), vel.get(), b0.get(), c.nx, c.ny,
                                            1, stream), "species B init");
    double *cf = f0.get(), *nf = f1.get(), *cA = a0.get(), *nA = a1.get(), *cB = b0.get(), *nB = b1.get();

    // diagnostics already on the device (diag) -> CSV row; fields -> VTK
    auto output = [&](int step) {
      check_engine(lbm_macro_fields_async(LBM_D2Q5, LBM_DOUBLE, cA, c.nx, c.ny, 1, ca.get(), nullptr, nullptr,
                                          stream), "C_A");
      check_engine(lbm_macro_fields_async(LBM_D2Q5, LBM_DOUBLE, cB, c.nx, c.ny, 1, cb.get(), nullptr, nullptr,
                                          stream), "C_B");
      check_engine(lbm_macro_fields_async(LBM_D2Q9, LBM_DOUBLE, cf, c.nx, c.ny, 1, nullptr, vel.get(), nullptr,
                                          stream), "velocity");
      check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
      const std::vector<double> d = diag.download(8);
      diagnostics << std::format("{},{:.17g},{:.17g},{:.17g},{:.17g},{:.17g},{:.17g},{:.17g},{:.17g}\n", step,
                                 d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7]);
      write_reaction_vtk(c.nx, c.ny, static_cast<std::size_t>(step), c.reaction_rate, ca.download(n),
                         cb.download(n), vel.download(2 * n));
    };

    KernelTimer timer(stream);
    const auto start = std::chrono::high_resolution_clock::now();
    check_engine(lbm_reactive_stats_async(LBM_D2Q5, LBM_DOUBLE, cA, cB, c.nx, c.ny, 1, c.reaction_rate,
                                          partials.get(), pb, diag.get(), stream), "statistics");
    output(0);
    timer.begin();
    for (int step = 1; step <= c.steps; ++step) {
      const bool out = step % c.output_frequency == 0;
      check_engine(lbm_fluid_reaction_ab_async(LBM_D2Q9, LBM_DOUBLE, LBM_BGK, cf, nf, cA, nA, cB, nB, c.nx, c.ny,
                                               1, omega, omega_c, c.reaction_rate,
                                               out ? partials.get() : nullptr, out ? pb : 0, stream),
                   "fluid + reaction step");
      std::swap(cf, nf);
      std::swap(cA, nA);
      std::swap(cB, nB);
      if (out) {
        check_engine(lbm_reactive_stats_finalize_async(LBM_D2Q9, LBM_DOUBLE, c.nx, c.ny, 1, c.reaction_rate,
                                                       partials.get(), pb, diag.get(), stream),
                     "statistics");
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
              << "Fluid lattice updates: " << updates / elapsed / 1.0e6 << " MLUPS\n"
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
