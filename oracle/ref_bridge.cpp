// Test infrastructure (oracle side). Builds LB-Cube's own CPU path, unmodified
// and in place, into oracle/_ref/libref.so and exposes it through a flat C ABI
// on raw [Q,Z,Y,X] arrays so that Python tests can run the reference itself on
// the same bits the CUDA engine sees.
//
// Entry points wrap, without changing any arithmetic:
//   step_cpu<L,Real,CT>            include/lattice_core.hpp:146-216
//   step_scalar_cpu<FL,SL,Real>    include/lattice_core.hpp:238-337
//   step_reaction_AB<FL,SL,Real>   include/lattice_core.hpp:357-474
//   compute_reactive_stats         include/lattice_io.hpp:256-338
//   compute_equilibrium            include/lattice_physics.hpp:267-290
//   mrt transforms                 include/lattice_mrt.hpp:439-534, :617-892, :1023-1225
//   write_vtk                      include/lattice_io.hpp:386-451 (writes lbm_<step>.vtk
//                                  into the current directory, as the reference does)
//
// Enum codes (shared with oracle/lbm_oracle.h and the engine's C ABI):
//   lattice: 0 D2Q9, 1 D3Q19, 2 D3Q27, 3 D2Q5, 4 D3Q7
//   precision: 0 float, 1 double
//   collision: 0 BGK, 1 TRT, 2 MRT, 3 RLBM
#include <cstddef>
#include <cstring>
#include <vector>

#include "lattice_core.hpp"
#include "lattice_io.hpp"
#include "lattice_memory.hpp"
#include "lattice_mrt.hpp"
#include "lattice_physics.hpp"
#include "lattice_traits.hpp"

namespace {

template <typename L, typename Real>
lbm::LatticeMemory<L, Real> make_memory(std::size_t nx, std::size_t ny, std::size_t nz) {
  if constexpr (L::D == 2) {
    return lbm::LatticeMemory<L, Real>{nx, ny};
  } else {
    return lbm::LatticeMemory<L, Real>{nx, ny, nz};
  }
}

template <typename L, typename Real>
void load(lbm::LatticeMemory<L, Real>& mem, const void* src) {
  auto view = mem.get_current_view();
  std::memcpy(view.data_handle(), src, mem.population_count() * sizeof(Real));
}

template <typename L, typename Real>
void store(const lbm::LatticeMemory<L, Real>& mem, void* dst) {
  const auto view = mem.get_current_view();
  std::memcpy(dst, view.data_handle(), mem.population_count() * sizeof(Real));
}

template <typename L, typename Real, lbm::CollisionType CT>
int run_step(const void* in, void* out, std::size_t nx, std::size_t ny, std::size_t nz,
             double omega, int steps) {
  auto mem = make_memory<L, Real>(nx, ny, nz);
  load(mem, in);
  for (int s = 0; s < steps; ++s) {
    lbm::step_cpu<L, Real, CT>(mem, static_cast<Real>(omega));
  }
  store(mem, out);
  return 0;
}

template <typename L, typename Real>
int dispatch_op(int op, const void* in, void* out, std::size_t nx, std::size_t ny,
                std::size_t nz, double omega, int steps) {
  switch (op) {
    case 0: return run_step<L, Real, lbm::CollisionType::BGK>(in, out, nx, ny, nz, omega, steps);
    case 1: return run_step<L, Real, lbm::CollisionType::TRT>(in, out, nx, ny, nz, omega, steps);
    case 2: return run_step<L, Real, lbm::CollisionType::MRT>(in, out, nx, ny, nz, omega, steps);
    case 3: return run_step<L, Real, lbm::CollisionType::RLBM>(in, out, nx, ny, nz, omega, steps);
    default: return -1;
  }
}

template <typename Real>
int dispatch_lattice(int lat, int op, const void* in, void* out, std::size_t nx,
                     std::size_t ny, std::size_t nz, double omega, int steps) {
  switch (lat) {
    case 0: return dispatch_op<lbm::D2Q9, Real>(op, in, out, nx, ny, 1, omega, steps);
    case 1: return dispatch_op<lbm::D3Q19, Real>(op, in, out, nx, ny, nz, omega, steps);
    case 2: return dispatch_op<lbm::D3Q27, Real>(op, in, out, nx, ny, nz, omega, steps);
    default: return -1;
  }
}

template <typename FL, typename SL, typename Real>
int run_scalar(const void* s_in, void* s_out, const void* fluid, std::size_t nx,
               std::size_t ny, std::size_t nz, double omega_c, double source, int steps) {
  auto smem = make_memory<SL, Real>(nx, ny, nz);
  auto fmem = make_memory<FL, Real>(nx, ny, nz);
  load(smem, s_in);
  load(fmem, fluid);
  for (int s = 0; s < steps; ++s) {
    lbm::step_scalar_cpu<FL, SL, Real>(smem, fmem, static_cast<Real>(omega_c),
                                       static_cast<Real>(source));
  }
  store(smem, s_out);
  return 0;
}

template <typename FL, typename SL, typename Real>
int run_reaction(const void* a_in, void* a_out, const void* b_in, void* b_out,
                 const void* fluid, std::size_t nx, std::size_t ny, std::size_t nz,
                 double omega_c, double k, int steps) {
  auto amem = make_memory<SL, Real>(nx, ny, nz);
  auto bmem = make_memory<SL, Real>(nx, ny, nz);
  auto fmem = make_memory<FL, Real>(nx, ny, nz);
  load(amem, a_in);
  load(bmem, b_in);
  load(fmem, fluid);
  for (int s = 0; s < steps; ++s) {
    lbm::step_reaction_AB<FL, SL, Real>(fmem, amem, bmem, static_cast<Real>(omega_c),
                                        static_cast<Real>(k));
  }
  store(amem, a_out);
  store(bmem, b_out);
  return 0;
}

// The reference driver's coupled loop (src/simulate_reaction.cpp:548-554):
// step_cpu on the fluid, then step_reaction_AB with the post-step fluid.
template <typename FL, typename SL, typename Real, lbm::CollisionType CT>
int run_coupled(void* fluid, void* a, void* b, std::size_t nx, std::size_t ny,
                std::size_t nz, double omega, double omega_c, double k, int steps) {
  auto amem = make_memory<SL, Real>(nx, ny, nz);
  auto bmem = make_memory<SL, Real>(nx, ny, nz);
  auto fmem = make_memory<FL, Real>(nx, ny, nz);
  load(amem, a);
  load(bmem, b);
  load(fmem, fluid);
  for (int s = 0; s < steps; ++s) {
    lbm::step_cpu<FL, Real, CT>(fmem, static_cast<Real>(omega));
    lbm::step_reaction_AB<FL, SL, Real>(fmem, amem, bmem, static_cast<Real>(omega_c),
                                        static_cast<Real>(k));
  }
  store(fmem, fluid);
  store(amem, a);
  store(bmem, b);
  return 0;
}

template <typename FL, typename SL, typename Real>
int coupled_op(int op, void* fluid, void* a, void* b, std::size_t nx, std::size_t ny,
               std::size_t nz, double omega, double omega_c, double k, int steps) {
  switch (op) {
    case 0: return run_coupled<FL, SL, Real, lbm::CollisionType::BGK>(fluid, a, b, nx, ny, nz, omega, omega_c, k, steps);
    case 1: return run_coupled<FL, SL, Real, lbm::CollisionType::TRT>(fluid, a, b, nx, ny, nz, omega, omega_c, k, steps);
    case 2: return run_coupled<FL, SL, Real, lbm::CollisionType::MRT>(fluid, a, b, nx, ny, nz, omega, omega_c, k, steps);
    default: return -1;
  }
}

template <typename SL, typename Real>
int run_stats(const void* a, const void* b, std::size_t nx, std::size_t ny, std::size_t nz,
              double k, double* out) {
  auto amem = make_memory<SL, Real>(nx, ny, nz);
  auto bmem = make_memory<SL, Real>(nx, ny, nz);
  load(amem, a);
  load(bmem, b);
  const auto d = lbm::compute_reactive_stats<SL, Real>(amem, bmem, static_cast<Real>(k));
  out[0] = d.mean_A;
  out[1] = d.mean_B;
  out[2] = d.var_A;
  out[3] = d.var_B;
  out[4] = d.covariance;
  out[5] = d.segregation_intensity;
  out[6] = d.true_reaction_rate;
  out[7] = d.mixed_reaction_rate;
  return 0;
}

template <typename L, typename Real>
void equilibrium(double rho, const double* u, void* out) {
  lbm::MacroState<L, Real> macro{};
  macro.density = static_cast<Real>(rho);
  for (int d = 0; d < L::D; ++d) macro.velocity[d] = static_cast<Real>(u[d]);
  Real* o = static_cast<Real*>(out);
  for (int i = 0; i < L::Q; ++i) o[i] = lbm::compute_equilibrium<L, Real>(i, macro);
}

template <typename SL, typename Real>
void scalar_equilibrium(double conc, const double* u, void* out) {
  Eigen::Matrix<Real, SL::D, 1> vel{};
  for (int d = 0; d < SL::D; ++d) vel[d] = static_cast<Real>(u[d]);
  Real* o = static_cast<Real*>(out);
  for (int i = 0; i < SL::Q; ++i) {
    o[i] = lbm::compute_scalar_equilibrium<SL, Real>(i, static_cast<Real>(conc), vel);
  }
}

template <typename L, typename Real>
int run_write_vtk(const void* f, std::size_t nx, std::size_t ny, std::size_t nz, std::size_t step) {
  auto mem = make_memory<L, Real>(nx, ny, nz);
  load(mem, f);
  lbm::write_vtk<L, Real>(mem, nx, ny, nz, step);
  return 0;
}

template <typename Real>
int write_vtk_lattice(int lattice, const void* f, std::size_t nx, std::size_t ny, std::size_t nz,
                      std::size_t step) {
  switch (lattice) {
    case 0: return run_write_vtk<lbm::D2Q9, Real>(f, nx, ny, nz, step);
    case 1: return run_write_vtk<lbm::D3Q19, Real>(f, nx, ny, nz, step);
    case 2: return run_write_vtk<lbm::D3Q27, Real>(f, nx, ny, nz, step);
    default: return -1;
  }
}

}  // namespace

extern "C" {

int ref_write_vtk(int lattice, int precision, const void* f, std::size_t nx, std::size_t ny,
                  std::size_t nz, std::size_t step) {
  if (precision == 0) return write_vtk_lattice<float>(lattice, f, nx, ny, nz, step);
  if (precision == 1) return write_vtk_lattice<double>(lattice, f, nx, ny, nz, step);
  return -1;
}

int ref_step(int lattice, int precision, int collision, const void* in, void* out,
             std::size_t nx, std::size_t ny, std::size_t nz, double omega, int steps) {
  if (precision == 0) return dispatch_lattice<float>(lattice, collision, in, out, nx, ny, nz, omega, steps);
  if (precision == 1) return dispatch_lattice<double>(lattice, collision, in, out, nx, ny, nz, omega, steps);
  return -1;
}

int ref_scalar_step(int fluid_lattice, int precision, const void* s_in, void* s_out,
                    const void* fluid, std::size_t nx, std::size_t ny, std::size_t nz,
                    double omega_c, double source, int steps) {
  if (fluid_lattice == 0) {
    if (precision == 0) return run_scalar<lbm::D2Q9, lbm::D2Q5, float>(s_in, s_out, fluid, nx, ny, nz, omega_c, source, steps);
    return run_scalar<lbm::D2Q9, lbm::D2Q5, double>(s_in, s_out, fluid, nx, ny, nz, omega_c, source, steps);
  }
  if (fluid_lattice == 1) {
    if (precision == 0) return run_scalar<lbm::D3Q19, lbm::D3Q7, float>(s_in, s_out, fluid, nx, ny, nz, omega_c, source, steps);
    return run_scalar<lbm::D3Q19, lbm::D3Q7, double>(s_in, s_out, fluid, nx, ny, nz, omega_c, source, steps);
  }
  if (fluid_lattice == 2) {
    if (precision == 0) return run_scalar<lbm::D3Q27, lbm::D3Q7, float>(s_in, s_out, fluid, nx, ny, nz, omega_c, source, steps);
    return run_scalar<lbm::D3Q27, lbm::D3Q7, double>(s_in, s_out, fluid, nx, ny, nz, omega_c, source, steps);
  }
  return -1;
}

int ref_reaction_ab(int fluid_lattice, int precision, const void* a_in, void* a_out,
                    const void* b_in, void* b_out, const void* fluid, std::size_t nx,
                    std::size_t ny, std::size_t nz, double omega_c, double k, int steps) {
  if (fluid_lattice == 0) {
    if (precision == 0) return run_reaction<lbm::D2Q9, lbm::D2Q5, float>(a_in, a_out, b_in, b_out, fluid, nx, ny, nz, omega_c, k, steps);
    return run_reaction<lbm::D2Q9, lbm::D2Q5, double>(a_in, a_out, b_in, b_out, fluid, nx, ny, nz, omega_c, k, steps);
  }
  if (fluid_lattice == 1) {
    if (precision == 0) return run_reaction<lbm::D3Q19, lbm::D3Q7, float>(a_in, a_out, b_in, b_out, fluid, nx, ny, nz, omega_c, k, steps);
    return run_reaction<lbm::D3Q19, lbm::D3Q7, double>(a_in, a_out, b_in, b_out, fluid, nx, ny, nz, omega_c, k, steps);
  }
  if (fluid_lattice == 2) {
    if (precision == 0) return run_reaction<lbm::D3Q27, lbm::D3Q7, float>(a_in, a_out, b_in, b_out, fluid, nx, ny, nz, omega_c, k, steps);
    return run_reaction<lbm::D3Q27, lbm::D3Q7, double>(a_in, a_out, b_in, b_out, fluid, nx, ny, nz, omega_c, k, steps);
  }
  return -1;
}

int ref_coupled_reaction(int fluid_lattice, int precision, int collision, void* fluid,
                         void* a, void* b, std::size_t nx, std::size_t ny, std::size_t nz,
                         double omega, double omega_c, double k, int steps) {
  if (fluid_lattice == 0) {
    if (precision == 0) return coupled_op<lbm::D2Q9, lbm::D2Q5, float>(collision, fluid, a, b, nx, ny, 1, omega, omega_c, k, steps);
    return coupled_op<lbm::D2Q9, lbm::D2Q5, double>(collision, fluid, a, b, nx, ny, 1, omega, omega_c, k, steps);
  }
  if (fluid_lattice == 1) {
    if (precision == 0) return coupled_op<lbm::D3Q19, lbm::D3Q7, float>(collision, fluid, a, b, nx, ny, nz, omega, omega_c, k, steps);
    return coupled_op<lbm::D3Q19, lbm::D3Q7, double>(collision, fluid, a, b, nx, ny, nz, omega, omega_c, k, steps);
  }
  if (fluid_lattice == 2) {
    if (precision == 0) return coupled_op<lbm::D3Q27, lbm::D3Q7, float>(collision, fluid, a, b, nx, ny, nz, omega, omega_c, k, steps);
    return coupled_op<lbm::D3Q27, lbm::D3Q7, double>(collision, fluid, a, b, nx, ny, nz, omega, omega_c, k, steps);
  }
  return -1;
}

int ref_reactive_stats(int scalar_lattice, int precision, const void* a, const void* b,
                       std::size_t nx, std::size_t ny, std::size_t nz, double k, double* out) {
  if (scalar_lattice == 3) {
    if (precision == 0) return run_stats<lbm::D2Q5, float>(a, b, nx, ny, 1, k, out);
    return run_stats<lbm::D2Q5, double>(a, b, nx, ny, 1, k, out);
  }
  if (scalar_lattice == 4) {
    if (precision == 0) return run_stats<lbm::D3Q7, float>(a, b, nx, ny, nz, k, out);
    return run_stats<lbm::D3Q7, double>(a, b, nx, ny, nz, k, out);
  }
  return -1;
}

int ref_equilibrium(int lattice, int precision, double rho, const double* u, void* out) {
  switch (lattice * 2 + precision) {
    case 0: equilibrium<lbm::D2Q9, float>(rho, u, out); return 0;
    case 1: equilibrium<lbm::D2Q9, double>(rho, u, out); return 0;
    case 2: equilibrium<lbm::D3Q19, float>(rho, u, out); return 0;
    case 3: equilibrium<lbm::D3Q19, double>(rho, u, out); return 0;
    case 4: equilibrium<lbm::D3Q27, float>(rho, u, out); return 0;
    case 5: equilibrium<lbm::D3Q27, double>(rho, u, out); return 0;
    case 6: scalar_equilibrium<lbm::D2Q5, float>(rho, u, out); return 0;
    case 7: scalar_equilibrium<lbm::D2Q5, double>(rho, u, out); return 0;
    case 8: scalar_equilibrium<lbm::D3Q7, float>(rho, u, out); return 0;
    case 9: scalar_equilibrium<lbm::D3Q7, double>(rho, u, out); return 0;
    default: return -1;
  }
}

// MRT moment transforms in double, for the golden identity vectors.
int ref_mrt_moments(int lattice, const double* f, double* m) {
  if (lattice == 0) {
    std::array<double, 9> a{};
    std::memcpy(a.data(), f, sizeof a);
    const auto r = lbm::mrt::compute_moments_d2q9<double>(a);
    std::memcpy(m, r.data(), sizeof r);
    return 0;
  }
  if (lattice == 1) {
    std::array<double, 19> a{};
    std::memcpy(a.data(), f, sizeof a);
    const auto r = lbm::mrt::compute_moments_d3q19<double>(a);
    std::memcpy(m, r.data(), sizeof r);
    return 0;
  }
  if (lattice == 2) {
    std::array<double, 27> a{};
    std::memcpy(a.data(), f, sizeof a);
    const auto r = lbm::mrt::transform_to_moments_d3q27<double>(a);
    std::memcpy(m, r.data(), sizeof r);
    return 0;
  }
  return -1;
}

int ref_mrt_populations(int lattice, const double* m, double* f) {
  if (lattice == 0) {
    std::array<double, 9> a{};
    std::memcpy(a.data(), m, sizeof a);
    const auto r = lbm::mrt::compute_populations_d2q9<double>(a);
    std::memcpy(f, r.data(), sizeof r);
    return 0;
  }
  if (lattice == 1) {
    std::array<double, 19> a{};
    std::memcpy(a.data(), m, sizeof a);
    const auto r = lbm::mrt::compute_populations_d3q19<double>(a);
    std::memcpy(f, r.data(), sizeof r);
    return 0;
  }
  if (lattice == 2) {
    std::array<double, 27> a{};
    std::memcpy(a.data(), m, sizeof a);
    const auto r = lbm::mrt::transform_to_populations_d3q27<double>(a);
    std::memcpy(f, r.data(), sizeof r);
    return 0;
  }
  return -1;
}

}  // extern "C"
