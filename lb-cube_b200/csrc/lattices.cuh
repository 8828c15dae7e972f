// Compile-time lattice descriptors for device code.
//
// The velocity sets, weights, cs^2 and opposite maps are LB-Cube's
// (include/lattice_traits.hpp:62-305); the [Q, Z, Y, X] population order is
// part of the data format shared with the reference, so the tables must be
// identical. They are plain C arrays read only inside constant expressions
// (indices come from `static_for`), so every lookup folds into an immediate
// and no table is ever odr-used in device code.
#pragma once

#include <cstdint>
#include <type_traits>
#include <utility>

namespace lbcube {

// Unrolled loop whose index is a compile-time constant: fn(std::integral_constant<int, I>).
template <class Fn, int... Is>
__host__ __device__ __forceinline__ void static_for_impl(Fn&& fn,
                                                         std::integer_sequence<int, Is...>) {
  (fn(std::integral_constant<int, Is>{}), ...);
}
template <int N, class Fn>
__host__ __device__ __forceinline__ void static_for(Fn&& fn) {
  static_for_impl(fn, std::make_integer_sequence<int, N>{});
}

enum LatticeId : int { kD2Q9 = 0, kD3Q19 = 1, kD3Q27 = 2, kD2Q5 = 3, kD3Q7 = 4 };

struct D2Q9 {
  static constexpr LatticeId id = kD2Q9;
  static constexpr int D = 2, Q = 9;
  static constexpr double cs2 = 1.0 / 3.0;
  static constexpr double w[Q] = {4.0 / 9.0,  1.0 / 9.0,  1.0 / 9.0,  1.0 / 9.0, 1.0 / 9.0,
                                  1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
  static constexpr int c[Q][3] = {{0, 0, 0},  {1, 0, 0},  {0, 1, 0},   {-1, 0, 0}, {0, -1, 0},
                                  {1, 1, 0},  {-1, 1, 0}, {-1, -1, 0}, {1, -1, 0}};
  static constexpr int opp[Q] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
};

struct D3Q19 {
  static constexpr LatticeId id = kD3Q19;
  static constexpr int D = 3, Q = 19;
  static constexpr double cs2 = 1.0 / 3.0;
  static constexpr double w[Q] = {1.0 / 3.0,  1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
                                  1.0 / 18.0, 1.0 / 18.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                                  1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                                  1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
  static constexpr int c[Q][3] = {{0, 0, 0},   {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
                                  {0, 0, 1},   {0, 0, -1}, {1, 1, 0},  {-1, 1, 0}, {1, -1, 0},
                                  {-1, -1, 0}, {1, 0, 1},  {-1, 0, 1}, {1, 0, -1}, {-1, 0, -1},
                                  {0, 1, 1},   {0, -1, 1}, {0, 1, -1}, {0, -1, -1}};
  static constexpr int opp[Q] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
};

struct D3Q27 {
  static constexpr LatticeId id = kD3Q27;
  static constexpr int D = 3, Q = 27;
  static constexpr double cs2 = 1.0 / 3.0;
  static constexpr double w[Q] = {
      8.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,
      1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,
      1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 216.0, 1.0 / 216.0,
      1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0};
  static constexpr int c[Q][3] = {
      {0, 0, 0},   {1, 0, 0},  {-1, 0, 0},  {0, 1, 0},   {0, -1, 0}, {0, 0, 1},   {0, 0, -1},
      {1, 1, 0},   {-1, 1, 0}, {1, -1, 0},  {-1, -1, 0}, {1, 0, 1},  {-1, 0, 1},  {1, 0, -1},
      {-1, 0, -1}, {0, 1, 1},  {0, -1, 1},  {0, 1, -1},  {0, -1, -1}, {1, 1, 1},  {-1, 1, 1},
      {1, -1, 1},  {-1, -1, 1}, {1, 1, -1}, {-1, 1, -1}, {1, -1, -1}, {-1, -1, -1}};
  static constexpr int opp[Q] = {0,  2,  1,  4,  3,  6,  5,  10, 9,  8,  7,  14, 13, 12,
                                 11, 18, 17, 16, 15, 26, 25, 24, 23, 22, 21, 20, 19};
};

struct D2Q5 {
  static constexpr LatticeId id = kD2Q5;
  static constexpr int D = 2, Q = 5;
  static constexpr double cs2 = 1.0 / 3.0;
  static constexpr double w[Q] = {1.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0};
  static constexpr int c[Q][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, -1, 0}};
  static constexpr int opp[Q] = {0, 3, 4, 1, 2};
};

struct D3Q7 {
  static constexpr LatticeId id = kD3Q7;
  static constexpr int D = 3, Q = 7;
  static constexpr double cs2 = 1.0 / 4.0;
  static constexpr double w[Q] = {1.0 / 4.0, 1.0 / 8.0, 1.0 / 8.0, 1.0 / 8.0,
                                  1.0 / 8.0, 1.0 / 8.0, 1.0 / 8.0};
  static constexpr int c[Q][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},
                                  {0, -1, 0}, {0, 0, 1},  {0, 0, -1}};
  static constexpr int opp[Q] = {0, 2, 1, 4, 3, 6, 5};
};

// Advection-diffusion lattice paired with each fluid lattice
// (the reference instantiates D2Q9/D2Q5, D3Q19/D3Q7, D3Q27/D3Q7; lattice_cuda.cu:912-1010).
template <class FL> struct ScalarOf;
template <> struct ScalarOf<D2Q9> { using type = D2Q5; };
template <> struct ScalarOf<D3Q19> { using type = D3Q7; };
template <> struct ScalarOf<D3Q27> { using type = D3Q7; };

enum Collision : int { kBGK = 0, kTRT = 1, kMRT = 2, kRLBM = 3 };

// Populations that cross a z face of a slab: zcount_of<L>() of them per face
// (c_z = +1 and c_z = -1 each); zslot_of<L>(i) is population i's place among
// those with the same c_z, in ascending i.
template <class L>
__host__ __device__ constexpr int zslot_of(int i) {
  int k = 0;
  for (int j = 0; j < i; ++j) k += L::c[j][2] == L::c[i][2] ? 1 : 0;
  return k;
}
template <class L>
__host__ __device__ constexpr int zcount_of() {
  int k = 0;
  for (int j = 0; j < L::Q; ++j) k += L::c[j][2] > 0 ? 1 : 0;
  return k;
}

}  // namespace lbcube
