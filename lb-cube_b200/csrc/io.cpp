// Host-side output formats.
//
// lbm_write_vtk_legacy writes the legacy ASCII VTK file of the reference's
// write_vtk (include/lattice_io.hpp:386-451) from macroscopic fields already
// on the host (lbm_macro_fields_async + one device-to-host copy of 2 + D values
// per cell): the same header lines, the density, velocity_magnitude and
// VECTORS velocity blocks in x-fastest order, every value printed as
// "{:.17g}" of the double widening of the population-precision value, and a
// zero z-component for 2-D lattices (velocity_component, :99-110). Numbers are
// formatted with std::to_chars (general, 17 significant digits: the
// printf("%.17g") text) by several threads in parallel, then written in order.
//
// lbm_write_populations / lbm_read_populations store a population field for
// restart: a 64-byte header (magic "LBCUBEP1", lattice, precision, extents,
// time step) followed by the raw [Q, Z, Y, X] values. No reference
// counterpart (the reference has no restart files).
#include <algorithm>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lbcube_b200.h"

namespace {

// Appends "{:.17g}" of v.
inline void put_g17(std::string& out, double v) {
  char buf[40];
  const auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::general, 17);
  out.append(buf, r.ptr);
}

template <class Real>
double at(const void* p, size_t i) {
  return static_cast<double>(static_cast<const Real*>(p)[i]);
}

// Formats rows [0, n) with `row(i, out)` on up to `threads` threads and writes
// the pieces in order.
template <class Row>
bool write_rows(FILE* fp, size_t n, Row row) {
  unsigned threads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  if (n < 65536) threads = 1;
  const size_t chunk = (n + threads - 1) / threads;
  std::vector<std::string> parts(threads);
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; ++t) {
    pool.emplace_back([&, t] {
      const size_t lo = t * chunk, hi = std::min(n, lo + chunk);
      std::string& s = parts[t];
      s.reserve((hi > lo ? hi - lo : 0) * 24);
      for (size_t i = lo; i < hi; ++i) row(i, s);
    });
  }
  for (auto& th : pool) th.join();
  for (const auto& s : parts)
    if (!s.empty() && fwrite(s.data(), 1, s.size(), fp) != s.size()) return false;
  return true;
}

template <class Real>
int write_vtk(const char* path, int dims, size_t nx, size_t ny, size_t nz, size_t step,
              const void* rho, const void* u, const void* speed) {
  if (dims == 2) nz = 1;
  const size_t n = nx * ny * nz;
  FILE* fp = fopen(path, "wb");
  if (fp == nullptr) return LBM_IO_OPEN_FAILED;
  std::string head;
  head += "# vtk DataFile Version 3.0\n";
  head += "LBM output step " + std::to_string(step) + "\n";
  head += "ASCII\n";
  head += "DATASET STRUCTURED_POINTS\n";
  head += "DIMENSIONS " + std::to_string(nx) + " " + std::to_string(ny) + " " + std::to_string(nz) + "\n";
  head += "ORIGIN 0 0 0\n";
  head += "SPACING 1 1 1\n";
  head += "POINT_DATA " + std::to_string(n) + "\n";
  head += "SCALARS density double 1\n";
  head += "LOOKUP_TABLE default\n";
  bool ok = fwrite(head.data(), 1, head.size(), fp) == head.size();
  ok = ok && write_rows(fp, n, [&](size_t i, std::string& s) {
         put_g17(s, at<Real>(rho, i));
         s += '\n';
       });
  const char* mid = "SCALARS velocity_magnitude double 1\nLOOKUP_TABLE default\n";
  ok = ok && fputs(mid, fp) >= 0;
  ok = ok && write_rows(fp, n, [&](size_t i, std::string& s) {
         put_g17(s, at<Real>(speed, i));
         s += '\n';
       });
  ok = ok && fputs("VECTORS velocity double\n", fp) >= 0;
  ok = ok && write_rows(fp, n, [&](size_t i, std::string& s) {
         put_g17(s, at<Real>(u, i));
         s += ' ';
         put_g17(s, at<Real>(u, n + i));
         s += ' ';
         put_g17(s, dims == 3 ? at<Real>(u, 2 * n + i) : static_cast<double>(Real(0)));
         s += '\n';
       });
  ok = (fclose(fp) == 0) && ok;
  return ok ? 0 : LBM_IO_WRITE_FAILED;
}

int q_of(int lattice) {
  switch (lattice) {
    case LBM_D2Q9: return 9;
    case LBM_D3Q19: return 19;
    case LBM_D3Q27: return 27;
    case LBM_D2Q5: return 5;
    case LBM_D3Q7: return 7;
    default: return 0;
  }
}

struct DumpHeader {
  char magic[8];
  int32_t lattice, precision;
  uint64_t nx, ny, nz, step;
  uint64_t reserved[2];
};
static_assert(sizeof(DumpHeader) == 64, "restart header is 64 bytes");

}  // namespace

extern "C" int lbm_write_vtk_legacy(const char* path, int dims, size_t x_extent, size_t y_extent,
                                    size_t z_extent, size_t time_step, int precision,
                                    const void* density, const void* velocity,
                                    const void* speed) {
  if (path == nullptr || density == nullptr || velocity == nullptr || speed == nullptr)
    return LBM_IO_BAD_ARGUMENT;
  if ((dims != 2 && dims != 3) || x_extent == 0 || y_extent == 0 || (dims == 3 && z_extent == 0))
    return LBM_IO_BAD_ARGUMENT;
  if (precision == LBM_FLOAT)
    return write_vtk<float>(path, dims, x_extent, y_extent, z_extent, time_step, density, velocity,
                            speed);
  if (precision == LBM_DOUBLE)
    return write_vtk<double>(path, dims, x_extent, y_extent, z_extent, time_step, density, velocity,
                             speed);
  return LBM_IO_BAD_ARGUMENT;
}

extern "C" int lbm_write_populations(const char* path, int lattice, int precision, size_t x_extent,
                                     size_t y_extent, size_t z_extent, size_t time_step,
                                     const void* populations) {
  const int q = q_of(lattice);
  if (path == nullptr || populations == nullptr || q == 0 ||
      (precision != LBM_FLOAT && precision != LBM_DOUBLE) || x_extent == 0 || y_extent == 0 ||
      z_extent == 0)
    return LBM_IO_BAD_ARGUMENT;
  DumpHeader h{};
  memcpy(h.magic, "LBCUBEP1", 8);
  h.lattice = lattice;
  h.precision = precision;
  h.nx = x_extent;
  h.ny = y_extent;
  h.nz = z_extent;
  h.step = time_step;
  const size_t bytes = (size_t)q * x_extent * y_extent * z_extent * (precision == LBM_FLOAT ? 4 : 8);
  FILE* fp = fopen(path, "wb");
  if (fp == nullptr) return LBM_IO_OPEN_FAILED;
  bool ok = fwrite(&h, sizeof(h), 1, fp) == 1 && fwrite(populations, 1, bytes, fp) == bytes;
  ok = (fclose(fp) == 0) && ok;
  return ok ? 0 : LBM_IO_WRITE_FAILED;
}

extern "C" int lbm_read_populations(const char* path, int lattice, int precision, size_t x_extent,
                                    size_t y_extent, size_t z_extent, size_t* time_step,
                                    void* populations) {
  const int q = q_of(lattice);
  if (path == nullptr || populations == nullptr || q == 0 ||
      (precision != LBM_FLOAT && precision != LBM_DOUBLE))
    return LBM_IO_BAD_ARGUMENT;
  FILE* fp = fopen(path, "rb");
  if (fp == nullptr) return LBM_IO_OPEN_FAILED;
  DumpHeader h{};
  const size_t bytes = (size_t)q * x_extent * y_extent * z_extent * (precision == LBM_FLOAT ? 4 : 8);
  int rc = 0;
  if (fread(&h, sizeof(h), 1, fp) != 1 || memcmp(h.magic, "LBCUBEP1", 8) != 0)
    rc = LBM_IO_BAD_FILE;
  else if (h.lattice != lattice || h.precision != precision || h.nx != x_extent ||
           h.ny != y_extent || h.nz != z_extent)
    rc = LBM_IO_MISMATCH;
  else if (fread(populations, 1, bytes, fp) != bytes)
    rc = LBM_IO_BAD_FILE;
  fclose(fp);
  if (rc == 0 && time_step != nullptr) *time_step = h.step;
  return rc;
}
