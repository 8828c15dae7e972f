// Test-infrastructure shim: a tiny GoogleTest stand-in (TEST, EXPECT_* with
// streamed messages, DISABLED_ skipping) so LB-Cube's own
// tests/test_validation.cpp can be compiled unmodified and re-run as a health
// check of the reference build. GoogleTest is not installed here. Prints one
// line per test and a summary; the exit status is the number of failed tests
// (capped at 255). An optional argv[1] substring filters tests by "Suite.Name".
#pragma once
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

namespace gtest_shim {
struct Case {
  const char* suite;
  const char* name;
  void (*fn)();
};
inline std::vector<Case>& registry() {
  static std::vector<Case> r;
  return r;
}
inline int& failures() {
  static int f = 0;
  return f;
}
struct Registrar {
  Registrar(const char* s, const char* n, void (*fn)()) { registry().push_back({s, n, fn}); }
};

// Outcome of one check: converts to true on success, carries text on failure.
struct Result {
  bool ok;
  std::string text;
  explicit operator bool() const { return ok; }
};

// Failure report; extra `<< message` parts are appended before it prints.
class Failure {
 public:
  Failure(const char* file, int line, std::string text) : file_(file), line_(line) {
    os_ << text;
  }
  ~Failure() {
    ++failures();
    std::printf("  FAILURE %s:%d: %s\n", file_, line_, os_.str().c_str());
  }
  template <typename T>
  Failure& operator<<(const T& v) {
    os_ << ' ' << v;
    return *this;
  }

 private:
  const char* file_;
  int line_;
  std::ostringstream os_;
};

inline std::string fmt(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}
inline Result cmp(bool ok, const char* what, double a, double b) {
  return {ok, ok ? std::string() : std::string(what) + " " + fmt(a) + " vs " + fmt(b)};
}
inline Result near(double a, double b, double tol) {
  const bool ok = std::fabs(a - b) <= tol;
  return {ok, ok ? std::string() : "EXPECT_NEAR " + fmt(a) + " vs " + fmt(b) + " tol " + fmt(tol)};
}
inline Result double_eq(double a, double b) {  // within 4 ULP, as GoogleTest
  const double ulp = std::fabs(std::nextafter(a, INFINITY) - a);
  return cmp(std::fabs(a - b) <= 4.0 * ulp, "EXPECT_DOUBLE_EQ", a, b);
}
}  // namespace gtest_shim

#define TEST(suite, name)                                                     \
  static void suite##_##name##_body();                                        \
  static gtest_shim::Registrar suite##_##name##_reg(#suite, #name,            \
                                                    &suite##_##name##_body);  \
  static void suite##_##name##_body()

#define GTEST_SHIM_EXPECT(res_expr)                                           \
  switch (0)                                                                  \
  case 0:                                                                     \
  default:                                                                    \
    if (const gtest_shim::Result gtest_r_ = (res_expr))                       \
      ;                                                                       \
    else                                                                      \
      gtest_shim::Failure(__FILE__, __LINE__, gtest_r_.text)

#define EXPECT_TRUE(c) GTEST_SHIM_EXPECT((gtest_shim::Result{bool(c), "EXPECT_TRUE(" #c ")"}))
#define EXPECT_FALSE(c) GTEST_SHIM_EXPECT((gtest_shim::Result{!bool(c), "EXPECT_FALSE(" #c ")"}))
#define EXPECT_LT(a, b) GTEST_SHIM_EXPECT(gtest_shim::cmp((a) < (b), "EXPECT_LT", (double)(a), (double)(b)))
#define EXPECT_GT(a, b) GTEST_SHIM_EXPECT(gtest_shim::cmp((a) > (b), "EXPECT_GT", (double)(a), (double)(b)))
#define EXPECT_GE(a, b) GTEST_SHIM_EXPECT(gtest_shim::cmp((a) >= (b), "EXPECT_GE", (double)(a), (double)(b)))
#define EXPECT_LE(a, b) GTEST_SHIM_EXPECT(gtest_shim::cmp((a) <= (b), "EXPECT_LE", (double)(a), (double)(b)))
#define EXPECT_NEAR(a, b, tol) GTEST_SHIM_EXPECT(gtest_shim::near((double)(a), (double)(b), (double)(tol)))
#define EXPECT_DOUBLE_EQ(a, b) GTEST_SHIM_EXPECT(gtest_shim::double_eq((double)(a), (double)(b)))

int main(int argc, char** argv) {
  int failed_tests = 0, run = 0, skipped = 0;
  const char* filter = argc > 1 ? argv[1] : nullptr;
  for (const auto& c : gtest_shim::registry()) {
    std::string full = std::string(c.suite) + "." + c.name;
    if (filter && full.find(filter) == std::string::npos) continue;
    if (std::strncmp(c.name, "DISABLED_", 9) == 0) {
      ++skipped;
      std::printf("[ SKIPPED ] %s\n", full.c_str());
      continue;
    }
    const int before = gtest_shim::failures();
    const auto t0 = std::chrono::steady_clock::now();
    c.fn();
    const double s =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    ++run;
    const bool ok = gtest_shim::failures() == before;
    if (!ok) ++failed_tests;
    std::printf("[ %s ] %s (%.2f s)\n", ok ? "     OK" : "FAILED ", full.c_str(), s);
    std::fflush(stdout);
  }
  std::printf("SUMMARY run=%d passed=%d failed=%d skipped=%d\n", run, run - failed_tests,
              failed_tests, skipped);
  return failed_tests > 255 ? 255 : failed_tests;
}
