/*
 * Test infrastructure only: a minimal, project-written harness exposing the
 * four GoogleTest macros the reference's unit tests use (TEST, EXPECT_EQ,
 * EXPECT_NEAR, EXPECT_FLOAT_EQ; src/*_test.cpp, src/test.cpp) so that those
 * tests compile unchanged against this machine, which has no GoogleTest.
 * EXPECT_FLOAT_EQ follows GoogleTest's documented rule: both values as float,
 * equal within 4 units in the last place.
 */
#ifndef AGD_ORACLE_MINI_GTEST_H
#define AGD_ORACLE_MINI_GTEST_H

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

namespace mini_gtest {

struct Case {
  const char *suite;
  const char *name;
  void (*fn)();
};

inline std::vector<Case> &registry() {
  static std::vector<Case> cases;
  return cases;
}

inline long &failures() {
  static long n = 0;
  return n;
}

inline long &checks() {
  static long n = 0;
  return n;
}

struct Registrar {
  Registrar(const char *suite, const char *name, void (*fn)()) {
    registry().push_back(Case{suite, name, fn});
  }
};

inline void report(const char *file, int line, const std::string &msg) {
  failures()++;
  if (failures() <= 50) std::fprintf(stderr, "%s:%d: Failure\n%s\n", file, line, msg.c_str());
}

template <typename A, typename B>
inline void expect_eq(const A &a, const B &b, const char *sa, const char *sb,
                      const char *file, int line) {
  checks()++;
  if (!(a == b)) {
    report(file, line,
           std::string("  Expected equality of ") + sa + " and " + sb);
  }
}

inline int32_t float_bits_biased(float f) {
  int32_t i;
  std::memcpy(&i, &f, sizeof(i));
  /* map sign-magnitude to a monotonic integer line */
  return i < 0 ? (int32_t)(0x80000000u - (uint32_t)i) : i;
}

inline void expect_float_eq(double a_in, double b_in, const char *sa,
                            const char *sb, const char *file, int line) {
  checks()++;
  float const a = (float)a_in;
  float const b = (float)b_in;
  bool ok;
  if (std::isnan(a) || std::isnan(b)) {
    ok = false;
  } else {
    int64_t const d = (int64_t)float_bits_biased(a) - (int64_t)float_bits_biased(b);
    ok = (d <= 4 && d >= -4);
  }
  if (!ok) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "  %s = %.9g vs %s = %.9g (float ULP check)", sa,
                  (double)a, sb, (double)b);
    report(file, line, buf);
  }
}

inline void expect_near(double a, double b, double tol, const char *sa,
                        const char *sb, const char *file, int line) {
  checks()++;
  if (!(std::fabs(a - b) <= tol)) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "  |%s - %s| = |%.17g - %.17g| > %g", sa, sb, a, b, tol);
    report(file, line, buf);
  }
}

// MINI_GTEST_SKIP: comma-separated Suite.Name entries to skip.
inline bool skipped(const Case &c) {
  const char *env = std::getenv("MINI_GTEST_SKIP");
  if (env == nullptr) return false;
  const std::string full = std::string(c.suite) + "." + c.name;
  const std::string list = std::string(",") + env + ",";
  return list.find("," + full + ",") != std::string::npos;
}

inline int run_all() {
  int failed_cases = 0;
  for (const Case &c : registry()) {
    if (skipped(c)) {
      std::printf("[ SKIPPED] %s.%s\n", c.suite, c.name);
      continue;
    }
    long const before = failures();
    c.fn();
    bool const ok = failures() == before;
    std::printf("[ %s ] %s.%s\n", ok ? "    OK" : "FAILED", c.suite, c.name);
    if (!ok) failed_cases++;
  }
  std::printf("%zu tests, %d failed, %ld checks, %ld failed checks\n",
              registry().size(), failed_cases, checks(), failures());
  return failed_cases == 0 ? 0 : 1;
}

}  // namespace mini_gtest

#define TEST(suite, name)                                                   \
  static void suite##_##name##_body();                                      \
  static mini_gtest::Registrar suite##_##name##_registrar(#suite, #name,    \
                                                          &suite##_##name##_body); \
  static void suite##_##name##_body()

#define EXPECT_EQ(a, b) mini_gtest::expect_eq((a), (b), #a, #b, __FILE__, __LINE__)
#define EXPECT_FLOAT_EQ(a, b) \
  mini_gtest::expect_float_eq((double)(a), (double)(b), #a, #b, __FILE__, __LINE__)
#define EXPECT_NEAR(a, b, tol)                                                \
  mini_gtest::expect_near((double)(a), (double)(b), (double)(tol), #a, #b, \
                          __FILE__, __LINE__)

#endif
