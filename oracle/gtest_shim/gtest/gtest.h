// Minimal GoogleTest stand-in used only to build the reference's own test
// files (tests/test_*.cpp of rezucch1/nbody-FMM) without network access.
// It supports the subset those files use: TEST, EXPECT_EQ/NE/LT/GT/NEAR/
// DOUBLE_EQ/TRUE and a main() that runs every registered test and returns
// the number of failed expectations (0 = pass).
//
// Test infrastructure only: nothing in the product links this header.
#pragma once
#include <cmath>
#include <cstdio>
#include <functional>
#include <iostream>
#include <string>
#include <vector>

namespace gshim {
struct Registry {
  std::vector<std::pair<std::string, std::function<void()>>> tests;
  int failures = 0;
  static Registry &get() { static Registry r; return r; }
};
struct Reg {
  Reg(const char *n, std::function<void()> f) { Registry::get().tests.emplace_back(n, std::move(f)); }
};
inline void fail(const char *file, int line, const std::string &what) {
  ++Registry::get().failures;
  std::fprintf(stderr, "%s:%d: expectation failed: %s\n", file, line, what.c_str());
}
}  // namespace gshim

#define TEST(suite, name)                                                        \
  static void suite##_##name##_body();                                           \
  static gshim::Reg suite##_##name##_reg(#suite "." #name, suite##_##name##_body); \
  static void suite##_##name##_body()

#define GSHIM_CHECK(cond, text) \
  do { if (!(cond)) gshim::fail(__FILE__, __LINE__, text); } while (0)
#define EXPECT_TRUE(a) GSHIM_CHECK((a), #a)
#define EXPECT_FALSE(a) GSHIM_CHECK(!(a), "!" #a)
#define EXPECT_EQ(a, b) GSHIM_CHECK((a) == (b), #a " == " #b)
#define EXPECT_NE(a, b) GSHIM_CHECK((a) != (b), #a " != " #b)
#define EXPECT_LT(a, b) GSHIM_CHECK((a) < (b), #a " < " #b)
#define EXPECT_GT(a, b) GSHIM_CHECK((a) > (b), #a " > " #b)
#define EXPECT_LE(a, b) GSHIM_CHECK((a) <= (b), #a " <= " #b)
#define EXPECT_GE(a, b) GSHIM_CHECK((a) >= (b), #a " >= " #b)
#define EXPECT_NEAR(a, b, tol) GSHIM_CHECK(std::fabs((double)(a) - (double)(b)) <= (tol), #a " ~ " #b)
#define EXPECT_DOUBLE_EQ(a, b) \
  GSHIM_CHECK(std::fabs((double)(a) - (double)(b)) <= 4 * 2.220446049250313e-16 * std::fmax(std::fabs((double)(a)), std::fabs((double)(b))), #a " == " #b)
#define ASSERT_EQ EXPECT_EQ
#define ASSERT_NEAR EXPECT_NEAR
#define ASSERT_TRUE EXPECT_TRUE

int main() {
  auto &r = gshim::Registry::get();
  for (auto &t : r.tests) {
    int before = r.failures;
    t.second();
    std::fprintf(stderr, "[%s] %s\n", r.failures == before ? "  OK  " : " FAIL ", t.first.c_str());
  }
  std::fprintf(stderr, "%d failed expectation(s)\n", r.failures);
  return r.failures == 0 ? 0 : 1;
}
