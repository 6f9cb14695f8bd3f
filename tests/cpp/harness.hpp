// A minimal test harness for the C++ drop-in tests (the reference uses
// Catch2, which is not available here).  TEST_CASE registers a test with tags;
// tests tagged [gpu] need a CUDA device.  main() runs `--cpu` (untagged),
// `--gpu` ([gpu] only) or everything, and prints one line per failure.
#pragma once
#include <cmath>
#include <cstdio>
#include <exception>
#include <functional>
#include <sstream>
#include <string>
#include <vector>

namespace harness {

struct Test {
  std::string name, tags;
  std::function<void()> fn;
};
inline std::vector<Test>& registry() {
  static std::vector<Test> r;
  return r;
}
struct Registrar {
  Registrar(const char* name, const char* tags, std::function<void()> fn) { registry().push_back({name, tags, fn}); }
};
struct Failure : std::exception {
  std::string msg;
  explicit Failure(std::string m) : msg(std::move(m)) {}
  const char* what() const noexcept override { return msg.c_str(); }
};

// Approx(x).margin(m): |a - x| <= margin, or within a relative 100 * DBL_EPSILON
// (stricter than Catch's default float-epsilon scale).
struct Approx {
  double value, margin_ = 0.0, eps = 2.220446049250313e-16 * 100;
  explicit Approx(double v) : value(v) {}
  Approx& margin(double m) {
    margin_ = m;
    return *this;
  }
  friend bool operator==(double a, const Approx& b) {
    const double d = std::fabs(a - b.value);
    return d <= b.margin_ || d <= b.eps * (std::fabs(b.value) + std::fabs(a)) * 0.5 + b.eps;
  }
  friend std::ostream& operator<<(std::ostream& os, const Approx& a) { return os << "Approx(" << a.value << ")"; }
};

}  // namespace harness

#define HARNESS_CAT2(a, b) a##b
#define HARNESS_CAT(a, b) HARNESS_CAT2(a, b)
#define TEST_CASE(name, tags)                                                                        \
  static void HARNESS_CAT(test_fn_, __LINE__)();                                                     \
  static harness::Registrar HARNESS_CAT(test_reg_, __LINE__)(name, tags, HARNESS_CAT(test_fn_, __LINE__)); \
  static void HARNESS_CAT(test_fn_, __LINE__)()

#define REQUIRE(...)                                                                                 \
  do {                                                                                               \
    if (!(__VA_ARGS__)) {                                                                            \
      std::ostringstream os_;                                                                        \
      os_ << __FILE__ << ":" << __LINE__ << ": REQUIRE(" #__VA_ARGS__ ") failed";                    \
      throw harness::Failure(os_.str());                                                             \
    }                                                                                                \
  } while (0)

#define REQUIRE_FALSE(...) REQUIRE(!(__VA_ARGS__))

#define REQUIRE_THROWS_AS(expr, type)                                                                \
  do {                                                                                               \
    bool caught_ = false;                                                                            \
    try {                                                                                            \
      (void)(expr);                                                                                  \
    } catch (const type&) {                                                                          \
      caught_ = true;                                                                                \
    } catch (const std::exception& e_) {                                                             \
      throw harness::Failure(std::string(__FILE__) + ":" + std::to_string(__LINE__) +               \
                             ": wrong exception from " #expr ": " + e_.what());                      \
    }                                                                                                \
    if (!caught_)                                                                                    \
      throw harness::Failure(std::string(__FILE__) + ":" + std::to_string(__LINE__) + ": " #expr     \
                             " did not throw " #type);                                               \
  } while (0)

#define REQUIRE_NOTHROW(...)                                                                         \
  do {                                                                                               \
    try {                                                                                            \
      (void)(__VA_ARGS__);                                                                           \
    } catch (const std::exception& e_) {                                                             \
      throw harness::Failure(std::string(__FILE__) + ":" + std::to_string(__LINE__) + ": " #__VA_ARGS__ \
                             " threw: " + e_.what());                                                \
    }                                                                                                \
  } while (0)
