// Runner for the C++ drop-in tests: `fem_cpp_tests [--cpu|--gpu]`.
#include <cstring>

#include "harness.hpp"

int main(int argc, char** argv) {
  const bool cpu_only = argc > 1 && std::strcmp(argv[1], "--cpu") == 0;
  const bool gpu_only = argc > 1 && std::strcmp(argv[1], "--gpu") == 0;
  int run = 0, failed = 0;
  for (const auto& t : harness::registry()) {
    const bool gpu = t.tags.find("[gpu]") != std::string::npos;
    if ((cpu_only && gpu) || (gpu_only && !gpu)) continue;
    ++run;
    try {
      t.fn();
    } catch (const std::exception& e) {
      ++failed;
      std::printf("FAILED %s: %s\n", t.name.c_str(), e.what());
    }
  }
  std::printf("%d tests, %d failed\n", run, failed);
  return failed ? 1 : 0;
}
