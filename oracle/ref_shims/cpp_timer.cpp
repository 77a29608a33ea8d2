// Test infrastructure for the oracle build only: definitions of zs::CppTimer and one
// missing Linux definition (see the end of this file); zs::CppTimer is
// (declared in the reference's profile/CppTimers.hpp) without the fmt dependency of the
// reference's profile/CppTimers.cpp.  The omp/seq policies construct a timer per launch
// and only print it when profiling is switched on.
#include <chrono>
#include <cstdio>
#include <string_view>
#include "zensim/profile/CppTimers.hpp"

namespace zs {
  static double zs_shim_now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
  }
  void CppTimer::tick() { last = zs_shim_now_ms(); }
  void CppTimer::tock() { cur = zs_shim_now_ms(); }
  float CppTimer::elapsed() const noexcept { return (float)(cur - last); }
  void CppTimer::tock(std::string_view tag) {
    tock();
    std::printf("%.*s: %.4f ms\n", (int)tag.size(), tag.data(), elapsed());
  }
}  // namespace zs

// The reference declares arena_virtual_memory_resource<host_mem_tag>::do_protect for every
// platform (memory/Allocator.h:304) but defines it only in its Windows branch
// (memory/Allocator.cpp:91).  The MPM path never changes page protection; report "not done".
#include "zensim/memory/Allocator.h"
namespace zs {
  bool arena_virtual_memory_resource<host_mem_tag>::do_protect(size_t, size_t, PageAccess) {
    return false;
  }
}  // namespace zs
