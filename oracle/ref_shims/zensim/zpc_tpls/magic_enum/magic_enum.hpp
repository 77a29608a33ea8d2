// Test infrastructure for the oracle build only (never linked into the product library).
//
// Minimal stand-in for the two magic_enum calls the reference's MPM headers make
// (execution/ExecutionPolicy.hpp:26 uses enum_integer, geometry/Structure.hpp:199 uses
// enum_name).  The reference vendors magic_enum in its zpc_tpls submodule, which is not
// checked out; neither call is on the arithmetic path.  geometry/SparseLevelSet.hpp:128
// also streams an enum, so an ostream operator for scoped enums is provided in namespace zs.
#pragma once
#include <ostream>
#include <string_view>
#include <type_traits>

namespace magic_enum {
  template <typename E> constexpr auto enum_integer(E e) noexcept {
    return static_cast<std::underlying_type_t<E>>(e);
  }
  template <typename E> constexpr std::string_view enum_name(E) noexcept { return "enum"; }
}  // namespace magic_enum

namespace zs {
  template <typename E, std::enable_if_t<std::is_enum_v<E>, int> = 0>
  std::ostream &operator<<(std::ostream &os, E e) {
    return os << static_cast<long long>(e);
  }
}  // namespace zs
