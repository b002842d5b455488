// Test infrastructure only: AMReX managed-arena stand-in (host malloc/free).
#ifndef AXREF_SHIM_AMREX_H
#define AXREF_SHIM_AMREX_H
#include <cstdlib>
namespace amrex {
struct Arena {
  void *alloc(std::size_t n) { return std::malloc(n); }
  void free(void *p) { std::free(p); }
};
inline Arena *The_Managed_Arena() {
  static Arena a;
  return &a;
}
} // namespace amrex
#endif
