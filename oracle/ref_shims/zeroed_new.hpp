// Test infrastructure: global operator new returning zeroed memory, for the programs built from
// the reference's sources (oracle/ref_cli.cpp, oracle/zpc_adapter_check.cpp; one translation unit
// per program includes this).
//
// zs::MemoryBackendRegistry::instance() (memory/MemoryBackend.cpp:12-15) allocates the registry
// with `new`, and its zs::Mutex member is a std::atomic<u32> without an initializer
// (execution/ConcurrencyPrimitive.hpp:59-69), so it starts with whatever the heap held at that
// address.  When that word is nonzero, the first Mutex::lock() (MemoryBackend.cpp:63-66, reached
// from the first container allocation) parks forever.  Zeroed allocations give the mutex its
// unlocked state; the reference's arithmetic is untouched.
#pragma once
#include <cstdlib>
#include <new>

void *operator new(std::size_t n) {
  if (void *p = std::calloc(1, n ? n : 1)) return p;
  throw std::bad_alloc();
}
void *operator new[](std::size_t n) {
  if (void *p = std::calloc(1, n ? n : 1)) return p;
  throw std::bad_alloc();
}
void operator delete(void *p) noexcept { std::free(p); }
void operator delete[](void *p) noexcept { std::free(p); }
void operator delete(void *p, std::size_t) noexcept { std::free(p); }
void operator delete[](void *p, std::size_t) noexcept { std::free(p); }
