// Project-written stand-in for the tlx header of the same name: one plus the
// index of the least significant set bit, 0 for 0 (POSIX ffs).
#pragma once
#include <cstdint>

namespace tlx {
inline unsigned ffs(uint64_t x) { return static_cast<unsigned>(__builtin_ffsll(static_cast<long long>(x))); }
inline unsigned ffs(uint32_t x) { return static_cast<unsigned>(__builtin_ffs(static_cast<int>(x))); }
inline unsigned ffs(int x) { return static_cast<unsigned>(__builtin_ffs(x)); }
inline unsigned ffs(uint8_t x) { return ffs(static_cast<uint32_t>(x)); }
} // namespace tlx
