// Project-written stand-in for the tlx header of the same name (the tlx
// submodule is not checked out): number of leading zero bits, 64 for 0.
#pragma once
#include <cstdint>

namespace tlx {
inline unsigned clz(uint64_t x) { return x ? static_cast<unsigned>(__builtin_clzll(x)) : 64u; }
inline unsigned clz(uint32_t x) { return x ? static_cast<unsigned>(__builtin_clz(x)) : 32u; }
} // namespace tlx
