// Project-written stand-in: floor/ceil of log2 for unsigned integers,
// computed with the compiler's count-leading-zeros builtin.
#pragma once
#include <cstdint>
namespace tlx {
template <typename T>
inline unsigned integer_log2_floor(T x) {
    return x <= 1 ? 0u : 63u - static_cast<unsigned>(__builtin_clzll(static_cast<unsigned long long>(x)));
}
template <typename T>
inline unsigned integer_log2_ceil(T x) {
    return x <= 1 ? 0u : integer_log2_floor(static_cast<unsigned long long>(x) - 1ull) + 1u;
}
} // namespace tlx
