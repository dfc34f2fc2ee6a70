// Project-written stand-in: swallow any arguments to silence unused warnings.
#pragma once
namespace tlx {
template <typename... Args>
inline void unused(Args &&...) {}
} // namespace tlx
