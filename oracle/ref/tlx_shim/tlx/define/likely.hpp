// Project-written stand-in for the tlx header of the same name: branch hints.
#pragma once
#define TLX_LIKELY(c) __builtin_expect(!!(c), 1)
#define TLX_UNLIKELY(c) __builtin_expect(!!(c), 0)
