// Project-written stand-in for the tlx header of the same name (the tlx
// submodule is not vendored with the reference). Only the macro the
// PageRank-path sources use is provided: it expands to its argument.
#pragma once
#define TLX_DEPRECATED(x) x
