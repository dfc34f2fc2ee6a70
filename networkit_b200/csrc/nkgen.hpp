// The generator library's C structure (shared by its sources): an in-CSR in
// malloc'd arrays that nkgen_free releases.
#pragma once
#include <cstdint>

extern "C" {
struct nkgen_csr {
    uint64_t z;
    uint64_t arcs;
    uint64_t *in_ptr;
    uint32_t *in_col;
    uint32_t *outdeg;
    double *w;
};
}

// Records the message that nkgen_last_error() returns on this thread.
void nkgen_set_error(const char *msg);
