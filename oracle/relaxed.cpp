// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
// C entry points of the relaxed BC1/BC7 decode (oracle_relaxed.h) for the
// differentiable-decode tests: parsing, and the relaxed decode and its
// adjoint in double precision (the finite-difference reference).
#include "oracle_relaxed.h"

using namespace oracle;

extern "C" void oracle_bc7_parse(const uint8_t* blocks, size_t n, uint32_t* meta, float* ep) {
    for (size_t i = 0; i < n; i++) relaxed::bc7_parse(blocks + 16 * i, meta + 8 * i, ep + 24 * i);
}

extern "C" void oracle_bc1_parse(const uint8_t* blocks, size_t n, uint32_t* meta, float* ep) {
    for (size_t i = 0; i < n; i++) relaxed::bc1_parse(blocks + 8 * i, meta + 2 * i, ep + 6 * i);
}

extern "C" void oracle_bc7_relaxed_f64(const uint32_t* meta, const double* ep, size_t n, double* out) {
    for (size_t i = 0; i < n; i++) relaxed::bc7_relaxed<double>(meta + 8 * i, ep + 24 * i, out + 64 * i);
}

extern "C" void oracle_bc7_adjoint_f64(const uint32_t* meta, const double* g, size_t n, double* gep) {
    for (size_t i = 0; i < n; i++) relaxed::bc7_adjoint<double>(meta + 8 * i, g + 64 * i, gep + 24 * i);
}

extern "C" void oracle_bc1_relaxed_f64(const uint32_t* meta, const double* ep, size_t n, double* out) {
    for (size_t i = 0; i < n; i++) relaxed::bc1_relaxed<double>(meta + 2 * i, ep + 6 * i, out + 64 * i);
}

extern "C" void oracle_bc1_adjoint_f64(const uint32_t* meta, const double* g, size_t n, double* gep) {
    for (size_t i = 0; i < n; i++) relaxed::bc1_adjoint<double>(meta + 2 * i, g + 64 * i, gep + 6 * i);
}
