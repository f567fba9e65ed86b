// gf_host.hpp -- host-side helpers shared by the C ABI translation units: error reporting,
// argument validation and the kernel dispatch tables.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "../../include/gfix.h"
#include "gf_device.cuh"

namespace gfb {

void set_error(const char *fmt, ...);
void clear_error();

// GF_OK if e == cudaSuccess, else records the message and returns GF_ERR_CUDA
int cuda_status(cudaError_t e, const char *what);
// checks the launch that just happened (cudaGetLastError)
int launch_status(const char *what);

// Validates extents (all even, >= 2, V < 2^31; COULOMB slices have size[0] == 1) and fills g.
int make_geom(const int32_t size[4], int gauge, bool plugin_slice, Geom &g);

inline bool valid_gauge(int gauge) { return gauge >= GF_LANDAU && gauge <= GF_U1XU1; }
inline bool valid_real(int real) { return real == GF_FP32 || real == GF_FP64; }

inline double prefactor_gff(int gauge) { return gauge == GF_COULOMB ? 1.0 / 9.0 : 1.0 / 12.0; }
inline double prefactor_a(int) { return 1.0 / 3.0; }

// compile-time dispatch of a functor over the gauge / algorithm template parameters
template <template <int, int> class K, typename... Args>
int dispatch_gauge_algo(int gauge, int algo, const Args &...args)
{
#define GFB_CASE_A(G)                                                   \
    switch (algo) {                                                     \
    case ALG_OR: return K<G, ALG_OR>::run(args...);                     \
    case ALG_MICRO: return K<G, ALG_MICRO>::run(args...);               \
    case ALG_SA: return K<G, ALG_SA>::run(args...);                     \
    case ALG_SR: return K<G, ALG_SR>::run(args...);                     \
    case ALG_RANDOM: return K<G, ALG_RANDOM>::run(args...);             \
    default: break;                                                     \
    }                                                                   \
    break;
    switch (gauge) {
    case LANDAU: GFB_CASE_A(LANDAU)
    case COULOMB: GFB_CASE_A(COULOMB)
    case MAG: GFB_CASE_A(MAG)
    case U1XU1: GFB_CASE_A(U1XU1)
    default: break;
    }
#undef GFB_CASE_A
    set_error("invalid gauge %d or algorithm %d", gauge, algo);
    return GF_ERR_INVALID;
}

}  // namespace gfb
