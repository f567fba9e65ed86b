// gf_noalloc.cu -- gauge quality (functional and theta) of a field without any allocation.
//
// gf_stats_generate needs reduction scratch that gf_stats_create obtains with cudaMalloc.  Some
// callers cannot call cudaMalloc: host frameworks that own all device memory through their own
// pool, and latency-critical loops where cudaMalloc's device-wide synchronisation is not
// acceptable.  gf_quality_noalloc runs the same fused quality kernel with its scratch in a
// file-scope __device__ array of fixed size instead: GF_NOALLOC_MAX_BLOCKS blocks of 256 sites,
// i.e. at most 256 * 65536 = 16,777,216 sites (64^4).  Every GPU that loads the library holds
// this ~1 MiB array until the process exits.
#include "gf_host.hpp"
#include "gf_kernels.cuh"

namespace gfb {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxBlocks = 65536;  // GF_NOALLOC_MAX_SITES / 256

// partials (2 doubles per block), then the 2 result doubles, then the ticket
struct NoAllocScratch {
    double partials[2 * kNoAllocMaxBlocks];
    double result[2];
    unsigned int ticket;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Host code may not use the symbol's host-side name as a device address.  The address is looked up
// on every call, with the caller's device current: the first lookup on a device may load this
// library's module there (so make that first call before any stream capture), later ones are a
// table lookup in the runtime.  Nothing is cached across calls, so after a cudaDeviceReset --
// which unloads the module and places the array anew when it is next loaded -- the next call
// uses the new address, never one kept from before the reset.
static int noalloc_scratch(NoAllocScratch **out)
{
    void *p = nullptr;
    const int st = cuda_status(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
    if (st) return st;
    *out = static_cast<NoAllocScratch *>(p);
    return GF_OK;
}

template <int GAUGE>
static int noalloc_launch(int real, const void *U, const Geom &g, QualityOut o, int stop_max, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((g.V + kNoAllocThreads - 1) / kNoAllocThreads);
    if (real == GF_FP64)
        k_quality<GAUGE, double, RefField<double>, kNoAllocThreads><<<blocks, kNoAllocThreads, 0, s>>>(
            RefField<double>{(double *)U, g.V}, g, o, stop_max, prefactor_gff(GAUGE), prefactor_a(GAUGE));
    else
        k_quality<GAUGE, float, RefField<float>, kNoAllocThreads><<<blocks, kNoAllocThreads, 0, s>>>(
            RefField<float>{(float *)U, g.V}, g, o, stop_max, prefactor_gff(GAUGE), prefactor_a(GAUGE));
    return launch_status("quality (no allocation)");
}

}  // namespace gfb

using namespace gfb;

extern "C" int gf_quality_noalloc(int gauge, int real, const void *U, const int32_t size[4], int stopping,
                                  void *stream, double *gff, double *theta)
{
    clear_error();
    if (!U || !valid_gauge(gauge) || !valid_real(real) || (stopping != GF_MAX && stopping != GF_AVERAGE)) {
        set_error("invalid argument to gf_quality_noalloc");
        return GF_ERR_INVALID;
    }
    Geom g;
    int st = make_geom(size, gauge, true, g);
    if (st) return st;
    if (g.V > (int64_t)kNoAllocThreads * kNoAllocMaxBlocks) {
        set_error("gf_quality_noalloc: lattice of %lld sites exceeds the fixed scratch limit of %lld sites",
                  (long long)g.V, (long long)kNoAllocThreads * kNoAllocMaxBlocks);
        return GF_ERR_INVALID;
    }
    NoAllocScratch *sc = nullptr;
    if ((st = noalloc_scratch(&sc))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    // the ticket must start at zero; a memset of the existing array allocates nothing
    if ((st = cuda_status(cudaMemsetAsync(&sc->ticket, 0, sizeof(unsigned int), s), "cudaMemsetAsync"))) return st;
    QualityOut o;
    o.partials = sc->partials;
    o.result = sc->result;
    o.ticket = &sc->ticket;
    o.gff_site = nullptr;
    o.theta_site = nullptr;
    const int stop_max = stopping == GF_MAX;
    switch (gauge) {
    case GF_LANDAU: st = noalloc_launch<LANDAU>(real, U, g, o, stop_max, s); break;
    case GF_COULOMB: st = noalloc_launch<COULOMB>(real, U, g, o, stop_max, s); break;
    case GF_MAG: st = noalloc_launch<MAG>(real, U, g, o, stop_max, s); break;
    default: st = noalloc_launch<U1XU1>(real, U, g, o, stop_max, s); break;
    }
    if (st) return st;
    double h[2];
    if ((st = cuda_status(cudaMemcpyAsync(h, sc->result, sizeof(h), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync")))
        return st;
    if ((st = cuda_status(cudaStreamSynchronize(s), "cudaStreamSynchronize"))) return st;
    if (gff) *gff = h[0];
    if (theta) *theta = h[1];
    return GF_OK;
}
