// gf_plugin.cu -- the plugin-level C ABI: the reference's static launch wrappers
// (LandauKernelsSU3, CoulombKernelsSU3, MAGKernelsSU3, U1xU1KernelsSU3, CommonKernelsSU3,
// GaugeFixingStats) as C functions that work in place on a GpuPattern device array.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>

#include "gf_host.hpp"
#include "gf_kernels.cuh"

namespace gfb {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

void clear_error() { g_err[0] = 0; }

int cuda_status(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return GF_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? GF_ERR_NOMEM : GF_ERR_CUDA;
}

int launch_status(const char *what) { return cuda_status(cudaGetLastError(), what); }

int make_geom(const int32_t size[4], int gauge, bool plugin_slice, Geom &g)
{
    if (!size) {
        set_error("size is NULL");
        return GF_ERR_INVALID;
    }
    int64_t V = 1;
    for (int i = 0; i < 4; i++) {
        const bool slice_t = plugin_slice && gauge == GF_COULOMB && i == 0;
        if (slice_t) {
            if (size[0] != 1) {
                set_error("Coulomb plugin calls take one timeslice: size[0] must be 1, got %d", size[0]);
                return GF_ERR_INVALID;
            }
        } else if (size[i] < 2 || (size[i] & 1)) {
            set_error("extent %d = %d: every extent must be even and >= 2", i, size[i]);
            return GF_ERR_INVALID;
        }
        g.n[i] = size[i];
        V *= size[i];
    }
    if (V >= (int64_t(1) << 31)) {
        set_error("lattice volume %lld exceeds 2^31 sites", (long long)V);
        return GF_ERR_INVALID;
    }
    // a warp updates an 8-site tile of one parity; four even extents always give V % 16 == 0, three
    // (a Coulomb timeslice) may not (6^3: 108 sites per parity).  The reference's kernels need a
    // whole number of 32-site blocks per parity (apps/CoulombGaugeFixingSU3_4D.cu:138).
    if ((V / 2) % 8 != 0) {
        set_error("volume %lld: each parity must hold a multiple of 8 sites (V %% 16 == 0)", (long long)V);
        return GF_ERR_INVALID;
    }
    g.V = V;
    g.Vh = V / 2;
    geom_init_div(g);
    return GF_OK;
}

// ---- parity pass on the reference layout ----------------------------------------------------
struct StepArgs {
    int real;
    void *U, *Udw;
    Geom g;
    int parity;
    AlgoParams p;
    cudaStream_t stream;
};

template <int GAUGE, int ALGO>
struct RefStep {
    template <typename R>
    static int go(const StepArgs &a)
    {
        RefField<R> fu{(R *)a.U, a.g.V};
        RefField<R> fd{(R *)(a.Udw ? a.Udw : a.U), a.g.V};
        const int64_t ntiles = a.g.Vh / 8;
        if constexpr (ALGO == ALG_OR && sizeof(R) == 4) {
            // FP32 OR, the drivers' hot loop: the persistent register-prefetch pass, one wave of
            // blocks (0.157 vs 0.160 ms per 32^4 sweep; in FP64 its 200 registers leave 8 warps per
            // SM and the direct pass is faster, 0.377 vs 0.436 ms)
            auto kern = k_parity_pass_rp<R, GAUGE, ALGO, RefField<R>>;
            static int per_sm = 0, sms = 0;  // resident blocks per SM of this instantiation, SMs
            if (per_sm <= 0) {
                int dev = 0, o = 0;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, 128, 0) != cudaSuccess || o < 1) o = 1;
                per_sm = o;
            }
            const int64_t need = (ntiles + 3) / 4;
            const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * per_sm));
            kern<<<blocks, 128, 0, a.stream>>>(fu, fd, a.g, a.parity, a.p);
            return launch_status("parity pass (register prefetch)");
        }
        if constexpr (ALGO == ALG_OR && sizeof(R) == 8) {
            // FP64 OR: the persistent pass with the next tile staged by cp.async, one wave of blocks
            auto kern = k_parity_pass_ref_staged<GAUGE, ALGO>;
            const size_t smem = ref_staged_smem_bytes(4);  // 48 KB: no opt-in needed
            static int per_sm = 0, sms = 0;
            if (per_sm <= 0) {
                int dev = 0, o = 0;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, 128, smem) != cudaSuccess || o < 1) o = 1;
                per_sm = o;
            }
            const int64_t need = (ntiles + 3) / 4;
            const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * per_sm));
            kern<<<blocks, 128, smem, a.stream>>>(fu, fd, a.g, a.parity, a.p);
            return launch_status("parity pass (cp.async pipelined)");
        }
        const int64_t threads = a.g.Vh * 4;
        const unsigned blocks = (unsigned)((threads + 127) / 128);
        k_parity_pass<R, GAUGE, ALGO, RefField<R>><<<blocks, 128, 0, a.stream>>>(fu, fd, a.g, a.parity, a.p);
        return launch_status("parity pass");
    }
    static int run(const StepArgs &a) { return a.real == GF_FP64 ? go<double>(a) : go<float>(a); }
};

static int plugin_step(int gauge, int real, int algo, void *U, void *Udw, const int32_t size[4], int parity,
                       float param, int seed, int counter, void *stream)
{
    clear_error();
    if (!valid_gauge(gauge) || !valid_real(real)) {
        set_error("invalid gauge %d or real type %d", gauge, real);
        return GF_ERR_INVALID;
    }
    if (!U || (gauge == GF_COULOMB && !Udw)) {
        set_error("field pointer is NULL (Coulomb needs both UtUp and UtDw)");
        return GF_ERR_INVALID;
    }
    if (parity != 0 && parity != 1) {
        set_error("parity must be 0 or 1, got %d", parity);
        return GF_ERR_INVALID;
    }
    StepArgs a;
    int st = make_geom(size, gauge, true, a.g);
    if (st) return st;
    a.real = real;
    a.U = U;
    a.Udw = gauge == GF_COULOMB ? Udw : U;
    a.parity = parity;
    a.p.param = param;
    a.p.seed = (uint32_t)seed;
    a.p.counter = (uint32_t)counter;
    a.p.counter_stride = 0;
    a.stream = (cudaStream_t)stream;
    return dispatch_gauge_algo<RefStep>(gauge, algo, a);
}

struct RangeArgs {
    StepArgs a;
    int64_t h_lo, h_hi;
    int64_t rng_site_offset;  // site h draws its random numbers as site h + rng_site_offset
};

template <int GAUGE, int ALGO>
struct RefStepRange {
    template <typename R>
    static int go(const RangeArgs &r)
    {
        if constexpr (GAUGE == COULOMB) {
            set_error("timeslice ranges are for the 4D gauges");
            return GF_ERR_INVALID;
        } else {
            RefField<R> fu{(R *)r.a.U, r.a.g.V};
            const int64_t warps = (r.h_hi - (r.h_lo & ~(int64_t)7) + 7) / 8;
            if (warps <= 0) return GF_OK;
            const unsigned blocks = (unsigned)((warps * 32 + 127) / 128);
            k_parity_pass_range<R, GAUGE, ALGO, RefField<R>><<<blocks, 128, 0, r.a.stream>>>(
                fu, r.a.g, r.a.parity, r.a.p, r.h_lo, r.h_hi, r.rng_site_offset);
            return launch_status("parity pass over timeslices");
        }
    }
    static int run(const RangeArgs &r) { return r.a.real == GF_FP64 ? go<double>(r) : go<float>(r); }
};

// ---- quality -----------------------------------------------------------------------------------
struct QualityArgs {
    int real;
    const void *U;
    Geom g;
    QualityOut o;
    int stop_max;
    cudaStream_t stream;
};

template <int GAUGE>
struct RefQuality {
    template <typename R>
    static int go(const QualityArgs &a)
    {
        RefField<R> f{(R *)a.U, a.g.V};
        const unsigned blocks = (unsigned)((a.g.V + 255) / 256);
        k_quality<GAUGE, R, RefField<R>, 256><<<blocks, 256, 0, a.stream>>>(f, a.g, a.o, a.stop_max,
                                                                           prefactor_gff(GAUGE), prefactor_a(GAUGE));
        return launch_status("quality");
    }
    static int run(const QualityArgs &a) { return a.real == GF_FP64 ? go<double>(a) : go<float>(a); }
};

static int quality_dispatch(int gauge, const QualityArgs &a)
{
    switch (gauge) {
    case GF_LANDAU: return RefQuality<LANDAU>::run(a);
    case GF_COULOMB: return RefQuality<COULOMB>::run(a);
    case GF_MAG: return RefQuality<MAG>::run(a);
    case GF_U1XU1: return RefQuality<U1XU1>::run(a);
    default: set_error("invalid gauge %d", gauge); return GF_ERR_INVALID;
    }
}

}  // namespace gfb

using namespace gfb;

struct gf_stats {
    int gauge, real, stop_max, device;
    Geom g;
    double *scratch;       // partials (2 per block) + result (2)
    unsigned int *ticket;
    unsigned blocks;
};

extern "C" {

const char *gf_last_error_string(void) { return gfb::g_err; }
const char *gf_version(void) { return "su3_ma_gauge_gpu_b200 0.2 (sm_100a)"; }

int gf_binary_arch(int *arch)
{
    clear_error();
    if (!arch) {
        set_error("NULL argument");
        return GF_ERR_INVALID;
    }
    cudaFuncAttributes a{};
    const int st = cuda_status(cudaFuncGetAttributes(&a, k_set_hot_ref<double>), "cudaFuncGetAttributes");
    if (st) return st;
    *arch = a.binaryVersion;
    return GF_OK;
}

int gf_or_step(int gauge, int real, void *U, void *Udw, const int32_t size[4], int parity, float or_parameter,
               void *stream)
{
    return plugin_step(gauge, real, ALG_OR, U, Udw, size, parity, or_parameter, 0, 0, stream);
}

int gf_micro_step(int gauge, int real, void *U, void *Udw, const int32_t size[4], int parity, void *stream)
{
    return plugin_step(gauge, real, ALG_MICRO, U, Udw, size, parity, 0.f, 0, 0, stream);
}

int gf_sa_step(int gauge, int real, void *U, void *Udw, const int32_t size[4], int parity, float temperature,
               int seed, int rng_counter, void *stream)
{
    return plugin_step(gauge, real, ALG_SA, U, Udw, size, parity, temperature, seed, rng_counter, stream);
}

int gf_sr_step(int gauge, int real, void *U, void *Udw, const int32_t size[4], int parity, float sr_parameter,
               int seed, int rng_counter, void *stream)
{
    return plugin_step(gauge, real, ALG_SR, U, Udw, size, parity, sr_parameter, seed, rng_counter, stream);
}

int gf_random_trafo(int gauge, int real, void *U, void *Udw, const int32_t size[4], int parity, int seed,
                    int rng_counter, void *stream)
{
    return plugin_step(gauge, real, ALG_RANDOM, U, Udw, size, parity, 0.f, seed, rng_counter, stream);
}

int gf_step_slices(int gauge, int real, int algo, void *U, const int32_t size[4], int parity, float param, int seed,
                   int rng_counter, int t_begin, int t_end, void *stream)
{
    return gf_step_slices_at(gauge, real, algo, U, size, parity, param, seed, rng_counter, t_begin, t_end, 0, stream);
}

int gf_step_slices_at(int gauge, int real, int algo, void *U, const int32_t size[4], int parity, float param,
                      int seed, int rng_counter, int t_begin, int t_end, long long rng_site_offset, void *stream)
{
    clear_error();
    if (!valid_gauge(gauge) || gauge == GF_COULOMB || !valid_real(real) || !U || (parity != 0 && parity != 1) ||
        algo < ALG_OR || algo > ALG_RANDOM) {
        set_error("invalid argument to gf_step_slices (4D gauges only)");
        return GF_ERR_INVALID;
    }
    RangeArgs r;
    int st = make_geom(size, gauge, false, r.a.g);
    if (st) return st;
    if (t_begin < 0 || t_end > size[0] || t_begin > t_end) {
        set_error("timeslice range [%d, %d) is not inside [0, %d)", t_begin, t_end, size[0]);
        return GF_ERR_INVALID;
    }
    const int64_t half_slice = r.a.g.V / size[0] / 2;
    r.h_lo = t_begin * half_slice;
    r.h_hi = t_end * half_slice;
    r.rng_site_offset = rng_site_offset;
    if (r.h_lo + rng_site_offset < 0) {
        set_error("rng_site_offset %lld puts site %lld before the lattice", rng_site_offset, (long long)r.h_lo);
        return GF_ERR_INVALID;
    }
    r.a.real = real;
    r.a.U = U;
    r.a.Udw = U;
    r.a.parity = parity;
    r.a.p.param = param;
    r.a.p.seed = (uint32_t)seed;
    r.a.p.counter = (uint32_t)rng_counter;
    r.a.p.counter_stride = 0;
    r.a.stream = (cudaStream_t)stream;
    return dispatch_gauge_algo<RefStepRange>(gauge, algo, r);
}

double gf_quality_prefactor_gff(int gauge) { return prefactor_gff(gauge); }
double gf_quality_prefactor_a(int gauge) { return prefactor_a(gauge); }

int gf_stats_create(int gauge, int real, const int32_t size[4], int stopping, gf_stats **out)
{
    clear_error();
    if (!out || !valid_gauge(gauge) || !valid_real(real) || (stopping != GF_MAX && stopping != GF_AVERAGE)) {
        set_error("invalid argument to gf_stats_create");
        return GF_ERR_INVALID;
    }
    *out = nullptr;
    Geom g;
    int st = make_geom(size, gauge, true, g);
    if (st) return st;
    gf_stats *s = new (std::nothrow) gf_stats();
    if (!s) {
        set_error("host allocation failed");
        return GF_ERR_NOMEM;
    }
    s->gauge = gauge;
    s->real = real;
    s->stop_max = stopping == GF_MAX;
    s->g = g;
    s->blocks = (unsigned)((g.V + 255) / 256);
    cudaGetDevice(&s->device);
    st = cuda_status(cudaMalloc(&s->scratch, sizeof(double) * (2 * (size_t)s->blocks + 2) + 256), "cudaMalloc");
    if (st) {
        delete s;
        return st;
    }
    s->ticket = (unsigned int *)(s->scratch + 2 * (size_t)s->blocks + 2);
    st = cuda_status(cudaMemset(s->ticket, 0, sizeof(unsigned int)), "cudaMemset");
    if (st) {
        cudaFree(s->scratch);
        delete s;
        return st;
    }
    *out = s;
    return GF_OK;
}

int gf_stats_generate(gf_stats *s, const void *U, void *stream, double *gff, double *theta)
{
    clear_error();
    if (!s || !U) {
        set_error("NULL stats object or field");
        return GF_ERR_INVALID;
    }
    QualityArgs a;
    a.real = s->real;
    a.U = U;
    a.g = s->g;
    a.o.partials = s->scratch;
    a.o.result = s->scratch + 2 * (size_t)s->blocks;
    a.o.ticket = s->ticket;
    a.o.gff_site = nullptr;
    a.o.theta_site = nullptr;
    a.stop_max = s->stop_max;
    a.stream = (cudaStream_t)stream;
    int st = quality_dispatch(s->gauge, a);
    if (st) return st;
    double h[2];
    st = cuda_status(cudaMemcpyAsync(h, a.o.result, sizeof(h), cudaMemcpyDeviceToHost, a.stream), "cudaMemcpyAsync");
    if (st) return st;
    st = cuda_status(cudaStreamSynchronize(a.stream), "cudaStreamSynchronize");
    if (st) return st;
    if (gff) *gff = h[0];
    if (theta) *theta = h[1];
    return GF_OK;
}

int gf_stats_destroy(gf_stats *s)
{
    if (!s) return GF_OK;
    cudaFree(s->scratch);
    delete s;
    return GF_OK;
}

int gf_quality_per_site(int gauge, int real, const void *U, const int32_t size[4], double *dGff, double *dA,
                        void *stream)
{
    gf_stats *s = nullptr;
    int st = gf_stats_create(gauge, real, size, GF_AVERAGE, &s);
    if (st) return st;
    QualityArgs a;
    a.real = real;
    a.U = U;
    a.g = s->g;
    a.o.partials = s->scratch;
    a.o.result = s->scratch + 2 * (size_t)s->blocks;
    a.o.ticket = s->ticket;
    a.o.gff_site = dGff;
    a.o.theta_site = dA;
    a.stop_max = 0;
    a.stream = (cudaStream_t)stream;
    st = U ? quality_dispatch(gauge, a) : (set_error("field is NULL"), GF_ERR_INVALID);
    if (!st) st = cuda_status(cudaStreamSynchronize(a.stream), "cudaStreamSynchronize");
    gf_stats_destroy(s);
    return st;
}

int gf_project_su3(int real, void *U, const int32_t size[4], void *stream)
{
    clear_error();
    if (!U || !valid_real(real)) {
        set_error("invalid field or real type");
        return GF_ERR_INVALID;
    }
    Geom g;
    int st = make_geom(size, GF_COULOMB, true, g);  // accepts full lattices and timeslices
    if (st && size && size[0] != 1) st = make_geom(size, GF_LANDAU, false, g);
    if (st) return st;
    clear_error();
    const unsigned blocks = (unsigned)((4 * g.V + 255) / 256);
    if (real == GF_FP64)
        k_project_ref<double><<<blocks, 256, 0, (cudaStream_t)stream>>>(RefField<double>{(double *)U, g.V});
    else
        k_project_ref<float><<<blocks, 256, 0, (cudaStream_t)stream>>>(RefField<float>{(float *)U, g.V});
    return launch_status("project");
}

int gf_set_hot(int real, void *U, const int32_t size[4], int seed, int rng_counter, void *stream)
{
    clear_error();
    if (!U || !valid_real(real)) {
        set_error("invalid field or real type");
        return GF_ERR_INVALID;
    }
    Geom g;
    int st = make_geom(size, GF_COULOMB, true, g);
    if (st && size && size[0] != 1) st = make_geom(size, GF_LANDAU, false, g);
    if (st) return st;
    clear_error();
    const unsigned blocks = (unsigned)((g.V + 255) / 256);
    if (real == GF_FP64)
        k_set_hot_ref<double><<<blocks, 256, 0, (cudaStream_t)stream>>>(RefField<double>{(double *)U, g.V},
                                                                          (uint32_t)seed, (uint32_t)rng_counter);
    else
        k_set_hot_ref<float><<<blocks, 256, 0, (cudaStream_t)stream>>>(RefField<float>{(float *)U, g.V},
                                                                         (uint32_t)seed, (uint32_t)rng_counter);
    return launch_status("set_hot");
}

}  // extern "C"
