// gf_engine.cu -- the context-level C ABI: batched, mixed-precision gauge fixing.
//
// A context holds one or more lattices ("instances": gauge copies, uneven extents), each in the
// packed 12-real layout, FP32 and/or FP64.  gf_fix runs the reference driver's schedule
// (apps/LandauGaugeFixingSU3_4D.cu:185-271: random trafo, SA + micro, OR with reproject and
// checks, closing reprojection) for all instances at once:
//  - every parity pass is ONE launch over all instances still sweeping in that precision;
//  - a check (quality + state transition) every check_precision sweeps decides on the device
//    whether an instance switches FP32 -> FP64 (theta < switch_theta) or is done
//    (theta < precision, or out of sweeps); converged instances drop out of later launches;
//  - the OR loop is captured as a CUDA graph of one check chunk and replayed; the host only
//    reads the per-instance states (pinned memory) one chunk behind.
#include <algorithm>
#include <array>
#include <cstring>
#include <new>
#include <vector>

#include "gf_engine.cuh"
#include "gf_host.hpp"

using namespace gfb;

namespace {

bool same_check(const CheckParams &a, const CheckParams &b)
{
    return a.want_state == b.want_state && a.chunk_sweeps == b.chunk_sweeps && a.max_sweeps == b.max_sweeps &&
           a.switch_theta == b.switch_theta && a.precision == b.precision && a.stop_max == b.stop_max &&
           a.transitions == b.transitions && a.stall_checks == b.stall_checks && a.fold == b.fold &&
           a.fold_exit == b.fold_exit;
}

// what a captured check chunk depends on besides the context's buffers and launch shapes
struct ChunkKey {
    int n = 0, has32 = 0, has64 = 0, persistent = 0;
    unsigned int missing = 0;
    unsigned long long budget_ns = 0;
    float omega = 0.f;
    std::vector<unsigned char> repro;
    CheckParams base{};
    bool operator==(const ChunkKey &o) const
    {
        return n == o.n && has32 == o.has32 && has64 == o.has64 && persistent == o.persistent &&
               missing == o.missing && budget_ns == o.budget_ns && omega == o.omega && repro == o.repro &&
               same_check(base, o.base);
    }
};

}  // namespace

struct gf_ctx {
    int gauge = 0, ninst = 0, mixed = 0, device = 0;
    int refine = 0;           // mixed mode 2: FP64 master + FP32 working copy + accumulated W
    int site_w = 0;           // refine with W in a separate array (Landau, MAG, U1xU1; a Coulomb slice
                              // keeps its W in its own mu = 0 planes)
    float2 *w = nullptr;      // site_w: columns 0, 1 of W of every instance (6 float2 planes of V each)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<InstDesc> h_inst;
    InstDesc *d_inst = nullptr;
    int64_t total_warps = 0, total_links = 0, total_qblocks = 0, max_V = 0;
    float4 *f32 = nullptr;
    double2 *f64 = nullptr;
    int *d_state = nullptr, *d_sweeps = nullptr, *d_sweeps64 = nullptr, *d_storage = nullptr;
    double *d_quality = nullptr, *d_partials = nullptr;
    double *d_trace = nullptr;    // OR check trace (gf_schedule.trace_checks), else null
    int *d_ntrace = nullptr;
    int trace_cap = 0;
    unsigned int *d_tickets = nullptr;
    int *h_state = nullptr;       // pinned (state, then storage: 2 * ninst)
    int *h_chunk = nullptr;       // pinned, two slots of 2 * ninst: the states after check chunk k land in
                                  // slot k & 1 while the host reads slot (k - 1) & 1
    double *h_quality = nullptr;  // pinned
    int *h_sweeps = nullptr;      // pinned (2 * ninst: sweeps, sweeps64)
    void *staging = nullptr;
    size_t staging_bytes = 0;
    cudaEvent_t ev_chunk[2] = {nullptr, nullptr};
    mutable long long launches = 0;  // kernels this context has launched (graph nodes per replay)
    int num_sms = 148;
    uint32_t counter_stride = 0;  // Philox streams of the batch (AlgoParams::counter_stride), set by gf_fix
    // persistent chunk kernel: grid-barrier state on the device, and the {error, barrier} words of the
    // last two chunks in pinned memory
    ChunkSync *d_sync = nullptr;
    unsigned int *h_sync = nullptr;
    // check chunks captured as graphs, kept for later gf_fix calls; dropped when the launch shapes or
    // the trace buffer change (the graphs hold both)
    struct Graph {
        ChunkKey key;
        cudaGraphExec_t exec;
        long long nodes;
    };
    std::vector<Graph> graphs;
    void drop_graphs()
    {
        for (auto &g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }
    // parity-pass launch shape per precision ([0] FP32, [1] FP64): variant 0 = one warp per
    // 8-site tile, 128 threads per block; variant 1 = pipelined (cp.async prefetch of the next
    // tile), `warps` warps per block, grid = num_sms * blocks_per_sm
    struct PassShape {
        int variant = 0, warps = 4, blocks_per_sm = 0;
        int alternate = 0;  // persistent variants (1, 3, 7): walk the tiles backwards on odd parities
        int capped = 0;     // variants 1 (4 warps per block) and 7: registers capped for more resident warps
        int stages = 2;     // variant 1 with 4 warps per block: cp.async stages per warp (2 or 3)
    } shape[2];
    int tuned[2] = {0, 0};
    // the lattices the caller passed: first instance and number of instances (Coulomb contexts
    // split every lattice into its Nt timeslices; the other gauges have one instance each)
    struct Lattice {
        int first, count;
        int64_t slice_reals;  // reals of one instance's GpuPattern array (V * 72)
    };
    std::vector<Lattice> lattices;
    double2 *t64 = nullptr;   // Coulomb: original temporal links of every timeslice

    EngineDev dev() const
    {
        EngineDev e;
        e.inst = d_inst;
        e.ninst = ninst;
        e.state = d_state;
        e.sweeps = d_sweeps;
        e.sweeps64 = d_sweeps64;
        e.storage = d_storage;
        e.quality = d_quality;
        e.partials = d_partials;
        e.tickets = d_tickets;
        e.best32 = d_quality + 2 * ninst;
        e.trace = d_trace;
        e.ntrace = d_ntrace;
        e.trace_cap = trace_cap;
        e.stall = d_state + 4 * ninst;
        return e;
    }
};

namespace {

constexpr int QNT = 256;

unsigned grid_for(int64_t threads, int block) { return (unsigned)((threads + block - 1) / block); }

// ---- batched kernel dispatch -------------------------------------------------------------------
struct PassArgs {
    const gf_ctx *c;
    int parity;
    AlgoParams p;
    int want_state;
    int reverse;  // persistent passes: walk the tiles backwards
};

template <typename R, int GAUGE, int ALGO, int WARPS, int MINB = 1, int STAGES = 2>
int launch_staged(const gf_ctx *c, const EngineDev &e, const PassArgs &a, int blocks_per_sm)
{
    const size_t smem = staged_smem_bytes<R>(WARPS, STAGES);
    auto kern = k_batched_pass_staged<R, GAUGE, ALGO, WARPS, MINB, STAGES>;
    static bool smem_opt_in = false;  // above 48 KB the dynamic shared memory must be opted in
    if (!smem_opt_in) {
        int st = cuda_status(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                             "cudaFuncSetAttribute");
        if (st) return st;
        smem_opt_in = true;
    }
    int occ = blocks_per_sm;
    if (occ <= 0) {
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, WARPS * 32, smem) != cudaSuccess || o < 1) o = 1;
        occ = o;
    }
    const int64_t need = (a.c->total_warps + WARPS - 1) / WARPS;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)c->num_sms * occ));
    kern<<<blocks, WARPS * 32, smem, a.c->stream>>>(e, a.c->total_warps, a.parity, a.p, a.want_state, a.reverse);
    return launch_status("batched parity pass (pipelined)");
}

template <typename R, int GAUGE, int ALGO, bool SITE_W>
int launch_rp(const gf_ctx *c, const EngineDev &e, const PassArgs &a, int blocks_per_sm)
{
    auto kern = k_batched_pass_rp<R, GAUGE, ALGO, SITE_W>;
    static int occ_cached = 0;  // resident blocks per SM of this instantiation
    int occ = blocks_per_sm;
    if (occ <= 0) {
        if (occ_cached <= 0) {
            int o = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, 128, 0) != cudaSuccess || o < 1) o = 1;
            occ_cached = o;
        }
        occ = occ_cached;
    }
    const int64_t need = (a.c->total_warps + 3) / 4;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)c->num_sms * occ));
    kern<<<blocks, 128, 0, a.c->stream>>>(e, a.c->total_warps, a.parity, a.p, a.want_state, a.reverse);
    return launch_status("batched parity pass (register prefetch)");
}

template <int GAUGE, int ALGO, bool SITE_W>
int launch_site_staged(const gf_ctx *c, const EngineDev &e, const PassArgs &a, int blocks_per_sm)
{
    const size_t smem = SiteStage<SITE_W>::bytes;
    auto kern = k_batched_pass_site_staged<GAUGE, ALGO, SITE_W>;
    static int occ_cached = 0;  // also marks the opt-in to more than 48 KB of dynamic shared memory
    if (occ_cached == 0) {
        int st = cuda_status(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                             "cudaFuncSetAttribute");
        if (st) return st;
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, 128, smem) != cudaSuccess || o < 1) o = 1;
        occ_cached = o;
    }
    const int occ = blocks_per_sm > 0 ? blocks_per_sm : occ_cached;
    const int64_t need = (a.c->total_warps * 8 + 127) / 128;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)c->num_sms * occ));
    kern<<<blocks, 128, smem, a.c->stream>>>(e, a.c->total_warps, a.parity, a.p, a.want_state);
    return launch_status("batched parity pass (thread per site, pipelined)");
}

template <typename R, int GAUGE, int ALGO, bool SITE_W, int MINB = 1>
int launch_pair_rp(const gf_ctx *c, const EngineDev &e, const PassArgs &a, int blocks_per_sm)
{
    auto kern = k_batched_pass_pair_rp<R, GAUGE, ALGO, SITE_W, MINB>;
    static int occ_cached = 0;  // resident blocks per SM of this instantiation
    int occ = blocks_per_sm;
    if (occ <= 0) {
        if (occ_cached <= 0) {
            int o = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, 128, 0) != cudaSuccess || o < 1) o = 1;
            occ_cached = o;
        }
        occ = occ_cached;
    }
    const int64_t need = ((a.c->total_warps + 1) / 2 + 3) / 4;  // 16-site pair tiles, 4 warps per block
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)c->num_sms * occ));
    kern<<<blocks, 128, 0, a.c->stream>>>(e, a.c->total_warps, a.parity, a.p, a.want_state, a.reverse);
    return launch_status("batched parity pass (two lanes per site, register prefetch)");
}

template <typename R, int GAUGE, int ALGO>
int launch_pass(const gf_ctx *c, const EngineDev &e, const PassArgs &a, const gf_ctx::PassShape &sh)
{
    // two lanes per site: 7 = persistent with register prefetch (OR), 6 = direct (every rule, and
    // the other rules when 7 is chosen); Coulomb slices too (no W tracking: theirs rides in the
    // temporal planes)
    if constexpr (ALGO == ALG_OR && sizeof(R) == 4) {  // FP64 would spill at 255 registers
        if (sh.variant == 7) {
            if constexpr (GAUGE != COULOMB) {
                if (c->site_w) {
                    if (sh.capped) return launch_pair_rp<R, GAUGE, ALGO, true, 3>(c, e, a, sh.blocks_per_sm);
                    return launch_pair_rp<R, GAUGE, ALGO, true>(c, e, a, sh.blocks_per_sm);
                }
            }
            // capped: 168 registers, 3 blocks of 4 warps per SM instead of 2
            if (sh.capped) return launch_pair_rp<R, GAUGE, ALGO, false, 3>(c, e, a, sh.blocks_per_sm);
            return launch_pair_rp<R, GAUGE, ALGO, false>(c, e, a, sh.blocks_per_sm);
        }
    }
    if (sh.variant == 6 || sh.variant == 7) {
        const unsigned blocks = grid_for((a.c->total_warps + 1) / 2 * 32, 128);
        if constexpr (sizeof(R) == 4) {
            bool done = false;
            if constexpr (GAUGE != COULOMB) {
                if (c->site_w) {
                    k_batched_pass_pair<R, GAUGE, ALGO, true, 4><<<blocks, 128, 0, a.c->stream>>>(
                        e, a.c->total_warps, a.parity, a.p, a.want_state);
                    done = true;
                }
            }
            if (!done)
                k_batched_pass_pair<R, GAUGE, ALGO, false, 4><<<blocks, 128, 0, a.c->stream>>>(
                    e, a.c->total_warps, a.parity, a.p, a.want_state);
        } else {
            k_batched_pass_pair<R, GAUGE, ALGO, false, 2><<<blocks, 128, 0, a.c->stream>>>(
                e, a.c->total_warps, a.parity, a.p, a.want_state);
        }
        return launch_status("batched parity pass (two lanes per site)");
    }
    if constexpr (sizeof(R) == 4 && GAUGE != COULOMB && ALGO == ALG_OR) {
        if (sh.variant == 5) {
            if (c->site_w) return launch_site_staged<GAUGE, ALGO, true>(c, e, a, sh.blocks_per_sm);
            return launch_site_staged<GAUGE, ALGO, false>(c, e, a, sh.blocks_per_sm);
        }
    }
    if constexpr (sizeof(R) == 4 && GAUGE != COULOMB) {
        if (sh.variant == 4 || sh.variant == 5) {  // one thread per site (FP32); 5 = OR-only pipelined
            const unsigned blocks = grid_for(a.c->total_warps * 8, 128);
            if (c->site_w)
                k_batched_pass_site<R, GAUGE, ALGO, true, 2><<<blocks, 128, 0, a.c->stream>>>(
                    e, a.c->total_warps, a.parity, a.p, a.want_state);
            else
                k_batched_pass_site<R, GAUGE, ALGO, false, 2><<<blocks, 128, 0, a.c->stream>>>(
                    e, a.c->total_warps, a.parity, a.p, a.want_state);
            return launch_status("batched parity pass (thread per site)");
        }
    }
    if constexpr (ALGO == ALG_OR) {
        if (sh.variant == 3) {  // also Coulomb slices (their W rides in the temporal planes)
            if constexpr (sizeof(R) == 4 && GAUGE != COULOMB) {
                if (c->site_w) return launch_rp<R, GAUGE, ALGO, true>(c, e, a, sh.blocks_per_sm);
            }
            return launch_rp<R, GAUGE, ALGO, false>(c, e, a, sh.blocks_per_sm);
        }
    }
    if constexpr (ALGO == ALG_OR) {
        if (sh.variant == 1 && !(sizeof(R) == 4 && c->site_w)) {
            switch (sh.warps) {
            case 2: return launch_staged<R, GAUGE, ALGO, 2>(c, e, a, sh.blocks_per_sm);
            case 8: return launch_staged<R, GAUGE, ALGO, 8>(c, e, a, sh.blocks_per_sm);
            default:
                if (sh.stages == 3) return launch_staged<R, GAUGE, ALGO, 4, 1, 3>(c, e, a, sh.blocks_per_sm);
                if (sh.capped) return launch_staged<R, GAUGE, ALGO, 4, 4>(c, e, a, sh.blocks_per_sm);  // 128 registers
                return launch_staged<R, GAUGE, ALGO, 4>(c, e, a, sh.blocks_per_sm);
            }
        }
    }
    const unsigned blocks = grid_for(a.c->total_warps * 32, 128);
    if constexpr (sizeof(R) == 4) {
        if (c->site_w) {
            if (sh.variant == 2)
                k_batched_pass<R, GAUGE, ALGO, true, 8><<<blocks, 128, 0, a.c->stream>>>(e, a.c->total_warps,
                                                                                      a.parity, a.p, a.want_state);
            else
                k_batched_pass<R, GAUGE, ALGO, true><<<blocks, 128, 0, a.c->stream>>>(e, a.c->total_warps, a.parity,
                                                                                     a.p, a.want_state);
            return launch_status("batched parity pass (refine)");
        }
        if (sh.variant == 2) {
            k_batched_pass<R, GAUGE, ALGO, false, 8><<<blocks, 128, 0, a.c->stream>>>(e, a.c->total_warps, a.parity,
                                                                                   a.p, a.want_state);
            return launch_status("batched parity pass (64 registers)");
        }
    }
    k_batched_pass<R, GAUGE, ALGO><<<blocks, 128, 0, a.c->stream>>>(e, a.c->total_warps, a.parity, a.p,
                                                                     a.want_state);
    return launch_status("batched parity pass");
}

template <int GAUGE, int ALGO>
struct BatchedPass {
    static int run(const PassArgs &a, const EngineDev &e, const gf_ctx::PassShape *shape)
    {
        if (a.want_state == ST_FP32) return launch_pass<float, GAUGE, ALGO>(a.c, e, a, shape[0]);
        return launch_pass<double, GAUGE, ALGO>(a.c, e, a, shape[1]);
    }
};

int launch_sweep_on(const gf_ctx *c, const EngineDev &e, const gf_ctx::PassShape *shape, int algo, int want_state,
                    float param, uint32_t seed, uint32_t counter_even, uint32_t counter_odd)
{
    for (int parity = 0; parity < 2; parity++) {
        const gf_ctx::PassShape &sh = shape[want_state == ST_FP32 ? 0 : 1];
        PassArgs a{c, parity, AlgoParams{param, seed, parity ? counter_odd : counter_even, c->counter_stride},
                   want_state, sh.alternate && parity == 1};
        int st = dispatch_gauge_algo<BatchedPass>(c->gauge, algo, a, e, shape);
        if (st) return st;
        c->launches++;
    }
    return GF_OK;
}

int launch_sweep(const gf_ctx *c, int algo, int want_state, float param, uint32_t seed, uint32_t counter_even,
                 uint32_t counter_odd)
{
    return launch_sweep_on(c, c->dev(), c->shape, algo, want_state, param, seed, counter_even, counter_odd);
}

int launch_quality(const gf_ctx *c, const CheckParams &cp)
{
    const unsigned blocks = (unsigned)c->total_qblocks;
    const EngineDev e = c->dev();
#define GFB_Q(G)                                                                                  \
    if (cp.want_state == ST_FP32)                                                                 \
        k_batched_quality<G, float, QNT><<<blocks, QNT, 0, c->stream>>>(e, c->total_qblocks, cp);  \
    else                                                                                          \
        k_batched_quality<G, double, QNT><<<blocks, QNT, 0, c->stream>>>(e, c->total_qblocks, cp);
    switch (c->gauge) {
    case LANDAU: GFB_Q(LANDAU) break;
    case MAG: GFB_Q(MAG) break;
    case U1XU1: GFB_Q(U1XU1) break;
    default: GFB_Q(COULOMB) break;
    }
#undef GFB_Q
    c->launches++;
    return launch_status("batched quality");
}

int launch_reunitarise(const gf_ctx *c, int want_state, bool to64)
{
    const unsigned blocks = grid_for(c->total_links, 256);
    if (c->refine && to64) {
        // refine switch: the FP64 master takes the accumulated W (an exact gauge transformation)
        if (c->site_w) k_apply_w<<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links);
        else k_apply_w_coulomb<false><<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links);
        c->launches++;
        return launch_status("apply W");
    }
    if (c->site_w && want_state == ST_FP32) {
        k_reunitarise_w<<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links, want_state);
        c->launches++;
        int st = launch_status("reunitarise W");
        if (st) return st;
    }
    if (to64)
        k_reunitarise<float, true><<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links, want_state);
    else if (want_state == ST_FP32)
        k_reunitarise<float, false><<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links, want_state);
    else
        k_reunitarise<double, false><<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links, want_state);
    c->launches++;
    return launch_status("reunitarise");
}

int sync_states(gf_ctx *c)
{
    int st = cuda_status(cudaMemcpyAsync(c->h_state, c->d_state, sizeof(int) * 2 * c->ninst,
                                         cudaMemcpyDeviceToHost, c->stream), "state copy");
    if (st) return st;
    return cuda_status(cudaStreamSynchronize(c->stream), "stream sync");
}

int check_ctx(gf_ctx *c)
{
    if (!c) {
        set_error("context is NULL");
        return GF_ERR_INVALID;
    }
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != c->device) {
        int st = cuda_status(cudaSetDevice(c->device), "cudaSetDevice");
        if (st) return st;
    }
    return GF_OK;
}

// One OR check chunk: nsweeps sweeps of the instances sweeping in FP32 (has32) and FP64
// (has64), each followed by a reprojection where reproject_after[k] is set (the drivers reproject
// right after sweep i when i % reproject == 0, apps/LandauGaugeFixingSU3_4D.cu:249-252), then the
// checks: FP64 first, then FP32 with the switch of the instances that crossed switch_theta (so a
// switched instance is not counted twice).
struct ChunkOpts {
    int persistent;                 // 1: one cooperative launch per precision for the chunk's sweeps
    unsigned long long budget_ns;   // bound of every grid-barrier wait
    unsigned int missing;           // barrier arrivals that never come (tests of the bounded wait)
};

template <typename R, int GAUGE>
int launch_chunk_g(gf_ctx *c, int want, int nsweeps, const ChunkReproject &rp, float omega, const ChunkOpts &po)
{
    auto kern = k_chunk_sweeps<R, GAUGE>;
    static int occ_cached = 0;  // co-resident blocks per SM: a cooperative grid may not exceed them
    if (occ_cached <= 0) {
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, 128, 0) != cudaSuccess || o < 1) o = 1;
        occ_cached = o;
    }
    const int64_t need = (c->total_warps + 3) / 4;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)c->num_sms * occ_cached));
    int st = cuda_status(cudaMemsetAsync(c->d_sync, 0, sizeof(ChunkSync), c->stream), "barrier reset");
    if (st) return st;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const AlgoParams p{omega, 0u, 0u, 0u};
    st = cuda_status(cudaLaunchKernelEx(&cfg, kern, c->dev(), c->total_warps, c->total_links, nsweeps, rp, p, want,
                                        c->d_sync, blocks + po.missing, po.budget_ns),
                     "persistent chunk launch");
    c->launches++;
    return st;
}

int launch_chunk(gf_ctx *c, int want, int nsweeps, const ChunkReproject &rp, float omega, const ChunkOpts &po)
{
    const bool f32 = want == ST_FP32;
    switch (c->gauge) {
    case LANDAU: return f32 ? launch_chunk_g<float, LANDAU>(c, want, nsweeps, rp, omega, po)
                            : launch_chunk_g<double, LANDAU>(c, want, nsweeps, rp, omega, po);
    case COULOMB: return f32 ? launch_chunk_g<float, COULOMB>(c, want, nsweeps, rp, omega, po)
                             : launch_chunk_g<double, COULOMB>(c, want, nsweeps, rp, omega, po);
    case MAG: return f32 ? launch_chunk_g<float, MAG>(c, want, nsweeps, rp, omega, po)
                         : launch_chunk_g<double, MAG>(c, want, nsweeps, rp, omega, po);
    default: return f32 ? launch_chunk_g<float, U1XU1>(c, want, nsweeps, rp, omega, po)
                        : launch_chunk_g<double, U1XU1>(c, want, nsweeps, rp, omega, po);
    }
}

int enqueue_or_chunk(gf_ctx *c, int nsweeps, float omega, const std::vector<unsigned char> &reproject_after,
                     const CheckParams &base, bool has32, bool has64, const ChunkOpts &po)
{
    int st = GF_OK;
    if (po.persistent) {
        ChunkReproject rp{};
        for (int k = 0; k < nsweeps; k++)
            if (reproject_after[k]) rp.bits[k >> 6] |= 1ull << (k & 63);
        if (has32) st = launch_chunk(c, ST_FP32, nsweeps, rp, omega, po);
        if (!st && has64) st = launch_chunk(c, ST_FP64, nsweeps, rp, omega, po);
    } else {
        for (int k = 0; k < nsweeps && !st; k++) {
            if (has32) st = launch_sweep(c, ALG_OR, ST_FP32, omega, 0, 0, 0);
            if (!st && has64) st = launch_sweep(c, ALG_OR, ST_FP64, omega, 0, 0, 0);
            if (!st && reproject_after[k]) {
                if (has32) st = launch_reunitarise(c, ST_FP32, false);
                if (!st && has64) st = launch_reunitarise(c, ST_FP64, false);
            }
        }
    }
    if (st) return st;
    CheckParams cp = base;
    cp.chunk_sweeps = nsweeps;
    cp.transitions = 1;
    if (has64) {
        cp.want_state = ST_FP64;
        if ((st = launch_quality(c, cp))) return st;
    }
    if (has32) {
        cp.want_state = ST_FP32;
        if ((st = launch_quality(c, cp))) return st;
        if (c->refine && cp.fold) {
            // iterative refinement: instances now in ST_FOLD fold W into the FP64 master, restart
            // the working copy, and are checked on the master (their sweeps are already counted)
            const unsigned blocks = grid_for(c->total_links, 256);
            if (c->site_w) {
                k_reunitarise_w<<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links, ST_FOLD);
                k_fold_apply<<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links);
                k_fold_reset_w<<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links);
                c->launches += 3;
            } else {  // Coulomb slices: W32 lives in the working copy's mu = 0 planes
                k_apply_w_coulomb<true><<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links);
                k_fold_coulomb_reset<<<blocks, 256, 0, c->stream>>>(c->dev(), c->total_links);
                c->launches += 2;
            }
            if ((st = launch_status("fold"))) return st;
            CheckParams cf = cp;
            cf.want_state = ST_FOLD;
            cf.chunk_sweeps = 0;
            if ((st = launch_quality(c, cf))) return st;
        }
        if ((st = launch_reunitarise(c, ST_SWITCH, true))) return st;
        k_finish_switch<<<grid_for(c->ninst, 128), 128, 0, c->stream>>>(c->dev());
        c->launches++;
        st = launch_status("finish switch");
    }
    return st;
}

}  // namespace

extern "C" {

int gf_create(const gf_ctx_params *p, gf_ctx **out)
{
    clear_error();
    if (!p || !out || p->ninstances < 1 || !p->sizes || !valid_gauge(p->gauge)) {
        set_error("invalid gf_ctx_params");
        return GF_ERR_INVALID;
    }
    if (p->mixed < 0 || p->mixed > 2) {
        set_error("mixed must be 0, 1 or 2");
        return GF_ERR_INVALID;
    }
    *out = nullptr;
    gf_ctx *c = new (std::nothrow) gf_ctx();
    if (!c) {
        set_error("host allocation failed");
        return GF_ERR_NOMEM;
    }
    c->gauge = p->gauge;
    c->mixed = p->mixed ? 1 : 0;
    c->refine = p->mixed == 2 ? 1 : 0;
    c->site_w = c->refine && p->gauge != GF_COULOMB;
    cudaGetDevice(&c->device);
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
    const bool coulomb = p->gauge == GF_COULOMB;
    // expand the lattices into instances (Coulomb: one per timeslice, geometry {1, Nx, Ny, Nz})
    std::vector<std::array<int32_t, 4>> inst_sizes;
    std::vector<int> inst_next;
    for (int l = 0; l < p->ninstances; l++) {
        const int32_t *sz = p->sizes + 4 * l;
        const int nt = coulomb ? sz[0] : 1;
        if (coulomb && (nt < 2 || (nt & 1))) {
            set_error("Coulomb lattice %d: Nt = %d must be even and >= 2", l, nt);
            delete c;
            return GF_ERR_INVALID;
        }
        const int first = (int)inst_sizes.size();
        const int64_t vol = coulomb ? (int64_t)sz[1] * sz[2] * sz[3] : (int64_t)sz[0] * sz[1] * sz[2] * sz[3];
        c->lattices.push_back({first, nt, vol * 72});
        for (int t = 0; t < nt; t++) {
            inst_sizes.push_back(coulomb ? std::array<int32_t, 4>{1, sz[1], sz[2], sz[3]}
                                         : std::array<int32_t, 4>{sz[0], sz[1], sz[2], sz[3]});
            inst_next.push_back(coulomb ? first + (t + 1) % nt : -1);
        }
    }
    c->ninst = (int)inst_sizes.size();
    int st = GF_OK;
    int64_t voff = 0, woff = 0, loff = 0, qoff = 0, toff = 0;
    for (int i = 0; i < c->ninst && !st; i++) {
        InstDesc d{};
        st = make_geom(inst_sizes[i].data(), p->gauge, coulomb, d.g);
        d.next = inst_next[i];
        d.t64 = coulomb ? reinterpret_cast<double2 *>(toff) : nullptr;  // rebased after allocation
        d.w = reinterpret_cast<float2 *>(toff);                           // 2 columns: 6 float2 per site
        toff += 6 * d.g.V;
        d.warp_begin = woff;
        d.link_begin = loff;
        d.qblock_begin = qoff;
        d.qblocks = (d.g.V + QNT - 1) / QNT;
        // site offset: instances start on 128-byte boundaries of every plane (V is even, so
        // rounding the offset up to 8 sites keeps float4 and double2 planes aligned)
        d.f32 = reinterpret_cast<float4 *>(voff);  // rebased after allocation
        d.f64 = reinterpret_cast<double2 *>(voff);
        voff += 12 * ((d.g.V + 7) / 8 * 8);        // 4 mu x 3 float4 (or x 6 double2 -> x2)
        woff += d.g.Vh / 8;
        loff += 4 * d.g.V;
        qoff += d.qblocks;
        c->max_V = std::max(c->max_V, d.g.V);
        c->h_inst.push_back(d);
    }
    if (st) {
        delete c;
        return st;
    }
    c->total_warps = woff;
    c->total_links = loff;
    c->total_qblocks = qoff;
    const size_t n32 = (size_t)voff;   // float4 count
    const size_t n64 = (size_t)voff * 2;  // double2 count
    auto fail = [&](int s) {
        gf_destroy(c);
        return s;
    };
    if (p->stream) {
        c->stream = (cudaStream_t)p->stream;
    } else {
        if ((st = cuda_status(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate")))
            return fail(st);
        c->own_stream = true;
    }
    if (c->mixed && (st = cuda_status(cudaMalloc(&c->f32, n32 * sizeof(float4)), "cudaMalloc FP32 field")))
        return fail(st);
    if ((st = cuda_status(cudaMalloc(&c->f64, n64 * sizeof(double2)), "cudaMalloc FP64 field"))) return fail(st);
    if (coulomb && (st = cuda_status(cudaMalloc(&c->t64, (size_t)toff * sizeof(double2)), "cudaMalloc temporal links")))
        return fail(st);
    if (c->site_w && (st = cuda_status(cudaMalloc(&c->w, (size_t)toff * sizeof(float2)), "cudaMalloc W")))
        return fail(st);
    for (auto &d : c->h_inst) {
        const size_t off = (size_t)reinterpret_cast<uintptr_t>(d.f32);
        d.f32 = c->mixed ? c->f32 + off : nullptr;
        d.f64 = c->f64 + 2 * off;
        if (coulomb) d.t64 = c->t64 + (size_t)reinterpret_cast<uintptr_t>(d.t64);
        d.w = c->site_w ? c->w + (size_t)reinterpret_cast<uintptr_t>(d.w) : nullptr;
    }
    const int n = c->ninst;
    if ((st = cuda_status(cudaMalloc(&c->d_inst, sizeof(InstDesc) * n), "cudaMalloc"))) return fail(st);
    // state, storage, sweeps, sweeps64, stall
    if ((st = cuda_status(cudaMalloc(&c->d_state, sizeof(int) * 5 * n), "cudaMalloc"))) return fail(st);
    c->d_storage = c->d_state + n;
    c->d_sweeps = c->d_state + 2 * n;
    c->d_sweeps64 = c->d_state + 3 * n;
    // functional, theta, best FP32 theta
    if ((st = cuda_status(cudaMalloc(&c->d_quality, sizeof(double) * 3 * n), "cudaMalloc"))) return fail(st);
    if ((st = cuda_status(cudaMalloc(&c->d_partials, sizeof(double) * 2 * c->total_qblocks), "cudaMalloc")))
        return fail(st);
    if ((st = cuda_status(cudaMalloc(&c->d_tickets, sizeof(unsigned) * n), "cudaMalloc"))) return fail(st);
    if ((st = cuda_status(cudaHostAlloc(&c->h_state, sizeof(int) * 2 * n, cudaHostAllocDefault), "cudaHostAlloc")))
        return fail(st);
    if ((st = cuda_status(cudaHostAlloc(&c->h_quality, sizeof(double) * 2 * n, cudaHostAllocDefault),
                          "cudaHostAlloc")))
        return fail(st);
    if ((st = cuda_status(cudaHostAlloc(&c->h_sweeps, sizeof(int) * 2 * n, cudaHostAllocDefault), "cudaHostAlloc")))
        return fail(st);
    if ((st = cuda_status(cudaHostAlloc(&c->h_chunk, sizeof(int) * 4 * n, cudaHostAllocDefault), "cudaHostAlloc")))
        return fail(st);
    for (int k = 0; k < 2; k++)
        if ((st = cuda_status(cudaEventCreateWithFlags(&c->ev_chunk[k], cudaEventDisableTiming), "cudaEventCreate")))
            return fail(st);
    if ((st = cuda_status(cudaMemcpyAsync(c->d_inst, c->h_inst.data(), sizeof(InstDesc) * n, cudaMemcpyHostToDevice,
                                          c->stream), "descriptor copy")))
        return fail(st);
    std::vector<int> init(5 * n, 0);
    for (int i = 0; i < n; i++) {
        init[i] = ST_DONE;                 // nothing imported yet
        init[n + i] = c->mixed ? 0 : 1;    // storage
    }
    if ((st = cuda_status(cudaMemcpyAsync(c->d_state, init.data(), sizeof(int) * 5 * n, cudaMemcpyHostToDevice,
                                          c->stream), "state init")))
        return fail(st);
    if ((st = cuda_status(cudaMemsetAsync(c->d_tickets, 0, sizeof(unsigned) * n, c->stream), "memset"))) return fail(st);
    if ((st = cuda_status(cudaStreamSynchronize(c->stream), "sync"))) return fail(st);
    *out = c;
    return GF_OK;
}

int gf_destroy(gf_ctx *c)
{
    if (!c) return GF_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->drop_graphs();
    cudaFree(c->d_sync);
    if (c->h_sync) cudaFreeHost(c->h_sync);
    cudaFree(c->f32);
    cudaFree(c->f64);
    cudaFree(c->t64);
    cudaFree(c->w);
    cudaFree(c->d_inst);
    cudaFree(c->d_state);
    cudaFree(c->d_quality);
    cudaFree(c->d_trace);
    cudaFree(c->d_ntrace);
    cudaFree(c->d_partials);
    cudaFree(c->d_tickets);
    cudaFree(c->staging);
    if (c->h_state) cudaFreeHost(c->h_state);
    if (c->h_quality) cudaFreeHost(c->h_quality);
    if (c->h_sweeps) cudaFreeHost(c->h_sweeps);
    if (c->h_chunk) cudaFreeHost(c->h_chunk);
    for (auto &e : c->ev_chunk)
        if (e) cudaEventDestroy(e);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return GF_OK;
}

static int ensure_staging(gf_ctx *c, size_t bytes)
{
    if (c->staging_bytes >= bytes) return GF_OK;
    cudaFree(c->staging);
    c->staging = nullptr;
    c->staging_bytes = 0;
    int st = cuda_status(cudaMalloc(&c->staging, bytes), "cudaMalloc staging");
    if (!st) c->staging_bytes = bytes;
    return st;
}

// Import lattice `lat` (GpuPattern; for Coulomb the GpuPatternTimeslice array of Nt slices,
// apps/CoulombGaugeFixingSU3_4D.cu:57-59,132-134) into its instances and reset their state.
int gf_import(gf_ctx *c, int lat, int real, const void *U, int on_host)
{
    clear_error();
    int st = check_ctx(c);
    if (st) return st;
    if (lat < 0 || lat >= (int)c->lattices.size() || !U || !valid_real(real)) {
        set_error("invalid lattice index, field or real type");
        return GF_ERR_INVALID;
    }
    const gf_ctx::Lattice &L = c->lattices[lat];
    const size_t es = real == GF_FP64 ? 8 : 4;
    const char *src = (const char *)U;
    if (on_host) {
        // only the 12 planes of rows 0,1 of every mu travel (GpuPattern keeps them contiguous)
        if ((st = ensure_staging(c, (size_t)L.slice_reals * L.count * es))) return st;
        for (int t = 0; t < L.count; t++) {
            const int64_t V = c->h_inst[L.first + t].g.V;
            for (int mu = 0; mu < 4; mu++) {
                const size_t off = ((size_t)t * L.slice_reals + (size_t)mu * 18 * V) * es;
                if ((st = cuda_status(cudaMemcpyAsync((char *)c->staging + off, (const char *)U + off, 12 * V * es,
                                                      cudaMemcpyHostToDevice, c->stream), "H2D")))
                    return st;
            }
        }
        src = (const char *)c->staging;
    }
    const int target = c->mixed ? ST_FP32 : ST_FP64;
    for (int t = 0; t < L.count; t++) {
        const int i = L.first + t;
        const InstDesc &d = c->h_inst[i];
        const unsigned blocks = grid_for(4 * d.g.V, 256);
        const void *sp = src + (size_t)t * L.slice_reals * es;
        if (c->site_w) {
            if (real == GF_FP64) k_import_refine<double><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (const double *)sp);
            else k_import_refine<float><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (const float *)sp);
        } else if (c->refine) {
            // Coulomb slice: FP64 master and FP32 working copy, each with W = 1 in its mu = 0 planes
            if (real == GF_FP64) {
                k_import<double, double><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (const double *)sp);
                k_import<double, float><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (const double *)sp);
            } else {
                k_import<float, double><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (const float *)sp);
                k_import<float, float><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (const float *)sp);
            }
            c->launches++;
        } else if (target == ST_FP32) {
            if (real == GF_FP64) k_import<double, float><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (const double *)sp);
            else k_import<float, float><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (const float *)sp);
        } else {
            if (real == GF_FP64) k_import<double, double><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (const double *)sp);
            else k_import<float, double><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (const float *)sp);
        }
        c->launches++;
        if ((st = launch_status("import"))) return st;
    }
    const int n = L.count;
    std::vector<int> states(n, target), stor(n, target == ST_FP32 ? 0 : 1), zeros(n, 0);
    if ((st = cuda_status(cudaMemcpyAsync(c->d_state + L.first, states.data(), sizeof(int) * n,
                                          cudaMemcpyHostToDevice, c->stream), "state")) ||
        (st = cuda_status(cudaMemcpyAsync(c->d_storage + L.first, stor.data(), sizeof(int) * n,
                                          cudaMemcpyHostToDevice, c->stream), "storage")) ||
        (st = cuda_status(cudaMemcpyAsync(c->d_sweeps + L.first, zeros.data(), sizeof(int) * n,
                                          cudaMemcpyHostToDevice, c->stream), "sweeps")) ||
        (st = cuda_status(cudaMemcpyAsync(c->d_sweeps64 + L.first, zeros.data(), sizeof(int) * n,
                                          cudaMemcpyHostToDevice, c->stream), "sweeps")))
        return st;
    return cuda_status(cudaStreamSynchronize(c->stream), "import sync");
}

// Export lattice `lat`, reunitarised in FP64 with row 2 rebuilt; Coulomb lattices get their
// temporal links transformed by the accumulated W of slices t and t+1.
int gf_export(gf_ctx *c, int lat, int real, void *U, int on_host)
{
    clear_error();
    int st = check_ctx(c);
    if (st) return st;
    if (lat < 0 || lat >= (int)c->lattices.size() || !U || !valid_real(real)) {
        set_error("invalid lattice index, field or real type");
        return GF_ERR_INVALID;
    }
    const gf_ctx::Lattice &L = c->lattices[lat];
    const size_t es = real == GF_FP64 ? 8 : 4;
    if ((st = sync_states(c))) return st;
    char *dst = (char *)U;
    if (on_host) {
        if ((st = ensure_staging(c, (size_t)L.slice_reals * L.count * es))) return st;
        dst = (char *)c->staging;
    }
    for (int t = 0; t < L.count; t++) {
        const int i = L.first + t;
        const InstDesc &d = c->h_inst[i];
        const unsigned blocks = grid_for(4 * d.g.V, 256);
        void *dp = dst + (size_t)t * L.slice_reals * es;
        if (c->gauge == GF_COULOMB) {
            if (real == GF_FP64)
                k_export_coulomb<double><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (double *)dp, c->refine, -1);
            else
                k_export_coulomb<float><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (float *)dp, c->refine, -1);
        } else if (c->h_state[c->ninst + i] == 0 && c->refine) {
            if (real == GF_FP64) k_export_refine<double><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (double *)dp);
            else k_export_refine<float><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (float *)dp);
        } else if (c->h_state[c->ninst + i] == 0) {
            if (real == GF_FP64) k_export<float, double><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (double *)dp);
            else k_export<float, float><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (float *)dp);
        } else {
            if (real == GF_FP64) k_export<double, double><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (double *)dp);
            else k_export<double, float><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (float *)dp);
        }
        c->launches++;
        if ((st = launch_status("export"))) return st;
    }
    if (on_host && (st = cuda_status(cudaMemcpyAsync(U, dst, (size_t)L.slice_reals * L.count * es,
                                                     cudaMemcpyDeviceToHost, c->stream), "D2H")))
        return st;
    return cuda_status(cudaStreamSynchronize(c->stream), "export sync");
}

// Coulomb gauge copies: export one lattice made of the timeslices of several copies -- slice t from
// lattice copy_of_slice[t] -- as the Coulomb app keeps the best copy of every timeslice
// (apps/CoulombGaugeFixingSU3_4D.cu:303-311).  Spatial links of slice t are copy a_t's; the temporal
// links are W_{a_t}(t) U_0(t) W_{a_{t+1}}(t+1)^dagger, which is what the app's slice-by-slice
// multiplications produce when slice t's best copy is a_t.  Every lattice must have the extents
// of the first; the copies must have been imported from the same configuration.
int gf_export_slices(gf_ctx *c, const int *copy_of_slice, int real, void *U, int on_host)
{
    clear_error();
    int st = check_ctx(c);
    if (st) return st;
    if (c->gauge != GF_COULOMB || !copy_of_slice || !U || !valid_real(real)) {
        set_error("gf_export_slices: a GF_COULOMB context, a slice-to-copy table and a field are needed");
        return GF_ERR_INVALID;
    }
    const gf_ctx::Lattice &L0 = c->lattices[0];
    const int nt = L0.count;
    for (int t = 0; t < nt; t++) {
        const int a = copy_of_slice[t];
        if (a < 0 || a >= (int)c->lattices.size() || c->lattices[a].count != nt ||
            c->lattices[a].slice_reals != L0.slice_reals ||
            std::memcmp(c->h_inst[c->lattices[a].first].g.n, c->h_inst[L0.first].g.n, sizeof(int32_t) * 4) != 0) {
            set_error("gf_export_slices: slice %d names copy %d, which is not a lattice of the same extents", t, a);
            return GF_ERR_INVALID;
        }
    }
    const size_t es = real == GF_FP64 ? 8 : 4;
    if ((st = sync_states(c))) return st;
    char *dst = (char *)U;
    if (on_host) {
        if ((st = ensure_staging(c, (size_t)L0.slice_reals * nt * es))) return st;
        dst = (char *)c->staging;
    }
    for (int t = 0; t < nt; t++) {
        const int i = c->lattices[copy_of_slice[t]].first + t;
        const int next = c->lattices[copy_of_slice[(t + 1) % nt]].first + (t + 1) % nt;
        const unsigned blocks = grid_for(4 * c->h_inst[i].g.V, 256);
        void *dp = dst + (size_t)t * L0.slice_reals * es;
        if (real == GF_FP64)
            k_export_coulomb<double><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (double *)dp, c->refine, next);
        else
            k_export_coulomb<float><<<blocks, 256, 0, c->stream>>>(c->dev(), i, (float *)dp, c->refine, next);
        c->launches++;
        if ((st = launch_status("export slices"))) return st;
    }
    if (on_host && (st = cuda_status(cudaMemcpyAsync(U, dst, (size_t)L0.slice_reals * nt * es, cudaMemcpyDeviceToHost,
                                                     c->stream), "D2H")))
        return st;
    return cuda_status(cudaStreamSynchronize(c->stream), "export sync");
}

}  // extern "C"

namespace {

// which precisions the instances sweep in, from the host copy of the states
void present_states(const gf_ctx *c, bool &has32, bool &has64)
{
    has32 = has64 = false;
    for (int i = 0; i < c->ninst; i++) {
        has32 |= c->h_state[i] == ST_FP32;
        has64 |= c->h_state[i] == ST_FP64;
    }
}

int sweeps_on(gf_ctx *c, int algo, int nsweeps, float param, int seed, int rng_counter, bool has32, bool has64)
{
    int st = GF_OK;
    uint32_t ctr = (uint32_t)rng_counter;
    for (int k = 0; k < nsweeps && !st; k++) {
        // the reference takes a fresh Philox counter per launch (PhiloxWrapper::getNextCounter)
        if (c->mixed && has32) st = launch_sweep(c, algo, ST_FP32, param, (uint32_t)seed, ctr, ctr + 1);
        if (!st && has64) st = launch_sweep(c, algo, ST_FP64, param, (uint32_t)seed, ctr, ctr + 1);
        ctr += 2;
    }
    return st;
}

}  // namespace

extern "C" {

int gf_sweeps(gf_ctx *c, int algo, int nsweeps, float param, int seed, int rng_counter)
{
    clear_error();
    int st = check_ctx(c);
    if (st) return st;
    if (algo < ALG_OR || algo > ALG_RANDOM || nsweeps < 0) {
        set_error("invalid algorithm %d or sweep count %d", algo, nsweeps);
        return GF_ERR_INVALID;
    }
    // launch only the precisions some instance is sweeping in (an empty pass still costs a grid)
    if ((st = sync_states(c))) return st;
    bool has32, has64;
    present_states(c, has32, has64);
    return sweeps_on(c, algo, nsweeps, param, seed, rng_counter, has32, has64);
}

int gf_reunitarize(gf_ctx *c)
{
    clear_error();
    int st = check_ctx(c);
    if (st) return st;
    if (c->mixed && (st = launch_reunitarise(c, ST_FP32, false))) return st;
    return launch_reunitarise(c, ST_FP64, false);
}

int gf_quality_all(gf_ctx *c, double *gff, double *theta)
{
    clear_error();
    int st = check_ctx(c);
    if (st) return st;
    CheckParams cp{};
    cp.stop_max = 0;
    cp.transitions = 0;
    if (c->mixed) {
        cp.want_state = ST_FP32;
        if ((st = launch_quality(c, cp))) return st;
    }
    cp.want_state = ST_FP64;
    if ((st = launch_quality(c, cp))) return st;
    if ((st = cuda_status(cudaMemcpyAsync(c->h_quality, c->d_quality, sizeof(double) * 2 * c->ninst,
                                          cudaMemcpyDeviceToHost, c->stream), "quality copy")))
        return st;
    if ((st = cuda_status(cudaStreamSynchronize(c->stream), "sync"))) return st;
    for (int i = 0; i < c->ninst; i++) {
        if (gff) gff[i] = c->h_quality[2 * i];
        if (theta) theta[i] = c->h_quality[2 * i + 1];
    }
    return GF_OK;
}

int gf_set_storage(gf_ctx *c, int real)
{
    clear_error();
    int st = check_ctx(c);
    if (st) return st;
    if (!valid_real(real) || (real == GF_FP32 && !c->mixed)) {
        set_error("FP32 storage needs a mixed context");
        return GF_ERR_INVALID;
    }
    if (real == GF_FP64 && c->mixed) {
        // FP32 -> FP64 with FP64 reunitarisation, as the mixed schedule does at the switch
        std::vector<int> sw(c->ninst);
        if ((st = sync_states(c))) return st;
        for (int i = 0; i < c->ninst; i++) sw[i] = c->h_state[c->ninst + i] == 0 ? ST_SWITCH : c->h_state[i];
        if ((st = cuda_status(cudaMemcpyAsync(c->d_state, sw.data(), sizeof(int) * c->ninst, cudaMemcpyHostToDevice,
                                              c->stream), "state")))
            return st;
        if ((st = launch_reunitarise(c, ST_SWITCH, true))) return st;
        k_finish_switch<<<grid_for(c->ninst, 128), 128, 0, c->stream>>>(c->dev());
        if ((st = launch_status("finish switch"))) return st;
        return sync_states(c);
    }
    return GF_OK;  // FP32 request on a mixed context: instances start in FP32 at import
}

namespace {

// the {error, barrier} words a persistent chunk left in slot `slot`
int chunk_timeout(gf_ctx *c, int slot, const ChunkOpts &po)
{
    if (!c->h_sync[2 * slot]) return GF_OK;
    set_error("persistent chunk kernel: a grid-barrier wait ran out of its %llu ns budget at barrier %u",
              (unsigned long long)po.budget_ns, c->h_sync[2 * slot + 1]);
    return GF_ERR_TIMEOUT;
}

}  // namespace

int gf_fix(gf_ctx *c, const gf_schedule *s, gf_report *rep)
{
    clear_error();
    int st = check_ctx(c);
    if (st) return st;
    if (!s || s->check_precision < 1 || s->reproject < 1 || s->or_max_iter < 0 || s->sa_steps < 0) {
        set_error("invalid schedule");
        return GF_ERR_INVALID;
    }
    if (s->autotune && (!c->tuned[1] || (c->mixed && !c->tuned[0])) && (st = gf_autotune(c, nullptr, nullptr)))
        return st;
    uint32_t ctr = s->rng_counter;
    // the SA temperatures.  sa_mode 0: the Landau/Coulomb apps' linear schedule
    // (apps/LandauGaugeFixingSU3_4D.cu:212-234); 1: geometric; 2: the MAG / U1xU1 apps' do-while, step
    // (max-min)/steps divided by sa_slow_factor inside [sa_slow_lo, sa_slow_hi] (the float temperature
    // compared with the double bounds, apps/MAGaugeFixingSU3_4D.cu:233-266).
    std::vector<float> temps;
    const int mode = s->sa_mode ? s->sa_mode : (s->sa_geometric ? 1 : 0);
    if (s->sa_steps > 0 && mode == 2) {
        float T = s->sa_max;
        const float base_step = (s->sa_max - s->sa_min) / (float)s->sa_steps;
        const float slow = s->sa_slow_factor > 0 ? s->sa_slow_factor : 1.f;
        do {
            const float step = ((double)T <= s->sa_slow_hi && (double)T >= s->sa_slow_lo) ? base_step / slow : base_step;
            temps.push_back(T);
            T -= step;
        } while (T >= s->sa_min && (int)temps.size() < 100 * s->sa_steps);
    } else if (s->sa_steps > 0) {
        float T = s->sa_max;
        const float dT = (s->sa_max - s->sa_min) / (float)s->sa_steps;
        const double ratio = s->sa_steps > 1 ? pow((double)s->sa_min / s->sa_max, 1.0 / (s->sa_steps - 1)) : 1.0;
        for (int i = 0; i < s->sa_steps; i++) {
            temps.push_back(mode == 1 ? (float)(s->sa_max * pow(ratio, (double)i)) : T);
            T -= dT;
        }
    }
    // Philox streams: rng_streams = 1 continues one stream through the instances, the way the apps
    // fix copies / timeslices one after the other -- instance i starts where instance i - 1's
    // random trafo and SA sweeps (two launch counters each) end.  That count must be known before
    // the run, so SR (whose length depends on convergence) is excluded.
    struct StreamGuard {
        gf_ctx *c;
        ~StreamGuard() { c->counter_stride = 0; }
    } stream_guard{c};
    if (s->rng_streams == 1) {
        if (s->sr_max_iter > 0) {
            set_error("rng_streams = 1 needs a schedule without SR (its length depends on convergence)");
            return GF_ERR_INVALID;
        }
        const int repeat_ = s->sa_repeat > 0 ? s->sa_repeat : 1;
        c->counter_stride = (uint32_t)(2 * (s->random_trafo ? 1 : 0) + 2 * repeat_ * (int)temps.size());
        if (c->counter_stride == 0) c->counter_stride = 1;  // nothing random: any non-zero stride
    } else if (s->rng_streams != 0) {
        set_error("rng_streams must be 0 or 1");
        return GF_ERR_INVALID;
    }
    // the precisions the instances sweep in before the OR phase (set by gf_import)
    if ((st = sync_states(c))) return st;
    bool pre32, pre64;
    present_states(c, pre32, pre64);
    auto gf_sweeps = [&](gf_ctx *cc, int algo, int n, float param, int seed, int counter) {
        return sweeps_on(cc, algo, n, param, seed, counter, pre32, pre64);
    };
    // random gauge transformation of every instance (apps/LandauGaugeFixingSU3_4D.cu:192-196)
    if (s->random_trafo) {
        if ((st = gf_sweeps(c, ALG_RANDOM, 1, 0.f, (int)s->seed, (int)ctr))) return st;
        ctr += 2;
    }
    // simulated annealing with microcanonical steps: every temperature runs sa_repeat SA sweeps,
    // each followed (every micro_every-th) by micro_updates microcanonical sweeps.
    int sa_done = 0;
    const int every = s->micro_every > 0 ? s->micro_every : 1;
    const int repeat = s->sa_repeat > 0 ? s->sa_repeat : 1;
    auto sa_temperature = [&](float T, int i) -> int {
        for (int r = 0; r < repeat; r++) {
            int q = gf_sweeps(c, ALG_SA, 1, T, (int)s->seed, (int)ctr);
            if (q) return q;
            ctr += 2;
            if (s->micro_updates > 0 && (sa_done % every) == every - 1 &&
                (q = gf_sweeps(c, ALG_MICRO, s->micro_updates, 0.f, 0, 0)))
                return q;
            sa_done++;
        }
        if (i % s->reproject == 0) return gf_reunitarize(c);
        return GF_OK;
    };
    for (size_t i = 0; i < temps.size(); i++)
        if ((st = sa_temperature(temps[i], (int)i))) return st;
    // stochastic relaxation (the MAG app, apps/MAGaugeFixingSU3_4D.cu:278-297): SR sweeps until
    // every instance has theta < max(precision, sr_stop_theta), checked every checkprecision sweeps
    int sr_done = 0;
    if (s->sr_max_iter > 0) {
        std::vector<double> th(c->ninst);
        for (int i = 0; i < s->sr_max_iter; i++) {
            if ((st = gf_sweeps(c, ALG_SR, 1, s->sr_parameter, (int)s->seed, (int)ctr))) return st;
            ctr += 2;
            sr_done++;
            if (i % s->reproject == 0 && (st = gf_reunitarize(c))) return st;
            if (i % s->check_precision == 0) {
                if ((st = gf_quality_all(c, nullptr, th.data()))) return st;
                bool all = true;
                for (double t : th) all &= (t < s->precision || t < s->sr_stop_theta);
                if (all) break;
            }
        }
    }
    // overrelaxation to theta < precision (:244-262).  The reference checks after sweep i when
    // i % checkprecision == 0 (i = 0, C, 2C, ...) and reprojects when i % reproject == 0, so the
    // first chunk is one sweep and the later ones C sweeps.  Every chunk shape is captured once
    // as a CUDA graph and replayed; the host reads the states of chunk k-1 while chunk k runs.
    CheckParams base{};
    base.max_sweeps = s->or_max_iter;
    base.switch_theta = c->mixed ? s->switch_theta : -1.0;
    base.precision = s->precision;
    base.stop_max = 0;
    base.stall_checks = s->stall_checks;
    base.fold = c->refine ? s->fold : 0;
    base.fold_exit = s->fold_exit > 0 ? s->fold_exit : 0.0;
    {
        std::vector<int> zeros(2 * c->ninst, 0);
        if ((st = cuda_status(cudaMemcpyAsync(c->d_sweeps, zeros.data(), sizeof(int) * 2 * c->ninst,
                                              cudaMemcpyHostToDevice, c->stream), "sweeps reset")))
            return st;
    }
    // optional check trace: (re)allocated for this run's capacity, or switched off
    if (s->trace_checks > 0 && s->trace_checks != c->trace_cap) {
        c->drop_graphs();
        cudaFree(c->d_trace);
        cudaFree(c->d_ntrace);
        c->d_trace = nullptr;
        c->d_ntrace = nullptr;
        c->trace_cap = 0;
        if ((st = cuda_status(cudaMalloc(&c->d_trace, sizeof(double) * 4 * (size_t)s->trace_checks * c->ninst),
                              "cudaMalloc trace")) ||
            (st = cuda_status(cudaMalloc(&c->d_ntrace, sizeof(int) * c->ninst), "cudaMalloc trace")))
            return st;
        c->trace_cap = s->trace_checks;
    } else if (s->trace_checks <= 0 && c->trace_cap) {
        c->drop_graphs();
        cudaFree(c->d_trace);
        cudaFree(c->d_ntrace);
        c->d_trace = nullptr;
        c->d_ntrace = nullptr;
        c->trace_cap = 0;
    }
    if (c->trace_cap && (st = cuda_status(cudaMemsetAsync(c->d_ntrace, 0, sizeof(int) * c->ninst, c->stream),
                                          "trace reset")))
        return st;
    if ((st = sync_states(c))) return st;
    const int C = s->check_precision;
    // one persistent launch per check chunk (schedule.persistent): not for contexts with the separate
    // W array, and at most 256 sweeps per chunk (the reprojection mask)
    ChunkOpts po{s->persistent ? 1 : 0, 1000000000ull, 0u};
    if (po.persistent) {
        if (c->site_w || C > 256 || s->wait_test_missing < 0) {
            set_error("persistent chunks need a context without the separate W array (plain FP64, FP32 storage or "
                      "Coulomb) and check_precision <= 256");
            return GF_ERR_UNSUPPORTED;
        }
        if (s->wait_budget_us > 0) po.budget_ns = 1000ull * (unsigned long long)s->wait_budget_us;
        po.missing = (unsigned int)s->wait_test_missing;
        if (!c->d_sync && (st = cuda_status(cudaMalloc(&c->d_sync, sizeof(ChunkSync)), "cudaMalloc barrier")))
            return st;
        if (!c->h_sync && (st = cuda_status(cudaHostAlloc(&c->h_sync, sizeof(unsigned int) * 4, cudaHostAllocDefault),
                                            "cudaHostAlloc")))
            return st;
        c->h_sync[0] = c->h_sync[2] = 0;
    }
    auto get_graph = [&](int n, const std::vector<unsigned char> &repro, int h32, int h64,
                         cudaGraphExec_t &out) -> int {
        ChunkKey key;
        key.n = n;
        key.has32 = h32;
        key.has64 = h64;
        key.persistent = po.persistent;
        key.missing = po.missing;
        key.budget_ns = po.budget_ns;
        key.omega = s->or_parameter;
        key.repro = repro;
        key.base = base;
        for (auto &v : c->graphs)
            if (v.key == key) {
                out = v.exec;
                c->launches += v.nodes;
                return GF_OK;
            }
        cudaGraph_t g = nullptr;
        int r = cuda_status(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        if (r) return r;
        const long long before = c->launches;
        r = enqueue_or_chunk(c, n, s->or_parameter, repro, base, h32, h64, po);
        const long long nodes = c->launches - before;
        const int r2 = cuda_status(cudaStreamEndCapture(c->stream, &g), "end capture");
        if (r || r2) {
            if (g) cudaGraphDestroy(g);
            return r ? r : r2;
        }
        cudaGraphExec_t ex = nullptr;
        r = cuda_status(cudaGraphInstantiate(&ex, g, 0), "graph instantiate");
        cudaGraphDestroy(g);
        if (r) return r;
        c->graphs.push_back(gf_ctx::Graph{key, ex, nodes});
        out = ex;
        return GF_OK;
    };
    auto scan = [&](const int *states, bool &any, bool &h32, bool &h64) {
        any = h32 = h64 = false;
        for (int i = 0; i < c->ninst; i++) {
            const int q = states[i];
            any |= q != ST_DONE;
            h32 |= q == ST_FP32;
            h64 |= q == ST_FP64 || q == ST_SWITCH;
        }
    };
    bool any_active, has32, has64;
    scan(c->h_state, any_active, has32, has64);
    int issued = 0, launched = 0;
    for (int k = 0; any_active && issued < s->or_max_iter && !st; k++) {
        const int n = k == 0 ? 1 : std::min(C, s->or_max_iter - issued);
        std::vector<unsigned char> repro(n);
        for (int k2 = 0; k2 < n; k2++) repro[k2] = ((issued + k2) % s->reproject) == 0;
        if (s->use_graphs) {
            cudaGraphExec_t ex = nullptr;
            if ((st = get_graph(n, repro, has32, has64, ex))) break;
            if ((st = cuda_status(cudaGraphLaunch(ex, c->stream), "graph launch"))) break;
        } else if ((st = enqueue_or_chunk(c, n, s->or_parameter, repro, base, has32, has64, po))) {
            break;
        }
        issued += n;
        if (po.persistent && (st = cuda_status(cudaMemcpyAsync(c->h_sync + 2 * (k & 1), &c->d_sync->error,
                                                               2 * sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                                               c->stream), "barrier status copy")))
            break;
        if ((st = cuda_status(cudaMemcpyAsync(c->h_chunk + (k & 1) * 2 * c->ninst, c->d_state,
                                              sizeof(int) * 2 * c->ninst, cudaMemcpyDeviceToHost, c->stream),
                              "state copy")))
            break;
        if ((st = cuda_status(cudaEventRecord(c->ev_chunk[k & 1], c->stream), "event"))) break;
        launched++;
        if (k >= 1) {
            // slot (k-1) & 1 holds the complete copy of chunk k-1 once its event has fired; chunk k's
            // copy lands in the other slot and is read in the next iteration
            if ((st = cuda_status(cudaEventSynchronize(c->ev_chunk[(k - 1) & 1]), "event sync"))) break;
            if (po.persistent && (st = chunk_timeout(c, (k - 1) & 1, po))) break;
            bool a2, h32b, h64b;
            scan(c->h_chunk + ((k - 1) & 1) * 2 * c->ninst, a2, h32b, h64b);
            any_active = a2;
            has32 = h32b;
            // an instance that switches to FP64 during chunk k is seen here after chunk k+1 was
            // launched without FP64 passes: it idles for that chunk and is not counted for it
            has64 = h64b;
        }
    }
    if (st) {
        cudaStreamSynchronize(c->stream);
        return st;
    }
    if ((st = cuda_status(cudaStreamSynchronize(c->stream), "sync"))) return st;
    if (po.persistent && launched > 0 && (st = chunk_timeout(c, (launched - 1) & 1, po))) return st;
    if (rep) {
        if ((st = cuda_status(cudaMemcpy(c->h_quality, c->d_quality, sizeof(double) * 2 * c->ninst,
                                         cudaMemcpyDeviceToHost), "quality copy")))
            return st;
        if ((st = cuda_status(cudaMemcpy(c->h_sweeps, c->d_sweeps, sizeof(int) * 2 * c->ninst, cudaMemcpyDeviceToHost),
                              "sweeps copy")))
            return st;
        if ((st = sync_states(c))) return st;
        for (int i = 0; i < c->ninst; i++) {
            rep[i].gff = c->h_quality[2 * i];
            rep[i].theta = c->h_quality[2 * i + 1];
            rep[i].or_sweeps = c->h_sweeps[i];
            rep[i].or_sweeps_fp64 = c->h_sweeps[c->ninst + i];
            rep[i].sa_sweeps = sa_done;
            rep[i].sr_sweeps = sr_done;
            rep[i].converged = rep[i].theta < s->precision;
            rep[i].chunks = launched;
        }
    }
    return GF_OK;
}

// Project-written autotuner: times every candidate launch shape of the OR parity pass on a scratch
// copy of the context's field (the field itself is not touched; the pass's memory access pattern
// does not depend on the link values) and keeps the fastest one per precision.
int gf_autotune(gf_ctx *c, int *choice_fp32, int *choice_fp64)
{
    clear_error();
    int st = check_ctx(c);
    if (st) return st;
    // direct; register prefetch (persistent); two lanes per site (direct, and persistent with register
    // prefetch); pipelined with 2, 4, 8 warps per block; (FP32 only) direct capped at 64 registers and
    // one thread per site (plain and pipelined).  Coulomb passes are direct, register prefetch or two lanes per site; refine-FP32 passes
    // (W tracking) are not the 4-lane pipelined one.
    static const gf_ctx::PassShape cands64[] = {{0, 4, 0, 0, 0}, {3, 4, 0, 0, 0}, {6, 4, 0, 0, 0},    {1, 4, 0, 1, 0},
                                                {1, 8, 0, 1, 0}, {1, 4, 0, 1, 1}, {3, 4, 0, 1, 0},    {1, 2, 0, 0, 0},
                                                {1, 4, 0, 0, 0}, {1, 8, 0, 0, 0}, {1, 4, 0, 1, 0, 3}, {1, 4, 0, 0, 0, 3}};
    static const gf_ctx::PassShape cands32[] = {{0, 4, 0, 0, 0}, {2, 4, 0, 0, 0}, {3, 4, 0, 0, 0}, {4, 4, 0, 0, 0},
                                                {5, 4, 0, 0, 0}, {6, 4, 0, 0, 0}, {7, 4, 0, 0, 0}, {7, 4, 0, 1, 0},
                                                {7, 4, 0, 1, 1}, {3, 4, 0, 1, 0}, {1, 2, 0, 0, 0}, {1, 4, 0, 0, 0},
                                                {1, 8, 0, 0, 0}};
    // Coulomb slices: direct; register prefetch with and without the alternating walk; two lanes per
    // site (direct, register prefetch with the alternating walk, the same register-capped; the
    // prefetching ones FP32 only, in FP64 they run as the direct one)
    static const gf_ctx::PassShape candsC[] = {{0, 4, 0, 0, 0}, {3, 4, 0, 0, 0}, {3, 4, 0, 1, 0},
                                               {6, 4, 0, 0, 0}, {7, 4, 0, 1, 0}, {7, 4, 0, 1, 1}};
    for (int prec = 0; prec < 2; prec++) {
        if (prec == 0 && !c->mixed) continue;
        const gf_ctx::PassShape *cands = c->gauge == GF_COULOMB ? candsC : prec == 0 ? cands32 : cands64;
        int ncand = prec == 0 ? 13 : 12;
        if (c->gauge == GF_COULOMB) ncand = prec == 0 ? 6 : 4;
        else if (prec == 0 && c->site_w) ncand = 10;
        // scratch field, descriptors and states for this precision
        const InstDesc &last = c->h_inst.back();
        const size_t span32 = (size_t)(reinterpret_cast<const char *>(last.f32 ? last.f32 : (float4 *)nullptr) -
                                       reinterpret_cast<const char *>(c->f32 ? c->f32 : (float4 *)nullptr)) +
                              (size_t)12 * last.g.V * sizeof(float4);
        // an instance holds 4 mu x 3 float4 planes (FP32) or 4 mu x 6 double2 planes (FP64) of V
        const size_t span64 = (size_t)(reinterpret_cast<const char *>(last.f64) - reinterpret_cast<const char *>(c->f64)) +
                              (size_t)24 * last.g.V * sizeof(double2);
        const size_t span = prec == 0 ? span32 : span64;
        void *scratch = nullptr;
        float2 *wscratch = nullptr;  // refine: the passes also update W, which must not be touched
        InstDesc *dinst = nullptr;
        int *dstate = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        auto cleanup = [&]() {
            cudaFree(scratch);
            cudaFree(wscratch);
            cudaFree(dinst);
            cudaFree(dstate);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        };
        if ((st = cuda_status(cudaMalloc(&scratch, span), "autotune scratch"))) {
            cleanup();
            return st;
        }
        const void *src = prec == 0 ? (const void *)c->f32 : (const void *)c->f64;
        cudaMemcpyAsync(scratch, src, span, cudaMemcpyDeviceToDevice, c->stream);
        std::vector<InstDesc> hi = c->h_inst;
        if (prec == 0 && c->site_w) {
            const size_t spanw = (size_t)(last.w - c->w) + (size_t)6 * last.g.V;  // float2 count
            if ((st = cuda_status(cudaMalloc(&wscratch, spanw * sizeof(float2)), "autotune W scratch"))) {
                cleanup();
                return st;
            }
            cudaMemcpyAsync(wscratch, c->w, spanw * sizeof(float2), cudaMemcpyDeviceToDevice, c->stream);
            for (auto &d : hi) d.w = wscratch + (d.w - c->w);
        }
        for (auto &d : hi) {
            if (prec == 0)
                d.f32 = reinterpret_cast<float4 *>((char *)scratch + ((char *)d.f32 - (char *)c->f32));
            else
                d.f64 = reinterpret_cast<double2 *>((char *)scratch + ((char *)d.f64 - (char *)c->f64));
        }
        std::vector<int> hs(c->ninst, prec == 0 ? ST_FP32 : ST_FP64);
        if ((st = cuda_status(cudaMalloc(&dinst, sizeof(InstDesc) * c->ninst), "cudaMalloc")) ||
            (st = cuda_status(cudaMalloc(&dstate, sizeof(int) * c->ninst), "cudaMalloc")) ||
            (st = cuda_status(cudaMemcpyAsync(dinst, hi.data(), sizeof(InstDesc) * c->ninst, cudaMemcpyHostToDevice,
                                              c->stream), "copy")) ||
            (st = cuda_status(cudaMemcpyAsync(dstate, hs.data(), sizeof(int) * c->ninst, cudaMemcpyHostToDevice,
                                              c->stream), "copy")) ||
            (st = cuda_status(cudaEventCreate(&e0), "event")) || (st = cuda_status(cudaEventCreate(&e1), "event"))) {
            cleanup();
            return st;
        }
        EngineDev e = c->dev();
        e.inst = dinst;
        e.state = dstate;
        const int want = prec == 0 ? ST_FP32 : ST_FP64;
        float best = 1e30f;
        int besti = 0;
        const long long keep = c->launches;
        // three rounds over all candidates, each candidate's time the fastest of its three: shapes a
        // few per cent apart (FP64 at 32^4) are not ranked by one sample taken while the clock ramps
        std::vector<float> tmin(ncand, 1e30f);
        for (int round = 0; round < 3 && !st; round++) {
            for (int k = 0; k < ncand && !st; k++) {
                gf_ctx::PassShape sh[2] = {c->shape[0], c->shape[1]};
                sh[prec] = cands[k];
                for (int w = 0; w < (round ? 1 : 2) && !st; w++) st = launch_sweep_on(c, e, sh, ALG_OR, want, 1.7f, 0, 0, 0);
                cudaEventRecord(e0, c->stream);
                for (int w = 0; w < 4 && !st; w++) st = launch_sweep_on(c, e, sh, ALG_OR, want, 1.7f, 0, 0, 0);
                cudaEventRecord(e1, c->stream);
                if (!st) st = cuda_status(cudaEventSynchronize(e1), "autotune sync");
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (!st) tmin[k] = std::min(tmin[k], ms);
            }
        }
        for (int k = 0; k < ncand; k++)
            if (tmin[k] < best) {
                best = tmin[k];
                besti = k;
            }
        c->launches = keep;
        cleanup();
        if (st) return st;
        c->shape[prec] = cands[besti];
        c->tuned[prec] = 1;
        c->drop_graphs();
    }
    auto code = [](const gf_ctx::PassShape &sh) {
        return (sh.stages == 3 ? 100000 : 0) + (sh.capped ? 10000 : 0) + (sh.alternate ? 1000 : 0) +
               (sh.variant == 1 ? sh.warps
               : sh.variant == 2 ? 64
               : sh.variant == 3 ? 100
               : sh.variant == 4 ? 32
               : sh.variant == 5 ? 33
               : sh.variant == 6 ? 16
               : sh.variant == 7 ? 116
                                 : 0);
    };
    if (choice_fp32) *choice_fp32 = c->mixed ? code(c->shape[0]) : -1;
    if (choice_fp64) *choice_fp64 = code(c->shape[1]);
    return GF_OK;
}

// Set the parity-pass launch shape by hand: variant 0 (one warp per tile), 1 (pipelined with
// `warps` = 2, 4 or 8 warps per block), 2 (FP32 direct capped at 64 registers), 3 (register
// prefetch, persistent), 4 (FP32, one thread per site), 5 (the same, pipelined with cp.async;
// OR only, other update rules fall back to variant 4), 6 (two lanes per site) or 7 (two lanes per
// site, persistent with register prefetch; FP32 OR only, the other cases run as 6).
int gf_set_pass_shape(gf_ctx *c, int real, int variant, int warps)
{
    clear_error();
    if (!c || !valid_real(real) || variant < 0 || variant > 7 || (warps != 2 && warps != 4 && warps != 8) ||
        (variant != 0 && variant != 2 && variant != 3 && variant != 6 && variant != 7 && c->gauge == GF_COULOMB) ||
        (variant == 1 && real == GF_FP32 && c->site_w) ||
        ((variant == 2 || variant == 4 || variant == 5) && real == GF_FP64)) {
        set_error("invalid pass shape (Coulomb passes are direct, 64-register, register prefetch or two lanes per "
                  "site; refine-FP32 passes are not pipelined; the 64-register and thread-per-site passes are FP32)");
        return GF_ERR_INVALID;
    }
    c->drop_graphs();
    c->shape[real].variant = variant;
    c->shape[real].warps = warps;
    c->shape[real].alternate = 0;
    c->shape[real].capped = 0;
    c->shape[real].stages = 2;
    c->shape[real].blocks_per_sm = 0;
    c->tuned[real] = 1;
    return GF_OK;
}

// Walk order of the persistent parity passes (variants 1, 3 and 7): alternate = 1 walks the tiles of
// odd-parity passes backwards, so every pass starts on the links the previous one touched last;
// capped = 1 caps the registers of variants 1 (4 warps per block: 128) and 7 (168) so that more
// warps are resident.
int gf_set_pass_order(gf_ctx *c, int real, int alternate, int capped)
{
    clear_error();
    if (!c || !valid_real(real) || (alternate != 0 && alternate != 1) || (capped != 0 && capped != 1)) {
        set_error("invalid argument to gf_set_pass_order");
        return GF_ERR_INVALID;
    }
    c->drop_graphs();
    c->shape[real].alternate = alternate;
    c->shape[real].capped = capped;
    return GF_OK;
}

// cp.async stages per warp of the pipelined pass (variant 1 with 4 warps per block): 2 keeps the
// next tile in flight while the current one is computed, 3 the next two.
int gf_set_pass_stages(gf_ctx *c, int real, int stages)
{
    clear_error();
    if (!c || !valid_real(real) || (stages != 2 && stages != 3) ||
        (stages == 3 && (c->shape[real].variant != 1 || c->shape[real].warps != 4))) {
        set_error("invalid argument to gf_set_pass_stages (three stages: the pipelined pass with 4 warps per block)");
        return GF_ERR_INVALID;
    }
    c->drop_graphs();
    c->shape[real].stages = stages;
    return GF_OK;
}

int gf_instances(gf_ctx *c) { return c ? c->ninst : 0; }

int gf_trace(gf_ctx *c, int instance, double *out, int max_entries, int *n)
{
    clear_error();
    int st = check_ctx(c);
    if (st) return st;
    if (instance < 0 || instance >= c->ninst || max_entries < 0 || (max_entries > 0 && !out) || !n) {
        set_error("invalid argument to gf_trace");
        return GF_ERR_INVALID;
    }
    *n = 0;
    if (!c->trace_cap) return GF_OK;
    int cnt = 0;
    if ((st = cuda_status(cudaMemcpyAsync(&cnt, c->d_ntrace + instance, sizeof(int), cudaMemcpyDeviceToHost,
                                          c->stream), "trace count")) ||
        (st = cuda_status(cudaStreamSynchronize(c->stream), "sync")))
        return st;
    *n = std::min(cnt, c->trace_cap);
    const int m = std::min(*n, max_entries);
    if (m > 0) {
        if ((st = cuda_status(cudaMemcpyAsync(out, c->d_trace + (size_t)instance * c->trace_cap * 4,
                                              sizeof(double) * 4 * m, cudaMemcpyDeviceToHost, c->stream),
                              "trace copy")))
            return st;
        return cuda_status(cudaStreamSynchronize(c->stream), "sync");
    }
    return GF_OK;
}

int gf_kernel_launches(gf_ctx *c, long long *count)
{
    if (!c || !count) {
        set_error("NULL argument");
        return GF_ERR_INVALID;
    }
    *count = c->launches;
    return GF_OK;
}

}  // extern "C"
