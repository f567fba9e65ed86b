// gf_engine.cuh -- batched kernels of the gauge-fixing engine: many lattices (gauge copies,
// uneven extents) in one launch, each in the packed 12-real layout, with per-instance state so
// converged instances drop out without host intervention.
//
// Instance state machine (one int per instance, written only by the quality / convert kernels
// at the end of a check chunk):
//   ST_FP32   sweeping on the FP32 field
//   ST_SWITCH theta fell below the switch threshold; the convert kernel moves the field to FP64
//   ST_FP64   sweeping on the FP64 field (FP64 polish, or plain FP64 runs)
//   ST_DONE   converged (theta < precision) or out of sweeps
#pragma once

#include "gf_kernels.cuh"

namespace gfb {

enum InstState : int { ST_FP32 = 0, ST_FP64 = 1, ST_DONE = 2, ST_SWITCH = 3, ST_FOLD = 4 };

struct InstDesc {
    Geom g;
    int64_t warp_begin;   // first warp of this instance in a batched parity pass
    int64_t link_begin;   // first link (s, mu) of this instance in a batched link kernel
    int64_t qblock_begin; // first block of this instance in the batched quality kernel
    int64_t qblocks;      // quality blocks of this instance
    float4 *f32;          // packed FP32 field (may be null in plain-FP64 contexts)
    double2 *f64;         // packed FP64 field
    double2 *t64;         // Coulomb: the slice's original temporal links (6 double2 planes), else null
    int next;             // Coulomb: instance of timeslice t+1 of the same lattice, else -1
    float2 *w;            // refine mode: accumulated gauge transformation, columns 0, 1 (6 float2 planes), else null
};

struct EngineDev {
    const InstDesc *inst;
    int ninst;
    int *state;           // per instance
    int *sweeps;          // per instance, sweeps done in the current phase machine
    int *sweeps64;        // per instance, FP64 sweeps
    int *storage;         // per instance: 0 = field lives in FP32, 1 = in FP64
    double *quality;      // per instance: functional, theta
    double *partials;     // per quality block: 2 doubles
    unsigned int *tickets;// per instance
    double *best32;       // per instance: smallest FP32 theta of the current gf_fix
    int *stall;           // per instance: checks in a row without beating 0.98 * best32
    double *trace;        // optional: trace_cap entries of 4 doubles per instance, else null
    int *ntrace;          // per instance: checks recorded (may exceed trace_cap)
    int trace_cap;
};

// Traversal order of a persistent pass: with `reverse` the tiles are walked from the last to the
// first.  Consecutive parity passes alternate direction, so a pass starts where the previous one
// ended, on the links still held in L2 (every pass touches every link once).
__device__ __forceinline__ int64_t ordered_tile(int64_t t, int64_t n, int reverse) { return reverse ? n - 1 - t : t; }

// index of the instance whose range [begin[i], begin[i+1]) holds x (ranges ascending)
template <typename F>
__device__ __forceinline__ int find_instance(const InstDesc *inst, int n, int64_t x, F begin_of)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (begin_of(inst[mid]) <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <typename R>
__device__ __forceinline__ PackedField<R> packed_of(const InstDesc &d);
template <>
__device__ __forceinline__ PackedField<float> packed_of<float>(const InstDesc &d) { return PackedField<float>{d.f32, d.g.V}; }
template <>
__device__ __forceinline__ PackedField<double> packed_of<double>(const InstDesc &d) { return PackedField<double>{d.f64, d.g.V}; }

// One parity pass over every instance in state want_state.  A warp handles 8 sites of one
// instance (instance ranges are whole warps).  seed_i = seed + instance, so instance 0 draws the
// reference's Philox stream and the others draw independent ones.
// MINB > 1 caps the registers (65536 / (128 * MINB) per thread) for more resident warps; the
// autotuner decides whether the spills that may cost are worth it
template <typename R, int GAUGE, int ALGO, bool SITE_W = false, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) k_batched_pass(EngineDev e, int64_t total_warps, int parity, AlgoParams p,
                                                           int want_state)
{
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= total_warps) return;
    const int i = find_instance(e.inst, e.ninst, warp, [](const InstDesc &d) { return d.warp_begin; });
    if (e.state[i] != want_state) return;
    const InstDesc d = e.inst[i];
    const PackedField<R> f = packed_of<R>(d);
    AlgoParams pi = p;
    pi.seed = inst_seed(p, i);
    pi.counter = inst_counter(p, i);
    parity_pass_warp<R, GAUGE, ALGO, PackedField<R>, GAUGE == COULOMB, SITE_W>(f, f, d.g, warp - d.warp_begin, parity,
                                                                               pi, d.w);
}

// The descriptors and states of the first kInstCache instances, copied into shared memory once per
// block: a persistent block looks its tile's instance up every iteration, and a chain of dependent
// global loads there would stall every warp for an L2 round trip per tile.  Instances beyond the
// cache are read from global memory.
constexpr int kInstCache = 8;
struct InstCache {
    InstDesc d[kInstCache];
    int state[kInstCache];
    int n;
};

__device__ __forceinline__ void fill_inst_cache(const EngineDev &e, InstCache &ic)
{
    const int n = e.ninst < kInstCache ? e.ninst : kInstCache;
    if (threadIdx.x < n) {
        ic.d[threadIdx.x] = e.inst[threadIdx.x];
        ic.state[threadIdx.x] = e.state[threadIdx.x];
    }
    if (threadIdx.x == 0) ic.n = n;
    __syncthreads();
}

__device__ __forceinline__ const InstDesc &inst_at(const EngineDev &e, const InstCache &ic, int i)
{
    return i < ic.n ? ic.d[i] : e.inst[i];
}

// the instance and half-lattice site of global site index gsite, or -1 (inactive / past the end)
__device__ __forceinline__ int site_of(const EngineDev &e, const InstCache &ic, int64_t gsite, int64_t total_sites,
                                       int want_state, int64_t &h)
{
    if (gsite >= total_sites) return -1;
    const int64_t w = gsite >> 3;
    int i;
    if (e.ninst <= kInstCache) {
        i = find_instance(ic.d, ic.n, w, [](const InstDesc &d) { return d.warp_begin; });
        if (ic.state[i] != want_state) return -1;
    } else {
        i = find_instance(e.inst, e.ninst, w, [](const InstDesc &d) { return d.warp_begin; });
        if (e.state[i] != want_state) return -1;
    }
    h = gsite - inst_at(e, ic, i).warp_begin * 8;
    return i;
}

// Persistent variant with register prefetch: every warp walks a strided list of 8-site tiles and
// issues the loads of tile t+1 (its lane's two links, and the W column in refine mode) into
// registers before it computes tile t, so each warp keeps a tile's worth of loads in flight
// through its arithmetic and shuffles.  Same site update as k_batched_pass.  COULOMB slices: the
// mu = 0 lane holds the slice's W (its temporal plane) as its up link and has no down link, as in
// parity_pass_warp.
template <typename R>
struct TileRegs {
    int inst;        // -1: nothing to do
    int64_t h, s, sd;
    R up[12], dn[12];
    float2 w[3];
};

template <typename R, int GAUGE, bool SITE_W>
__device__ __forceinline__ void fetch_tile_regs(const EngineDev &e, const InstCache &ic, int64_t tile, int parity,
                                                int want_state, TileRegs<R> &t)
{
    t.inst = -1;
    int i;
    if (e.ninst <= kInstCache) {
        i = find_instance(ic.d, ic.n, tile, [](const InstDesc &d) { return d.warp_begin; });
        if (ic.state[i] != want_state) return;
    } else {
        i = find_instance(e.inst, e.ninst, tile, [](const InstDesc &d) { return d.warp_begin; });
        if (e.state[i] != want_state) return;
    }
    const InstDesc &d = inst_at(e, ic, i);
    const int lane = threadIdx.x & 31, mu = lane >> 3;
    t.inst = i;
    t.h = (tile - d.warp_begin) * 8 + (lane & 7);
    int32_t c[4];
    site_coords(d.g, t.h, parity, c);
    t.s = t.h + (parity ? d.g.Vh : 0);
    const bool wlane = GAUGE == COULOMB && mu == 0;
    t.sd = wlane ? t.s : neighbour_down(d.g, c, mu);
    const PackedField<R> f = packed_of<R>(d);
    f.load12(t.s, mu, t.up);
    if (!wlane) f.load12(t.sd, mu, t.dn);
    if (SITE_W) {
        const int k = mu & 1;
#pragma unroll
        for (int r = 0; r < 3; r++) t.w[r] = d.w[(int64_t)(k * 3 + r) * d.g.V + t.s];
    }
}

template <typename R, int GAUGE, int ALGO, bool SITE_W>
__global__ void __launch_bounds__(128) k_batched_pass_rp(EngineDev e, int64_t total_warps, int parity, AlgoParams p,
                                                         int want_state, int reverse)
{
    static_assert(GAUGE != COULOMB || !SITE_W, "Coulomb slices carry W in their temporal planes");
    __shared__ InstCache ic;
    fill_inst_cache(e, ic);
    const int mu = (threadIdx.x & 31) >> 3;
    const bool wlane = GAUGE == COULOMB && mu == 0;
    const int64_t stride = (int64_t)gridDim.x * 4;
    int64_t tile = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    TileRegs<R> cur;
    cur.inst = -1;
    if (tile < total_warps)
        fetch_tile_regs<R, GAUGE, SITE_W>(e, ic, ordered_tile(tile, total_warps, reverse), parity, want_state, cur);
    for (; tile < total_warps; tile += stride) {
        TileRegs<R> nxt;
        nxt.inst = -1;
        if (tile + stride < total_warps)
            fetch_tile_regs<R, GAUGE, SITE_W>(e, ic, ordered_tile(tile + stride, total_warps, reverse), parity,
                                              want_state, nxt);
        if (cur.inst >= 0) {
            const InstDesc &d = inst_at(e, ic, cur.inst);
            Link<R> up, dn;
            unpack12(up, cur.up);
            reconstruct(up);
            if (wlane) {  // the slice's W rides as the up link; no down link
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) dn.e[a][b] = cx<R>(a == b ? (R)1 : (R)0, (R)0);
            } else {
                unpack12(dn, cur.dn);
                reconstruct(dn);
            }
            Rng<R> rng;
            if (ALGO == ALG_SA || ALGO == ALG_SR || ALGO == ALG_RANDOM)
                rng.init(ref_rng_tid(cur.h), inst_seed(p, cur.inst), inst_counter(p, cur.inst));
            Cx<R> wcol[3];
            if (SITE_W) {
#pragma unroll
                for (int r = 0; r < 3; r++) wcol[r] = cx<R>((R)cur.w[r].x, (R)cur.w[r].y);
            }
            site_update<GAUGE, ALGO, R, SITE_W>(up, dn, mu, p, rng, &wcol);
            const PackedField<R> f = packed_of<R>(d);
            store_link<R>(f, cur.s, mu, up);
            if (!wlane) store_link<R>(f, cur.sd, mu, dn);
            if (SITE_W && mu < 2) {
#pragma unroll
                for (int r = 0; r < 3; r++)
                    d.w[(int64_t)(mu * 3 + r) * d.g.V + cur.s] = make_float2((float)wcol[r].x, (float)wcol[r].y);
            }
        }
        cur = nxt;
    }
}

// One thread per site: a warp updates 32 consecutive sites of a parity, each thread all 8 links
// of its site (4 up, 4 down) in registers.  Every load and store of a plane is 32 consecutive
// 16-byte chunks, there are no shuffles, and the subgroup quaternion and its update are computed
// once per site instead of once per lane.  Not for COULOMB (its slices keep W in the temporal
// planes and use the 4-lane pass).
template <typename R, int GAUGE, int ALGO, bool SITE_W, int MINB>
__global__ void __launch_bounds__(128, MINB) k_batched_pass_site(EngineDev e, int64_t total_warps, int parity,
                                                                 AlgoParams p, int want_state)
{
    static_assert(GAUGE != COULOMB, "Coulomb slices use k_batched_pass");
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // one site per thread
    if (t >= total_warps * 8) return;
    const int i = find_instance(e.inst, e.ninst, t >> 3, [](const InstDesc &d) { return d.warp_begin; });
    if (e.state[i] != want_state) return;
    const InstDesc &d = e.inst[i];
    const int64_t h = t - d.warp_begin * 8;
    int32_t c[4];
    site_coords(d.g, h, parity, c);
    const int64_t s = h + (parity ? d.g.Vh : 0);
    const PackedField<R> f = packed_of<R>(d);
    Link<R> up[4], dn[4];
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
        R r[12];
        f.load12(s, mu, r);
        unpack12(up[mu], r);
    }
    int64_t sd[4];
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
        sd[mu] = neighbour_down(d.g, c, mu);
        R r[12];
        f.load12(sd[mu], mu, r);
        unpack12(dn[mu], r);
    }
    Cx<R> wc[2][3];
    if (SITE_W) {
#pragma unroll
        for (int k = 0; k < 2; k++)
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const float2 v = d.w[(int64_t)(k * 3 + r) * d.g.V + s];
                wc[k][r] = cx<R>((R)v.x, (R)v.y);
            }
    }
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
        reconstruct(up[mu]);
        reconstruct(dn[mu]);
    }
    Rng<R> rng;
    if (ALGO == ALG_SA || ALGO == ALG_SR || ALGO == ALG_RANDOM) rng.init(ref_rng_tid(h), inst_seed(p, i), inst_counter(p, i));
    site_update_thread<GAUGE, ALGO, R, SITE_W>(up, dn, p, rng, &wc);
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
        store_link<R>(f, s, mu, up[mu]);
        store_link<R>(f, sd[mu], mu, dn[mu]);
    }
    if (SITE_W) {
#pragma unroll
        for (int k = 0; k < 2; k++)
#pragma unroll
            for (int r = 0; r < 3; r++)
                d.w[(int64_t)(k * 3 + r) * d.g.V + s] = make_float2((float)wc[k][r].x, (float)wc[k][r].y);
    }
}

// cp.async: 16-byte copies bypass L1 (.cg); 8-byte copies must go through it (.ca)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

// ---- two lanes per site --------------------------------------------------------------------------
// A warp updates 16 sites: lanes 0-7 and 16-23 the sites of 8-site tile 2T, lanes 8-15 and 24-31
// those of tile 2T + 1.  Lane `role` = lane >> 4 of a site holds directions 2 role and 2 role + 1
// (their up links at x and down links at x - mu), so a site's 8 links are in 2 lanes instead of 4:
// half the shuffles, the SU(2) update computed twice per site instead of four times, and each of
// the two tracked columns of W updated by one lane.  A tile's two lanes of a site are lane and
// lane ^ 16, always in the same tile, so an idle tile (past the end, or an instance in another
// state) only ever exchanges with itself.  COULOMB slices: direction 0 of role 0 is the slice's W
// (its temporal plane), held as the up link with the identity as its down link, which is neither
// loaded nor stored (as in parity_pass_warp); refine mode keeps no separate W array there.
template <typename R>
__device__ __forceinline__ void set_identity(Link<R> &L)
{
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) L.e[a][b] = cx<R>(a == b ? (R)1 : (R)0, (R)0);
}
struct PairSite {
    int inst;           // -1: idle
    int64_t h, s, sd[2];
};

__device__ __forceinline__ PairSite pair_site(const InstDesc &d, int i, int64_t tile, int parity)
{
    const int lane = threadIdx.x & 31, role = lane >> 4;
    PairSite ps;
    ps.inst = i;
    ps.h = (tile - d.warp_begin) * 8 + (lane & 7);
    int32_t c[4];
    site_coords(d.g, ps.h, parity, c);
    ps.s = ps.h + (parity ? d.g.Vh : 0);
#pragma unroll
    for (int j = 0; j < 2; j++) ps.sd[j] = neighbour_down(d.g, c, 2 * role + j);
    return ps;
}

template <typename R, int GAUGE, int ALGO, bool SITE_W, int MINB>
__global__ void __launch_bounds__(128, MINB) k_batched_pass_pair(EngineDev e, int64_t total_tiles, int parity,
                                                                 AlgoParams p, int want_state)
{
    static_assert(GAUGE != COULOMB || !SITE_W, "Coulomb slices carry W in their temporal planes");
    const int lane = threadIdx.x & 31, role = lane >> 4;
    const bool wlane = GAUGE == COULOMB && role == 0;  // its direction 0 is the slice's W
    const int64_t tile = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 2 + ((lane >> 3) & 1);
    int i = -1;
    if (tile < total_tiles) {
        i = find_instance(e.inst, e.ninst, tile, [](const InstDesc &d) { return d.warp_begin; });
        if (e.state[i] != want_state) i = -1;
    }
    if (!__any_sync(0xffffffffu, i >= 0)) return;
    Link<R> up[2], dn[2];
    Cx<R> wcol[3];
    PairSite ps{-1, 0, 0, {0, 0}};
    PackedField<R> f{nullptr, 0};
    float2 *W = nullptr;
    if (i >= 0) {
        const InstDesc &d = e.inst[i];
        ps = pair_site(d, i, tile, parity);
        f = packed_of<R>(d);
        W = d.w;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            load_link<R>(f, ps.s, 2 * role + j, up[j]);
            if (wlane && j == 0)
                set_identity(dn[j]);
            else
                load_link<R>(f, ps.sd[j], 2 * role + j, dn[j]);
        }
        if (SITE_W) {
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const float2 v = W[(int64_t)(role * 3 + r) * f.V + ps.s];
                wcol[r] = cx<R>((R)v.x, (R)v.y);
            }
        }
    } else {  // idle tile: no coupling, so every update leaves the (unstored) links alone
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) up[j].e[a][b] = dn[j].e[a][b] = cx<R>((R)0, (R)0);
#pragma unroll
        for (int r = 0; r < 3; r++) wcol[r] = cx<R>((R)0, (R)0);
    }
    Rng<R> rng;
    if (ALGO == ALG_SA || ALGO == ALG_SR || ALGO == ALG_RANDOM)
        rng.init(ref_rng_tid(ps.h), inst_seed(p, i < 0 ? 0 : i), inst_counter(p, i < 0 ? 0 : i));
    site_update_pair<GAUGE, ALGO, R, SITE_W>(up, dn, role, p, rng, &wcol);
    if (i < 0) return;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        store_link<R>(f, ps.s, 2 * role + j, up[j]);
        if (!(wlane && j == 0)) store_link<R>(f, ps.sd[j], 2 * role + j, dn[j]);
    }
    if (SITE_W) {
#pragma unroll
        for (int r = 0; r < 3; r++)
            W[(int64_t)(role * 3 + r) * f.V + ps.s] = make_float2((float)wcol[r].x, (float)wcol[r].y);
    }
}

// Persistent form with register prefetch: each warp walks a strided list of 16-site pair tiles and
// loads the next one's links into registers before it updates the current one.  In refine mode the
// next tile's W column goes to shared memory instead (cp.async, two stages per warp), which keeps
// its registers free for the occupancy the register cap buys.
template <typename R>
struct PairRegs {
    PairSite ps;
    R up[2][12], dn[2][12];
};

template <typename R, int GAUGE, bool SITE_W>
__device__ __forceinline__ void fetch_pair_regs(const EngineDev &e, const InstCache &ic, int64_t tile,
                                                int64_t total_tiles, int parity, int want_state, PairRegs<R> &t,
                                                float2 *wstage)
{
    t.ps.inst = -1;
    if (tile >= total_tiles) return;
    int i;
    if (e.ninst <= kInstCache) {
        i = find_instance(ic.d, ic.n, tile, [](const InstDesc &d) { return d.warp_begin; });
        if (ic.state[i] != want_state) return;
    } else {
        i = find_instance(e.inst, e.ninst, tile, [](const InstDesc &d) { return d.warp_begin; });
        if (e.state[i] != want_state) return;
    }
    const InstDesc &d = inst_at(e, ic, i);
    const int role = (threadIdx.x & 31) >> 4;
    t.ps = pair_site(d, i, tile, parity);
    const PackedField<R> f = packed_of<R>(d);
#pragma unroll
    for (int j = 0; j < 2; j++) {
        f.load12(t.ps.s, 2 * role + j, t.up[j]);
        if (!(GAUGE == COULOMB && role == 0 && j == 0)) f.load12(t.ps.sd[j], 2 * role + j, t.dn[j]);
    }
    if (SITE_W) {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int r = 0; r < 3; r++) cp_async8(wstage + r * 32 + lane, d.w + (int64_t)(role * 3 + r) * d.g.V + t.ps.s);
    }
}

template <typename R, int GAUGE, int ALGO, bool SITE_W, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) k_batched_pass_pair_rp(EngineDev e, int64_t total_tiles, int parity,
                                                              AlgoParams p, int want_state, int reverse)
{
    static_assert(GAUGE != COULOMB || !SITE_W, "Coulomb slices carry W in their temporal planes");
    __shared__ InstCache ic;
    // refine: this warp's two stages of the W column, [warp][stage][r][lane] (each lane reads back
    // only what it copied, so the per-thread cp.async.wait_group is the only synchronisation)
    __shared__ float2 wst[SITE_W ? 4 * 2 * 3 * 32 : 1];
    fill_inst_cache(e, ic);
    const int lane = threadIdx.x & 31, role = lane >> 4, half = (lane >> 3) & 1;
    const bool wlane = GAUGE == COULOMB && role == 0;  // its direction 0 is the slice's W
    const int64_t npair = (total_tiles + 1) / 2;                 // 16-site pair tiles
    const int64_t stride = (int64_t)gridDim.x * 4;
    int64_t pt = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);   // this warp's pair tile
    float2 *const wbase = wst + (SITE_W ? (threadIdx.x >> 5) * 2 * 3 * 32 : 0);
    int wcur = 0;
    PairRegs<R> cur;
    cur.ps.inst = -1;
    if (pt < npair)
        fetch_pair_regs<R, GAUGE, SITE_W>(e, ic, ordered_tile(pt, npair, reverse) * 2 + half, total_tiles, parity,
                                          want_state, cur, wbase);
    if (SITE_W) cp_async_commit();
    // every lane of a warp runs the same iterations (pt is warp-uniform), so the shuffles are safe
    for (; pt < npair; pt += stride) {
        PairRegs<R> nxt;
        nxt.ps.inst = -1;
        if (pt + stride < npair)
            fetch_pair_regs<R, GAUGE, SITE_W>(e, ic, ordered_tile(pt + stride, npair, reverse) * 2 + half, total_tiles,
                                              parity, want_state, nxt, wbase + (wcur ^ 1) * 3 * 32);
        if (SITE_W) {
            cp_async_commit();
            cp_async_wait<1>();  // this lane's W column of the current tile has landed
        }
        const int i = cur.ps.inst;
        if (__any_sync(0xffffffffu, i >= 0)) {
            Link<R> up[2], dn[2];
            Cx<R> wcol[3];
#pragma unroll
            for (int j = 0; j < 2; j++) {
                if (i >= 0) {
                    unpack12(up[j], cur.up[j]);
                    reconstruct(up[j]);
                    if (wlane && j == 0) {
                        set_identity(dn[j]);
                    } else {
                        unpack12(dn[j], cur.dn[j]);
                        reconstruct(dn[j]);
                    }
                } else {
#pragma unroll
                    for (int a = 0; a < 3; a++)
#pragma unroll
                        for (int b = 0; b < 3; b++) up[j].e[a][b] = dn[j].e[a][b] = cx<R>((R)0, (R)0);
                }
            }
#pragma unroll
            for (int r = 0; r < 3; r++) {
                wcol[r] = cx<R>((R)0, (R)0);
                if (SITE_W && i >= 0) {
                    const float2 v = wbase[wcur * 3 * 32 + r * 32 + lane];
                    wcol[r] = cx<R>((R)v.x, (R)v.y);
                }
            }
            Rng<R> rng;
            if (ALGO == ALG_SA || ALGO == ALG_SR || ALGO == ALG_RANDOM)
                rng.init(ref_rng_tid(cur.ps.h), inst_seed(p, i < 0 ? 0 : i), inst_counter(p, i < 0 ? 0 : i));
            site_update_pair<GAUGE, ALGO, R, SITE_W>(up, dn, role, p, rng, &wcol);
            if (i >= 0) {
                const InstDesc &d = inst_at(e, ic, i);
                const PackedField<R> f = packed_of<R>(d);
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    store_link<R>(f, cur.ps.s, 2 * role + j, up[j]);
                    if (!(wlane && j == 0)) store_link<R>(f, cur.ps.sd[j], 2 * role + j, dn[j]);
                }
                if (SITE_W) {
#pragma unroll
                    for (int r = 0; r < 3; r++)
                        d.w[(int64_t)(role * 3 + r) * d.g.V + cur.ps.s] =
                            make_float2((float)wcol[r].x, (float)wcol[r].y);
                }
            }
        }
        cur = nxt;
        wcur ^= 1;
    }
    if (SITE_W) cp_async_wait<0>();
}

// ---- refine mode: FP64 master + FP32 working copy + accumulated W --------------------------------
// W(x) is kept as the first two columns of D = W - 1 (6 float2 planes of V): storing the
// deviation from the identity keeps FP32 relative accuracy on the small rotations of the late
// sweeps, when every fold resets W to 1.  The third column of W is conj(c0 x c1), which holds
// for every SU(3) matrix; W stays in SU(3) because every factor g is (reprojection at the
// reference's cadence removes the FP32 drift).  The sweeps only update columns 0 and 1.
__device__ __forceinline__ void load_w_f64(const InstDesc &d, int64_t s, Link<double> &W)
{
#pragma unroll
    for (int k = 0; k < 2; k++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
            const float2 v = d.w[(int64_t)(k * 3 + r) * d.g.V + s];
            W.e[r][k] = cx<double>((double)v.x + (r == k ? 1.0 : 0.0), v.y);
        }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int j = (i + 1) % 3, k = (i + 2) % 3;
        const Cx<double> a = cmul(W.e[j][0], W.e[k][1]), b = cmul(W.e[k][0], W.e[j][1]);
        W.e[i][2] = cx<double>(a.x - b.x, -(a.y - b.y));
    }
}

__device__ __forceinline__ void store_w(const InstDesc &d, int64_t s, const Link<double> &W)
{
#pragma unroll
    for (int k = 0; k < 2; k++)
#pragma unroll
        for (int r = 0; r < 3; r++)
            d.w[(int64_t)(k * 3 + r) * d.g.V + s] =
                make_float2((float)(W.e[r][k].x - (r == k ? 1.0 : 0.0)), (float)W.e[r][k].y);
}

// import of a refine instance: FP64 master and FP32 working copy of the links, W = 1
template <typename Rin>
__global__ void __launch_bounds__(256) k_import_refine(EngineDev e, int i, const Rin *U)
{
    const InstDesc d = e.inst[i];
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * d.g.V) return;
    const int mu = (int)(idx / d.g.V);
    const int64_t s = idx - mu * d.g.V;
    Rin r[12];
    RefField<Rin>{(Rin *)U, d.g.V}.load12(s, mu, r);
    double m[12];
    float f[12];
#pragma unroll
    for (int k = 0; k < 12; k++) {
        m[k] = (double)r[k];
        f[k] = (float)r[k];
    }
    packed_of<double>(d).store12(s, mu, m);
    packed_of<float>(d).store12(s, mu, f);
    if (mu == 0) {
        Link<double> W;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) W.e[a][b] = cx<double>(a == b ? 1.0 : 0.0, 0.0);
        store_w(d, s, W);
    }
}

// reunitarise W (FP64 arithmetic) of every instance in state want_state
__global__ void __launch_bounds__(256) k_reunitarise_w(EngineDev e, int64_t total_links, int want_state)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total_links) return;
    const int i = find_instance(e.inst, e.ninst, idx, [](const InstDesc &d) { return d.link_begin; });
    if (e.state[i] != want_state) return;
    const InstDesc d = e.inst[i];
    const int64_t l = idx - d.link_begin;
    if (l >= d.g.V) return;  // one thread per site: the first quarter of the instance's links
    Link<double> W;
    load_w_f64(d, l, W);
    project_rows(W);
    store_w(d, l, W);
}

// U64_mu(x) <- W(x) U64_mu(x) W(x+mu)^dagger, reunitarised, in FP64 (W reunitarised first unless
// the caller has projected every W of the instance already)
__device__ __forceinline__ void apply_w_link(const InstDesc &d, int64_t s, int mu, Link<double> &L,
                                             bool project_w = true)
{
    const int parity = s >= d.g.Vh;
    int32_t c[4];
    site_coords(d.g, s - (parity ? d.g.Vh : 0), parity, c);
    const int64_t sf = neighbour_up(d.g, c, mu);
    Link<double> W, Wf, T;
    load_w_f64(d, s, W);
    load_w_f64(d, sf, Wf);
    if (project_w) {
        project_rows(W);
        project_rows(Wf);
    }
    load_link_f64<double>(packed_of<double>(d), s, mu, T);
    Link<double> M;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            Cx<double> acc = cx<double>(0, 0);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const Cx<double> t = cmul(W.e[a][k], T.e[k][b]);
                acc.x += t.x;
                acc.y += t.y;
            }
            M.e[a][b] = acc;
        }
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            Cx<double> acc = cx<double>(0, 0);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const Cx<double> w = Wf.e[b][k];
                const Cx<double> t = cmul(M.e[a][k], cx<double>(w.x, -w.y));
                acc.x += t.x;
                acc.y += t.y;
            }
            L.e[a][b] = acc;
        }
    project_rows(L);
}

// refine switch: the FP64 master of every instance in ST_SWITCH becomes W U64 W^dagger
__global__ void __launch_bounds__(256) k_apply_w(EngineDev e, int64_t total_links)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total_links) return;
    const int i = find_instance(e.inst, e.ninst, idx, [](const InstDesc &d) { return d.link_begin; });
    if (e.state[i] != ST_SWITCH) return;
    const InstDesc d = e.inst[i];
    const int64_t l = idx - d.link_begin;
    const int mu = (int)(l / d.g.V);
    const int64_t s = l - mu * d.g.V;
    Link<double> L;
    apply_w_link(d, s, mu, L);
    double r[12];
    pack12(L, r);
    packed_of<double>(d).store12(s, mu, r);  // each thread reads and writes only its own link
}

// iterative refinement (refine contexts, fold mode): every instance in ST_FOLD folds its
// accumulated W into the FP64 master and restarts the FP32 working copy from it, so the rounding
// of the FP32 sweeps never accumulates past one check chunk.  k_reunitarise_w projects each W
// once before (instead of twice per link here); W is reset by k_fold_reset_w in a separate
// launch, because this one reads W(x + mu) of neighbouring sites.
__global__ void __launch_bounds__(256) k_fold_apply(EngineDev e, int64_t total_links)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total_links) return;
    const int i = find_instance(e.inst, e.ninst, idx, [](const InstDesc &d) { return d.link_begin; });
    if (e.state[i] != ST_FOLD) return;
    const InstDesc d = e.inst[i];
    const int64_t l = idx - d.link_begin;
    const int mu = (int)(l / d.g.V);
    const int64_t s = l - mu * d.g.V;
    Link<double> L;
    apply_w_link(d, s, mu, L, false);  // k_reunitarise_w has projected every W of the instance
    double r[12];
    float f[12];
    pack12(L, r);
#pragma unroll
    for (int k = 0; k < 12; k++) f[k] = (float)r[k];
    packed_of<double>(d).store12(s, mu, r);
    packed_of<float>(d).store12(s, mu, f);
}

__global__ void __launch_bounds__(256) k_fold_reset_w(EngineDev e, int64_t total_links)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total_links) return;
    const int i = find_instance(e.inst, e.ninst, idx, [](const InstDesc &d) { return d.link_begin; });
    if (e.state[i] != ST_FOLD) return;
    const InstDesc d = e.inst[i];
    const int64_t l = idx - d.link_begin;
    if (l >= d.g.V) return;  // one thread per site
#pragma unroll
    for (int k = 0; k < 2; k++)
#pragma unroll
        for (int r = 0; r < 3; r++) d.w[(int64_t)(k * 3 + r) * d.g.V + l] = make_float2(0.f, 0.f);  // D = 0
}

// export of a refine instance still in FP32: W U64 W^dagger on the fly
template <typename Rout>
__global__ void __launch_bounds__(256) k_export_refine(EngineDev e, int i, Rout *U)
{
    const InstDesc d = e.inst[i];
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * d.g.V) return;
    const int mu = (int)(idx / d.g.V);
    const int64_t s = idx - mu * d.g.V;
    Link<double> L;
    apply_w_link(d, s, mu, L);
    Link<Rout> o;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) o.e[a][b] = cx<Rout>((Rout)L.e[a][b].x, (Rout)L.e[a][b].y);
    RefField<Rout>{U, d.g.V}.store18(s, mu, o);
}

// ---- refine mode for Coulomb timeslices ----------------------------------------------------------
// A Coulomb slice already keeps its accumulated gauge transformation in its mu = 0 planes (the
// TRACK_W parity pass), so refine mode needs no separate W array: the FP64 master holds the spatial
// links and W64, the product of every transformation folded in so far; the FP32 working copy holds
// its spatial links and W32, the transformation since the last fold.  A fold (and the switch to FP64
// sweeps) applies W32 exactly to the master:
//   U64_i(x) <- W32(x) U64_i(x) W32(x + i)^dagger  (i = 1..3, x + i inside the slice),
//   W64(x)   <- W32(x) W64(x),
// with every W32 reunitarised in FP64 first, so the master's spatial links stay on their gauge orbit
// and W64 stays the exact product the export applies to the temporal links.
__device__ __forceinline__ void mul33(const Link<double> &A, const Link<double> &B, Link<double> &C)
{
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            Cx<double> acc = cx<double>(0, 0);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const Cx<double> t = cmul(A.e[a][k], B.e[k][b]);
                acc.x += t.x;
                acc.y += t.y;
            }
            C.e[a][b] = acc;
        }
}

// C = A B^dagger
__device__ __forceinline__ void mul33_adj(const Link<double> &A, const Link<double> &B, Link<double> &C)
{
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            Cx<double> acc = cx<double>(0, 0);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const Cx<double> t = cmul(A.e[a][k], cx<double>(B.e[b][k].x, -B.e[b][k].y));
                acc.x += t.x;
                acc.y += t.y;
            }
            C.e[a][b] = acc;
        }
}

// W32(s) of a Coulomb slice's working copy, reunitarised in FP64
__device__ __forceinline__ void coulomb_w32(const InstDesc &d, int64_t s, Link<double> &W)
{
    load_link_f64<float>(packed_of<float>(d), s, 0, W);
    project_rows(W);
}

// spatial link mu of the master with the working copy's W32 applied: W32(s) U64_mu(s) W32(s + mu)^dagger
__device__ __forceinline__ void coulomb_apply_w32(const InstDesc &d, int64_t s, int mu, Link<double> &L)
{
    const int parity = s >= d.g.Vh;
    int32_t c[4];
    site_coords(d.g, s - (parity ? d.g.Vh : 0), parity, c);
    Link<double> W, Wf, U, M;
    coulomb_w32(d, s, W);
    coulomb_w32(d, neighbour_up(d.g, c, mu), Wf);
    load_link_f64<double>(packed_of<double>(d), s, mu, U);
    mul33(W, U, M);
    mul33_adj(M, Wf, L);
    project_rows(L);
}

// The fold (FOLD = true: instances in ST_FOLD; the working copy's spatial links restart from the new
// master) or the switch (ST_SWITCH) of refine Coulomb slices, one thread per link.  The working copy's
// W32 is reset to 1 by k_fold_coulomb_reset in a separate launch: this one reads W32 of neighbours.
template <bool FOLD>
__global__ void __launch_bounds__(256) k_apply_w_coulomb(EngineDev e, int64_t total_links)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total_links) return;
    const int i = find_instance(e.inst, e.ninst, idx, [](const InstDesc &d) { return d.link_begin; });
    if (e.state[i] != (FOLD ? ST_FOLD : ST_SWITCH)) return;
    const InstDesc d = e.inst[i];
    const int64_t l = idx - d.link_begin;
    const int mu = (int)(l / d.g.V);
    const int64_t s = l - mu * d.g.V;
    Link<double> L;
    if (mu == 0) {
        Link<double> W, W64;
        coulomb_w32(d, s, W);
        load_link_f64<double>(packed_of<double>(d), s, 0, W64);
        mul33(W, W64, L);
        project_rows(L);
    } else {
        coulomb_apply_w32(d, s, mu, L);
    }
    double r[12];
    pack12(L, r);
    packed_of<double>(d).store12(s, mu, r);  // each thread reads and writes only its own master link
    if (FOLD && mu != 0) {
        float f[12];
#pragma unroll
        for (int k = 0; k < 12; k++) f[k] = (float)r[k];
        packed_of<float>(d).store12(s, mu, f);
    }
}

__global__ void __launch_bounds__(256) k_fold_coulomb_reset(EngineDev e, int64_t total_links)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total_links) return;
    const int i = find_instance(e.inst, e.ninst, idx, [](const InstDesc &d) { return d.link_begin; });
    if (e.state[i] != ST_FOLD) return;
    const InstDesc d = e.inst[i];
    const int64_t l = idx - d.link_begin;
    if (l >= d.g.V) return;  // one thread per site: the mu = 0 planes
    float one[12];
#pragma unroll
    for (int k = 0; k < 12; k++) one[k] = (k == 0 || k == 8) ? 1.f : 0.f;  // rows 0,1 of 1
    packed_of<float>(d).store12(l, 0, one);
}

// ---- software-pipelined parity pass --------------------------------------------------------------
// Same site update as k_batched_pass, but every warp walks a strided list of 8-site tiles and
// prefetches the 2 links of its lane for tile t+1 into shared memory with cp.async (16-byte,
// L2-only) while it computes tile t.  Each lane reads back only the chunks it copied, so the
// per-thread cp.async.wait_group is the only synchronisation.  Shared memory per warp:
// 2 stages x NCH chunks x 32 lanes x 16 B (NCH = 6 for FP32, 12 for FP64).
template <typename R>
struct Chunks {
    static constexpr int per_link = (int)(12 * sizeof(R) / 16);  // 3 (FP32) or 6 (FP64)
    static constexpr int per_lane = 2 * per_link;
};


struct TileRef {
    int inst;      // -1: nothing to do
    int64_t h;     // half-lattice index of this lane's site
    int64_t s, sd; // up-link site and down-link site
};

template <typename R>
__device__ __forceinline__ const uint4 *link_chunks(const InstDesc &d, int64_t s, int mu, int k);
template <>
__device__ __forceinline__ const uint4 *link_chunks<float>(const InstDesc &d, int64_t s, int mu, int k)
{
    return reinterpret_cast<const uint4 *>(d.f32 + ((int64_t)(mu * 3 + k)) * d.g.V + s);
}
template <>
__device__ __forceinline__ const uint4 *link_chunks<double>(const InstDesc &d, int64_t s, int mu, int k)
{
    return reinterpret_cast<const uint4 *>(d.f64 + ((int64_t)(mu * 6 + k)) * d.g.V + s);
}

template <typename R>
__device__ __forceinline__ TileRef prefetch_tile(const EngineDev &e, int64_t tile, int parity, int want_state,
                                                 uint4 *stage)
{
    TileRef t{-1, 0, 0, 0};
    const int i = find_instance(e.inst, e.ninst, tile, [](const InstDesc &d) { return d.warp_begin; });
    if (e.state[i] != want_state) return t;
    const InstDesc &d = e.inst[i];
    const int lane = threadIdx.x & 31, mu = lane >> 3;
    t.inst = i;
    t.h = (tile - d.warp_begin) * 8 + (lane & 7);
    int32_t c[4];
    site_coords(d.g, t.h, parity, c);
    t.s = t.h + (parity ? d.g.Vh : 0);
    t.sd = neighbour_down(d.g, c, mu);
    constexpr int P = Chunks<R>::per_link;
#pragma unroll
    for (int k = 0; k < P; k++) {
        cp_async16(stage + k * 32 + lane, link_chunks<R>(d, t.s, mu, k));
        cp_async16(stage + (P + k) * 32 + lane, link_chunks<R>(d, t.sd, mu, k));
    }
    return t;
}

template <typename R>
__device__ __forceinline__ void unstage_link(const uint4 *stage, int first, Link<R> &L)
{
    const int lane = threadIdx.x & 31;
    R r[12];
    constexpr int P = Chunks<R>::per_link;
#pragma unroll
    for (int k = 0; k < P; k++) {
        const uint4 v = stage[(first + k) * 32 + lane];
        const R *pv = reinterpret_cast<const R *>(&v);
#pragma unroll
        for (int q = 0; q < (int)(16 / sizeof(R)); q++) r[k * (16 / sizeof(R)) + q] = pv[q];
    }
    unpack12(L, r);
    reconstruct(L);
}

// STAGES = 2: the next tile is in flight while the current one is computed; STAGES = 3: the next two
// (a ring of three stages per warp, twice the bytes in flight for the same warps).
template <typename R, int GAUGE, int ALGO, int WARPS, int MINB = 1, int STAGES = 2>
__global__ void __launch_bounds__(WARPS * 32, MINB) k_batched_pass_staged(EngineDev e, int64_t total_warps, int parity,
                                                                      AlgoParams p, int want_state, int reverse)
{
    static_assert(STAGES == 2 || STAGES == 3, "two or three stages");
    extern __shared__ uint4 smem[];
    constexpr int NCH = Chunks<R>::per_lane;
    const int w = threadIdx.x >> 5;
    uint4 *const wbase = smem + (STAGES * w) * NCH * 32;  // this warp's stages, NCH * 32 chunks apart
    const int64_t stride = (int64_t)gridDim.x * WARPS;
    int64_t tile = (int64_t)blockIdx.x * WARPS + w;
    // prefetch tile tt into stage st and close its cp.async group (an empty group past the end)
    auto issue = [&](int64_t tt, int st) -> TileRef {
        const TileRef r = tt < total_warps ? prefetch_tile<R>(e, ordered_tile(tt, total_warps, reverse), parity,
                                                              want_state, wbase + st * NCH * 32)
                                           : TileRef{-1, 0, 0, 0};
        cp_async_commit();
        return r;
    };
    int cur = 0;
    TileRef t = issue(tile, 0);
    TileRef t1{-1, 0, 0, 0};
    if (STAGES == 3) t1 = issue(tile + stride, 1);
    for (; tile < total_warps; tile += stride) {
        // the stage consumed in the previous iteration receives the tile STAGES - 1 strides ahead
        const TileRef n = issue(tile + (STAGES - 1) * stride, (cur + STAGES - 1) % STAGES);
        cp_async_wait<STAGES - 1>();  // this tile's group (the oldest in flight) has landed
        if (t.inst >= 0) {
            const InstDesc &d = e.inst[t.inst];
            const int mu = (threadIdx.x & 31) >> 3;
            Link<R> up, dn;
            unstage_link<R>(wbase + cur * NCH * 32, 0, up);
            unstage_link<R>(wbase + cur * NCH * 32, Chunks<R>::per_link, dn);
            Rng<R> rng;
            if (ALGO == ALG_SA || ALGO == ALG_SR || ALGO == ALG_RANDOM)
                rng.init(ref_rng_tid(t.h), inst_seed(p, t.inst), inst_counter(p, t.inst));
            site_update<GAUGE, ALGO>(up, dn, mu, p, rng);
            const PackedField<R> f = packed_of<R>(d);
            store_link<R>(f, t.s, mu, up);
            store_link<R>(f, t.sd, mu, dn);
        }
        __syncwarp();  // every lane is done with the current stage before it is refilled
        if (STAGES == 3) {
            t = t1;
            t1 = n;
        } else {
            t = n;
        }
        cur = (cur + 1) % STAGES;
    }
    cp_async_wait<0>();
}

template <typename R>
constexpr size_t staged_smem_bytes(int warps, int stages = 2)
{
    return (size_t)warps * stages * Chunks<R>::per_lane * 32 * 16;
}

// ---- one thread per site, pipelined: FP32 only ---------------------------------------------------
// Persistent blocks of 128 threads walk 128-site tiles; every thread prefetches the 8 links of its
// site in the next tile (24 chunks of 16 B) and, in refine mode, the 6 complex floats of its W
// columns (3 slots of 16 B, filled by 8-byte copies) into shared memory with cp.async while it
// updates its site of the current tile.  Slot j of a thread is at [stage][j][thread], so the
// copies and the reads back are conflict-free and each thread only reads what it copied itself.
template <bool SITE_W>
struct SiteStage {
    static constexpr int slots = 24 + (SITE_W ? 3 : 0);
    static constexpr size_t bytes = (size_t)2 * slots * 128 * 16;
};

template <bool SITE_W>
__device__ __forceinline__ void prefetch_site(const EngineDev &e, const InstCache &ic, int i, int64_t h, int parity,
                                              uint4 *stage)
{
    const InstDesc &d = inst_at(e, ic, i);
    int32_t c[4];
    site_coords(d.g, h, parity, c);
    const int64_t s = h + (parity ? d.g.Vh : 0);
    const int t = threadIdx.x;
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
        const int64_t sd = neighbour_down(d.g, c, mu);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            cp_async16(stage + (mu * 3 + k) * 128 + t, d.f32 + (int64_t)(mu * 3 + k) * d.g.V + s);
            cp_async16(stage + (12 + mu * 3 + k) * 128 + t, d.f32 + (int64_t)(mu * 3 + k) * d.g.V + sd);
        }
    }
    if (SITE_W) {
        float2 *ws = reinterpret_cast<float2 *>(stage + 24 * 128);
#pragma unroll
        for (int q = 0; q < 6; q++)  // slot q/2, half q%2
            cp_async8(ws + ((q >> 1) * 128 + t) * 2 + (q & 1), d.w + (int64_t)q * d.g.V + s);
    }
}

__device__ __forceinline__ void unstage_link_f32(const uint4 *stage, int first, Link<float> &L)
{
    float r[12];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float4 v = reinterpret_cast<const float4 *>(stage)[(first + k) * 128 + threadIdx.x];
        r[4 * k] = v.x;
        r[4 * k + 1] = v.y;
        r[4 * k + 2] = v.z;
        r[4 * k + 3] = v.w;
    }
    unpack12(L, r);
}

template <int GAUGE, int ALGO, bool SITE_W>
__global__ void __launch_bounds__(128, 2) k_batched_pass_site_staged(EngineDev e, int64_t total_warps, int parity,
                                                                     AlgoParams p, int want_state)
{
    static_assert(GAUGE != COULOMB, "Coulomb slices use k_batched_pass");
    extern __shared__ uint4 smem[];
    __shared__ InstCache ic;
    fill_inst_cache(e, ic);
    constexpr int SL = SiteStage<SITE_W>::slots;
    // stage k starts at smem + k * SL * 128 (pointer arithmetic: an array of the two stage
    // pointers indexed by the loop's stage bit would live in local memory)
    const int64_t total_sites = total_warps * 8;
    const int64_t stride = (int64_t)gridDim.x * 128;
    int64_t gsite = (int64_t)blockIdx.x * 128 + threadIdx.x;
    int64_t h = 0;
    int inst = site_of(e, ic, gsite, total_sites, want_state, h);
    if (inst >= 0) prefetch_site<SITE_W>(e, ic, inst, h, parity, smem);
    cp_async_commit();
    int cur = 0;
    // every thread of the block runs the same number of iterations (the tile loop is uniform)
    for (int64_t tile0 = (int64_t)blockIdx.x * 128; tile0 < total_sites; tile0 += stride) {
        int64_t hn = 0;
        const int next = site_of(e, ic, gsite + stride, total_sites, want_state, hn);
        uint4 *const stage_cur = smem + cur * (SL * 128);
        uint4 *const stage_next = smem + (cur ^ 1) * (SL * 128);
        if (next >= 0) prefetch_site<SITE_W>(e, ic, next, hn, parity, stage_next);
        cp_async_commit();
        cp_async_wait<1>();
        if (inst >= 0) {
            const InstDesc &d = inst_at(e, ic, inst);
            int32_t c[4];
            site_coords(d.g, h, parity, c);
            const int64_t s = h + (parity ? d.g.Vh : 0);
            Link<float> up[4], dn[4];
#pragma unroll
            for (int mu = 0; mu < 4; mu++) {
                unstage_link_f32(stage_cur, mu * 3, up[mu]);
                unstage_link_f32(stage_cur, 12 + mu * 3, dn[mu]);
                reconstruct(up[mu]);
                reconstruct(dn[mu]);
            }
            Cx<float> wc[2][3];
            if (SITE_W) {
                const float2 *ws = reinterpret_cast<const float2 *>(stage_cur + 24 * 128);
#pragma unroll
                for (int q = 0; q < 6; q++) {
                    const float2 v = ws[((q >> 1) * 128 + threadIdx.x) * 2 + (q & 1)];
                    wc[q / 3][q % 3] = cx<float>(v.x, v.y);
                }
            }
            Rng<float> rng;
            if (ALGO == ALG_SA || ALGO == ALG_SR || ALGO == ALG_RANDOM)
                rng.init(ref_rng_tid(h), inst_seed(p, inst), inst_counter(p, inst));
            site_update_thread<GAUGE, ALGO, float, SITE_W>(up, dn, p, rng, &wc);
            const PackedField<float> f = packed_of<float>(d);
#pragma unroll
            for (int mu = 0; mu < 4; mu++) {
                store_link<float>(f, s, mu, up[mu]);
                store_link<float>(f, neighbour_down(d.g, c, mu), mu, dn[mu]);
            }
            if (SITE_W) {
#pragma unroll
                for (int q = 0; q < 6; q++)
                    d.w[(int64_t)q * d.g.V + s] = make_float2(wc[q / 3][q % 3].x, wc[q / 3][q % 3].y);
            }
        }
        gsite += stride;
        h = hn;
        inst = next;
        cur ^= 1;
    }
    cp_async_wait<0>();
}

// ---- one persistent launch per check chunk --------------------------------------------------------
// A cooperative launch (every block resident) runs all parity passes of a check chunk -- and the
// reprojections the drivers do inside it -- with a grid-wide barrier between them, instead of one
// launch per pass: for small lattices the launches, not the passes, set the time per sweep.
// Every wait of the barrier is bounded: a block that waits longer than budget_ns records the
// barrier in ChunkSync and leaves the kernel, and every other block leaves at its next wait, so the
// host gets an error status (GF_ERR_TIMEOUT) and the context stays usable.
struct ChunkSync {
    unsigned int count;   // barrier arrivals since the launch (zeroed before it; only grows)
    unsigned int unused;
    unsigned int error;   // 1: a wait ran out of its budget
    unsigned int where;   // index of that barrier
};

struct ChunkReproject {
    unsigned long long bits[4];  // bit k: reproject after sweep k of the chunk (k < 256)
    __device__ __forceinline__ bool after(int k) const { return (bits[k >> 6] >> (k & 63)) & 1ull; }
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_add_gpu(unsigned int *p, unsigned int v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier `index` (0, 1, 2, ... within a launch): thread 0 of each block adds its arrival to
// the counter with release semantics (after the block's bar.sync, so it publishes every thread's
// writes of the pass) and polls the counter with acquire loads until all `arrivals` blocks have
// arrived at this barrier, count >= (index + 1) * arrivals.  One L2 round trip after the last
// arrival releases everyone: no reset, no generation word, no full fences.  `arrivals` is
// gridDim.x (more only when a test makes the wait run out).  The wait is bounded: a block that
// waits longer than budget_ns records the barrier and leaves, and every other block leaves at its
// next poll of the error word.  Returns false when the block must leave the kernel.
__device__ __forceinline__ bool grid_barrier(ChunkSync *sy, unsigned int arrivals, unsigned long long budget_ns,
                                             unsigned int index)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned int target = (index + 1) * arrivals;
        red_release_add_gpu(&sy->count, 1u);
        if (ld_acquire_gpu(&sy->count) < target) {
            const unsigned long long t0 = global_ns();
            for (unsigned int spin = 1; ld_acquire_gpu(&sy->count) < target; spin++) {
                if (spin & 31u) continue;  // poll the counter; the error word and the clock less often
                if (ld_acquire_gpu(&sy->error)) {
                    ok = 0;
                    break;
                }
                if (global_ns() - t0 > budget_ns) {
                    if (atomicExch(&sy->error, 1u) == 0u) sy->where = index;
                    ok = 0;
                    break;
                }
            }
        }
        if (ok && ld_acquire_gpu(&sy->error)) ok = 0;  // another block gave up: leave with it
    }
    __syncthreads();
    return ok != 0;
}

template <typename R>
__device__ __forceinline__ PackedFieldL2<R> packed_l2_of(const InstDesc &d);
template <>
__device__ __forceinline__ PackedFieldL2<float> packed_l2_of<float>(const InstDesc &d)
{
    return PackedFieldL2<float>{d.f32, d.g.V};
}
template <>
__device__ __forceinline__ PackedFieldL2<double> packed_l2_of<double>(const InstDesc &d)
{
    return PackedFieldL2<double>{d.f64, d.g.V};
}

// nsweeps OR sweeps of every instance in want_state (a context without the separate W array:
// plain FP64, FP32 storage, Coulomb slices with W in their temporal planes), each pass the
// 4-lane site update of k_batched_pass, reprojecting after sweep k where repro.after(k).
template <typename R, int GAUGE>
__global__ void __launch_bounds__(128) k_chunk_sweeps(EngineDev e, int64_t total_warps, int64_t total_links,
                                                      int nsweeps, ChunkReproject repro, AlgoParams p,
                                                      int want_state, ChunkSync *sy, unsigned int arrivals,
                                                      unsigned long long budget_ns)
{
    // the states cannot change inside a chunk (only its check moves them), so the descriptors and
    // states of the first instances are read once per launch instead of once per tile and pass
    __shared__ InstCache ic;
    fill_inst_cache(e, ic);
    const int64_t wstride = (int64_t)gridDim.x * 4;
    const int64_t wfirst = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    unsigned int bar = 0;
    for (int k = 0; k < nsweeps; k++) {
        for (int parity = 0; parity < 2; parity++) {
            for (int64_t warp = wfirst; warp < total_warps; warp += wstride) {
                int i;
                if (e.ninst <= kInstCache) {
                    i = find_instance(ic.d, ic.n, warp, [](const InstDesc &d) { return d.warp_begin; });
                    if (ic.state[i] != want_state) continue;  // warp-uniform: a tile lies in one instance
                } else {
                    i = find_instance(e.inst, e.ninst, warp, [](const InstDesc &d) { return d.warp_begin; });
                    if (e.state[i] != want_state) continue;
                }
                const InstDesc &d = inst_at(e, ic, i);
                const PackedFieldL2<R> f = packed_l2_of<R>(d);
                parity_pass_warp<R, GAUGE, ALG_OR, PackedFieldL2<R>, GAUGE == COULOMB, false>(
                    f, f, d.g, warp - d.warp_begin, parity, p, nullptr);
            }
            const bool last = k == nsweeps - 1 && parity == 1 && !repro.after(k);
            if (!last && !grid_barrier(sy, arrivals, budget_ns, bar++)) return;
        }
        if (repro.after(k)) {
            for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total_links;
                 idx += (int64_t)gridDim.x * blockDim.x) {
                const int i = e.ninst <= kInstCache
                                  ? find_instance(ic.d, ic.n, idx, [](const InstDesc &d) { return d.link_begin; })
                                  : find_instance(e.inst, e.ninst, idx, [](const InstDesc &d) { return d.link_begin; });
                if ((i < ic.n ? ic.state[i] : e.state[i]) != want_state) continue;
                const InstDesc &d = inst_at(e, ic, i);
                const int64_t l = idx - d.link_begin;
                const int mu = (int)(l / d.g.V);
                const int64_t s = l - mu * d.g.V;
                Link<double> L;
                load_link_f64<R>(packed_l2_of<R>(d), s, mu, L);
                project_rows(L);
                R o[12];
#pragma unroll
                for (int a = 0; a < 2; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) {
                        o[2 * (3 * a + b)] = (R)L.e[a][b].x;
                        o[2 * (3 * a + b) + 1] = (R)L.e[a][b].y;
                    }
                packed_of<R>(d).store12(s, mu, o);
            }
            if (k < nsweeps - 1 && !grid_barrier(sy, arrivals, budget_ns, bar++)) return;
        }
    }
}

// Quality of every instance in state want_state, with the state transitions of the check:
//  ST_FP32 -> ST_SWITCH when theta < switch_theta (mixed runs) or when theta has stopped
//  falling in FP32 (stall_checks), ST_FP64 -> ST_DONE when
//  theta < precision; either -> ST_DONE when the sweep budget is spent.  chunk_sweeps is added
//  to the instance's sweep count first.  Per-instance tickets make the last block of each
//  instance reduce that instance's partials in block order (deterministic).
struct CheckParams {
    int want_state;
    int chunk_sweeps;
    int max_sweeps;
    double switch_theta;  // <= 0: never switch
    double precision;
    int stop_max;
    int transitions;      // 0: only measure
    int stall_checks;     // ST_FP32 -> ST_SWITCH also after this many checks without progress
    int fold;             // refine contexts: ST_FP32 -> ST_FOLD (not ST_SWITCH) below switch_theta
    double fold_exit;     // ST_FOLD -> ST_FP64 once theta < fold_exit * precision (0: off)
};

// progress of an instance's theta: a new best when it falls below 0.98 x the best so far;
// returns the number of checks in a row without one
__device__ __forceinline__ int track_progress(EngineDev e, int i, double tn)
{
    double best = e.best32[i];
    int stall = e.stall[i];
    if (tn < 0.98 * best) {
        best = tn;
        stall = 0;
    } else {
        stall++;
    }
    e.best32[i] = best;
    e.stall[i] = stall;
    return stall;
}

template <int GAUGE, typename R, int NT = 256>
__global__ void __launch_bounds__(NT) k_batched_quality(EngineDev e, int64_t total_blocks, CheckParams cp)
{
    const int64_t b = blockIdx.x;
    const int i = find_instance(e.inst, e.ninst, b, [](const InstDesc &d) { return d.qblock_begin; });
    // with transitions: the instances sweeping in this precision; without: every instance whose
    // field lives in this precision (uniform over the block)
    if (cp.transitions ? (e.state[i] != cp.want_state) : (e.storage[i] != (sizeof(R) == 8 ? 1 : 0))) return;
    const InstDesc d = e.inst[i];
    const int64_t lb = b - d.qblock_begin;
    const int64_t s = lb * NT + threadIdx.x;
    double gv = 0, tv = 0;
    if (s < d.g.V) quality_site<GAUGE, R>(packed_of<R>(d), d.g, s, gv, tv);
    block_reduce2<NT>(gv, tv, cp.stop_max != 0);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        e.partials[2 * b] = gv;
        e.partials[2 * b + 1] = tv;
        __threadfence();
        last = atomicAdd(&e.tickets[i], 1u) == (unsigned)d.qblocks - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double G = 0, T = 0;
    for (int64_t k = threadIdx.x; k < d.qblocks; k += NT) {
        G += __ldcg(&e.partials[2 * (d.qblock_begin + k)]);
        const double t = __ldcg(&e.partials[2 * (d.qblock_begin + k) + 1]);
        T = cp.stop_max ? fmax(T, t) : T + t;
    }
    block_reduce2<NT>(G, T, cp.stop_max != 0);
    if (threadIdx.x == 0) {
        const double gn = G * prefactor_gff_dev(GAUGE) / (double)d.g.V;
        double tn = T * (1.0 / 3.0);
        if (!cp.stop_max) tn = tn / (double)d.g.V;
        e.quality[2 * i] = gn;
        e.quality[2 * i + 1] = tn;
        e.tickets[i] = 0;
        if (cp.transitions) {
            const int sw = e.sweeps[i] + cp.chunk_sweeps;
            e.sweeps[i] = sw;
            if (e.trace) {
                const int k = e.ntrace[i]++;
                if (k < e.trace_cap) {
                    double *t = e.trace + ((int64_t)i * e.trace_cap + k) * 4;
                    t[0] = sw;
                    t[1] = cp.want_state;
                    t[2] = gn;
                    t[3] = tn;
                }
            }
            if (cp.want_state == ST_FP64) e.sweeps64[i] += cp.chunk_sweeps;
            int st = cp.want_state;
            if (cp.want_state == ST_FP32) {
                if (sw == cp.chunk_sweeps) {  // first check of this gf_fix
                    e.best32[i] = 1e300;
                    e.stall[i] = 0;
                }
                if (cp.switch_theta > 0 && tn < cp.switch_theta)
                    st = cp.fold ? ST_FOLD : ST_SWITCH;
                else if (track_progress(e, i, tn) >= cp.stall_checks && cp.stall_checks > 0 && cp.switch_theta > 0)
                    st = ST_SWITCH;  // FP32 rounding floor: no 2% gain within stall_checks checks
            } else if (cp.want_state == ST_FOLD) {
                // theta of the FP64 master right after a fold: done; or within fold_exit of the
                // target, where the FP32 rounding noise (~1e-12) is a visible part of it, or with
                // the folds no longer gaining 2% within stall_checks folds: polish with FP64
                // sweeps; else keep refining in FP32
                if (tn < cp.precision) {
                    st = ST_DONE;
                    e.storage[i] = 1;
                } else if (tn < cp.fold_exit * cp.precision ||
                           (track_progress(e, i, tn) >= cp.stall_checks && cp.stall_checks > 0)) {
                    st = ST_FP64;
                    e.storage[i] = 1;
                } else {
                    st = ST_FP32;
                }
            }
            if (st == ST_FP64 && tn < cp.precision) st = ST_DONE;
            if (sw >= cp.max_sweeps) st = ST_DONE;
            e.state[i] = st;
        }
    }
}

// ---- link-wise kernels over all instances -----------------------------------------------------
// import: reference GpuPattern (rows 0,1) -> packed field of type R
template <typename Rin, typename R>
__global__ void __launch_bounds__(256) k_import(EngineDev e, int i, const Rin *U)
{
    const InstDesc d = e.inst[i];
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * d.g.V) return;
    const int mu = (int)(idx / d.g.V);
    const int64_t s = idx - mu * d.g.V;
    RefField<Rin> src{(Rin *)U, d.g.V};
    Rin r[12];
    src.load12(s, mu, r);
    R o[12];
#pragma unroll
    for (int k = 0; k < 12; k++) o[k] = (R)r[k];
    if (d.t64 && mu == 0) {
        // Coulomb: keep the temporal link in FP64 and start W at the identity
        double t[12];
#pragma unroll
        for (int k = 0; k < 12; k++) t[k] = (double)r[k];
        PackedField<double>{d.t64, d.g.V}.store12(s, 0, t);
#pragma unroll
        for (int k = 0; k < 12; k++) o[k] = (k == 0 || k == 8) ? (R)1 : (R)0;  // rows 0,1 of 1
    }
    packed_of<R>(d).store12(s, mu, o);
}

// export: packed field of type R -> reference GpuPattern, reunitarised in FP64 with row 2
// rebuilt (the reference's closing projectSU3, apps/LandauGaugeFixingSU3_4D.cu:271)
template <typename R, typename Rout>
__global__ void __launch_bounds__(256) k_export(EngineDev e, int i, Rout *U)
{
    const InstDesc d = e.inst[i];
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * d.g.V) return;
    const int mu = (int)(idx / d.g.V);
    const int64_t s = idx - mu * d.g.V;
    Link<double> L;
    load_link_f64<R>(packed_of<R>(d), s, mu, L);
    project_rows(L);
    Link<Rout> o;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) o.e[a][b] = cx<Rout>((Rout)L.e[a][b].x, (Rout)L.e[a][b].y);
    RefField<Rout>{U, d.g.V}.store18(s, mu, o);
}

// The accumulated transformation W(s) of Coulomb slice i, from the storage its field lives in; a
// refine slice whose FP32 working copy is current has W = W32 W64 (working copy after master).
__device__ __forceinline__ void coulomb_w_total(const EngineDev &e, int i, int64_t s, bool refine, Link<double> &W)
{
    const InstDesc d = e.inst[i];
    if (e.storage[i] == 1) {
        load_link_f64<double>(packed_of<double>(d), s, 0, W);
    } else if (!refine) {
        load_link_f64<float>(packed_of<float>(d), s, 0, W);
    } else {
        Link<double> W32, W64;
        coulomb_w32(d, s, W32);
        load_link_f64<double>(packed_of<double>(d), s, 0, W64);
        mul33(W32, W64, W);
    }
}

// Coulomb export of timeslice i: spatial links as k_export (a refine slice whose working copy is
// current exports its master with W32 applied); temporal links
// U_0(t,x) <- W(t,x) U_0(t,x) W(t+1,x)^dagger, W read from each slice's current storage; W(t+1) is
// that of instance `next` when next >= 0 (slice t+1 taken from another gauge copy), else of the
// lattice's own slice t+1.
template <typename Rout>
__global__ void __launch_bounds__(256) k_export_coulomb(EngineDev e, int i, Rout *U, int refine, int next)
{
    const InstDesc d = e.inst[i];
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * d.g.V) return;
    const int mu = (int)(idx / d.g.V);
    const int64_t s = idx - mu * d.g.V;
    Link<double> L;
    const bool own64 = e.storage[i] == 1;
    if (mu != 0) {
        if (own64) load_link_f64<double>(packed_of<double>(d), s, mu, L);
        else if (refine) coulomb_apply_w32(d, s, mu, L);
        else load_link_f64<float>(packed_of<float>(d), s, mu, L);
    } else {
        Link<double> W, Wn, T;
        coulomb_w_total(e, i, s, refine != 0, W);
        coulomb_w_total(e, next >= 0 ? next : d.next, s, refine != 0, Wn);
        load_link_f64<double>(PackedField<double>{d.t64, d.g.V}, s, 0, T);
        Link<double> M;  // W T
        mul33(W, T, M);
        mul33_adj(M, Wn, L);  // rows 0,1 are what project_rows reads; row 2 is rebuilt there
    }
    project_rows(L);
    Link<Rout> o;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) o.e[a][b] = cx<Rout>((Rout)L.e[a][b].x, (Rout)L.e[a][b].y);
    RefField<Rout>{U, d.g.V}.store18(s, mu, o);
}

// reunitarise (FP64 arithmetic) the packed field of every instance in state want_state; with
// to64 = true, instances in ST_SWITCH are read from FP32 and written to FP64 instead
template <typename R, bool TO64>
__global__ void __launch_bounds__(256) k_reunitarise(EngineDev e, int64_t total_links, int want_state)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total_links) return;
    const int i = find_instance(e.inst, e.ninst, idx, [](const InstDesc &d) { return d.link_begin; });
    if (e.state[i] != want_state) return;
    const InstDesc d = e.inst[i];
    const int64_t l = idx - d.link_begin;
    const int mu = (int)(l / d.g.V);
    const int64_t s = l - mu * d.g.V;
    Link<double> L;
    load_link_f64<R>(packed_of<R>(d), s, mu, L);
    project_rows(L);
    double r[12];
    pack12(L, r);
    if (TO64) {
        packed_of<double>(d).store12(s, mu, r);
    } else {
        R o[12];
#pragma unroll
        for (int k = 0; k < 12; k++) o[k] = (R)r[k];
        packed_of<R>(d).store12(s, mu, o);
    }
}

__global__ void k_finish_switch(EngineDev e)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < e.ninst && e.state[i] == ST_SWITCH) {
        e.state[i] = ST_FP64;
        e.storage[i] = 1;
    }
}

}  // namespace gfb
