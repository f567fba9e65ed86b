// gf_kernels.cuh -- kernel templates shared by the plugin entry points (reference layout, in
// place) and the batched engine (packed layout): parity pass, gauge quality with a deterministic
// FP64 reduction, reprojection and random start.
#pragma once

#include "gf_field.cuh"

namespace gfb {

// functional normalisation 1/(Nc*Nd), Coulomb 1/(Nc*(Nd-1)) (LandauKernelsSU3.hxx:79-82,
// CoulombKernelsSU3.hxx:75-78); theta is normalised by 1/Nc
__host__ __device__ constexpr double prefactor_gff_dev(int gauge) { return gauge == COULOMB ? 1.0 / 9.0 : 1.0 / 12.0; }

// ---- one parity pass ---------------------------------------------------------------------------
// 4 lanes per site (lane = 8*mu + site-in-warp), 8 sites per warp.  Vh is a multiple of 8 for
// even extents, so a warp is either fully inside the parity half or fully outside.
// Fup holds the up links and every down link except, for COULOMB, the temporal down link, which
// comes from the slice t-1 field Fdw at the same spatial site (CoulombKernelsSU3.hxx:226-234).
// TRACK_W (batched Coulomb): the mu = 0 planes of a timeslice hold W(x), the gauge transformation
// accumulated at that site, instead of temporal links.  Lane mu = 0 left-multiplies W by every g
// (W <- g W) and has no down link; the temporal links themselves are transformed once, at the end,
// as U_0(t,x) <- W(t,x) U_0(t,x) W(t+1,x)^dagger (the product of the reference's per-sweep left and
// right multiplications, CoulombKernelsSU3.hxx:226-247), so timeslices share no memory while they
// sweep.
// W columns of the refine mode: float2 planes W[(k*3 + r)*V + s] = W(s)_{r,k}; lane mu < 3 of a
// site carries column mu through the three subgroup steps (W <- g W), lane 3 carries none.
template <typename R, int GAUGE, int ALGO, class F, bool TRACK_W = false, bool SITE_W = false>
__device__ __forceinline__ void parity_pass_warp(const F &Fup, const F &Fdw, const Geom &g, int64_t warp, int parity,
                                                 const AlgoParams &p, float2 *Wsite = nullptr)
{
    const int lane = threadIdx.x & 31;
    const int mu = lane >> 3;
    const int64_t h = warp * 8 + (lane & 7);
    int32_t c[4];
    site_coords(g, h, parity, c);
    const int64_t s = h + (parity ? g.Vh : 0);
    const bool tdown = (GAUGE == COULOMB) && (mu == 0);
    const bool wlane = TRACK_W && tdown;
    const int64_t sd = tdown ? s : neighbour_down(g, c, mu);
    Link<R> up, dn;
    load_link<R>(Fup, s, mu, up);
    if (wlane) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) dn.e[i][j] = cx<R>(i == j ? (R)1 : (R)0, (R)0);
    } else if (tdown) {
        load_link<R>(Fdw, sd, mu, dn);
    } else {
        load_link<R>(Fup, sd, mu, dn);
    }
    Rng<R> rng;
    if (ALGO == ALG_SA || ALGO == ALG_SR || ALGO == ALG_RANDOM) rng.init(ref_rng_tid(h), p.seed, p.counter);
    Cx<R> wcol[3];
    if (SITE_W) {
        const int k = mu & 1;  // lanes mu = 0, 1 own columns 0, 1 of W; 2, 3 re-read them
#pragma unroll
        for (int r = 0; r < 3; r++) {
            const float2 v = Wsite[(int64_t)(k * 3 + r) * g.V + s];
            wcol[r] = cx<R>((R)v.x, (R)v.y);
        }
    }
    site_update<GAUGE, ALGO, R, SITE_W>(up, dn, mu, p, rng, &wcol);
    store_link<R>(Fup, s, mu, up);
    if (SITE_W && mu < 2) {
#pragma unroll
        for (int r = 0; r < 3; r++) Wsite[(int64_t)(mu * 3 + r) * g.V + s] = make_float2((float)wcol[r].x, (float)wcol[r].y);
    }
    if (wlane) return;
    if (tdown)
        store_link<R>(Fdw, sd, mu, dn);
    else
        store_link<R>(Fup, sd, mu, dn);
}

template <typename R, int GAUGE, int ALGO, class F>
__global__ void __launch_bounds__(128) k_parity_pass(F Fup, F Fdw, Geom g, int parity, AlgoParams p)
{
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp * 8 >= g.Vh) return;
    parity_pass_warp<R, GAUGE, ALGO>(Fup, Fdw, g, warp, parity, p);
}

// The same pass as a persistent kernel with register prefetch: each warp walks a strided list of
// 8-site tiles and loads its lane's two links of the next tile into registers before it updates
// the current one, so a tile's loads are in flight through the arithmetic of the previous one.
// Odd parities walk the tiles backwards: a driver that calls parity 0 and then parity 1 finds the
// links the first pass touched last still in L2.  Same site update and stores as k_parity_pass.
template <typename R, int GAUGE, int ALGO, class F>
__global__ void __launch_bounds__(128) k_parity_pass_rp(F Fup, F Fdw, Geom g, int parity, AlgoParams p)
{
    const int lane = threadIdx.x & 31, mu = lane >> 3;
    const bool tdown = (GAUGE == COULOMB) && (mu == 0);  // the temporal down link is in slice t-1
    const int64_t ntiles = g.Vh / 8;
    const int64_t stride = (int64_t)gridDim.x * 4;
    int64_t t = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    struct Tile {
        int64_t h, s, sd;
        R up[12], dn[12];
    };
    auto fetch = [&](int64_t k, Tile &r) {
        const int64_t tile = parity ? ntiles - 1 - k : k;
        r.h = tile * 8 + (lane & 7);
        int32_t c[4];
        site_coords(g, r.h, parity, c);
        r.s = r.h + (parity ? g.Vh : 0);
        r.sd = tdown ? r.s : neighbour_down(g, c, mu);
        Fup.load12(r.s, mu, r.up);
        if (tdown)
            Fdw.load12(r.sd, mu, r.dn);
        else
            Fup.load12(r.sd, mu, r.dn);
    };
    Tile cur;
    if (t < ntiles) fetch(t, cur);
    for (; t < ntiles; t += stride) {  // warp-uniform: every lane of a warp runs the same tiles
        Tile nxt;
        if (t + stride < ntiles) fetch(t + stride, nxt);
        Link<R> up, dn;
        unpack12(up, cur.up);
        reconstruct(up);
        unpack12(dn, cur.dn);
        reconstruct(dn);
        Rng<R> rng;
        if (ALGO == ALG_SA || ALGO == ALG_SR || ALGO == ALG_RANDOM) rng.init(ref_rng_tid(cur.h), p.seed, p.counter);
        site_update<GAUGE, ALGO>(up, dn, mu, p, rng);
        store_link<R>(Fup, cur.s, mu, up);
        if (tdown)
            store_link<R>(Fdw, cur.sd, mu, dn);
        else
            store_link<R>(Fup, cur.sd, mu, dn);
        cur = nxt;
    }
}

// FP64 on the reference layout: the same persistent pass with the next tile staged in shared
// memory by cp.async instead of registers (the register form holds 200 registers in FP64).  In
// the reference layout every real of a link is its own plane, so a lane copies its two links as
// 24 eight-byte chunks; chunk k of a lane sits at [stage][k][lane] (conflict-free), and each lane
// reads back only what it copied, so its own cp.async.wait_group is the only synchronisation.
constexpr int kRefStageDoubles = 24;  // two links x rows 0, 1 (12 reals each) per lane
constexpr size_t ref_staged_smem_bytes(int warps) { return (size_t)warps * 2 * kRefStageDoubles * 32 * 8; }

__device__ __forceinline__ void cp_async8_ref(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

template <int GAUGE, int ALGO>
__global__ void __launch_bounds__(128) k_parity_pass_ref_staged(RefField<double> Fup, RefField<double> Fdw, Geom g,
                                                                int parity, AlgoParams p)
{
    extern __shared__ double ref_stage[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, mu = lane >> 3;
    const bool tdown = (GAUGE == COULOMB) && (mu == 0);  // the temporal down link is in slice t-1
    const int64_t ntiles = g.Vh / 8;
    const int64_t stride = (int64_t)gridDim.x * 4;
    double *const wbase = ref_stage + (size_t)w * 2 * kRefStageDoubles * 32;  // this warp's two stages
    struct Tile {
        int64_t h, s, sd;
        bool valid;
    };
    auto issue = [&](int64_t k, int st) -> Tile {
        Tile r{0, 0, 0, k < ntiles};
        if (r.valid) {
            const int64_t tile = parity ? ntiles - 1 - k : k;
            r.h = tile * 8 + (lane & 7);
            int32_t c[4];
            site_coords(g, r.h, parity, c);
            r.s = r.h + (parity ? g.Vh : 0);
            r.sd = tdown ? r.s : neighbour_down(g, c, mu);
            double *dst = wbase + (size_t)st * kRefStageDoubles * 32;
            const double *up = Fup.U + (int64_t)mu * 18 * g.V + r.s;
            const double *dn = (tdown ? Fdw.U : Fup.U) + (int64_t)mu * 18 * g.V + r.sd;
#pragma unroll
            for (int q = 0; q < 12; q++) {
                cp_async8_ref(dst + q * 32 + lane, up + (int64_t)q * g.V);
                cp_async8_ref(dst + (12 + q) * 32 + lane, dn + (int64_t)q * g.V);
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        return r;
    };
    int64_t t = (int64_t)blockIdx.x * 4 + w;
    int cur = 0;
    Tile tc = issue(t, 0);
    for (; t < ntiles; t += stride) {  // warp-uniform: every lane of a warp runs the same tiles
        const Tile tn = issue(t + stride, cur ^ 1);
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this tile's copies have landed
        const double *src = wbase + (size_t)cur * kRefStageDoubles * 32;
        double ru[12], rd[12];
#pragma unroll
        for (int q = 0; q < 12; q++) {
            ru[q] = src[q * 32 + lane];
            rd[q] = src[(12 + q) * 32 + lane];
        }
        Link<double> up, dn;
        unpack12(up, ru);
        reconstruct(up);
        unpack12(dn, rd);
        reconstruct(dn);
        Rng<double> rng;
        if (ALGO == ALG_SA || ALGO == ALG_SR || ALGO == ALG_RANDOM) rng.init(ref_rng_tid(tc.h), p.seed, p.counter);
        site_update<GAUGE, ALGO>(up, dn, mu, p, rng);
        store_link<double>(Fup, tc.s, mu, up);
        if (tdown)
            store_link<double>(Fdw, tc.sd, mu, dn);
        else
            store_link<double>(Fup, tc.sd, mu, dn);
        __syncwarp();  // every lane is done with this stage before the next iteration refills it
        tc = tn;
        cur ^= 1;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// One parity pass over the sites of timeslices [t_begin, t_end) only (4D gauges): in the
// parity-split order those sites are the contiguous run h in [t_begin Vs/2, t_end Vs/2), so the
// warps cover that run from its 8-aligned start and leave the sites outside it alone.  A t-slab
// rank updates its interior slices with it while the boundary links are on their way.
template <typename R, int GAUGE, int ALGO, class F>
__global__ void __launch_bounds__(128) k_parity_pass_range(F f, Geom g, int parity, AlgoParams p, int64_t h_lo,
                                                           int64_t h_hi, int64_t rng_site_offset)
{
    static_assert(GAUGE != COULOMB, "timeslice ranges are for the 4D gauges");
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, mu = lane >> 3;
    const int64_t h0 = (h_lo & ~(int64_t)7) + warp * 8;
    if (h0 >= h_hi) return;  // warp-uniform
    const int64_t h = h0 + (lane & 7);
    const bool active = h >= h_lo && h < h_hi;  // the same for the 4 lanes of a site
    int64_t s = 0, sd = 0;
    Link<R> up, dn;
    if (active) {
        int32_t c[4];
        site_coords(g, h, parity, c);
        s = h + (parity ? g.Vh : 0);
        sd = neighbour_down(g, c, mu);
        load_link<R>(f, s, mu, up);
        load_link<R>(f, sd, mu, dn);
    } else {  // no coupling: the update leaves these (unstored) links alone
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) up.e[i][j] = dn.e[i][j] = cx<R>((R)0, (R)0);
    }
    Rng<R> rng;
    if (ALGO == ALG_SA || ALGO == ALG_SR || ALGO == ALG_RANDOM)
        rng.init(ref_rng_tid(h + rng_site_offset), p.seed, p.counter);  // the whole lattice's stream for a part of it
    site_update<GAUGE, ALGO>(up, dn, mu, p, rng);
    if (active) {
        store_link<R>(f, s, mu, up);
        store_link<R>(f, sd, mu, dn);
    }
}

// ---- gauge quality ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void rows_f64(const R r[12], Link<double> &L)
{
    double d[12];
#pragma unroll
    for (int k = 0; k < 12; k++) d[k] = (double)r[k];
    unpack12(L, d);
    reconstruct(L);
}

template <typename R, class F>
__device__ __forceinline__ void load_link_f64(const F &f, int64_t s, int mu, Link<double> &L)
{
    R r[12];
    f.load12(s, mu, r);
    rows_f64(r, L);
}

// Visit the up link U_mu(x), then the down link U_mu(x - mu), of every direction mu >= mu0, in
// FP64, in the order mu = mu0 .. 3 (so the arithmetic of the visitors runs in that order).  FP32
// fields load the rows of all these links (at most 96 floats) before any arithmetic, so the eight
// loads of a site are in flight together; FP64 fields load one link at a time.
template <typename R, int MU0, class F, class Up, class Down>
__device__ __forceinline__ void visit_site_links(const F &f, const Geom &g, int64_t s, const int32_t c[4], Up up,
                                                 Down down)
{
    if constexpr (sizeof(R) == 4) {
        R ru[4][12], rd[4][12];
#pragma unroll
        for (int mu = MU0; mu < 4; mu++) {
            f.load12(s, mu, ru[mu]);
            f.load12(neighbour_down(g, c, mu), mu, rd[mu]);
        }
#pragma unroll
        for (int mu = MU0; mu < 4; mu++) {
            Link<double> u;
            rows_f64(ru[mu], u);
            up(u);
            rows_f64(rd[mu], u);
            down(u);
        }
    } else {
#pragma unroll 1
        for (int mu = MU0; mu < 4; mu++) {
            Link<double> u;
            load_link_f64<R>(f, s, mu, u);
            up(u);
            load_link_f64<R>(f, neighbour_down(g, c, mu), mu, u);
            down(u);
        }
    }
}

// Per-site functional and theta, computed in FP64 from the stored rows:
//  LANDAU/U1XU1 (LandauKernelsSU3.hxx:114-191, U1xU1KernelsSU3.hxx:114-191) and COULOMB
//  (CoulombKernelsSU3.hxx:110-183, mu = 1..3): gff = sum_mu Re tr U_mu(x);
//  theta = sum_ij |(A - A^dagger)_ij|^2, A = D - tr(D)/3, D = sum_mu U_mu(x) - U_mu(x-mu).
//  MAG (MAGKernelsSU3.hxx:116-223): gff = sum_mu sum_j |U_mu(x)_jj|^2, theta = sum_k |X_k|.
template <int GAUGE, typename R, class F>
__device__ __forceinline__ void quality_site(const F &f, const Geom &g, int64_t s, double &gff, double &th)
{
    const int parity = s >= g.Vh;
    int32_t c[4];
    site_coords(g, s - (parity ? g.Vh : 0), parity, c);
    gff = 0;
    if (GAUGE == MAG) {
        double X[3][2] = {{0, 0}, {0, 0}, {0, 0}};
        Link<double> u;
        visit_site_links<R, 0>(f, g, s, c, [&](const Link<double> &l) { u = l; }, [&](const Link<double> &d) {
            gff += abs2(u.e[0][0]) + abs2(u.e[1][1]) + abs2(u.e[2][2]);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const int i = k == 2 ? 1 : 0, j = k == 0 ? 1 : 2;  // (0,1), (0,2), (1,2)
                const Cx<double> a = u.e[i][i], b = u.e[i][j], cc = u.e[j][i], e = u.e[j][j];
                // up: m00 conj(m10) - m01 conj(m11)
                X[k][0] += (a.x * cc.x + a.y * cc.y) - (b.x * e.x + b.y * e.y);
                X[k][1] += (a.y * cc.x - a.x * cc.y) - (b.y * e.x - b.x * e.y);
                // down, hermitian submatrix: conj(d_ii) d_ij - conj(d_ji) d_jj
                const Cx<double> p = d.e[i][i], q = d.e[i][j], r = d.e[j][i], t = d.e[j][j];
                X[k][0] += (p.x * q.x + p.y * q.y) - (r.x * t.x + r.y * t.y);
                X[k][1] += (p.x * q.y - p.y * q.x) - (r.x * t.y - r.y * t.x);
            }
        });
        th = sqrt(X[0][0] * X[0][0] + X[0][1] * X[0][1]) + sqrt(X[1][0] * X[1][0] + X[1][1] * X[1][1]) +
             sqrt(X[2][0] * X[2][0] + X[2][1] * X[2][1]);
    } else {
        Cx<double> D[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) D[i][j] = cx<double>(0, 0);
        visit_site_links<R, GAUGE == COULOMB ? 1 : 0>(
            f, g, s, c,
            [&](const Link<double> &u) {
                gff += u.e[0][0].x + u.e[1][1].x + u.e[2][2].x;
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        D[i][j].x += u.e[i][j].x;
                        D[i][j].y += u.e[i][j].y;
                    }
            },
            [&](const Link<double> &d) {
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        D[i][j].x -= d.e[i][j].x;
                        D[i][j].y -= d.e[i][j].y;
                    }
            });
        const double trx = (D[0][0].x + D[1][1].x + D[2][2].x) / 3.0;
        const double try_ = (D[0][0].y + D[1][1].y + D[2][2].y) / 3.0;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            D[i][i].x -= trx;
            D[i][i].y -= try_;
        }
        double acc = 0;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const double rx = D[i][j].x - D[j][i].x;  // (A - A^dagger)_ij = A_ij - conj(A_ji)
                const double ry = D[i][j].y + D[j][i].y;
                acc += rx * rx + ry * ry;
            }
        th = acc;
    }
}

// Fixed-order block reduction (warp butterfly, then warps in order): deterministic for a fixed
// launch shape.  Result valid in thread 0.
template <int NT>
__device__ __forceinline__ void block_reduce2(double &a, double &b, bool b_is_max)
{
    __shared__ double sa[NT / 32], sb[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        const double ob = __shfl_xor_sync(0xffffffffu, b, o);
        b = b_is_max ? fmax(b, ob) : b + ob;
    }
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        sa[w] = a;
        sb[w] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = sa[0];
        b = sb[0];
#pragma unroll
        for (int k = 1; k < NT / 32; k++) {
            a += sa[k];
            b = b_is_max ? fmax(b, sb[k]) : b + sb[k];
        }
    }
}

struct QualityOut {
    double *partials;    // 2 doubles per block
    unsigned int *ticket; // zero before the launch; the last block resets it
    double *result;      // [0] = functional, [1] = theta (normalised as the reference does)
    double *gff_site;    // optional per-site arrays (generateGaugeQualityPerSite), may be null
    double *theta_site;
};

// GaugeFixingStats::generateGaugeQuality (GaugeFixingStats.hxx:186-232) in one launch: per-site
// values, per-block partial sums, and the last block to finish sums the partials in block
// order and applies the normalisation gff*preG/V, theta*preA (/V for AVERAGE).
template <int GAUGE, typename R, class F, int NT = 256>
__global__ void __launch_bounds__(NT) k_quality(F f, Geom g, QualityOut o, int stop_max, double preG, double preA)
{
    const int64_t s = (int64_t)blockIdx.x * NT + threadIdx.x;
    double gv = 0, tv = 0;
    if (s < g.V) {
        quality_site<GAUGE, R>(f, g, s, gv, tv);
        if (o.gff_site) o.gff_site[s] = gv;
        if (o.theta_site) o.theta_site[s] = tv;
    }
    block_reduce2<NT>(gv, tv, stop_max != 0);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        o.partials[2 * blockIdx.x] = gv;
        o.partials[2 * blockIdx.x + 1] = tv;
        __threadfence();
        last = atomicAdd(o.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double G = 0, T = 0;
    for (unsigned int k = threadIdx.x; k < gridDim.x; k += NT) {
        G += __ldcg(&o.partials[2 * k]);
        const double t = __ldcg(&o.partials[2 * k + 1]);
        T = stop_max ? fmax(T, t) : T + t;
    }
    block_reduce2<NT>(G, T, stop_max != 0);
    if (threadIdx.x == 0) {
        double gn = G * preG / (double)g.V;
        double tn = T * preA;
        if (!stop_max) tn = tn / (double)g.V;
        o.result[0] = gn;
        o.result[1] = tn;
        *o.ticket = 0;
    }
}

// ---- reprojection (SU3::projectSU3, lattice/SU3.hxx:536-583) in FP64 ---------------------------
__device__ __forceinline__ void project_rows(Link<double> &L)
{
    double nu = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) nu += abs2(L.e[0][i]);
    nu = 1.0 / sqrt(nu);
#pragma unroll
    for (int i = 0; i < 3; i++) L.e[0][i] = cx<double>(L.e[0][i].x * nu, L.e[0][i].y * nu);
    Cx<double> sp = cx<double>(0, 0);  // sum_i row1_i conj(row0_i)
#pragma unroll
    for (int i = 0; i < 3; i++) {
        sp.x += L.e[1][i].x * L.e[0][i].x + L.e[1][i].y * L.e[0][i].y;
        sp.y += L.e[1][i].y * L.e[0][i].x - L.e[1][i].x * L.e[0][i].y;
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const Cx<double> t = cmul(L.e[0][i], sp);
        L.e[1][i].x -= t.x;
        L.e[1][i].y -= t.y;
    }
    double nv = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) nv += abs2(L.e[1][i]);
    nv = 1.0 / sqrt(nv);
#pragma unroll
    for (int i = 0; i < 3; i++) L.e[1][i] = cx<double>(L.e[1][i].x * nv, L.e[1][i].y * nv);
    reconstruct(L);
}

template <typename R>
__global__ void __launch_bounds__(256) k_project_ref(RefField<R> f)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * f.V) return;
    const int mu = (int)(idx / f.V);
    const int64_t s = idx - mu * f.V;
    Link<double> L;
    load_link_f64<R>(f, s, mu, L);
    project_rows(L);
    Link<R> o;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) o.e[i][j] = cx<R>((R)L.e[i][j].x, (R)L.e[i][j].y);
    f.store18(s, mu, o);
}

// ---- random start (COMKSU3::setHot, CommonKernelsSU3.hxx:92-130) -------------------------------
template <int I, int J, typename R>
__device__ __forceinline__ void hot_subgroup(Link<R> &M, Rng<R> &rng)
{
    R q[4];
    q[0] = (R)(rng.rand() * 2.0 - 1.0);
    q[1] = (R)(rng.rand() * 2.0 - 1.0);
    q[2] = (R)(rng.rand() * 2.0 - 1.0);
    q[3] = (R)(rng.rand() * 2.0 - 1.0);
    const R det = rsq(q[0] * q[0] + q[3] * q[3] + q[2] * q[2] + q[1] * q[1]);  // Quaternion::projectSU2
    q[0] *= det;
    q[1] *= det;
    q[2] *= det;
    q[3] *= det;
    right_mult<I, J>(M, q);
}

template <typename R>
__global__ void __launch_bounds__(256) k_set_hot_ref(RefField<R> f, uint32_t seed, uint32_t counter)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= f.V) return;
    Rng<R> rng;
    rng.init((uint32_t)s, seed, counter);
#pragma unroll 1
    for (int mu = 0; mu < 4; mu++) {
        Link<R> M;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) M.e[i][j] = cx<R>(i == j ? (R)1 : (R)0, (R)0);
        hot_subgroup<0, 1>(M, rng);
        hot_subgroup<0, 2>(M, rng);
        hot_subgroup<1, 2>(M, rng);
        f.store18(s, mu, M);
    }
}

}  // namespace gfb
