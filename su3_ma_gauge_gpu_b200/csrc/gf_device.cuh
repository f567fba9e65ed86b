// gf_device.cuh -- device-side building blocks of the B200 gauge-fixing sweep.
//
// SU(3) links live in registers as 3x3 complex matrices; only rows 0 and 1 travel to and from
// HBM, row 2 is rebuilt in registers (the reference's 12-parameter trick, lattice/SU3.hxx:639-676).
// A site update is done by FOUR lanes of a warp, one per direction mu: each lane holds the
// up link U_mu(x) and the down link U_mu(x-mu), so the 8 links of a site are spread over 4 lanes
// and the SU(2) subgroup sums are combined with two warp-shuffle butterflies (xor 8, xor 16)
// instead of the reference's shared-memory atomics and __syncthreads rounds
// (gaugefixing/GaugeFixingSubgroupStep.hxx:74-237).  The butterfly gives every lane of a site a
// bit-identical sum, so all four lanes compute the same SU(2) element without a broadcast.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gfb {

// gauge and algorithm codes: the gauge order is the reference's enum GaugeType
// (lattice/datatype/lattice_typedefs.h:43)
enum Gauge : int { LANDAU = 0, COULOMB = 1, MAG = 2, U1XU1 = 3 };
enum Algo : int { ALG_OR = 0, ALG_MICRO = 1, ALG_SA = 2, ALG_SR = 3, ALG_RANDOM = 4 };

template <typename R>
struct Cx {
    R x, y;
};

template <typename R>
__device__ __forceinline__ Cx<R> cx(R x, R y) { return Cx<R>{x, y}; }
template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) { return cx<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename R>
__device__ __forceinline__ Cx<R> cmulcc(Cx<R> a, Cx<R> b)  // conj(a) * conj(b)
{
    return cx<R>(a.x * b.x - a.y * b.y, -(a.x * b.y + a.y * b.x));
}
template <typename R>
__device__ __forceinline__ R abs2(Cx<R> a) { return a.x * a.x + a.y * a.y; }

__device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
__device__ __forceinline__ float sq(float x) { return sqrtf(x); }
__device__ __forceinline__ double sq(double x) { return sqrt(x); }
__device__ __forceinline__ float lg(float x) { return logf(x); }
__device__ __forceinline__ double lg(double x) { return log(x); }
__device__ __forceinline__ float cpi(float x) { return cospif(x); }
__device__ __forceinline__ double cpi(double x) { return cospi(x); }
__device__ __forceinline__ float spi(float x) { return sinpif(x); }
__device__ __forceinline__ double spi(double x) { return sinpi(x); }

template <typename R>
struct Link {
    Cx<R> e[3][3];
};

// row 2 = conj(row0 x row1), normalised (SU3::reconstructThirdLine, lattice/SU3.hxx:655-664)
template <typename R>
__device__ __forceinline__ void reconstruct(Link<R> &L)
{
    Cx<R> a = cmulcc(L.e[0][1], L.e[1][2]), a2 = cmulcc(L.e[0][2], L.e[1][1]);
    Cx<R> b = cmulcc(L.e[0][2], L.e[1][0]), b2 = cmulcc(L.e[0][0], L.e[1][2]);
    Cx<R> c = cmulcc(L.e[0][0], L.e[1][1]), c2 = cmulcc(L.e[0][1], L.e[1][0]);
    a.x -= a2.x; a.y -= a2.y;
    b.x -= b2.x; b.y -= b2.y;
    c.x -= c2.x; c.y -= c2.y;
    R n = rsq(abs2(a) + abs2(b) + abs2(c));
    L.e[2][0] = cx<R>(a.x * n, a.y * n);
    L.e[2][1] = cx<R>(b.x * n, b.y * n);
    L.e[2][2] = cx<R>(c.x * n, c.y * n);
}

template <typename R>
__device__ __forceinline__ void unpack12(Link<R> &L, const R r[12])
{
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) L.e[i][j] = cx<R>(r[2 * (3 * i + j)], r[2 * (3 * i + j) + 1]);
}

template <typename R>
__device__ __forceinline__ void pack12(const Link<R> &L, R r[12])
{
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            r[2 * (3 * i + j)] = L.e[i][j].x;
            r[2 * (3 * i + j) + 1] = L.e[i][j].y;
        }
}

// SU(2) quaternion q of the (I,J) 2x2 block, unnormalised (SU3::getSubgroupQuaternion,
// lattice/SU3.hxx:193-217); the SU(2) <-> 2x2 map is Quaternion::get (Quaternion.hxx:100-131):
// [[q0+i q3, q2+i q1], [-q2+i q1, q0-i q3]]
template <int I, int J, typename R>
__device__ __forceinline__ void subq(const Link<R> &L, R q[4])
{
    q[0] = L.e[I][I].x + L.e[J][J].x;
    q[3] = L.e[I][I].y - L.e[J][J].y;
    q[2] = L.e[I][J].x - L.e[J][I].x;
    q[1] = L.e[I][J].y + L.e[J][I].y;
}

// rows (I,J) <- g * rows (SU3::leftSubgroupMult, lattice/SU3.hxx:702-714)
template <int I, int J, typename R>
__device__ __forceinline__ void left_mult(Link<R> &L, const R g[4])
{
    const Cx<R> g00 = cx<R>(g[0], g[3]), g01 = cx<R>(g[2], g[1]);
    const Cx<R> g10 = cx<R>(-g[2], g[1]), g11 = cx<R>(g[0], -g[3]);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        Cx<R> a = cmul(g00, L.e[I][k]), b = cmul(g01, L.e[J][k]);
        Cx<R> c = cmul(g10, L.e[I][k]), d = cmul(g11, L.e[J][k]);
        L.e[I][k] = cx<R>(a.x + b.x, a.y + b.y);
        L.e[J][k] = cx<R>(c.x + d.x, c.y + d.y);
    }
}

// cols (I,J) <- cols * h (SU3::rightSubgroupMult, lattice/SU3.hxx:682-697)
template <int I, int J, typename R>
__device__ __forceinline__ void right_mult(Link<R> &L, const R h[4])
{
    const Cx<R> h00 = cx<R>(h[0], h[3]), h01 = cx<R>(h[2], h[1]);
    const Cx<R> h10 = cx<R>(-h[2], h[1]), h11 = cx<R>(h[0], -h[3]);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        Cx<R> a = cmul(h00, L.e[k][I]), b = cmul(h10, L.e[k][J]);
        Cx<R> c = cmul(h01, L.e[k][I]), d = cmul(h11, L.e[k][J]);
        L.e[k][I] = cx<R>(a.x + b.x, a.y + b.y);
        L.e[k][J] = cx<R>(c.x + d.x, c.y + d.y);
    }
}

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ---------------------------------------
// Not inlined: a heat-bath site update draws from up to eight call sites per subgroup, three
// subgroups per update, and inlined copies of the ten rounds made the kernel's code outgrow the
// instruction cache (the SA pass stalled on instruction fetch more than on anything else).
static __device__ __noinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k.x += 0x9E3779B9u;
            k.y += 0xBB67AE85u;
        }
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

// The reference's per-thread generator (lattice/rng/PhiloxWrapper.hxx:92-137): key = (tid, seed),
// counter = (k, launch counter, 0x12345678, 0xabcdef09), the k = 0 block discarded; floats are
// drawn i[3], i[2], i[1], i[0] from each block, doubles i64[1], i64[0].
template <typename R>
struct Rng {
    uint2 key;
    uint4 ctr;
    uint4 res;
    int local;
    __device__ __forceinline__ void init(uint32_t tid, uint32_t seed, uint32_t counter)
    {
        key = make_uint2(tid, seed);
        ctr = make_uint4(0u, counter, 0x12345678u, 0xabcdef09u);
        local = 0;
    }
    __device__ __forceinline__ R rand();
};

// u01_open_open_32_24 / _64_53 of Random123's u01.h: (1 + (i >> 8)) * 0x1.fffffep-25f and
// (1 + (i >> 11)) * 0x1.fffffffffffffp-54
template <>
__device__ __forceinline__ float Rng<float>::rand()
{
    if (local == 0) {
        local = 3;
        ctr.x++;
        res = philox4x32_10(ctr, key);
    } else {
        local--;
    }
    const uint32_t v = local == 3 ? res.w : (local == 2 ? res.z : (local == 1 ? res.y : res.x));
    return (float)(1u + (v >> 8)) * 0x1.fffffep-25f;
}

template <>
__device__ __forceinline__ double Rng<double>::rand()
{
    if (local == 0) {
        local = 1;
        ctr.x++;
        res = philox4x32_10(ctr, key);
    } else {
        local--;
    }
    const uint64_t v = local == 1 ? (((uint64_t)res.w << 32) | res.z) : (((uint64_t)res.y << 32) | res.x);
    return (double)(1ull + (v >> 11)) * 0x1.fffffffffffffp-54;
}

// ---- update rules on the accumulated 4-vector (gaugefixing/algorithms/*Update.hxx) ----------
struct AlgoParams {
    float param;      // OR omega, SA temperature, SR probability
    uint32_t seed;
    uint32_t counter;
    uint32_t counter_stride;  // batches: 0 = instance i draws key word seed + i; > 0 = every instance draws
                              // key word seed, instance i from launch counter counter + i * counter_stride
};

// Philox key word and launch counter of instance i of a batch.  By default every instance has a
// stream of its own (key word seed + i, the same counters).  With counter_stride > 0 the instances
// continue one stream, as the reference apps do when they fix gauge copies or timeslices one after
// the other (PhiloxWrapper::getNextCounter is one process-wide counter, lattice/rng/PhiloxWrapper.hxx:
// 90,142-145): key word seed, instance i starting counter_stride launches after instance i - 1.
__host__ __device__ __forceinline__ uint32_t inst_seed(const AlgoParams &p, int i)
{
    return p.counter_stride ? p.seed : p.seed + (uint32_t)i;
}
__host__ __device__ __forceinline__ uint32_t inst_counter(const AlgoParams &p, int i)
{
    return p.counter + (uint32_t)i * p.counter_stride;
}

// OrUpdate::calculateUpdate (OrUpdate.hxx:66-75)
template <typename R>
__device__ __forceinline__ void upd_or(R a[4], float omega)
{
    const R ai_sq = a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
    const R a0_sq = a[0] * a[0];
    if (!(a0_sq + ai_sq > (R)0)) {  // no coupling (every contribution cancelled): leave the site
        a[0] = 1;
        a[1] = a[2] = a[3] = 0;
        return;
    }
    const R b = (omega * a0_sq + ai_sq) / (a0_sq + ai_sq);
    const R c = rsq(a0_sq + b * b * ai_sq);
    const R bc = b * c;
    a[0] *= c;
    a[1] *= bc;
    a[2] *= bc;
    a[3] *= bc;
}

// MicroUpdate::calculateUpdate (MicroUpdate.hxx:55-64)
template <typename R>
__device__ __forceinline__ void upd_micro(R a[4])
{
    const R ai_sq = a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
    const R a0_sq = a[0] * a[0];
    const R n = a0_sq + ai_sq;
    if (!(n > (R)0)) {  // no coupling: the reflection is undefined, leave the site
        a[0] = 1;
        a[1] = a[2] = a[3] = 0;
        return;
    }
    const R b = (R)2. * a[0] / n;
    a[0] = (a0_sq - ai_sq) / n;
    a[1] *= b;
    a[2] *= b;
    a[3] *= b;
}

// Kennedy-Pendleton heat-bath, SaUpdate::calculateUpdate (SaUpdate.hxx:103-146).  The literal
// types follow the reference (double constants, cospi of a double argument), so the FP32
// variant promotes where the reference promotes.  Every rejection loop is bounded (2^16 draws).
// The inner loops accept with probability >= 0.9999 per draw; the outer one accepts rarely when
// p0 = T/|a| is large (a site whose subgroup coupling |a| is tiny against the temperature), and
// there the reference would keep drawing.  Such a site -- the outer bound exhausted, or |a| = 0
// -- takes a0 from the p0 -> infinity limit of the same distribution, the Haar measure (density
// proportional to sqrt(1 - a0^2), sampled by rejection), instead of the unaccepted 1 - delta,
// whose square root below would be NaN for delta > 2.
template <typename R>
__device__ __forceinline__ void upd_sa(R a[4], float temperature, Rng<R> &rng)
{
    R e0 = a[0], e1 = -a[1], e2 = -a[2], e3 = -a[3];
    const R nrm2 = e0 * e0 + e1 * e1 + e2 * e2 + e3 * e3;
    const bool flat = !(nrm2 > (R)0);  // no coupling: the local distribution is Haar
    const R dk = flat ? (R)1 : rsq(nrm2);
    if (flat) {
        e0 = 1;
        e1 = e2 = e3 = 0;
    }
    const R p0 = dk * temperature;
    R r1, r2, r3, r4, delta = 0;
    bool accepted = false;
    int guard = 0;
    if (!flat) {
        do {
            int g1 = 0, g2 = 0;
            do { r1 = rng.rand(); } while (r1 < 0.0001 && ++g1 < 65536);
            r1 = -lg(r1) * p0;
            do { r2 = rng.rand(); } while (r2 < 0.0001 && ++g2 < 65536);
            r2 = -lg(r2) * p0;
            r3 = (R)cospi(2.0 * (double)rng.rand());
            r3 = r3 * r3;
            delta = r2 + r1 * r3;
            r4 = rng.rand();
            accepted = !(r4 * r4 > (1.0 - 0.5 * delta));
        } while (!accepted && ++guard < 65536);
    }
    R a0 = (R)(1.0 - delta);
    if (!accepted) {
        int g = 0;
        do {
            a0 = (R)(2.0 * rng.rand() - 1.0);
            r4 = rng.rand();
        } while (r4 * r4 > (R)1 - a0 * a0 && ++g < 64);
    }
    const R cos_theta = (R)(2.0 * rng.rand() - 1.0);
    const R sin_theta = (R)sqrt(1.0 - (double)(cos_theta * cos_theta));
    const R sin_alpha = sq((R)(1 - a0 * a0));
    const R phi = (R)(2.0 * rng.rand());
    const R a1 = sin_alpha * sin_theta * cpi(phi);
    const R a2 = sin_alpha * sin_theta * spi(phi);
    const R a3 = sin_alpha * cos_theta;
    e0 *= dk;
    e1 *= dk;
    e2 *= dk;
    e3 *= dk;
    a[0] = a0 * e0 + a3 * e3 + a2 * e2 + e1 * a1;
    a[3] = e0 * a3 - e3 * a0 + a1 * e2 - a2 * e1;
    a[2] = a3 * e1 - a0 * e2 + a2 * e0 - a1 * e3;
    a[1] = a2 * e3 + a1 * e0 - a3 * e2 - e1 * a0;
}

// SrUpdate::calculateUpdate (SrUpdate.hxx:76-94): with probability p square the quaternion
template <typename R>
__device__ __forceinline__ void upd_sr(R a[4], float p, Rng<R> &rng)
{
    const R u = rng.rand();
    const R a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3];
    if (u < p) {
        a[0] = a0 * a0 - a1 * a1 - a2 * a2 - a3 * a3;
        a[1] = (R)(2.0 * a0 * a1);
        a[2] = (R)(2.0 * a0 * a2);
        a[3] = (R)(2.0 * a0 * a3);
    }
    const R c = rsq(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3]);
    a[0] *= c;
    a[1] *= c;
    a[2] *= c;
    a[3] *= c;
}

// RandomUpdate::calculateUpdate (RandomUpdate.hxx:47-59): uniform random SU(2) element
template <typename R>
__device__ __forceinline__ void upd_random(R a[4], Rng<R> &rng)
{
    const R alpha = rng.rand();
    const R phi = (R)(2.0 * rng.rand());
    const R cos_theta = (R)(2.0 * rng.rand() - 1.0);
    const R sin_theta = (R)sqrt(1.0 - (double)(cos_theta * cos_theta));
    const R sin_alpha = spi(alpha);
    a[0] = cpi(alpha);
    a[1] = sin_alpha * sin_theta * cpi(phi);
    a[2] = sin_alpha * sin_theta * spi(phi);
    a[3] = sin_alpha * cos_theta;
}

template <int ALGO, typename R>
__device__ __forceinline__ void apply_algo(R a[4], const AlgoParams &p, Rng<R> &rng)
{
    if (ALGO == ALG_OR) upd_or(a, p.param);
    else if (ALGO == ALG_MICRO) upd_micro(a);
    else if (ALGO == ALG_SA) upd_sa(a, p.param, rng);
    else if (ALGO == ALG_SR) upd_sr(a, p.param, rng);
    else upd_random(a, rng);
}

// sum over the four lanes of one site (lanes l, l^8, l^16, l^24); the butterfly leaves the same
// bits in all four lanes
template <typename R>
__device__ __forceinline__ R site_sum(R v)
{
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    return v;
}

// One SU(2) subgroup step of GaugeFixingSubgroupStep::subgroup for the gauge GAUGE, done by the
// lane that holds direction mu of the site (LANDAU/COULOMB :99-237, U1xU1 :238-353, MAG :354-589).
// Refine mode: column k of D = W - 1, the deviation of the site's accumulated gauge
// transformation from the identity, under W <- g W:  D' = D + (g - 1)(1 + D) on rows (I, J).
// g - 1 is formed without cancellation (g0 - 1 = -|g_vec|^2 / (1 + g0)), so near convergence, where
// the folds keep W close to 1, D carries the small rotations to FP32 relative accuracy instead of
// rounding them against the unit diagonal.
template <int I, int J, typename R>
__device__ __forceinline__ void left_mult_dcolumn(Cx<R> (&col)[3], const R g[4], int k)
{
    const R v2 = g[1] * g[1] + g[2] * g[2] + g[3] * g[3];
    const R em = g[0] >= (R)0 ? -v2 / ((R)1 + g[0]) : g[0] - (R)1;
    const Cx<R> a = cx<R>(col[I].x + (k == I ? (R)1 : (R)0), col[I].y);
    const Cx<R> b = cx<R>(col[J].x + (k == J ? (R)1 : (R)0), col[J].y);
    const Cx<R> p0 = cmul(cx<R>(em, g[3]), a), p1 = cmul(cx<R>(g[2], g[1]), b);
    const Cx<R> q0 = cmul(cx<R>(-g[2], g[1]), a), q1 = cmul(cx<R>(em, -g[3]), b);
    col[I] = cx<R>(col[I].x + (p0.x + p1.x), col[I].y + (p0.y + p1.y));
    col[J] = cx<R>(col[J].x + (q0.x + q1.x), col[J].y + (q0.y + q1.y));
}

// Contribution of direction mu (its up link U_mu(x) and down link U_mu(x-mu)) to the subgroup
// quaternion w of the site, before the sum over mu (GaugeFixingSubgroupStep.hxx:99-237 Landau and
// Coulomb, :238-353 U1xU1, :354-589 MAG; MAG's factor 2 and square root follow the sum).
template <int GAUGE, int I, int J, typename R>
__device__ __forceinline__ void subgroup_contrib(const Link<R> &up, const Link<R> &dn, int mu, R v[4])
{
    if (GAUGE == MAG) {
        const Cx<R> u00 = up.e[I][I], u01 = up.e[I][J], u10 = up.e[J][I], u11 = up.e[J][J];
        const Cx<R> d00 = dn.e[I][I], d01 = dn.e[I][J], d10 = dn.e[J][I], d11 = dn.e[J][J];
        const R Du = abs2(u00) - abs2(u01) - abs2(u10) + abs2(u11);
        const R Dd = abs2(d00) - abs2(d01) - abs2(d10) + abs2(d11);
        // up:   c = m00 conj(m10) - m01 conj(m11);  down: c = conj(m00) m01 - conj(m10) m11
        const R cux = (u00.x * u10.x + u00.y * u10.y) - (u01.x * u11.x + u01.y * u11.y);
        const R cuy = (u00.y * u10.x - u00.x * u10.y) - (u01.y * u11.x - u01.x * u11.y);
        const R cdx = (d00.x * d01.x + d00.y * d01.y) - (d10.x * d11.x + d10.y * d11.y);
        const R cdy = (d00.x * d01.y - d00.y * d01.x) - (d10.x * d11.y - d10.y * d11.x);
        v[0] = Du + Dd;
        v[1] = cuy + cdy;
        v[2] = cux + cdx;
        v[3] = 0;
    } else {
        R qu[4], qd[4];
        subq<I, J>(up, qu);
        subq<I, J>(dn, qd);
        const bool skip = (GAUGE == COULOMB) && (mu == 0);  // Coulomb: mu = 0 not in the sum
        if (GAUGE == U1XU1) {
            v[0] = qu[0] + qd[0];
            v[1] = 0;
            v[2] = 0;
            v[3] = qd[3] - qu[3];
        } else {
            v[0] = skip ? (R)0 : qu[0] + qd[0];
            v[1] = skip ? (R)0 : qd[1] - qu[1];
            v[2] = skip ? (R)0 : qd[2] - qu[2];
            v[3] = skip ? (R)0 : qd[3] - qu[3];
        }
    }
}

// From the summed quaternion to the update g (in place): MAG's factor 2 and square root, the
// update rule, and the U1xU1 / MAG renormalisation.
template <int GAUGE, int ALGO, typename R>
__device__ __forceinline__ void subgroup_finish(R w[4], const AlgoParams &p, Rng<R> &rng)
{
    if (GAUGE == MAG) {
        w[1] *= (R)2.;  // the factor 2 of GaugeFixingSubgroupStep.hxx:535-536
        w[2] *= (R)2.;
        w[3] = 0;
        w[0] = w[0] + sq(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    } else if (GAUGE == U1XU1) {
        w[1] = 0;
        w[2] = 0;
    }
    apply_algo<ALGO>(w, p, rng);
    if (GAUGE == U1XU1) {
        w[1] = 0;
        w[2] = 0;
        const R n = rsq(w[0] * w[0] + w[3] * w[3]);
        w[0] *= n;
        w[3] *= n;
    } else if (GAUGE == MAG) {
        w[3] = 0;
        const R n = rsq(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        w[0] *= n;
        w[1] *= n;
        w[2] *= n;
    }
}

template <int GAUGE, int ALGO, int I, int J, typename R, bool SITE_W = false>
__device__ __forceinline__ void subgroup_step(Link<R> &up, Link<R> &dn, int mu, const AlgoParams &p, Rng<R> &rng,
                                              Cx<R> (*wcol)[3] = nullptr)
{
    R v[4], w[4];
    subgroup_contrib<GAUGE, I, J>(up, dn, mu, v);
    w[0] = site_sum(v[0]);
    w[1] = (GAUGE == U1XU1) ? (R)0 : site_sum(v[1]);
    w[2] = (GAUGE == U1XU1) ? (R)0 : site_sum(v[2]);
    w[3] = (GAUGE == MAG) ? (R)0 : site_sum(v[3]);
    subgroup_finish<GAUGE, ALGO>(w, p, rng);
    left_mult<I, J>(up, w);
    const R h[4] = {w[0], -w[1], -w[2], -w[3]};
    right_mult<I, J>(dn, h);
    if (SITE_W) left_mult_dcolumn<I, J>(*wcol, w, mu & 1);
}

// One thread per site: the same subgroup step with all 8 links of the site in the thread.  The
// sum over mu is taken in the order of the 4-lane butterfly, (v0 + v1) + (v2 + v3), so both
// layouts do the same arithmetic (the compiler may still contract a product differently in the
// two kernels).  With SITE_W the thread applies g to both tracked columns of D = W - 1.
template <int GAUGE, int ALGO, int I, int J, typename R, bool SITE_W = false>
__device__ __forceinline__ void subgroup_step_site(Link<R> (&up)[4], Link<R> (&dn)[4], const AlgoParams &p,
                                                   Rng<R> &rng, Cx<R> (*wcols)[2][3] = nullptr)
{
    R v[4][4], w[4];
#pragma unroll
    for (int mu = 0; mu < 4; mu++) subgroup_contrib<GAUGE, I, J>(up[mu], dn[mu], mu, v[mu]);
#pragma unroll
    for (int k = 0; k < 4; k++) w[k] = (v[0][k] + v[1][k]) + (v[2][k] + v[3][k]);
    if (GAUGE == U1XU1) w[1] = w[2] = 0;
    if (GAUGE == MAG) w[3] = 0;
    subgroup_finish<GAUGE, ALGO>(w, p, rng);
    const R h[4] = {w[0], -w[1], -w[2], -w[3]};
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
        left_mult<I, J>(up[mu], w);
        right_mult<I, J>(dn[mu], h);
    }
    if (SITE_W) {
        left_mult_dcolumn<I, J>((*wcols)[0], w, 0);
        left_mult_dcolumn<I, J>((*wcols)[1], w, 1);
    }
}

// Two lanes per site: lane `role` (0 or 1; its partner is lane ^ 16) holds directions 2*role and
// 2*role + 1, each as its up link U_mu(x) and down link U_mu(x - mu).  The quaternion sum is
// (v0 + v1) + (v2 + v3) -- the additions of the 4-lane butterfly, in the same order -- and both
// lanes compute the same g.  Each lane then updates its four links, and with SITE_W column `role`
// of the site's D = W - 1, so no lane repeats another's work except the SU(2) update itself.
template <int GAUGE, int ALGO, int I, int J, typename R, bool SITE_W>
__device__ __forceinline__ void subgroup_step_pair(Link<R> (&up)[2], Link<R> (&dn)[2], int role, const AlgoParams &p,
                                                   Rng<R> &rng, Cx<R> (*wcol)[3])
{
    R a[4], b[4], w[4];
    subgroup_contrib<GAUGE, I, J>(up[0], dn[0], 2 * role, a);
    subgroup_contrib<GAUGE, I, J>(up[1], dn[1], 2 * role + 1, b);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const bool zero = (GAUGE == U1XU1 && (k == 1 || k == 2)) || (GAUGE == MAG && k == 3);
        const R v = a[k] + b[k];
        w[k] = zero ? (R)0 : v + __shfl_xor_sync(0xffffffffu, v, 16);
    }
    subgroup_finish<GAUGE, ALGO>(w, p, rng);
    const R h[4] = {w[0], -w[1], -w[2], -w[3]};
#pragma unroll
    for (int j = 0; j < 2; j++) {
        left_mult<I, J>(up[j], w);
        right_mult<I, J>(dn[j], h);
    }
    if (SITE_W) left_mult_dcolumn<I, J>(*wcol, w, role);
}

template <int GAUGE, int ALGO, typename R, bool SITE_W = false>
__device__ __forceinline__ void site_update_pair(Link<R> (&up)[2], Link<R> (&dn)[2], int role, const AlgoParams &p,
                                                 Rng<R> &rng, Cx<R> (*wcol)[3] = nullptr)
{
    subgroup_step_pair<GAUGE, ALGO, 0, 2, R, SITE_W>(up, dn, role, p, rng, wcol);
    subgroup_step_pair<GAUGE, ALGO, 1, 2, R, SITE_W>(up, dn, role, p, rng, wcol);
    subgroup_step_pair<GAUGE, ALGO, 0, 1, R, SITE_W>(up, dn, role, p, rng, wcol);
}

// the three subgroups in the reference order (0,2), (1,2), (0,1) (SU3::perSubgroup, SU3.hxx:762-771);
// with SITE_W the lane also applies every g to its column (mu & 1) of the site's D = W - 1
template <int GAUGE, int ALGO, typename R, bool SITE_W = false>
__device__ __forceinline__ void site_update(Link<R> &up, Link<R> &dn, int mu, const AlgoParams &p, Rng<R> &rng,
                                            Cx<R> (*wcol)[3] = nullptr)
{
    subgroup_step<GAUGE, ALGO, 0, 2, R, SITE_W>(up, dn, mu, p, rng, wcol);
    subgroup_step<GAUGE, ALGO, 1, 2, R, SITE_W>(up, dn, mu, p, rng, wcol);
    subgroup_step<GAUGE, ALGO, 0, 1, R, SITE_W>(up, dn, mu, p, rng, wcol);
}

template <int GAUGE, int ALGO, typename R, bool SITE_W = false>
__device__ __forceinline__ void site_update_thread(Link<R> (&up)[4], Link<R> (&dn)[4], const AlgoParams &p,
                                                   Rng<R> &rng, Cx<R> (*wcols)[2][3] = nullptr)
{
    subgroup_step_site<GAUGE, ALGO, 0, 2, R, SITE_W>(up, dn, p, rng, wcols);
    subgroup_step_site<GAUGE, ALGO, 1, 2, R, SITE_W>(up, dn, p, rng, wcols);
    subgroup_step_site<GAUGE, ALGO, 0, 1, R, SITE_W>(up, dn, p, rng, wcols);
}

// ---- lattice geometry -----------------------------------------------------------------------
// Division by a lattice extent without a divide instruction: for 0 <= n < 2^31 and d >= 1,
// q = (umulhi(n, m) + n) >> s with s = ceil(log2 d), m = floor(2^32 (2^s - d) / d) + 1
// (Granlund & Montgomery, "Division by invariant integers using multiplication", PLDI 1994).
struct FastDiv {
    uint32_t d, m, s;
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const { return (__umulhi_any(n, m) + n) >> s; }

  private:
    __host__ __device__ static __forceinline__ uint32_t __umulhi_any(uint32_t a, uint32_t b)
    {
#ifdef __CUDA_ARCH__
        return __umulhi(a, b);
#else
        return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
    }
};

inline FastDiv make_fastdiv(uint32_t d)
{
    uint32_t s = 0;
    while ((1ull << s) < d) s++;
    const uint64_t m = ((uint64_t(1) << 32) * ((uint64_t(1) << s) - d)) / d + 1;
    return FastDiv{d, (uint32_t)m, s};
}

// Parity-split site order of the reference (SiteCoord.hxx:104-175): lexicographic l =
// ((t*Nx + x)*Ny + y)*Nz + z, s = l/2 (+V/2 for odd t+x+y+z).  All extents must be even and
// V < 2^31, so site arithmetic is 32-bit.
struct Geom {
    int32_t n[4];   // Nt, Nx, Ny, Nz
    int64_t V, Vh;
    FastDiv dx, dy, dz;
};

inline void geom_init_div(Geom &g)
{
    g.dx = make_fastdiv((uint32_t)g.n[1]);
    g.dy = make_fastdiv((uint32_t)g.n[2]);
    g.dz = make_fastdiv((uint32_t)g.n[3]);
}

__device__ __forceinline__ void site_coords(const Geom &g, int64_t h64, int parity, int32_t c[4])
{
    uint32_t l = 2u * (uint32_t)h64;
    uint32_t q = g.dz.div(l);
    c[3] = (int32_t)(l - q * g.dz.d);
    l = q;
    q = g.dy.div(l);
    c[2] = (int32_t)(l - q * g.dy.d);
    l = q;
    q = g.dx.div(l);
    c[1] = (int32_t)(l - q * g.dx.d);
    c[0] = (int32_t)q;
    if (((c[0] + c[1] + c[2] + c[3]) & 1) != parity) c[3] += 1;
}

__device__ __forceinline__ int64_t site_index(const Geom &g, const int32_t c[4])
{
    const uint32_t l = (((uint32_t)c[0] * g.n[1] + c[1]) * g.n[2] + c[2]) * g.n[3] + c[3];
    return (int64_t)(l >> 1) + (((c[0] + c[1] + c[2] + c[3]) & 1) ? g.Vh : 0);
}

// forward neighbour x + mu of the site with coordinates c
__device__ __forceinline__ int64_t neighbour_up(const Geom &g, const int32_t c[4], int mu)
{
    int32_t d[4];
#pragma unroll
    for (int k = 0; k < 4; k++) d[k] = (mu == k) ? ((c[k] + 1 == g.n[k]) ? 0 : c[k] + 1) : c[k];
    return site_index(g, d);
}

// backward neighbour x - mu of the site with coordinates c (mu is lane-dependent, so the
// coordinate arrays are only ever indexed with constants: no local-memory spill)
__device__ __forceinline__ int64_t neighbour_down(const Geom &g, const int32_t c[4], int mu)
{
    int32_t d[4];
#pragma unroll
    for (int k = 0; k < 4; k++) d[k] = (mu == k) ? ((c[k] == 0 ? g.n[k] : c[k]) - 1) : c[k];
    return site_index(g, d);
}

}  // namespace gfb
