/*
 * gf_oracle.c -- CPU restatement of the cuLGT gauge-fixing sweep (TEST INFRASTRUCTURE ONLY).
 * See gf_oracle.h.  Built by oracle/Makefile into oracle/liborc.so; loaded only by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg.
 */
#include "gf_oracle.h"
#include "orc_math.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>

/* ---- Philox4x32-10 --------------------------------------------------------------------------
 * The published algorithm (J. Salmon, M. Moraes, R. Dror, D. Shaw, "Parallel random numbers:
 * as easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplications with the constants
 * 0xD2511F53 / 0xCD9E8D57, key bumped by the Weyl constants 0x9E3779B9 / 0xBB67AE85 between
 * rounds.  The reference reaches it through the vendored Random123 header
 * (lattice/rng/PhiloxWrapper.hxx:30-31,98); the known-answer check against that header is in
 * tests/test_oracle_pin.py. */
void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

/* Uniform (0,1) conversions of Random123's u01.h as used by PhiloxWrapper::rand
 * (PhiloxWrapper.hxx:116,128): (1 + (i >> 8)) * 0x1.fffffep-25f and
 * (1 + (i >> 11)) * 0x1.fffffffffffffp-54. */
float orc_u01_open_open_32_24(uint32_t i)
{
    const float f = 16777215.f * (1.f / 16777216.f) * (1.f / 16777216.f);
    return (float)(1 + (i >> 8)) * f;
}

double orc_u01_open_open_64_53(uint64_t i)
{
    const double p53 = 1. / (4294967296. * 2097152.);
    const double f = 9007199254740991. * p53 * p53;
    return (double)(1 + (i >> 11)) * f;
}

/* ---- layout helpers -------------------------------------------------------------------------- */
static int64_t volume(const int32_t size[4])
{
    return (int64_t)size[0] * size[1] * size[2] * size[3];
}

/* SiteCoord::getLatticeIndex, FULL_SPLIT (lattice/SiteCoord.hxx:104-129) */
int64_t orc_site_index(const int32_t size[4], const int32_t x[4])
{
    int64_t parity = 0, index = 0;
    for (int i = 0; i < 4; i++) parity += x[i];
    for (int i = 0; i < 4; i++) index = index * size[i] + x[i];
    if (parity % 2 == 0) return index / 2;
    return index / 2 + volume(size) / 2;
}

/* SiteCoord::setLatticeIndex, FULL_SPLIT (lattice/SiteCoord.hxx:147-175) */
void orc_site_coords(const int32_t size[4], int64_t s, int32_t x[4])
{
    const int64_t V = volume(size);
    int cur;
    if (s >= V / 2) {
        s = (s - V / 2) * 2;
        cur = 1;
    } else {
        s = s * 2;
        cur = 0;
    }
    int64_t parity = 0;
    for (int i = 3; i >= 0; i--) {
        x[i] = (int32_t)(s % size[i]);
        parity += x[i];
        s /= size[i];
    }
    if (parity % 2 != cur) x[3]++;
}

/* SiteCoord::setNeighbour (lattice/SiteCoord.hxx:405-427) */
int64_t orc_neighbour(const int32_t size[4], int64_t s, int mu, int up)
{
    int32_t x[4];
    orc_site_coords(size, s, x);
    x[mu] += up ? 1 : -1;
    if (x[mu] >= size[mu]) x[mu] -= size[mu];
    if (x[mu] < 0) x[mu] += size[mu];
    return orc_site_index(size, x);
}

/* SiteIndex::calculateNeighbourTable (lattice/SiteIndex.hxx:256-284):
 * nn[(2*mu+up)*V + s] = neighbour of s in direction mu (up = 0 backward, 1 forward). */
void orc_neighbour_table(const int32_t size[4], int32_t *nn)
{
    const int64_t V = volume(size);
    for (int64_t l = 0; l < V; l++) {
        int32_t x[4];
        int64_t t = l;
        for (int j = 3; j >= 0; j--) {
            x[j] = (int32_t)(t % size[j]);
            t /= size[j];
        }
        const int64_t s = orc_site_index(size, x);
        for (int j = 0; j < 4; j++) {
            int32_t y[4] = {x[0], x[1], x[2], x[3]};
            y[j]--;
            if (y[j] < 0) y[j] += size[j];
            nn[(2 * j) * V + s] = (int32_t)orc_site_index(size, y);
            y[j] = x[j] + 1;
            if (y[j] >= size[j]) y[j] -= size[j];
            nn[(2 * j + 1) * V + s] = (int32_t)orc_site_index(size, y);
        }
    }
}

/* ---- the two precisions ---------------------------------------------------------------------- */
#define REAL double
#define SFX _f64
#define ORC_IS_DOUBLE 1
#define R_SQRT sqrt
#define R_RSQRT orc_rsqrt_d
#define R_LOG log
#define R_COSPI orc_cospi_d
#define R_SINPI orc_sinpi_d
#include "gf_oracle_impl.h"
#undef REAL
#undef SFX
#undef ORC_IS_DOUBLE
#undef R_SQRT
#undef R_RSQRT
#undef R_LOG
#undef R_COSPI
#undef R_SINPI

#define REAL float
#define SFX _f32
#define ORC_IS_DOUBLE 0
#define R_SQRT sqrtf
#define R_RSQRT orc_rsqrt_f
#define R_LOG logf
#define R_COSPI orc_cospi_f
#define R_SINPI orc_sinpi_f
#include "gf_oracle_impl.h"
