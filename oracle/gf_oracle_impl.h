/*
 * gf_oracle_impl.h -- precision-generic body of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 * Included twice by gf_oracle.c, with REAL = double / float and SFX = _f64 / _f32.
 *
 * Expression order and C type promotion follow the reference's device code line by line so
 * that the FP64 build is bit-identical to the reference's host-compiled templates (checked by
 * tests/test_oracle_pin.py).  Citations are paths inside the reference's src/ tree.
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)
#define CPX FN(orc_cpx)
#define MAT FN(orc_mat)
#define RNG FN(orc_rng)

typedef struct { REAL x, y; } CPX;            /* lattice/Complex.hxx:28-48 */
typedef struct { CPX m[3][3]; } MAT;          /* lattice/Matrix.hxx (row-major 3x3) */

static inline CPX FN(cmake)(REAL x, REAL y) { CPX c; c.x = x; c.y = y; return c; }
static inline CPX FN(conj)(CPX a) { return FN(cmake)(a.x, -a.y); }
/* Complex::operator*= (Complex.hxx:148-154): x = re*a.x - im*a.y; y = re*a.y + im*a.x */
static inline CPX FN(cmul)(CPX a, CPX b) { return FN(cmake)(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
static inline CPX FN(cadd)(CPX a, CPX b) { return FN(cmake)(a.x + b.x, a.y + b.y); }
static inline CPX FN(csub)(CPX a, CPX b) { return FN(cmake)(a.x - b.x, a.y - b.y); }
static inline REAL FN(abs2)(CPX a) { return a.x * a.x + a.y * a.y; }

/* ---- Philox-driven rand() of lattice/rng/PhiloxWrapper.hxx:92-137 ---------------------- */
typedef struct {
    uint32_t key[2], ctr[4], res[4];
    int local;
} RNG;

static void FN(rng_init)(RNG *r, uint32_t tid, uint32_t seed, uint32_t counter)
{
    /* PhiloxWrapper.hxx:92-102: key = (tid, seed); ctr = (0, counter, 0x12345678, 0xabcdef09);
     * the block for ctr[0] = 0 is computed and then discarded by the first rand(). */
    r->key[0] = tid;
    r->key[1] = seed;
    r->ctr[0] = 0;
    r->ctr[1] = counter;
    r->ctr[2] = 0x12345678u;
    r->ctr[3] = 0xabcdef09u;
    orc_philox4x32_10(r->ctr, r->key, r->res);
    r->local = 0;
}

static REAL FN(rng_rand)(RNG *r)
{
#if ORC_IS_DOUBLE
    /* PhiloxWrapper.hxx:108-117: two doubles per block, i64[1] first, then i64[0] */
    if (r->local == 0) {
        r->local = 1;
        r->ctr[0]++;
        orc_philox4x32_10(r->ctr, r->key, r->res);
    } else {
        r->local--;
    }
    uint64_t v = (uint64_t)r->res[2 * r->local] | ((uint64_t)r->res[2 * r->local + 1] << 32);
    return orc_u01_open_open_64_53(v);
#else
    /* PhiloxWrapper.hxx:121-129: four floats per block, i[3], i[2], i[1], i[0] */
    if (r->local == 0) {
        r->local = 3;
        r->ctr[0]++;
        orc_philox4x32_10(r->ctr, r->key, r->res);
    } else {
        r->local--;
    }
    return orc_u01_open_open_32_24(r->res[r->local]);
#endif
}

void FN(orc_rand_sequence)(uint32_t tid, uint32_t seed, uint32_t counter, int n, double *out)
{
    RNG r;
    FN(rng_init)(&r, tid, seed, counter);
    for (int i = 0; i < n; i++) out[i] = (double)FN(rng_rand)(&r);
}

/* ---- link load/store in the GpuPattern layout ------------------------------------------- */
/* GpuPattern::getIndex (access_pattern/GpuPattern.hxx:53-56):
 *   idx = s + V*(c + 2*(j + 3*(i + 3*mu))) */
static inline int64_t FN(gidx)(int64_t V, int64_t s, int mu, int i, int j, int c)
{
    return s + V * (int64_t)(c + 2 * (j + 3 * (i + 3 * mu)));
}

/* SU3::reconstructThirdLine (lattice/SU3.hxx:639-676): row2 = conj(row0 x row1), normalised */
static void FN(reconstruct)(MAT *M)
{
    CPX a = FN(csub)(FN(cmul)(FN(conj)(M->m[0][1]), FN(conj)(M->m[1][2])),
                     FN(cmul)(FN(conj)(M->m[0][2]), FN(conj)(M->m[1][1])));
    CPX b = FN(csub)(FN(cmul)(FN(conj)(M->m[0][2]), FN(conj)(M->m[1][0])),
                     FN(cmul)(FN(conj)(M->m[0][0]), FN(conj)(M->m[1][2])));
    CPX c = FN(csub)(FN(cmul)(FN(conj)(M->m[0][0]), FN(conj)(M->m[1][1])),
                     FN(cmul)(FN(conj)(M->m[0][1]), FN(conj)(M->m[1][0])));
    REAL norm = FN(abs2)(a) + FN(abs2)(b) + FN(abs2)(c);
    norm = 1. / R_SQRT(norm);
    M->m[2][0] = FN(cmake)(a.x * norm, a.y * norm);
    M->m[2][1] = FN(cmake)(b.x * norm, b.y * norm);
    M->m[2][2] = FN(cmake)(c.x * norm, c.y * norm);
}

/* SU3::assignWithoutThirdLine from a Link (SU3.hxx:320-328, Link.hxx:111-127) + reconstruct */
static void FN(load12)(const REAL *U, int64_t V, int64_t s, int mu, MAT *M)
{
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 3; j++)
            M->m[i][j] = FN(cmake)(U[FN(gidx)(V, s, mu, i, j, 0)], U[FN(gidx)(V, s, mu, i, j, 1)]);
    FN(reconstruct)(M);
}

static void FN(store12)(REAL *U, int64_t V, int64_t s, int mu, const MAT *M)
{
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 3; j++) {
            U[FN(gidx)(V, s, mu, i, j, 0)] = M->m[i][j].x;
            U[FN(gidx)(V, s, mu, i, j, 1)] = M->m[i][j].y;
        }
}

/* ---- SU(2) subgroup helpers --------------------------------------------------------------- */
/* SU3::getSubgroupQuaternion (SU3.hxx:193-217) */
static void FN(subq)(const MAT *M, int i, int j, REAL q[4])
{
    CPX t = M->m[i][i];
    q[0] = t.x;
    q[3] = t.y;
    t = M->m[j][j];
    q[0] += t.x;
    q[3] -= t.y;
    t = M->m[i][j];
    q[2] = t.x;
    q[1] = t.y;
    t = M->m[j][i];
    q[2] -= t.x;
    q[1] += t.y;
}

/* Quaternion::get (Quaternion.hxx:100-131): [[q0+iq3, q2+iq1], [-q2+iq1, q0-iq3]] */
static inline CPX FN(qget)(const REAL q[4], int i, int j)
{
    if (i == 0) return j == 0 ? FN(cmake)(q[0], q[3]) : FN(cmake)(q[2], q[1]);
    return j == 0 ? FN(cmake)(-q[2], q[1]) : FN(cmake)(q[0], -q[3]);
}

/* SU3::leftSubgroupMult (SU3.hxx:702-714): rows (i,j) <- q * rows */
static void FN(left_mult)(MAT *M, int i, int j, const REAL q[4])
{
    for (int k = 0; k < 3; k++) {
        CPX IK = FN(cmul)(FN(qget)(q, 0, 0), M->m[i][k]);
        IK = FN(cadd)(IK, FN(cmul)(FN(qget)(q, 0, 1), M->m[j][k]));
        CPX JK = FN(cmul)(FN(qget)(q, 1, 0), M->m[i][k]);
        JK = FN(cadd)(JK, FN(cmul)(FN(qget)(q, 1, 1), M->m[j][k]));
        M->m[i][k] = IK;
        M->m[j][k] = JK;
    }
}

/* SU3::rightSubgroupMult (SU3.hxx:682-697): cols (i,j) <- cols * q */
static void FN(right_mult)(MAT *M, int i, int j, const REAL q[4])
{
    for (int k = 0; k < 3; k++) {
        CPX KI = FN(cmul)(FN(qget)(q, 0, 0), M->m[k][i]);
        KI = FN(cadd)(KI, FN(cmul)(FN(qget)(q, 1, 0), M->m[k][j]));
        CPX KJ = FN(cmul)(FN(qget)(q, 0, 1), M->m[k][i]);
        KJ = FN(cadd)(KJ, FN(cmul)(FN(qget)(q, 1, 1), M->m[k][j]));
        M->m[k][i] = KI;
        M->m[k][j] = KJ;
    }
}

/* ---- update rules (gaugefixing/algorithms/{Or,Micro,Sa,Sr,Random}Update.hxx, the non-USE_DP_* branches) -------------- */
static void FN(algo_or)(REAL a[4], float omega)
{
    /* OrUpdate.hxx:66-75 */
    REAL ai_sq = a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
    REAL a0_sq = a[0] * a[0];
    REAL b = (omega * a0_sq + ai_sq) / (a0_sq + ai_sq);
    REAL c = R_RSQRT(a0_sq + b * b * ai_sq);
    a[0] *= c;
    a[1] *= b * c;
    a[2] *= b * c;
    a[3] *= b * c;
}

static void FN(algo_micro)(REAL a[4])
{
    /* MicroUpdate.hxx:55-64 */
    REAL ai_sq = a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
    REAL a0_sq = a[0] * a[0];
    REAL b = (REAL)2. * a[0] / (a0_sq + ai_sq);
    a[0] = (a0_sq - ai_sq) / (a0_sq + ai_sq);
    a[1] *= b;
    a[2] *= b;
    a[3] *= b;
}

static void FN(algo_sa)(REAL a[4], float temperature, RNG *rng)
{
    /* SaUpdate.hxx:103-146 (Kennedy-Pendleton heat-bath) */
    REAL e0, e1, e2, e3, dk, p0;
    REAL r1, r2, r3, r4;
    REAL a0, a1, a2, a3;
    REAL delta, phi, sin_alpha, sin_theta, cos_theta;
    e0 = a[0];
    e1 = -a[1];
    e2 = -a[2];
    e3 = -a[3];
    dk = R_RSQRT(e0 * e0 + e1 * e1 + e2 * e2 + e3 * e3);
    p0 = (dk * temperature);
    do {
        do; while ((r1 = FN(rng_rand)(rng)) < 0.0001);
        r1 = -R_LOG(r1) * p0;
        do; while ((r2 = FN(rng_rand)(rng)) < 0.0001);
        r2 = -R_LOG(r2) * p0;
        r3 = orc_cospi_d(2.0 * FN(rng_rand)(rng));
        r3 = r3 * r3;
        delta = r2 + r1 * r3;
        r4 = FN(rng_rand)(rng);
    } while (r4 * r4 > (1.0 - 0.5 * delta));
    a0 = 1.0 - delta;
    cos_theta = 2.0 * FN(rng_rand)(rng) - 1.0;
    sin_theta = sqrt(1.0 - cos_theta * cos_theta);
    sin_alpha = R_SQRT(1 - a0 * a0);
    phi = 2.0 * FN(rng_rand)(rng);
    a1 = sin_alpha * sin_theta * R_COSPI(phi);
    a2 = sin_alpha * sin_theta * R_SINPI(phi);
    a3 = sin_alpha * cos_theta;

    e0 *= dk;
    e1 *= dk;
    e2 *= dk;
    e3 *= dk;

    a[0] = a0 * e0 + a3 * e3 + a2 * e2 + e1 * a1;
    a[3] = e0 * a3 - e3 * a0 + a1 * e2 - a2 * e1;
    a[2] = a3 * e1 - a0 * e2 + a2 * e0 - a1 * e3;
    a[1] = a2 * e3 + a1 * e0 - a3 * e2 - e1 * a0;
}

static void FN(algo_sr)(REAL a[4], float p, RNG *rng)
{
    /* SrUpdate.hxx:76-94 */
    REAL rand = FN(rng_rand)(rng);
    REAL a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3], c;
    a[0] = (rand >= p) * a0 + (rand < p) * (a0 * a0 - a1 * a1 - a2 * a2 - a3 * a3);
    a[1] = (rand >= p) * a1 + (rand < p) * (2.0 * a0 * a1);
    a[2] = (rand >= p) * a2 + (rand < p) * (2.0 * a0 * a2);
    a[3] = (rand >= p) * a3 + (rand < p) * (2.0 * a0 * a3);
    c = R_RSQRT(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3]);
    a[0] *= c;
    a[1] *= c;
    a[2] *= c;
    a[3] *= c;
}

static void FN(algo_random)(REAL a[4], RNG *rng)
{
    /* RandomUpdate.hxx:47-59 */
    REAL alpha, phi, cos_theta, sin_theta, sin_alpha;
    alpha = FN(rng_rand)(rng);
    phi = 2.0 * FN(rng_rand)(rng);
    cos_theta = 2.0 * FN(rng_rand)(rng) - 1.0;
    sin_theta = sqrt(1.0 - cos_theta * cos_theta);
    sin_alpha = R_SINPI(alpha);
    a[0] = R_COSPI(alpha);
    a[1] = sin_alpha * sin_theta * R_COSPI(phi);
    a[2] = sin_alpha * sin_theta * R_SINPI(phi);
    a[3] = sin_alpha * cos_theta;
}

static void FN(algo_apply)(REAL a[4], int algo, float param, RNG *rng)
{
    switch (algo) {
    case ORC_OR: FN(algo_or)(a, param); break;
    case ORC_MICRO: FN(algo_micro)(a); break;
    case ORC_SA: FN(algo_sa)(a, param, rng); break;
    case ORC_SR: FN(algo_sr)(a, param, rng); break;
    default: FN(algo_random)(a, rng); break;
    }
}

/* ---- one site update: GaugeFixingSubgroupStep::subgroup for the 3 subgroups -------------- */
/* M[0..3] = up links U_mu(x), M[4..7] = down links U_mu(x-mu).  The accumulation order is the
 * serialised (non-atomic) order of the DP build: up mu=0..3, then down mu=0..3
 * (GaugeFixingSubgroupStep.hxx:127-207). */
static void FN(subgroup)(MAT M[8], int i, int j, int gauge, int algo, float param, RNG *rng)
{
    REAL a[4] = {0, 0, 0, 0};
    REAL q[4];
    if (gauge == ORC_LANDAU || gauge == ORC_COULOMB) {
        /* GaugeFixingSubgroupStep.hxx:99-237 */
        for (int mu = 0; mu < 4; mu++) {
            if (gauge == ORC_COULOMB && mu == 0) continue;
            FN(subq)(&M[mu], i, j, q);
            a[0] += q[0];
            a[1] -= q[1];
            a[2] -= q[2];
            a[3] -= q[3];
        }
        for (int mu = 0; mu < 4; mu++) {
            if (gauge == ORC_COULOMB && mu == 0) continue;
            FN(subq)(&M[4 + mu], i, j, q);
            a[0] += q[0];
            a[1] += q[1];
            a[2] += q[2];
            a[3] += q[3];
        }
        FN(algo_apply)(a, algo, param, rng);
        q[0] = a[0];
        q[1] = a[1];
        q[2] = a[2];
        q[3] = a[3];
    } else if (gauge == ORC_U1XU1) {
        /* GaugeFixingSubgroupStep.hxx:238-353: only q0 and q3 enter, g normalised */
        for (int mu = 0; mu < 4; mu++) {
            FN(subq)(&M[mu], i, j, q);
            a[0] += q[0];
            a[3] -= q[3];
        }
        for (int mu = 0; mu < 4; mu++) {
            FN(subq)(&M[4 + mu], i, j, q);
            a[0] += q[0];
            a[3] += q[3];
        }
        a[1] = 0.0;
        a[2] = 0.0;
        FN(algo_apply)(a, algo, param, rng);
        q[0] = a[0];
        q[1] = 0.0;
        q[2] = 0.0;
        q[3] = a[3];
        REAL norm = R_RSQRT(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        q[0] *= norm;
        q[1] *= norm;
        q[2] *= norm;
        q[3] *= norm;
    } else {
        /* MAG, GaugeFixingSubgroupStep.hxx:354-589 */
        for (int ud = 0; ud < 2; ud++) {
            for (int mu = 0; mu < 4; mu++) {
                const MAT *L = &M[4 * ud + mu];
                /* getSubgroupMatrix (SU3.hxx:219-229) */
                CPX s00 = L->m[i][i], s01 = L->m[i][j], s10 = L->m[j][i], s11 = L->m[j][j];
                a[0] += FN(abs2)(s00) - FN(abs2)(s01) - FN(abs2)(s10) + FN(abs2)(s11);
                CPX c;
                if (ud == 0)
                    c = FN(csub)(FN(cmul)(s00, FN(conj)(s10)), FN(cmul)(s01, FN(conj)(s11)));
                else
                    c = FN(csub)(FN(cmul)(FN(conj)(s00), s01), FN(cmul)(FN(conj)(s10), s11));
                a[1] += c.y;
                a[2] += c.x;
            }
        }
        a[1] *= 2.;
        a[2] *= 2.;
        a[3] = 0;
        a[0] = a[0] + R_SQRT(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        FN(algo_apply)(a, algo, param, rng);
        q[0] = a[0];
        q[1] = a[1];
        q[2] = a[2];
        q[3] = 0;
        REAL norm = R_RSQRT(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        q[0] *= norm;
        q[1] *= norm;
        q[2] *= norm;
        q[3] *= norm;
    }
    /* up links: leftSubgroupMult(g); down links: rightSubgroupMult(g^dagger) */
    for (int mu = 0; mu < 4; mu++) FN(left_mult)(&M[mu], i, j, q);
    REAL qh[4] = {q[0], -q[1], -q[2], -q[3]};
    for (int mu = 0; mu < 4; mu++) FN(right_mult)(&M[4 + mu], i, j, qh);
}

/* One parity pass (the apply() of LandauKernelsSU3.hxx:216-256, CoulombKernelsSU3.hxx:208-250,
 * MAGKernelsSU3.hxx:248-293, U1xU1KernelsSU3.hxx:216-256), serial over sites, over the sites h in
 * [h_lo, h_hi) of the parity.  Site h draws its random numbers as site h + rng_site_offset of the
 * lattice would: a part of a larger lattice (a t-slab) then draws the whole lattice's stream. */
void FN(orc_step_range_at)(REAL *Uup, REAL *Udw, const int32_t size[4], int gauge, int algo, int parity,
                           float param, uint32_t seed, uint32_t counter, int64_t h_lo, int64_t h_hi,
                           int64_t rng_site_offset, int nthreads)
{
    const int64_t V = (int64_t)size[0] * size[1] * size[2] * size[3];
    const int64_t Vh = V / 2;
    if (nthreads < 1) nthreads = 1;
    if (Udw == 0) Udw = Uup;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int64_t h = h_lo; h < h_hi; h++) {
        const int64_t s = h + (parity ? Vh : 0);
        MAT M[8];
        int64_t site[8];
        REAL *arr[8];
        for (int mu = 0; mu < 4; mu++) {
            site[mu] = s;
            arr[mu] = Uup;
            if (gauge == ORC_COULOMB && mu == 0) {
                site[4 + mu] = s; /* temporal down link from slice t-1, same spatial site */
                arr[4 + mu] = Udw;
            } else {
                site[4 + mu] = orc_neighbour(size, s, mu, 0);
                arr[4 + mu] = Uup;
            }
        }
        for (int k = 0; k < 8; k++) FN(load12)(arr[k], V, site[k], k & 3, &M[k]);
        RNG rng;
        if (algo == ORC_SA || algo == ORC_SR || algo == ORC_RANDOM) {
            /* key of the (mu=0, up) thread: blockIdx.x*blockDim.x + threadIdx.x with
             * NSB = 32 sites and 256 threads per block (apps/Makefile:36) */
            const int64_t hr = h + rng_site_offset;
            uint32_t tid = (uint32_t)((hr / 32) * 256 + (hr % 32));
            FN(rng_init)(&rng, tid, seed, counter);
        }
        /* SU3::perSubgroup (SU3.hxx:762-771): (0,2), (1,2), (0,1) */
        FN(subgroup)(M, 0, 2, gauge, algo, param, &rng);
        FN(subgroup)(M, 1, 2, gauge, algo, param, &rng);
        FN(subgroup)(M, 0, 1, gauge, algo, param, &rng);
        for (int k = 0; k < 8; k++) FN(store12)(arr[k], V, site[k], k & 3, &M[k]);
    }
}

void FN(orc_step_range)(REAL *Uup, REAL *Udw, const int32_t size[4], int gauge, int algo, int parity,
                        float param, uint32_t seed, uint32_t counter, int64_t h_lo, int64_t h_hi, int nthreads)
{
    FN(orc_step_range_at)(Uup, Udw, size, gauge, algo, parity, param, seed, counter, h_lo, h_hi, 0, nthreads);
}

void FN(orc_step)(REAL *Uup, REAL *Udw, const int32_t size[4], int gauge, int algo, int parity,
                  float param, uint32_t seed, uint32_t counter, int nthreads)
{
    const int64_t Vh = (int64_t)size[0] * size[1] * size[2] * size[3] / 2;
    FN(orc_step_range)(Uup, Udw, size, gauge, algo, parity, param, seed, counter, 0, Vh, nthreads);
}

/* ---- gauge quality ------------------------------------------------------------------------- */
/* Landau / U1xU1 / Coulomb per-site values: LandauKernelsSU3.hxx:114-191,
 * CoulombKernelsSU3.hxx:110-183 (mu = 1..3). */
static void FN(quality_site_landau)(const REAL *U, const int32_t size[4], int64_t V, int64_t s,
                                    int mu0, double *gff, double *dA)
{
    MAT Sum, T;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Sum.m[i][j] = FN(cmake)(0, 0);
    for (int mu = mu0; mu < 4; mu++) {
        FN(load12)(U, V, s, mu, &T);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) Sum.m[i][j] = FN(cadd)(Sum.m[i][j], T.m[i][j]);
        FN(load12)(U, V, orc_neighbour(size, s, mu, 0), mu, &T);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) Sum.m[i][j] = FN(csub)(Sum.m[i][j], T.m[i][j]);
    }
    /* Sum -= Sum.trace()/Real(3.)  (diagonal only, Matrix.hxx operator-=(T)) */
    CPX tr = FN(cmake)(0, 0);
    for (int i = 0; i < 3; i++) tr = FN(cadd)(tr, Sum.m[i][i]);
    tr.x /= (REAL)3.;
    tr.y /= (REAL)3.;
    for (int i = 0; i < 3; i++) Sum.m[i][i] = FN(csub)(Sum.m[i][i], tr);
    MAT H;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) H.m[j][i] = FN(conj)(Sum.m[i][j]);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Sum.m[i][j] = FN(csub)(Sum.m[i][j], H.m[i][j]);
    double prec = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) prec += FN(abs2)(Sum.m[i][j]);
    *dA = prec;
    double result = 0;
    for (int mu = mu0; mu < 4; mu++) {
        FN(load12)(U, V, s, mu, &T);
        CPX t = FN(cmake)(0, 0);
        for (int i = 0; i < 3; i++) t = FN(cadd)(t, T.m[i][i]);
        result += t.x;
    }
    *gff = result;
}

/* MAG per-site values: MAGKernelsSU3.hxx:116-223 */
static void FN(quality_site_mag)(const REAL *U, const int32_t size[4], int64_t V, int64_t s,
                                 double *gff, double *dA)
{
    double Xx[3] = {0, 0, 0}, Xy[3] = {0, 0, 0};
    double g = 0.0;
    for (int mu = 0; mu < 4; mu++) {
        MAT up, dw;
        FN(load12)(U, V, s, mu, &up);
        FN(load12)(U, V, orc_neighbour(size, s, mu, 0), mu, &dw);
        for (int j = 0; j < 3; j++) g += FN(abs2)(up.m[j][j]);
        for (int i = 0; i < 2; i++)
            for (int j = i + 1; j < 3; j++) {
                CPX m00 = up.m[i][i], m01 = up.m[i][j], m10 = up.m[j][i], m11 = up.m[j][j];
                CPX c = FN(csub)(FN(cmul)(m00, FN(conj)(m10)), FN(cmul)(m01, FN(conj)(m11)));
                Xx[i + j - 1] += (double)c.x;
                Xy[i + j - 1] += (double)c.y;
                /* getSubgroupMatrixHermitian (SU3.hxx:231-241) */
                m00 = FN(conj)(dw.m[i][i]);
                m01 = FN(conj)(dw.m[j][i]);
                m10 = FN(conj)(dw.m[i][j]);
                m11 = FN(conj)(dw.m[j][j]);
                c = FN(csub)(FN(cmul)(m00, FN(conj)(m10)), FN(cmul)(m01, FN(conj)(m11)));
                Xx[i + j - 1] += (double)c.x;
                Xy[i + j - 1] += (double)c.y;
            }
    }
    *gff = g;
    *dA = sqrt(Xx[0] * Xx[0] + Xy[0] * Xy[0]) + sqrt(Xx[1] * Xx[1] + Xy[1] * Xy[1]) +
          sqrt(Xx[2] * Xx[2] + Xy[2] * Xy[2]);
}

void FN(orc_quality)(const REAL *U, const int32_t size[4], int gauge, int stop_max, double *gff,
                     double *theta, double *gff_site, double *theta_site, int nthreads)
{
    const int64_t V = (int64_t)size[0] * size[1] * size[2] * size[3];
    double *g = gff_site ? gff_site : (double *)malloc(sizeof(double) * V);
    double *a = theta_site ? theta_site : (double *)malloc(sizeof(double) * V);
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int64_t s = 0; s < V; s++) {
        if (gauge == ORC_MAG)
            FN(quality_site_mag)(U, size, V, s, &g[s], &a[s]);
        else
            FN(quality_site_landau)(U, size, V, s, gauge == ORC_COULOMB ? 1 : 0, &g[s], &a[s]);
    }
    /* reduceGaugeQuality (GaugeFixingStats.hxx:655-668): serial sum (or max) in site order */
    double G = 0, A = 0;
    for (int64_t s = 0; s < V; s++) {
        G += g[s];
        A = stop_max ? (A > a[s] ? A : a[s]) : A + a[s];
    }
    /* normalisation (GaugeFixingStats.hxx:203-206) with the plugin prefactors
     * (LandauKernelsSU3.hxx:75-82, CoulombKernelsSU3.hxx:75-78, MAGKernelsSU3.hxx:77-84) */
    const int Nc = 3, Nd = 4;
    double preG = gauge == ORC_COULOMB ? 1. / (double)(Nc * (Nd - 1)) : 1. / (double)(Nc * Nd);
    double preA = 1. / (double)Nc;
    G = G * preG / (double)V;
    A = A * preA;
    if (!stop_max) A = A / (double)V;
    *gff = G;
    *theta = A;
    if (!gff_site) free(g);
    if (!theta_site) free(a);
}

/* ---- reunitarisation: SU3::projectSU3 (SU3.hxx:536-583) on every link ------------------- */
static void FN(project_link)(MAT *M)
{
    REAL abs_u = 0, abs_v = 0;
    CPX sp = FN(cmake)(0., 0.);
    for (int i = 0; i < 3; i++) abs_u += FN(abs2)(M->m[0][i]);
    abs_u = R_SQRT(abs_u);
    for (int i = 0; i < 3; i++) M->m[0][i] = FN(cmake)(M->m[0][i].x / abs_u, M->m[0][i].y / abs_u);
    for (int i = 0; i < 3; i++) sp = FN(cadd)(sp, FN(cmul)(M->m[1][i], FN(conj)(M->m[0][i])));
    for (int i = 0; i < 3; i++) M->m[1][i] = FN(csub)(M->m[1][i], FN(cmul)(M->m[0][i], sp));
    for (int i = 0; i < 3; i++) abs_v += FN(abs2)(M->m[1][i]);
    abs_v = R_SQRT(abs_v);
    for (int i = 0; i < 3; i++) M->m[1][i] = FN(cmake)(M->m[1][i].x / abs_v, M->m[1][i].y / abs_v);
    FN(reconstruct)(M);
}

void FN(orc_project)(REAL *U, const int32_t size[4], int nthreads)
{
    const int64_t V = (int64_t)size[0] * size[1] * size[2] * size[3];
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int64_t s = 0; s < V; s++) {
        for (int mu = 0; mu < 4; mu++) {
            MAT M;
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                    M.m[i][j] = FN(cmake)(U[FN(gidx)(V, s, mu, i, j, 0)], U[FN(gidx)(V, s, mu, i, j, 1)]);
            FN(project_link)(&M);
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    U[FN(gidx)(V, s, mu, i, j, 0)] = M.m[i][j].x;
                    U[FN(gidx)(V, s, mu, i, j, 1)] = M.m[i][j].y;
                }
        }
    }
}

/* ---- random start: COMKSU3::setHot (CommonKernelsSU3.hxx:92-130) -------------------------- */
void FN(orc_set_hot)(REAL *U, const int32_t size[4], uint32_t seed, uint32_t counter, int nthreads)
{
    const int64_t V = (int64_t)size[0] * size[1] * size[2] * size[3];
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int64_t s = 0; s < V; s++) {
        RNG rng;
        FN(rng_init)(&rng, (uint32_t)s, seed, counter);
        for (int mu = 0; mu < 4; mu++) {
            MAT M;
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) M.m[i][j] = FN(cmake)(i == j ? 1 : 0, 0);
            for (int i = 0; i < 2; i++)
                for (int j = i + 1; j < 3; j++) {
                    REAL q[4];
                    q[0] = FN(rng_rand)(&rng) * 2.0 - 1.0;
                    q[1] = FN(rng_rand)(&rng) * 2.0 - 1.0;
                    q[2] = FN(rng_rand)(&rng) * 2.0 - 1.0;
                    q[3] = FN(rng_rand)(&rng) * 2.0 - 1.0;
                    /* Quaternion::projectSU2 (Quaternion.hxx:220-228) */
                    REAL det = R_RSQRT(q[0] * q[0] + q[3] * q[3] + q[2] * q[2] + q[1] * q[1]);
                    q[0] *= det;
                    q[1] *= det;
                    q[2] *= det;
                    q[3] *= det;
                    FN(right_mult)(&M, i, j, q);
                }
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    U[FN(gidx)(V, s, mu, i, j, 0)] = M.m[i][j].x;
                    U[FN(gidx)(V, s, mu, i, j, 1)] = M.m[i][j].y;
                }
        }
    }
}

/* ---- whole-run driver: apps/LandauGaugeFixingSU3_4D.cu:185-271 (one copy) --------------- */
void FN(orc_fix)(REAL *U, const int32_t size[4], int gauge, const orc_schedule *sc, uint32_t *counter,
                 orc_result *res, int nthreads)
{
    double gff = 0, theta = 0;
    if (sc->random_trafo) {
        FN(orc_step)(U, U, size, gauge, ORC_RANDOM, 0, 0.f, sc->seed, (*counter)++, nthreads);
        FN(orc_step)(U, U, size, gauge, ORC_RANDOM, 1, 0.f, sc->seed, (*counter)++, nthreads);
    }
    FN(orc_quality)(U, size, gauge, 0, &gff, &theta, 0, 0, nthreads);
    float temperature = sc->sa_max;
    float tempStep = sc->sa_steps > 0 ? (sc->sa_max - sc->sa_min) / (float)sc->sa_steps : 0.f;
    for (int i = 0; i < sc->sa_steps; i++) {
        FN(orc_step)(U, U, size, gauge, ORC_SA, 0, temperature, sc->seed, (*counter)++, nthreads);
        FN(orc_step)(U, U, size, gauge, ORC_SA, 1, temperature, sc->seed, (*counter)++, nthreads);
        for (int m = 0; m < sc->micro_updates; m++) {
            FN(orc_step)(U, U, size, gauge, ORC_MICRO, 0, 0.f, 0, 0, nthreads);
            FN(orc_step)(U, U, size, gauge, ORC_MICRO, 1, 0.f, 0, 0, nthreads);
        }
        if (i % sc->reproject == 0) FN(orc_project)(U, size, nthreads);
        if (i % sc->check_precision == 0) FN(orc_quality)(U, size, gauge, 0, &gff, &theta, 0, 0, nthreads);
        temperature -= tempStep;
    }
    int it = 0;
    for (int i = 0; i < sc->or_max_iter; i++) {
        FN(orc_step)(U, U, size, gauge, ORC_OR, 0, sc->or_parameter, 0, 0, nthreads);
        FN(orc_step)(U, U, size, gauge, ORC_OR, 1, sc->or_parameter, 0, 0, nthreads);
        it = i + 1;
        if (i % sc->reproject == 0) FN(orc_project)(U, size, nthreads);
        if (i % sc->check_precision == 0) {
            FN(orc_quality)(U, size, gauge, 0, &gff, &theta, 0, 0, nthreads);
            if (theta < sc->precision) break;
        }
    }
    FN(orc_project)(U, size, nthreads);
    res->gff = gff;
    res->theta = theta;
    res->or_iterations = it;
}

/* orc_fix_app: see gf_oracle.h.  The loops follow apps/LandauGaugeFixingSU3_4D.cu:204-271 (sa_mode 0,
 * also the Coulomb app's slice body, apps/CoulombGaugeFixingSU3_4D.cu:216-301) and
 * apps/MAGaugeFixingSU3_4D.cu:222-333 (sa_mode 2 and the SR loop). */
void FN(orc_fix_app)(REAL *U, REAL *Udw, const int32_t size[4], int gauge, const orc_app_schedule *sc,
                     uint32_t *counter, orc_app_result *res, int nthreads)
{
    const int coulomb = gauge == ORC_COULOMB;
    REAL *dw = coulomb ? Udw : U;
    double gff = 0, theta = 0;
    int sa_done = 0;
#define ORC_PROJECT()                                               \
    do {                                                            \
        FN(orc_project)(U, size, nthreads);                         \
        if (coulomb) FN(orc_project)(Udw, size, nthreads);          \
    } while (0)
    if (sc->random_trafo) {
        FN(orc_step)(U, dw, size, gauge, ORC_RANDOM, 0, 0.f, sc->seed, (*counter)++, nthreads);
        FN(orc_step)(U, dw, size, gauge, ORC_RANDOM, 1, 0.f, sc->seed, (*counter)++, nthreads);
    }
    const int repeat = sc->sa_repeat > 0 ? sc->sa_repeat : 1;
    float temperature = sc->sa_max;
    const float base = sc->sa_steps > 0 ? (sc->sa_max - sc->sa_min) / (float)sc->sa_steps : 0.f;
    int i = 0;
    for (;;) {
        if (sc->sa_steps <= 0) break;
        if (sc->sa_mode != 2 && i >= sc->sa_steps) break;
        float step = base;
        if (sc->sa_mode == 2 && (double)temperature <= sc->sa_slow_hi && (double)temperature >= sc->sa_slow_lo)
            step = base / sc->sa_slow_factor;
        for (int r = 0; r < repeat; r++) {
            FN(orc_step)(U, dw, size, gauge, ORC_SA, 0, temperature, sc->seed, (*counter)++, nthreads);
            FN(orc_step)(U, dw, size, gauge, ORC_SA, 1, temperature, sc->seed, (*counter)++, nthreads);
            sa_done++;
            for (int m = 0; m < sc->micro_updates; m++) {
                FN(orc_step)(U, dw, size, gauge, ORC_MICRO, 0, 0.f, 0, 0, nthreads);
                FN(orc_step)(U, dw, size, gauge, ORC_MICRO, 1, 0.f, 0, 0, nthreads);
            }
        }
        if (i % sc->reproject == 0) ORC_PROJECT();
        temperature -= step;
        i++;
        if (sc->sa_mode == 2 && !(temperature >= sc->sa_min)) break;
    }
    int sr = 0;
    for (int k = 0; k < sc->sr_max_iter; k++) {
        FN(orc_step)(U, dw, size, gauge, ORC_SR, 0, sc->sr_parameter, sc->seed, (*counter)++, nthreads);
        FN(orc_step)(U, dw, size, gauge, ORC_SR, 1, sc->sr_parameter, sc->seed, (*counter)++, nthreads);
        sr = k + 1;
        if (k % sc->reproject == 0) ORC_PROJECT();
        if (k % sc->check_precision == 0) {
            FN(orc_quality)(U, size, gauge, 0, &gff, &theta, 0, 0, nthreads);
            if (theta < sc->precision || theta < sc->sr_stop_theta) break;
        }
    }
    int it = 0;
    for (int k = 0; k < sc->or_max_iter; k++) {
        FN(orc_step)(U, dw, size, gauge, ORC_OR, 0, sc->or_parameter, 0, 0, nthreads);
        FN(orc_step)(U, dw, size, gauge, ORC_OR, 1, sc->or_parameter, 0, 0, nthreads);
        it = k + 1;
        if (k % sc->reproject == 0) ORC_PROJECT();
        if (k % sc->check_precision == 0) {
            FN(orc_quality)(U, size, gauge, 0, &gff, &theta, 0, 0, nthreads);
            if (theta < sc->precision) break;
        }
    }
    ORC_PROJECT();
#undef ORC_PROJECT
    res->gff = gff;
    res->theta = theta;
    res->or_iterations = it;
    res->sa_sweeps = sa_done;
    res->sr_iterations = sr;
}

void FN(orc_fix_coulomb)(REAL *U, const int32_t size[4], const orc_app_schedule *sc, uint32_t *counter,
                         orc_app_result *res, int nthreads)
{
    const int32_t ss[4] = {1, size[1], size[2], size[3]};
    const int64_t slice = (int64_t)72 * size[1] * size[2] * size[3];
    for (int t = 0; t < size[0]; t++) {
        const int tdw = t > 0 ? t - 1 : size[0] - 1;
        FN(orc_fix_app)(U + slice * t, U + slice * tdw, ss, ORC_COULOMB, sc, counter, &res[t], nthreads);
    }
}

#undef CPX
#undef MAT
#undef RNG
#undef FN
#undef CAT
#undef CAT2
