/*
 * ref_pin.cpp -- runs the reference's OWN site-update code on the host, to pin the C oracle.
 * TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against the reference tree (read in
 * place, never copied) into oracle/_ref/libref_pin_{f64,f32}.so.
 *
 * What comes from the reference, unmodified, through #include:
 *   gaugefixing/GaugeFixingSubgroupStep.hxx   (the cooperative 8-threads-per-site update)
 *   gaugefixing/algorithms/{Or,Micro,Sa,Sr,Random}Update.hxx
 *   lattice/{SU3,Matrix,Complex,Quaternion,Link,SiteIndex,SiteCoord}.hxx, access_pattern/GpuPattern.hxx
 *   lattice/rng/PhiloxWrapper.hxx + external/Random123 (philox.h, u01.h)
 * What this file adds (the reference's *KernelsSU3.hxx cannot be compiled by a host compiler
 * because of their <<<>>> launch wrappers):
 *   - a tiny CUDA-on-host emulation: one std::thread per CUDA thread of a 256-thread block,
 *     __shared__ as a function-static array, __syncthreads() as a std::barrier, atomicAdd under
 *     a mutex, rsqrt/cospi/sinpi from orc_math.h;
 *   - restatements of the thin kernel bodies that call that code: apply() of
 *     LandauKernelsSU3.hxx:216-256 (and the Coulomb/MAG/U1xU1 twins), the per-site quality of
 *     LandauKernelsSU3.hxx:114-191 / CoulombKernelsSU3.hxx:110-183 / MAGKernelsSU3.hxx:116-223,
 *     COMKSU3::projectSU3 and COMKSU3::setHot (CommonKernelsSU3.hxx:71-130), with runtime
 *     extents instead of the reference's compile-time ones.
 */
#include <barrier>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <thread>
#include <vector>

#include "orc_math.h"

/* ---- CUDA-on-host emulation ---------------------------------------------------------------- */
#define __device__
#define __host__
#define __global__
#define __constant__
#define __shared__ static
#define __forceinline__ inline

static std::barrier<> *g_block_barrier = nullptr;
static inline void __syncthreads() { g_block_barrier->arrive_and_wait(); }
static std::mutex g_atomic_mutex;
static inline float atomicAdd(float *a, float v)
{
    std::lock_guard<std::mutex> lock(g_atomic_mutex);
    float old = *a;
    *a = old + v;
    return old;
}
static inline double atomicAdd(double *a, double v)
{
    std::lock_guard<std::mutex> lock(g_atomic_mutex);
    double old = *a;
    *a = old + v;
    return old;
}
static inline float rsqrt(float x) { return orc_rsqrt_f(x); }
static inline double rsqrt(double x) { return orc_rsqrt_d(x); }
static inline float cospi(float x) { return orc_cospi_f(x); }
static inline double cospi(double x) { return orc_cospi_d(x); }
static inline float sinpi(float x) { return orc_sinpi_f(x); }
static inline double sinpi(double x) { return orc_sinpi_d(x); }

/* compile-time extents are only needed to make GlobalConstants.h compile; all lattice
 * geometry below is runtime.  NSB keeps the reference default of 32 sites per block. */
#define _X_ 4
#define _T_ 4
#include "gaugefixing/GlobalConstants.h"
#include "lattice/datatype/datatypes.h"
#include "lattice/datatype/lattice_typedefs.h"
#include "lattice/Complex.hxx"
#include "lattice/Matrix.hxx"
#include "lattice/Quaternion.hxx"
#include "lattice/SU3.hxx"
#include "lattice/Link.hxx"
#include "lattice/SiteIndex.hxx"
#include "lattice/SiteCoord.hxx"
#include "lattice/access_pattern/GpuPattern.hxx"
#include "lattice/rng/PhiloxWrapper.hxx"
#include "gaugefixing/GaugeFixingSubgroupStep.hxx"
#include "gaugefixing/algorithms/OrUpdate.hxx"
#include "gaugefixing/algorithms/MicroUpdate.hxx"
#include "gaugefixing/algorithms/SaUpdate.hxx"
#include "gaugefixing/algorithms/SrUpdate.hxx"
#include "gaugefixing/algorithms/RandomUpdate.hxx"

#ifdef DOUBLEPRECISION
#define REF_SFX(name) name##_f64
#else
#define REF_SFX(name) name##_f32
#endif

typedef GpuPattern<SiteIndex<4, FULL_SPLIT>, 4, 3> GpuIndex;
typedef Link<GpuIndex, SiteIndex<4, FULL_SPLIT>, 4, 3> TLinkIndex;
typedef GpuPattern<SiteCoord<4, FULL_SPLIT>, 4, 3> GpuCoord;
typedef Link<GpuCoord, SiteCoord<4, FULL_SPLIT>, 4, 3> TLinkCoord;
typedef SU3<Matrix<Complex<Real>, 3>> LocalSU3;

/* apply() of the gauge plugins, for CUDA thread t of block b (LandauKernelsSU3.hxx:216-256;
 * CoulombKernelsSU3.hxx:208-250 for the temporal down link from UtDw). */
template <class Algorithm, GaugeType G>
static void ref_apply(Real *Uup, Real *Udw, lat_index_t *nn, const lat_coord_t size[4], bool parity,
                      int b, int t, Algorithm algorithm)
{
    SiteIndex<4, FULL_SPLIT> s(size);
    s.nn = nn;
    const bool updown = t / (4 * NSB);
    const short mu = (t % (4 * NSB)) / NSB;
    const short id = (t % (4 * NSB)) % NSB;
    int site = b * NSB + id;
    if (parity == 1) site += s.getLatticeSize() / 2;
    s.setLatticeIndex(site);
    Real *U = Uup;
    if (G == COULOMB) {
        if ((mu != 0) && (updown == true)) s.setNeighbour(mu, false);
        if ((mu == 0) && (updown == true)) U = Udw;
    } else if (updown == 1) {
        s.setNeighbour(mu, false);
    }
    Matrix<Complex<Real>, 3> locMat;
    LocalSU3 locU(locMat);
    TLinkIndex link(U, s, mu);
    SU3<TLinkIndex> globU(link);
    locU.assignWithoutThirdLine(globU);
    locU.reconstructThirdLine();
    GaugeFixingSubgroupStep<LocalSU3, Algorithm, G> subgroupStep(&locU, algorithm, id, mu, updown);
    /* SU3::perSubgroup (SU3.hxx:762-771) is device-only; its order is (0,2), (1,2), (0,1) */
    subgroupStep.subgroup(0, 2);
    subgroupStep.subgroup(1, 2);
    subgroupStep.subgroup(0, 1);
    globU.assignWithoutThirdLine(locU);
}

template <GaugeType G>
static void ref_thread(Real *Uup, Real *Udw, lat_index_t *nn, const lat_coord_t size[4], int parity,
                       int algo, float param, int seed, unsigned counter, int nblocks, int t)
{
    for (int b = 0; b < nblocks; b++) {
        const int tid = b * 8 * NSB + t; /* blockIdx.x * blockDim.x + threadIdx.x */
        switch (algo) {
        case 0: ref_apply<OrUpdate, G>(Uup, Udw, nn, size, parity, b, t, OrUpdate(param)); break;
        case 1: ref_apply<MicroUpdate, G>(Uup, Udw, nn, size, parity, b, t, MicroUpdate()); break;
        case 2: {
            PhiloxWrapper rng(tid, seed, counter);
            ref_apply<SaUpdate, G>(Uup, Udw, nn, size, parity, b, t, SaUpdate(param, &rng));
            break;
        }
        case 3: {
            PhiloxWrapper rng(tid, seed, counter);
            ref_apply<SrUpdate, G>(Uup, Udw, nn, size, parity, b, t, SrUpdate(param, &rng));
            break;
        }
        default: {
            PhiloxWrapper rng(tid, seed, counter);
            ref_apply<RandomUpdate, G>(Uup, Udw, nn, size, parity, b, t, RandomUpdate(&rng));
            break;
        }
        }
        g_block_barrier->arrive_and_wait();
    }
}

extern "C" {

/* One parity pass of the reference kernel (orStep/microStep/saStep/srStep/randomTrafo) with
 * V/2/NSB blocks of 8*NSB threads.  size = {Nt,Nx,Ny,Nz} ({1,Nx,Ny,Nz} for COULOMB). */
int REF_SFX(ref_step)(Real *Uup, Real *Udw, const int32_t size_in[4], int gauge, int algo, int parity,
                      float param, uint32_t seed, uint32_t counter)
{
    lat_coord_t size[4];
    for (int i = 0; i < 4; i++) size[i] = (lat_coord_t)size_in[i];
    SiteIndex<4, FULL_SPLIT> s(size);
    const int V = s.getLatticeSize();
    if ((V / 2) % NSB != 0) return -1;
    std::vector<lat_index_t> nn((size_t)8 * V);
    s.calculateNeighbourTable(nn.data());
    if (Udw == nullptr) Udw = Uup;
    const int nblocks = V / 2 / NSB;
    const int nthreads = 8 * NSB;
    std::barrier<> bar(nthreads);
    g_block_barrier = &bar;
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; t++) {
        switch (gauge) {
        case LANDAU:
            pool.emplace_back(ref_thread<LANDAU>, Uup, Udw, nn.data(), size, parity, algo, param, (int)seed, counter, nblocks, t);
            break;
        case COULOMB:
            pool.emplace_back(ref_thread<COULOMB>, Uup, Udw, nn.data(), size, parity, algo, param, (int)seed, counter, nblocks, t);
            break;
        case MAG:
            pool.emplace_back(ref_thread<MAG>, Uup, Udw, nn.data(), size, parity, algo, param, (int)seed, counter, nblocks, t);
            break;
        default:
            pool.emplace_back(ref_thread<U1xU1>, Uup, Udw, nn.data(), size, parity, algo, param, (int)seed, counter, nblocks, t);
            break;
        }
    }
    for (auto &th : pool) th.join();
    g_block_barrier = nullptr;
    return 0;
}

/* Per-site quality, LandauKernelsSU3.hxx:114-191 (mu from mu0; mu0 = 1 is the Coulomb variant
 * CoulombKernelsSU3.hxx:110-183) and MAGKernelsSU3.hxx:116-223. */
void REF_SFX(ref_quality_sites)(Real *U, const int32_t size_in[4], int gauge, double *dGff, double *dA)
{
    lat_coord_t size[4];
    for (int i = 0; i < 4; i++) size[i] = (lat_coord_t)size_in[i];
    SiteCoord<4, FULL_SPLIT> s(size);
    const int V = s.getLatticeSize();
    for (int site = 0; site < V; site++) {
        if (gauge == MAG) {
            Complex<double> X[3];
            dGff[site] = 0.0;
            for (int mu = 0; mu < 4; mu++) {
                s.setLatticeIndex(site);
                TLinkCoord linkUp(U, s, mu);
                SU3<TLinkCoord> globUp(linkUp);
                SU3<Matrix<Complex<Real>, 3>> locUp;
                locUp.assignWithoutThirdLine(globUp);
                locUp.reconstructThirdLine();
                s.setNeighbour(mu, false);
                TLinkCoord linkDw(U, s, mu);
                SU3<TLinkCoord> globDw(linkDw);
                SU3<Matrix<Complex<Real>, 3>> locDw;
                locDw.assignWithoutThirdLine(globDw);
                locDw.reconstructThirdLine();
                for (int j = 0; j < 3; j++) dGff[site] += locUp.get(j, j).abs_squared();
                Matrix<Complex<Real>, 2> mat;
                Complex<Real> c;
                for (int i = 0; i < 2; i++)
                    for (int j = i + 1; j < 3; j++) {
                        mat = locUp.getSubgroupMatrix(i, j);
                        c = mat.get(0, 0) * mat.get(1, 0).conj() - mat.get(0, 1) * mat.get(1, 1).conj();
                        X[i + j - 1].x += (double)c.x;
                        X[i + j - 1].y += (double)c.y;
                        mat = locDw.getSubgroupMatrixHermitian(i, j);
                        c = mat.get(0, 0) * mat.get(1, 0).conj() - mat.get(0, 1) * mat.get(1, 1).conj();
                        X[i + j - 1].x += (double)c.x;
                        X[i + j - 1].y += (double)c.y;
                    }
            }
            dA[site] = X[0].abs() + X[1].abs() + X[2].abs();
            continue;
        }
        const int mu0 = (gauge == COULOMB) ? 1 : 0;
        Matrix<Complex<Real>, 3> locMatSum;
        SU3<Matrix<Complex<Real>, 3>> Sum(locMatSum);
        Sum.zero();
        for (int mu = mu0; mu < 4; mu++) {
            s.setLatticeIndex(site);
            Matrix<Complex<Real>, 3> locMat;
            SU3<Matrix<Complex<Real>, 3>> temp(locMat);
            TLinkCoord linkUp(U, s, mu);
            SU3<TLinkCoord> globUp(linkUp);
            temp.assignWithoutThirdLine(globUp);
            temp.reconstructThirdLine();
            Sum += temp;
            s.setNeighbour(mu, false);
            TLinkCoord linkDw(U, s, mu);
            SU3<TLinkCoord> globDw(linkDw);
            temp.assignWithoutThirdLine(globDw);
            temp.reconstructThirdLine();
            Sum -= temp;
        }
        Sum -= Sum.trace() / Real(3.);
        Matrix<Complex<Real>, 3> locMatSumHerm;
        SU3<Matrix<Complex<Real>, 3>> SumHerm(locMatSumHerm);
        SumHerm = Sum;
        SumHerm.hermitian();
        Sum -= SumHerm;
        double prec = 0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) prec += Sum.get(i, j).abs_squared();
        dA[site] = prec;
        s.setLatticeIndex(site);
        double result = 0;
        Matrix<Complex<Real>, 3> locTemp;
        SU3<Matrix<Complex<Real>, 3>> temp(locTemp);
        for (int mu = mu0; mu < 4; mu++) {
            TLinkCoord linkUp(U, s, mu);
            SU3<TLinkCoord> globUp(linkUp);
            temp.assignWithoutThirdLine(globUp);
            temp.reconstructThirdLine();
            result += temp.trace().x;
        }
        dGff[site] = result;
    }
}

/* COMKSU3::projectSU3 (CommonKernelsSU3.hxx:71-90): SU3<Link>::projectSU3 on every link */
void REF_SFX(ref_project)(Real *U, const int32_t size_in[4])
{
    lat_coord_t size[4];
    for (int i = 0; i < 4; i++) size[i] = (lat_coord_t)size_in[i];
    SiteIndex<4, FULL_SPLIT> s(size);
    const int V = s.getLatticeSize();
    for (int site = 0; site < V; site++) {
        s.setLatticeIndex(site);
        for (int mu = 0; mu < 4; mu++) {
            TLinkIndex linkUp(U, s, mu);
            SU3<TLinkIndex> globUp(linkUp);
            globUp.projectSU3();
        }
    }
}

/* COMKSU3::setHot (CommonKernelsSU3.hxx:92-130) */
void REF_SFX(ref_set_hot)(Real *U, const int32_t size_in[4], uint32_t seed, uint32_t counter)
{
    lat_coord_t size[4];
    for (int i = 0; i < 4; i++) size[i] = (lat_coord_t)size_in[i];
    SiteIndex<4, FULL_SPLIT> s(size);
    const int V = s.getLatticeSize();
    for (int site = 0; site < V; site++) {
        s.setLatticeIndex(site);
        PhiloxWrapper rng(site, (int)seed, counter);
        Quaternion<Real> q;
        for (int mu = 0; mu < 4; mu++) {
            TLinkIndex linkUp(U, s, mu);
            SU3<TLinkIndex> globUp(linkUp);
            Matrix<Complex<Real>, 3> locMat;
            SU3<Matrix<Complex<Real>, 3>> locU(locMat);
            locU.identity();
            for (int i = 0; i < 2; i++)
                for (int j = i + 1; j < 3; j++) {
                    q[0] = rng.rand() * 2.0 - 1.0;
                    q[1] = rng.rand() * 2.0 - 1.0;
                    q[2] = rng.rand() * 2.0 - 1.0;
                    q[3] = rng.rand() * 2.0 - 1.0;
                    q.projectSU2();
                    locU.rightSubgroupMult(i, j, &q);
                }
            globUp = locU;
        }
    }
}

/* PhiloxWrapper::rand() sequence for one thread (PhiloxWrapper.hxx:92-137) */
void REF_SFX(ref_rand_sequence)(uint32_t tid, uint32_t seed, uint32_t counter, int n, double *out)
{
    PhiloxWrapper rng((int)tid, (int)seed, counter);
    for (int i = 0; i < n; i++) out[i] = (double)rng.rand();
}

/* the vendored Random123 Philox4x32-10 and u01 conversions */
void REF_SFX(ref_philox4x32_10)(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    philox4x32_ctr_t c = {{ctr[0], ctr[1], ctr[2], ctr[3]}};
    philox4x32_key_t k = {{key[0], key[1]}};
    philox4x32_ctr_t r = philox4x32(c, k);
    for (int i = 0; i < 4; i++) out[i] = r.v[i];
}

float REF_SFX(ref_u01_32_24)(uint32_t i) { return u01_open_open_32_24(i); }
double REF_SFX(ref_u01_64_53)(uint64_t i) { return u01_open_open_64_53(i); }

} /* extern "C" */
