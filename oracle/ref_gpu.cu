// ref_gpu.cu -- boost-free host harness around the reference's OWN CUDA kernels
// (TEST INFRASTRUCTURE ONLY).  Compiled by oracle/Makefile, per lattice extent and precision,
// against the reference tree read in place, into oracle/_ref/libref_gpu_<X>x<T>_<prec>.so.
//
// The reference's apps need boost and MPI, which this image does not have; everything below the
// app layer -- the plugin classes (gaugefixing/*KernelsSU3.hxx), CommonKernelsSU3,
// GaugeFixingStats, the lattice templates and GlobalConstants.cu -- compiles unchanged for
// sm_100a.  This file only exposes the static launch wrappers through a C ABI, with the launch
// geometry the reference apps use (apps/LandauGaugeFixingSU3_4D.cu:119-120: V/2/NSB blocks of
// 8*NSB threads; CoulombGaugeFixingSU3_4D.cu:137-138 with the timeslice volume).  Extents are
// compile-time (-D_X_ -D_T_), as in the reference (gaugefixing/GlobalConstants.h:35-56).
// U1xU1KernelsSU3.hxx reuses the include guard of LandauKernelsSU3.hxx and the shared headers
// define non-inline symbols, so the U(1)xU(1) plugin is built as a library of its own
// (-DREFGPU_U1); both libraries export the same entry points.
#include <cstdio>

#include "lattice/access_pattern/GpuPattern.hxx"
#include "lattice/SiteCoord.hxx"
#include "lattice/SiteIndex.hxx"
#include "gaugefixing/GlobalConstants.h"
#include "gaugefixing/GaugeFixingStats.hxx"
#ifdef REFGPU_U1
#include "gaugefixing/U1xU1KernelsSU3.hxx"
#else
#include "gaugefixing/LandauKernelsSU3.hxx"
#include "gaugefixing/CoulombKernelsSU3.hxx"
#include "gaugefixing/MAGKernelsSU3.hxx"
#endif
#include "gaugefixing/CommonKernelsSU3.hxx"

namespace {

int volume() { return Nt * Nx * Ny * Nz; }
int timeslice_volume() { return Nx * Ny * Nz; }

template <class G>
void step(int algo, Real *U, lat_index_t *nn, bool parity, float param, int seed, int counter)
{
    const int a = volume() / 2 / NSB, b = 8 * NSB;
    switch (algo) {
    case 0: G::orStep(a, b, U, nn, parity, param); break;
    case 1: G::microStep(a, b, U, nn, parity); break;
    case 2: G::saStep(a, b, U, nn, parity, param, seed, counter); break;
    default: G::randomTrafo(a, b, U, nn, parity, seed, counter); break;
    }
}

}  // namespace

extern "C" {

// extents this library was built for: {Nt, Nx, Ny, Nz}; returns sizeof(Real)
int refgpu_config(int *size)
{
    size[0] = Nt;
    size[1] = Nx;
    size[2] = Ny;
    size[3] = Nz;
    return (int)sizeof(Real);
}

// reference neighbour table of the full lattice (timeslice = 0) or of one timeslice (= 1)
void refgpu_neighbour_table(int timeslice, lat_index_t *nn_host)
{
    SiteIndex<4, FULL_SPLIT> s(timeslice ? HOST_CONSTANTS::SIZE_TIMESLICE : HOST_CONSTANTS::SIZE);
    s.calculateNeighbourTable(nn_host);
}

// One parity pass with the reference kernels.  gauge: 0 Landau, 1 Coulomb (UtUp = U, UtDw),
// 2 MAG, 3 U1xU1; algo: 0 OR, 1 micro, 2 SA, 3 SR (MAG only), 4 random trafo.
int refgpu_step(int gauge, int algo, Real *U, Real *Udw, lat_index_t *nn, int parity, float param, int seed,
                int counter)
{
    const bool p = parity != 0;
#ifdef REFGPU_U1
    if (gauge != 3 || algo == 3) return -1;
    step<U1xU1KernelsSU3>(algo, U, nn, p, param, seed, counter);
    (void)Udw;
#else
    if (gauge == 1) {
        const int a = timeslice_volume() / 2 / NSB, b = 8 * NSB;
        switch (algo) {
        case 0: CoulombKernelsSU3::orStep(a, b, U, Udw, nn, p, param); break;
        case 1: CoulombKernelsSU3::microStep(a, b, U, Udw, nn, p); break;
        case 2: CoulombKernelsSU3::saStep(a, b, U, Udw, nn, p, param, seed, counter); break;
        case 4: CoulombKernelsSU3::randomTrafo(a, b, U, Udw, nn, p, seed, counter); break;
        default: return -1;
        }
    } else if (gauge == 2) {
        if (algo == 3)
            MAGKernelsSU3::srStep(volume() / 2 / NSB, 8 * NSB, U, nn, p, param, seed, counter);
        else
            step<MAGKernelsSU3>(algo, U, nn, p, param, seed, counter);
    } else if (gauge == 0) {
        if (algo == 3) return -1;
        step<LandauKernelsSU3>(algo, U, nn, p, param, seed, counter);
    } else {
        return -1;
    }
#endif
    return (int)cudaGetLastError();
}

// GaugeFixingStats<4,3,GType,AVERAGE>::generateGaugeQuality (blocking).  The reference's
// destructor calls cudaFree(&dGff) (GaugeFixingStats.hxx:116-120), which fails with
// cudaErrorInvalidValue and leaks the two V-double arrays; that error is cleared here and the
// kernels' status is reported through cudaDeviceSynchronize.
static int quality_status()
{
    cudaGetLastError();
    return (int)cudaDeviceSynchronize();
}

int refgpu_quality(int gauge, Real *U, double *gff, double *theta)
{
#ifdef REFGPU_U1
    if (gauge != 3) return -1;
    {
    GaugeFixingStats<4, 3, U1xU1KernelsSU3, AVERAGE> st(U, HOST_CONSTANTS::SIZE);
    st.generateGaugeQuality();
    *gff = st.getCurrentGff();
    *theta = st.getCurrentA();
    }
    return quality_status();
#else
    switch (gauge) {
    case 0: {
        GaugeFixingStats<4, 3, LandauKernelsSU3, AVERAGE> st(U, HOST_CONSTANTS::SIZE);
        st.generateGaugeQuality();
        *gff = st.getCurrentGff();
        *theta = st.getCurrentA();
        break;
    }
    case 1: {
        GaugeFixingStats<4, 3, CoulombKernelsSU3, AVERAGE> st(U, HOST_CONSTANTS::SIZE_TIMESLICE);
        st.generateGaugeQuality();
        *gff = st.getCurrentGff();
        *theta = st.getCurrentA();
        break;
    }
    case 2: {
        GaugeFixingStats<4, 3, MAGKernelsSU3, AVERAGE> st(U, HOST_CONSTANTS::SIZE);
        st.generateGaugeQuality();
        *gff = st.getCurrentGff();
        *theta = st.getCurrentA();
        break;
    }
    default: return -1;
    }
    return quality_status();
#endif
}

// CommonKernelsSU3::projectSU3 over the full lattice (timeslice = 0) or one timeslice (= 1)
int refgpu_project(int timeslice, Real *U)
{
    if (timeslice)
        CommonKernelsSU3::projectSU3(timeslice_volume() / 32, 32, U, HOST_CONSTANTS::getPtrToDeviceSizeTimeslice());
    else
        CommonKernelsSU3::projectSU3(volume() / 32, 32, U, HOST_CONSTANTS::getPtrToDeviceSize());
    return (int)cudaGetLastError();
}

}  // extern "C"

#ifndef REFGPU_U1
namespace {

// The overrelaxation phase of the apps' per-copy loop, on the reference's own kernels:
// apps/LandauGaugeFixingSU3_4D.cu:244-271 (MAG: apps/MAGaugeFixingSU3_4D.cu:300-329) -- orStep for
// parity 0 and 1; projectSU3 when i % reproject == 0; generateGaugeQuality when
// i % checkprecision == 0, leaving the loop once A < precision (a float, as the apps' option);
// the closing projectSU3.  One GaugeFixingStats serves the whole loop, as the apps' gaugeStats does.
template <class G>
int or_loop(Real *U, lat_index_t *nn, float omega, float precision, int check, int reproject, int max_iter,
            double *gff, double *theta, int *sweeps, float *ms)
{
    const int a = volume() / 2 / NSB, b = 8 * NSB;
    GaugeFixingStats<4, 3, G, AVERAGE> st(U, HOST_CONSTANTS::SIZE);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    int done = 0;
    for (int i = 0; i < max_iter; i++) {
        G::orStep(a, b, U, nn, 0, omega);
        G::orStep(a, b, U, nn, 1, omega);
        if (i % reproject == 0) CommonKernelsSU3::projectSU3(volume() / 32, 32, U, HOST_CONSTANTS::getPtrToDeviceSize());
        done = i + 1;
        if (i % check == 0) {
            st.generateGaugeQuality();
            if (st.getCurrentA() < precision) break;
        }
    }
    CommonKernelsSU3::projectSU3(volume() / 32, 32, U, HOST_CONSTANTS::getPtrToDeviceSize());
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *gff = st.getCurrentGff();
    *theta = st.getCurrentA();
    *sweeps = done;
    return quality_status();
}

}  // namespace

extern "C" int refgpu_or_loop(int gauge, Real *U, lat_index_t *nn, float omega, float precision, int check,
                              int reproject, int max_iter, double *gff, double *theta, int *sweeps, float *ms)
{
    if (check < 1 || reproject < 1) return -1;
    if (gauge == 0) return or_loop<LandauKernelsSU3>(U, nn, omega, precision, check, reproject, max_iter, gff, theta,
                                                     sweeps, ms);
    if (gauge == 2) return or_loop<MAGKernelsSU3>(U, nn, omega, precision, check, reproject, max_iter, gff, theta,
                                                  sweeps, ms);
    return -1;
}
#endif
