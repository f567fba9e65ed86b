/*
 * gfix_culgt.hpp -- header-only C++ shim with the reference's plugin classes on top of gfix.h.
 *
 * A driver written against cuLGT's gauge-fixing headers recompiles unchanged against this
 * header: it provides LandauKernelsSU3, CoulombKernelsSU3, MAGKernelsSU3, U1xU1KernelsSU3,
 * CommonKernelsSU3 and GaugeFixingStats with the reference's static member names and argument
 * lists (gaugefixing/LandauKernelsSU3.hxx:55-106, CoulombKernelsSU3.hxx:53-101,
 * MAGKernelsSU3.hxx:57-111, U1xU1KernelsSU3.hxx:55-106, CommonKernelsSU3.hxx:38-61,
 * GaugeFixingStats.hxx:55-70) and forwards every call to the C ABI.
 *
 * Like the reference, the lattice extents and the precision are compile-time: -D_X_ -D_T_
 * [-D_Y_ -D_Z_] and -DDOUBLEPRECISION (gaugefixing/GlobalConstants.h:35-56,
 * lattice/datatype/datatypes.h:26-33).  The launch geometry arguments (a, b) and the
 * neighbour table are accepted and ignored.  The reference's wrappers return void; a failing
 * call here prints gf_last_error_string() and sets gfix_culgt::last_status.
 */
#ifndef GFIX_CULGT_HPP
#define GFIX_CULGT_HPP

#include <cstdio>

#include "gfix.h"

#ifndef _X_
#error "define _X_ and _T_ (lattice extents), as for the reference"
#endif

namespace gfix_culgt {

#ifdef DOUBLEPRECISION
typedef double real_t;
static const int kReal = GF_FP64;
#else
typedef float real_t;
static const int kReal = GF_FP32;
#endif
typedef int lat_index_t;
typedef short lat_coord_t;

#ifdef _Y_
static const int kNy = _Y_;
#else
static const int kNy = _X_;
#endif
#ifdef _Z_
static const int kNz = _Z_;
#else
static const int kNz = _X_;
#endif

inline const int32_t *lattice_size()
{
    static const int32_t s[4] = {_T_, _X_, kNy, kNz};
    return s;
}

inline const int32_t *timeslice_size()
{
    static const int32_t s[4] = {1, _X_, kNy, kNz};
    return s;
}

static int last_status = GF_OK;

inline void check(int st, const char *what)
{
    last_status = st;
    if (st != GF_OK) std::fprintf(stderr, "gfix: %s failed (%d): %s\n", what, st, gf_last_error_string());
}

template <int GAUGE>
struct GaugePlugin {
    static const int gauge = GAUGE;
    static void initCacheConfig() {}
    static void generateGaugeQualityPerSite(int, int, real_t *U, double *dGff, double *dA)
    {
        check(gf_quality_per_site(GAUGE, kReal, U, GAUGE == GF_COULOMB ? timeslice_size() : lattice_size(), dGff,
                                  dA, 0),
              "generateGaugeQualityPerSite");
    }
    static double getGaugeQualityPrefactorA() { return gf_quality_prefactor_a(GAUGE); }
    static double getGaugeQualityPrefactorGff() { return gf_quality_prefactor_gff(GAUGE); }
    static void restoreThirdLine(int, int, real_t *U, lat_index_t *)
    {
        check(gf_project_su3(kReal, U, GAUGE == GF_COULOMB ? timeslice_size() : lattice_size(), 0), "restoreThirdLine");
    }
};

template <int GAUGE>
struct LatticePlugin : GaugePlugin<GAUGE> {
    static void randomTrafo(int, int, real_t *U, lat_index_t *, bool parity, int rngSeed, int rngCounter)
    {
        check(gf_random_trafo(GAUGE, kReal, U, 0, lattice_size(), parity, rngSeed, rngCounter, 0), "randomTrafo");
    }
    static void orStep(int, int, real_t *U, lat_index_t *, bool parity, float orParameter)
    {
        check(gf_or_step(GAUGE, kReal, U, 0, lattice_size(), parity, orParameter, 0), "orStep");
    }
    static void microStep(int, int, real_t *U, lat_index_t *, bool parity)
    {
        check(gf_micro_step(GAUGE, kReal, U, 0, lattice_size(), parity, 0), "microStep");
    }
    static void saStep(int, int, real_t *U, lat_index_t *, bool parity, float temperature, int rngSeed,
                       int rngCounter)
    {
        check(gf_sa_step(GAUGE, kReal, U, 0, lattice_size(), parity, temperature, rngSeed, rngCounter, 0), "saStep");
    }
};

}  // namespace gfix_culgt

class LandauKernelsSU3 : public gfix_culgt::LatticePlugin<GF_LANDAU> {};
class U1xU1KernelsSU3 : public gfix_culgt::LatticePlugin<GF_U1XU1> {};

class MAGKernelsSU3 : public gfix_culgt::LatticePlugin<GF_MAG> {
public:
    static void srStep(int, int, gfix_culgt::real_t *U, gfix_culgt::lat_index_t *, bool parity, float srParameter,
                       int rngSeed, int rngCounter)
    {
        gfix_culgt::check(gf_sr_step(GF_MAG, gfix_culgt::kReal, U, 0, gfix_culgt::lattice_size(), parity, srParameter,
                                     rngSeed, rngCounter, 0),
                          "srStep");
    }
};

class CoulombKernelsSU3 : public gfix_culgt::GaugePlugin<GF_COULOMB> {
public:
    typedef gfix_culgt::real_t real_t;
    typedef gfix_culgt::lat_index_t lat_index_t;
    static void randomTrafo(int, int, real_t *UtUp, real_t *UtDw, lat_index_t *, bool parity, int rngSeed,
                            int rngCounter)
    {
        gfix_culgt::check(gf_random_trafo(GF_COULOMB, gfix_culgt::kReal, UtUp, UtDw, gfix_culgt::timeslice_size(),
                                          parity, rngSeed, rngCounter, 0),
                          "randomTrafo");
    }
    static void orStep(int, int, real_t *UtUp, real_t *UtDw, lat_index_t *, bool parity, float orParameter)
    {
        gfix_culgt::check(gf_or_step(GF_COULOMB, gfix_culgt::kReal, UtUp, UtDw, gfix_culgt::timeslice_size(), parity,
                                     orParameter, 0),
                          "orStep");
    }
    static void microStep(int, int, real_t *UtUp, real_t *UtDw, lat_index_t *, bool parity)
    {
        gfix_culgt::check(gf_micro_step(GF_COULOMB, gfix_culgt::kReal, UtUp, UtDw, gfix_culgt::timeslice_size(),
                                        parity, 0),
                          "microStep");
    }
    static void saStep(int, int, real_t *UtUp, real_t *UtDw, lat_index_t *, bool parity, float temperature,
                       int rngSeed, int rngCounter)
    {
        gfix_culgt::check(gf_sa_step(GF_COULOMB, gfix_culgt::kReal, UtUp, UtDw, gfix_culgt::timeslice_size(), parity,
                                     temperature, rngSeed, rngCounter, 0),
                          "saStep");
    }
};

class CommonKernelsSU3 {
public:
    static void initCacheConfig() {}
    // the reference passes a device pointer to the extents; the shim uses the compile-time ones
    // (the full lattice, or the timeslice when the caller passes the timeslice size pointer)
    static void projectSU3(int a, int b, gfix_culgt::real_t *U, const void *ptrToDeviceSize, bool timeslice = false)
    {
        (void)a;
        (void)b;
        (void)ptrToDeviceSize;
        gfix_culgt::check(gf_project_su3(gfix_culgt::kReal, U,
                                         timeslice ? gfix_culgt::timeslice_size() : gfix_culgt::lattice_size(), 0),
                          "projectSU3");
    }
    static void setHot(int, int, gfix_culgt::real_t *U, const void *, int rngSeed, int rngCounter)
    {
        gfix_culgt::check(gf_set_hot(gfix_culgt::kReal, U, gfix_culgt::lattice_size(), rngSeed, rngCounter, 0),
                          "setHot");
    }
};

/* GaugeFixingStats<Ndim, Nc, GType, ma>(U, size): ma = 0 (MAX) or 1 (AVERAGE), the values of
 * the reference's enum StoppingCrit (lattice/datatype/lattice_typedefs.h:46). */
template <int Ndim, int Nc, class GType, int ma>
class GaugeFixingStats {
public:
    GaugeFixingStats(gfix_culgt::real_t *U, const gfix_culgt::lat_coord_t *size) : U_(U)
    {
        int32_t s[4];
        for (int i = 0; i < 4; i++) s[i] = size[i];
        gfix_culgt::check(gf_stats_create(GType::gauge, gfix_culgt::kReal, s, ma, &h_), "GaugeFixingStats");
    }
    ~GaugeFixingStats() { gf_stats_destroy(h_); }
    void setPointer(gfix_culgt::real_t *U) { U_ = U; }
    void generateGaugeQuality()
    {
        gfix_culgt::check(gf_stats_generate(h_, U_, 0, &gff_, &a_), "generateGaugeQuality");
    }
    double getCurrentGff() { return gff_; }
    double getCurrentA() { return a_; }

private:
    GaugeFixingStats(const GaugeFixingStats &);
    GaugeFixingStats &operator=(const GaugeFixingStats &);
    gfix_culgt::real_t *U_;
    gf_stats *h_ = nullptr;
    double gff_ = 0, a_ = 0;
};

#endif /* GFIX_CULGT_HPP */
