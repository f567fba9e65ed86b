/*
 * gfix.h -- C ABI of su3_ma_gauge_gpu_b200, a B200-native (sm_100a) SU(3) gauge-fixing sweep.
 *
 * The library is a drop-in for the gauge-fixing "plugin" classes of cuLGT
 * (ilyakudrov/SU3_MA_gauge_GPU): LandauKernelsSU3, CoulombKernelsSU3, MAGKernelsSU3,
 * U1xU1KernelsSU3, CommonKernelsSU3 and GaugeFixingStats.  Those are C++ classes of static
 * launch wrappers over compile-time lattice extents; here every entry point is a plain C
 * function with runtime extents, an explicit precision and an explicit CUDA stream, returning a
 * status code (GF_OK = 0).  Nothing calls exit().
 *
 * Field layout at the boundary: the reference device layout GpuPattern
 * (lattice/access_pattern/GpuPattern.hxx:53-56), i.e. for a lattice of V = Nt*Nx*Ny*Nz sites
 *     U[s + V*(c + 2*(j + 3*(i + 3*mu)))],  s = parity-split site index (SiteCoord.hxx:104-129),
 * mu = 0..3 (t, x, y, z), row i, column j, c = 0 (re) / 1 (im); float or double.  The sweeps
 * read and write rows 0 and 1 only and rebuild row 2 in registers, like the reference.
 * Coulomb entry points take one timeslice (size = {1, Nx, Ny, Nz}) plus the slice t-1 array.
 * All extents must be even and V < 2^31.  Pointers named U are device pointers.
 * The neighbour table of the reference (lat_index_t* nn) is not needed: neighbours are computed
 * from coordinates on the fly.
 */
#ifndef GFIX_H
#define GFIX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------- */
#define GF_OK 0
#define GF_ERR_INVALID 1     /* invalid argument: extents, pointers, enum values */
#define GF_ERR_CUDA 2        /* a CUDA call failed; gf_last_error_string() has the message */
#define GF_ERR_TIMEOUT 3     /* a bounded device-side wait gave up */
#define GF_ERR_NOMEM 4       /* device or host allocation failed */
#define GF_ERR_UNSUPPORTED 5 /* valid request that this build does not support */

/* gauge: the order of the reference's enum GaugeType (lattice/datatype/lattice_typedefs.h:43) */
#define GF_LANDAU 0
#define GF_COULOMB 1
#define GF_MAG 2
#define GF_U1XU1 3

/* arithmetic type of the field array */
#define GF_FP32 0
#define GF_FP64 1

/* stopping criterion: the order of the reference's enum StoppingCrit (lattice_typedefs.h:46) */
#define GF_MAX 0
#define GF_AVERAGE 1

/* Message of the last failing call on this host thread ("" if none). */
const char *gf_last_error_string(void);
/* Library version string. */
const char *gf_version(void);

/* ---- plugin level: one parity pass, in place on a GpuPattern device array ------------------
 * stream: a cudaStream_t, or NULL for the default stream.  Launches are asynchronous.
 * Udw: the slice t-1 array for GF_COULOMB (CoulombKernelsSU3::orStep(.., UtUp, UtDw, ..),
 *      CoulombKernelsSU3.hxx:88-91); ignored (may be NULL) for the other gauges. */

/* LandauKernelsSU3::orStep (LandauKernelsSU3.hxx:92-95) and its Coulomb/MAG/U1xU1 twins
 * (CoulombKernelsSU3.hxx:88-91, MAGKernelsSU3.hxx:93-96, U1xU1KernelsSU3.hxx:92-95) */
int gf_or_step(int gauge, int real, void *U, void *Udw, const int32_t size[4], int parity,
               float or_parameter, void *stream);
/* *KernelsSU3::microStep (LandauKernelsSU3.hxx:96-99) */
int gf_micro_step(int gauge, int real, void *U, void *Udw, const int32_t size[4], int parity,
                  void *stream);
/* *KernelsSU3::saStep (LandauKernelsSU3.hxx:100-103): Philox key (thread id, seed), counter
 * (k, rng_counter, 0x12345678, 0xabcdef09) exactly as lattice/rng/PhiloxWrapper.hxx:92-102 */
int gf_sa_step(int gauge, int real, void *U, void *Udw, const int32_t size[4], int parity,
               float temperature, int seed, int rng_counter, void *stream);
/* MAGKernelsSU3::srStep (MAGKernelsSU3.hxx:97-100); accepted for every gauge */
int gf_sr_step(int gauge, int real, void *U, void *Udw, const int32_t size[4], int parity,
               float sr_parameter, int seed, int rng_counter, void *stream);
/* *KernelsSU3::randomTrafo (LandauKernelsSU3.hxx:88-91) */
int gf_random_trafo(int gauge, int real, void *U, void *Udw, const int32_t size[4], int parity,
                    int seed, int rng_counter, void *stream);

/* *KernelsSU3::generateGaugeQualityPerSite (LandauKernelsSU3.hxx:71-74): per-site functional
 * and theta terms into device arrays of V doubles (either may be NULL). */
int gf_quality_per_site(int gauge, int real, const void *U, const int32_t size[4], double *dGff,
                        double *dA, void *stream);
/* *KernelsSU3::getGaugeQualityPrefactorGff / getGaugeQualityPrefactorA (LandauKernelsSU3.hxx:75-82) */
double gf_quality_prefactor_gff(int gauge);
double gf_quality_prefactor_a(int gauge);

/* CommonKernelsSU3::projectSU3 (CommonKernelsSU3.hxx:51-54): reunitarise every link and
 * rebuild row 2 (also the reference's "restore third line" at the end of a run); FP64 math. */
int gf_project_su3(int real, void *U, const int32_t size[4], void *stream);
/* CommonKernelsSU3::setHot (CommonKernelsSU3.hxx:56-59): random start, same Philox mapping. */
int gf_set_hot(int real, void *U, const int32_t size[4], int seed, int rng_counter, void *stream);

/* ---- GaugeFixingStats (GaugeFixingStats.hxx:55-70) ----------------------------------------
 * gf_stats_create allocates the reduction scratch (like the reference constructor, :83-99);
 * gf_stats_generate runs generateGaugeQuality (:186-232) -- one fused kernel with a
 * deterministic FP64 reduction -- and returns the normalised functional and theta (blocking,
 * like the reference's cudaMemcpy).  stopping = GF_MAX or GF_AVERAGE. */
typedef struct gf_stats gf_stats;
int gf_stats_create(int gauge, int real, const int32_t size[4], int stopping, gf_stats **out);
int gf_stats_generate(gf_stats *st, const void *U, void *stream, double *gff, double *theta);
int gf_stats_destroy(gf_stats *st);

#ifdef __cplusplus
}
#endif
#endif /* GFIX_H */
