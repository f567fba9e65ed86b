/*
 * gf_oracle.h -- CPU restatement of the cuLGT gauge-fixing sweep (TEST INFRASTRUCTURE ONLY).
 *
 * This is the parity oracle for the CUDA kernels of su3_ma_gauge_gpu_b200.  Only the tests,
 * the smoke check and the CPU-baseline leg of bench.py may load it.  The product library never
 * links it and never falls back to it.
 *
 * It restates, in plain C, the device code of the reference (ilyakudrov/SU3_MA_gauge_GPU, i.e.
 * cuLGT) for one parity pass of the red/black site update, the gauge quality and the
 * reprojection.  Every function names the reference file:line it follows.  Fields are held in
 * the reference device layout (GpuPattern, 18 reals per link, parity-split site order).
 *
 * Parity of this oracle is pinned two ways (tests/test_oracle_pin.py):
 *   - bit-exact against the reference's own host-compilable templates (lattice/SU3.hxx,
 *     Quaternion.hxx, Matrix.hxx, Complex.hxx, algorithms/{Or,Micro,Sa,Sr,Random}Update.hxx) and the vendored Random123
 *     Philox, compiled from the reference tree by oracle/Makefile into oracle/_ref/;
 *   - against golden vectors generated from that build (tests/golden/).
 */
#ifndef GF_ORACLE_H
#define GF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Gauge and algorithm codes.  The gauge order is the reference's enum GaugeType
 * (lattice/datatype/lattice_typedefs.h:43). */
enum { ORC_LANDAU = 0, ORC_COULOMB = 1, ORC_MAG = 2, ORC_U1XU1 = 3 };
enum { ORC_OR = 0, ORC_MICRO = 1, ORC_SA = 2, ORC_SR = 3, ORC_RANDOM = 4 };

/* Philox4x32-10 (Salmon et al., SC'11), as used through lattice/rng/PhiloxWrapper.hxx:92-137. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float orc_u01_open_open_32_24(uint32_t i);
double orc_u01_open_open_64_53(uint64_t i);
/* the first n values PhiloxWrapper::rand() returns for a thread key tid (test hook) */
void orc_rand_sequence_f64(uint32_t tid, uint32_t seed, uint32_t counter, int n, double *out);
void orc_rand_sequence_f32(uint32_t tid, uint32_t seed, uint32_t counter, int n, double *out);

/* Layout helpers: parity-split site index (SiteCoord.hxx:104-129), coordinates
 * (SiteCoord.hxx:147-175), neighbours and the reference neighbour table (SiteIndex.hxx:247-284).
 * size = {Nt, Nx, Ny, Nz}; x = {t, x, y, z}. */
int64_t orc_site_index(const int32_t size[4], const int32_t x[4]);
void orc_site_coords(const int32_t size[4], int64_t s, int32_t x[4]);
int64_t orc_neighbour(const int32_t size[4], int64_t s, int mu, int up);
void orc_neighbour_table(const int32_t size[4], int32_t *nn);

/* One parity pass of one update algorithm (a17: *KernelsSU3::orStep/microStep/saStep/srStep/
 * randomTrafo).  For COULOMB, size = {1, Nx, Ny, Nz}, Uup is the slice-t array and Udw the
 * slice-(t-1) array (CoulombKernelsSU3.hxx:208-250); for the other gauges Udw is ignored.
 * param = OR omega, SA temperature or SR probability (a float, as in the reference signatures).
 * seed / counter feed the Philox key/counter exactly as the reference kernels do. */
void orc_step_f64(double *Uup, double *Udw, const int32_t size[4], int gauge, int algo, int parity,
                  float param, uint32_t seed, uint32_t counter, int nthreads);
void orc_step_f32(float *Uup, float *Udw, const int32_t size[4], int gauge, int algo, int parity,
                  float param, uint32_t seed, uint32_t counter, int nthreads);

/* The same pass over the half-lattice sites h in [h_lo, h_hi) only (a timeslice range of a t-slab). */
void orc_step_range_f64(double *Uup, double *Udw, const int32_t size[4], int gauge, int algo, int parity,
                        float param, uint32_t seed, uint32_t counter, int64_t h_lo, int64_t h_hi, int nthreads);
void orc_step_range_f32(float *Uup, float *Udw, const int32_t size[4], int gauge, int algo, int parity,
                        float param, uint32_t seed, uint32_t counter, int64_t h_lo, int64_t h_hi, int nthreads);
/* The same with site h drawing its random numbers as site h + rng_site_offset (a t-slab's sites
 * draw the whole lattice's stream). */
void orc_step_range_at_f64(double *Uup, double *Udw, const int32_t size[4], int gauge, int algo, int parity,
                           float param, uint32_t seed, uint32_t counter, int64_t h_lo, int64_t h_hi,
                           int64_t rng_site_offset, int nthreads);
void orc_step_range_at_f32(float *Uup, float *Udw, const int32_t size[4], int gauge, int algo, int parity,
                           float param, uint32_t seed, uint32_t counter, int64_t h_lo, int64_t h_hi,
                           int64_t rng_site_offset, int nthreads);

/* Gauge quality (a18, a19): per-site arrays (optional, may be NULL) and the normalised
 * functional and theta as GaugeFixingStats::generateGaugeQuality (GaugeFixingStats.hxx:186-232)
 * returns them.  stop_max = 0 -> AVERAGE, 1 -> MAX.  For COULOMB pass the slice array with
 * size = {1, Nx, Ny, Nz}. */
void orc_quality_f64(const double *U, const int32_t size[4], int gauge, int stop_max,
                     double *gff, double *theta, double *gff_site, double *theta_site, int nthreads);
void orc_quality_f32(const float *U, const int32_t size[4], int gauge, int stop_max,
                     double *gff, double *theta, double *gff_site, double *theta_site, int nthreads);

/* Reunitarisation of every link, third row rebuilt (a20: CommonKernelsSU3.hxx:71-90). */
void orc_project_f64(double *U, const int32_t size[4], int nthreads);
void orc_project_f32(float *U, const int32_t size[4], int nthreads);

/* Random start (CommonKernelsSU3.hxx:92-130). */
void orc_set_hot_f64(double *U, const int32_t size[4], uint32_t seed, uint32_t counter, int nthreads);
void orc_set_hot_f32(float *U, const int32_t size[4], uint32_t seed, uint32_t counter, int nthreads);

/* Whole-run driver for one configuration of the Landau-type gauges (a21), following the
 * per-copy body of apps/LandauGaugeFixingSU3_4D.cu:185-271 (random trafo -> SA+micro loop ->
 * OR loop with reproject and check -> final projectSU3).  *counter is the host Philox counter
 * (PhiloxWrapper::getNextCounter) and is advanced as the reference advances it. */
typedef struct orc_schedule {
    int random_trafo;      /* 0/1 */
    int sa_steps;          /* sasteps */
    float sa_min, sa_max;  /* samin, samax */
    int micro_updates;     /* microupdates */
    int or_max_iter;       /* ormaxiter */
    float or_parameter;    /* orparameter */
    float precision;       /* precision (stored as float in the reference) */
    int check_precision;   /* checkprecision */
    int reproject;         /* reproject */
    uint32_t seed;         /* seed */
} orc_schedule;

typedef struct orc_result {
    double gff, theta;     /* last quality computed inside the OR loop */
    int or_iterations;     /* OR sweeps performed */
} orc_result;

void orc_fix_f64(double *U, const int32_t size[4], int gauge, const orc_schedule *sched,
                 uint32_t *counter, orc_result *res, int nthreads);
void orc_fix_f32(float *U, const int32_t size[4], int gauge, const orc_schedule *sched,
                 uint32_t *counter, orc_result *res, int nthreads);

/* Whole-run driver of one gauge copy as the apps run it, for every gauge:
 *   apps/LandauGaugeFixingSU3_4D.cu:185-271 (and U1xU1), apps/MAGaugeFixingSU3_4D.cu:197-333,
 *   the per-slice body of apps/CoulombGaugeFixingSU3_4D.cu:216-301 --
 * random gauge transformation; simulated annealing, either the Landau/Coulomb apps' for-loop over
 * sa_steps linearly falling temperatures (sa_mode 0) or the MAG/U1xU1 apps' do-while whose step is
 * divided by sa_slow_factor while the temperature lies in [sa_slow_lo, sa_slow_hi] (sa_mode 2),
 * each temperature running sa_repeat SA sweeps, each followed by micro_updates microcanonical
 * sweeps, with a reprojection at every temperature index i with i % reproject == 0; stochastic
 * relaxation (MAG) until theta < precision or theta < sr_stop_theta, checked at i % checkprecision
 * == 0; overrelaxation with the same check and reprojection cadence; the closing projectSU3.
 * For ORC_COULOMB, U is the slice-t array and Udw the slice-(t-1) array (size = {1, Nx, Ny, Nz});
 * both are reprojected, as the Coulomb app does.  *counter is the host Philox counter
 * (PhiloxWrapper::getNextCounter), advanced as the apps advance it. */
typedef struct orc_app_schedule {
    int random_trafo;
    int sa_steps;
    float sa_min, sa_max;
    int micro_updates;
    int sa_mode;            /* 0: for-loop, linear (Landau, Coulomb); 2: do-while with slowed window */
    int sa_repeat;          /* SA (+ micro) sweeps per temperature (MAG app: 5) */
    double sa_slow_lo, sa_slow_hi;
    float sa_slow_factor;
    int sr_max_iter;
    float sr_parameter;
    double sr_stop_theta;   /* MAG app: 1e-6 */
    int or_max_iter;
    float or_parameter;
    float precision;
    int check_precision;
    int reproject;
    uint32_t seed;
} orc_app_schedule;

typedef struct orc_app_result {
    double gff, theta;      /* last quality computed (OR loop, or SR loop if OR never checked) */
    int or_iterations, sa_sweeps, sr_iterations;
} orc_app_result;

void orc_fix_app_f64(double *U, double *Udw, const int32_t size[4], int gauge, const orc_app_schedule *sched,
                     uint32_t *counter, orc_app_result *res, int nthreads);
void orc_fix_app_f32(float *U, float *Udw, const int32_t size[4], int gauge, const orc_app_schedule *sched,
                     uint32_t *counter, orc_app_result *res, int nthreads);

/* The Coulomb app's slice loop (apps/CoulombGaugeFixingSU3_4D.cu:199-311) for one gauge copy:
 * timeslices t = 0 .. Nt-1 one after the other, each fixed by orc_fix_app with UtUp = slice t
 * and UtDw = slice t-1 (periodic) of the GpuPatternTimeslice array U (slice t at offset
 * 72 * Vs * t), the Philox counter running on from slice to slice.  res has Nt entries. */
void orc_fix_coulomb_f64(double *U, const int32_t size[4], const orc_app_schedule *sched, uint32_t *counter,
                         orc_app_result *res, int nthreads);
void orc_fix_coulomb_f32(float *U, const int32_t size[4], const orc_app_schedule *sched, uint32_t *counter,
                         orc_app_result *res, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
