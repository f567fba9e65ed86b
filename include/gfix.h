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
/* Compute capability the device code that runs on the current device was built for, as
 * major * 10 + minor (100 for sm_100a), from cudaFuncGetAttributes.  No counterpart in the
 * reference (its apps are built per architecture by their Makefile); needs a GPU. */
int gf_binary_arch(int *arch);

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

/* One parity pass of update rule `algo` (0 OR, 1 micro, 2 SA, 3 SR, 4 random) over the sites of
 * timeslices [t_begin, t_end) only, 4D gauges: the slab pass of the reference's MPI driver split
 * into boundary and interior (apps/MultiGPU_MPI/MultiGPU_MPI_Communicator.hxx:351-430), so the
 * interior runs while the boundary links are exchanged.  Philox as gf_sa_step. */
int gf_step_slices(int gauge, int real, int algo, void *U, const int32_t size[4], int parity, float param,
                   int seed, int rng_counter, int t_begin, int t_end, void *stream);
/* The same, with site h of the lattice drawing its random numbers as site h + rng_site_offset
 * (parity-split order): a t-slab of a larger lattice passes the offset of its first owned
 * timeslice, ((global t of local slice 0) x Vs / 2), so its heat bath draws the whole lattice's
 * stream and SA over slabs equals SA on the whole lattice. */
int gf_step_slices_at(int gauge, int real, int algo, void *U, const int32_t size[4], int parity, float param,
                      int seed, int rng_counter, int t_begin, int t_end, long long rng_site_offset, void *stream);
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

/* Gauge quality without any allocation.  No counterpart in the reference: it is
 * gf_stats_generate for callers that cannot call cudaMalloc -- host frameworks that own all
 * device memory through their own pool, or latency-critical loops where cudaMalloc's
 * device-wide synchronisation is not acceptable.  Its reduction scratch is a fixed array in
 * device memory (about 1 MiB, held by every GPU that loads the library until the process
 * exits), so lattices are limited to 16,777,216 sites (64^4); larger ones return
 * GF_ERR_INVALID.  Every call looks up that array's device address on the caller's current
 * device (nothing is kept across calls, so a device reset in between is harmless); the first
 * call on a device may load the library's module there: make it once before latency matters,
 * and before any stream capture.  All calls share the one array:
 * calls whose kernels overlap on the GPU (different streams or threads at the same time) race
 * and must be serialised by the caller.  Blocking, like gf_stats_generate; stopping = GF_MAX or GF_AVERAGE. */
int gf_quality_noalloc(int gauge, int real, const void *U, const int32_t size[4], int stopping,
                       void *stream, double *gff, double *theta);

/* ---- context level: batched, mixed-precision gauge fixing --------------------------------
 * A context holds one or more lattices ("instances": gauge copies, lattices of uneven extents)
 * in this library's packed 12-real layout.  Every parity pass is one launch over all instances;
 * convergence is decided per instance on the device, and converged instances drop out.
 * mixed = 1: instances sweep in FP32 until theta < switch_theta, then move (reunitarised in
 * FP64) to FP64 storage for the polish to theta < precision; mixed = 0: FP64 throughout.
 * The gauge functional and theta always accumulate in FP64.
 * This replaces the per-copy loop of the reference drivers
 * (apps/LandauGaugeFixingSU3_4D.cu:185-283, apps/MAGaugeFixingSU3_4D.cu:197-333), which fix
 * one configuration of compile-time extents at a time.
 * GF_COULOMB: every lattice is split into its Nt timeslices, which are fixed as independent
 * instances in the same launches (the reference fixes them one after the other,
 * apps/CoulombGaugeFixingSU3_4D.cu:199-311).  Their temporal links are not touched while they
 * sweep: each slice accumulates its gauge transformation W(t,x) instead, and gf_export applies
 * U_0(t,x) <- W(t,x) U_0(t,x) W(t+1,x)^dagger, which equals the reference's per-sweep left and
 * right multiplications of U_0 (CoulombKernelsSU3.hxx:226-247). */
typedef struct gf_ctx gf_ctx;

typedef struct gf_ctx_params {
    int gauge;             /* GF_LANDAU, GF_COULOMB, GF_MAG or GF_U1XU1 */
    int ninstances;        /* number of lattices, >= 1 */
    const int32_t *sizes;  /* 4 * ninstances extents {Nt, Nx, Ny, Nz}, all even */
    int mixed;             /* 0: FP64 only; 1: FP32 storage for the bulk, converted to FP64 for the
                              polish; 2 ("refine"): an FP64 master field plus an FP32 working copy
                              that also accumulates the gauge transformation W(x); at the switch
                              the master becomes W(x) U(x) W(x+mu)^dagger, so rounding in the FP32
                              phase never moves the field off its gauge orbit.  A GF_COULOMB slice
                              keeps its W in its own temporal planes: the fold applies the working
                              copy's W32 to the master's spatial links and multiplies it into the
                              master's W64, which gf_export applies to the temporal links */
    void *stream;          /* cudaStream_t to run on, or NULL for a stream of the context's own */
} gf_ctx_params;

/* the knobs of the reference's ProgramOptions (apps/program_options/ProgramOptions.hxx:223-266)
 * that drive the per-copy loop, plus the mixed-precision switch */
typedef struct gf_schedule {
    int random_trafo;      /* randomtrafo: random gauge transformation first */
    uint32_t seed;         /* seed (Philox key word 1; see rng_streams) */
    uint32_t rng_counter;  /* first Philox launch counter (PhiloxWrapper::getNextCounter) */
    int sa_steps;          /* sasteps */
    float sa_min, sa_max;  /* samin, samax */
    int sa_geometric;      /* 0: linear temperature steps (reference), 1: geometric */
    int micro_updates;     /* microupdates after each (micro_every-th) SA sweep */
    int or_max_iter;       /* ormaxiter: OR sweep budget (FP32 + FP64) */
    float or_parameter;    /* orparameter (omega) */
    double precision;      /* stop when theta < precision */
    double switch_theta;   /* mixed contexts: FP32 -> FP64 when theta < switch_theta */
    int check_precision;   /* checkprecision: sweeps between checks */
    int reproject;         /* reproject: sweeps between reunitarisations */
    int use_graphs;        /* 1: replay check chunks from CUDA graphs */
    int autotune;          /* 1: gf_autotune first if the context is not tuned yet */
    int micro_every;       /* micro steps after every micro_every-th SA sweep (reference: 1) */
    int sa_mode;           /* 0: linear (Landau/Coulomb apps), 1: geometric, 2: the MAG/U1xU1 apps'
                              do-while with a slowed window; 0 with sa_geometric = 1 means 1 */
    int sa_repeat;         /* SA (+ micro) sweeps per temperature (MAG app: 5) */
    double sa_slow_lo, sa_slow_hi; /* sa_mode 2: step / sa_slow_factor for T in [lo, hi] (the apps
                              compare the float T with double constants) */
    float sa_slow_factor;
    int sr_max_iter;       /* srmaxiter: stochastic relaxation sweeps before OR (MAG app) */
    float sr_parameter;    /* srparameter */
    double sr_stop_theta;  /* SR stops below max(precision, this) (MAG app: 1e-6) */
    int stall_checks;      /* mixed contexts: an FP32 instance also moves to FP64 after this many
                              checks in a row without theta falling below 0.98 x its best FP32
                              theta -- FP32 rounding has become the floor (MAG's theta stalls
                              near 2e-7 in FP32, far above any useful switch_theta); 0: off */
    int fold;              /* refine contexts (mixed = 2): 1 = iterative refinement -- below
                              switch_theta the FP32 working copy keeps sweeping, and after every
                              check W is folded into the FP64 master (U64 <- W U64 W^dagger), the
                              working copy restarts from the master, and theta is measured on the
                              master in FP64; FP64 sweeps only if folds stop gaining (stall_checks).
                              0 = switch to FP64 sweeps at switch_theta */
    int trace_checks;      /* > 0: record up to this many OR checks per instance (gf_trace); the
                              reference prints the same line at every check */
    double fold_exit;      /* fold mode: once the master's theta after a fold is below fold_exit x
                              precision, the instance finishes with FP64 sweeps.  The FP32 working
                              copy leaves a rounding-noise floor of about 1e-12 in the master's
                              theta that only FP64 sweeps remove (they do so within ~20 sweeps);
                              0: fold until theta < precision or the folds stall */
    int rng_streams;       /* Philox streams of the instances: 0 = instance i draws key word seed + i
                              (independent streams, the same launch counters); 1 = the reference
                              apps' one stream (lattice/rng/PhiloxWrapper.hxx:90,142-145): every
                              instance draws key word seed, instance i starting after the counters
                              instances 0 .. i-1 would have used fixed one after the other (random
                              trafo and SA; not with sr_max_iter > 0) -- for a Coulomb lattice the
                              timeslices then draw exactly what apps/CoulombGaugeFixingSU3_4D.cu
                              draws for them */
    int persistent;        /* 1: each check chunk's OR sweeps (and its reprojections) run as ONE
                              cooperative launch per precision, the parity passes separated by a
                              grid-wide barrier, instead of one launch per pass (the apps' loop,
                              apps/LandauGaugeFixingSU3_4D.cu:244-262, launches two kernels per
                              sweep); for small lattices, whose passes are shorter than a launch.
                              Contexts without the separate W array only (plain FP64, mixed = 1,
                              GF_COULOMB), check_precision <= 256; else GF_ERR_UNSUPPORTED */
    int wait_budget_us;    /* persistent: bound of every barrier wait (0: 1 s); a wait that runs out
                              stops the kernel and gf_fix returns GF_ERR_TIMEOUT, the context usable */
    int wait_test_missing; /* persistent: barrier arrivals that never come -- only for testing the
                              bounded wait; 0 in use */
} gf_schedule;

typedef struct gf_report {
    double gff, theta;     /* FP64 functional and theta at the last check */
    int or_sweeps;         /* OR sweeps done (FP32 + FP64) */
    int or_sweeps_fp64;    /* of which in FP64 */
    int sa_sweeps;         /* SA sweeps done */
    int converged;         /* theta < precision */
    int chunks;            /* check chunks launched */
    int sr_sweeps;         /* SR sweeps done */
} gf_report;

int gf_create(const gf_ctx_params *params, gf_ctx **out);
int gf_destroy(gf_ctx *ctx);
/* Load lattice `lattice` (0 .. ninstances-1) from a GpuPattern array (float or double; device
 * memory, or host memory with on_host = 1, in which case only rows 0,1 are copied); for
 * GF_COULOMB the array holds its Nt timeslices one after the other (GpuPatternTimeslice,
 * access_pattern/GpuPatternTimeslice.hxx:57-62).  Resets the state of its instances. */
int gf_import(gf_ctx *ctx, int lattice, int real, const void *U, int on_host);
/* Write lattice `lattice` back in the same layout, reunitarised in FP64 with row 2 rebuilt
 * (the reference's closing projectSU3, apps/LandauGaugeFixingSU3_4D.cu:271). */
int gf_export(gf_ctx *ctx, int lattice, int real, void *U, int on_host);
/* GF_COULOMB contexts holding gauge copies of one configuration (one lattice per copy): write the
 * lattice whose timeslice t is that of copy copy_of_slice[t] -- the best copy of every timeslice,
 * as apps/CoulombGaugeFixingSU3_4D.cu:303-311 keeps it -- with temporal links
 * W_a(t) U_0(t) W_b(t+1)^dagger for a = copy_of_slice[t], b = copy_of_slice[t+1]. */
int gf_export_slices(gf_ctx *ctx, const int *copy_of_slice, int real, void *U, int on_host);
/* nsweeps full sweeps (both parities) of one algorithm (0 OR, 1 micro, 2 SA, 3 SR, 4 random
 * trafo) on every instance still sweeping; Philox counters rng_counter, rng_counter+1, ... */
int gf_sweeps(gf_ctx *ctx, int algo, int nsweeps, float param, int seed, int rng_counter);
/* FP64 functional and theta of every instance (one per lattice, or per timeslice for
 * GF_COULOMB: arrays of that many doubles). */
int gf_quality_all(gf_ctx *ctx, double *gff, double *theta);
/* Reunitarise every instance in its current storage (FP64 arithmetic). */
int gf_reunitarize(gf_ctx *ctx);
/* Move every FP32 instance of a mixed context to FP64 storage (reunitarised in FP64). */
int gf_set_storage(gf_ctx *ctx, int real);
/* The whole per-copy schedule for all instances; reports has one entry per instance (per
 * timeslice for GF_COULOMB), or NULL. */
int gf_fix(gf_ctx *ctx, const gf_schedule *schedule, gf_report *reports);
/* Autotuner: times the candidate launch shapes of the OR parity pass (one warp per 8-site tile;
 * the same capped at 64 registers (FP32); persistent with the next tile prefetched into
 * registers; FP32 with one thread per site; pipelined with cp.async prefetch and 2, 4 or 8 warps
 * per block; two lanes per site, direct and persistent with register prefetch) on a scratch copy of
 * the field (and of W in refine contexts) and keeps the fastest per precision.  Outputs: 0 = direct,
 * 64 = direct with 64 registers, 100 = register prefetch, 32 = thread per site, 33 = thread per site
 * pipelined with cp.async, 2/4/8 = warps per block of the pipelined pass, 16 = two lanes per site,
 * 116 = two lanes per site with register prefetch, each + 1000 when the passes alternate their walk
 * order, + 10000 with capped registers (gf_set_pass_order) and + 100000 with three cp.async stages
 * (gf_set_pass_stages) (-1: precision not used). */
int gf_autotune(gf_ctx *ctx, int *choice_fp32, int *choice_fp64);
/* Fix the launch shape instead: variant 0 (direct), 1 (pipelined, warps = 2, 4 or 8), 2 (FP32
 * direct capped at 64 registers), 3 (register prefetch), 4 (FP32, one thread per site), 5 (FP32,
 * one thread per site pipelined; OR, the other rules run as 4), 6 (two lanes per site) or 7 (two
 * lanes per site with register prefetch; OR, the other rules run as 6).  GF_COULOMB: 0, 2, 3, 6 or 7;
 * refine FP32: not 1. */
int gf_set_pass_shape(gf_ctx *ctx, int real, int variant, int warps);
/* Walk order and occupancy of the persistent passes (variants 1, 3, 7): alternate = 1 walks the
 * tiles of every odd-parity pass from the last to the first, so each pass begins on the links the
 * previous pass touched last and still finds them in L2; capped = 1 caps the registers of variants 1
 * (4 warps per block) and 7 so that more warps are resident.  gf_set_pass_shape resets both to 0. */
int gf_set_pass_order(gf_ctx *ctx, int real, int alternate, int capped);
/* cp.async stages per warp of the pipelined pass (variant 1 with 4 warps per block): 2 (default)
 * keeps the next 8-site tile in flight while the current one is computed, 3 the next two (twice the
 * bytes in flight for the same resident warps; the FP64 pass's choice on a B200).  GF_ERR_INVALID
 * for 3 with any other launch shape; gf_set_pass_shape resets it to 2. */
int gf_set_pass_stages(gf_ctx *ctx, int real, int stages);
/* Number of instances (lattices, or timeslices for GF_COULOMB). */
int gf_instances(gf_ctx *ctx);
/* The OR checks of the last gf_fix with schedule.trace_checks > 0: for instance `instance`, up to
 * max_entries entries of 4 doubles {OR sweeps so far, precision of the check (0 = FP32 working
 * copy, 1 = FP64, 4 = FP64 master right after an iterative-refinement fold), functional, theta};
 * *n = entries available (at most trace_checks: the first ones are kept); call with max_entries =
 * 0 to size the buffer. */
int gf_trace(gf_ctx *ctx, int instance, double *out, int max_entries, int *n);
/* Number of kernels this context has launched so far (each node of a replayed graph counts). */
int gf_kernel_launches(gf_ctx *ctx, long long *count);

/* ---- configuration files (lattice/LinkFile.hxx, lattice/filetypes/, apps/ildg.cpp, apps/qcdstag.cpp)
 * Read a configuration into / write one from the array U (18 reals per link, like the plugin
 * entry points) of the given precision, on the device (on_device = 1) or in host memory, in the
 * layout GF_LAYOUT_GPU (GpuPattern, access_pattern/GpuPattern.hxx:53-56) or GF_LAYOUT_TIMESLICE
 * (GpuPatternTimeslice, access_pattern/GpuPatternTimeslice.hxx:57-62: the Nt timeslices one
 * after the other, each the GpuPattern array of its {1, Nx, Ny, Nz} lattice -- what the Coulomb
 * drivers and gf_import of a GF_COULOMB context use; the reference's readILDG_timeslice /
 * readQCDSTAG_timeslice, apps/ildg.cpp:240-451, apps/qcdstag.cpp:123-227).  The payload is
 * transcoded on the GPU in one pass.
 *  GF_FILE_PLAIN       StandardPattern array of file_real reals, no header (LinkFile.hxx:83-167)
 *  GF_FILE_HEADERONLY  header of (file size - payload) bytes, then PLAIN; on writing, the header
 *                      is copied from template_path (FileHeaderOnly.hxx:72-103)
 *  GF_FILE_VOGT        7 shorts {4, 3, Nt, Nx, Ny, Nz, sizeof(real)}, then PLAIN (FileVogt.hxx:60-108)
 *  GF_FILE_ILDG        LIME container, "ildg-binary-data" in big-endian doubles, x fastest, file
 *                      directions (x,y,z,t) = internal (1,2,3,0); on writing, every other record of
 *                      template_path is copied and "xlf-info" gets " SA steps <sa_steps>" appended
 *                      (apps/ildg.cpp:26-238)
 *  GF_FILE_QCDSTAG     native doubles, direction-major, x fastest, directions as stored
 *                      (apps/qcdstag.cpp:17-67)
 * ILDG and QCDSTAG are always double; file_real is used by PLAIN / HEADERONLY / VOGT.  Blocking. */
#define GF_FILE_PLAIN 0
#define GF_FILE_HEADERONLY 1
#define GF_FILE_VOGT 2
#define GF_FILE_ILDG 3
#define GF_FILE_QCDSTAG 4
#define GF_LAYOUT_GPU 0
#define GF_LAYOUT_TIMESLICE 1
int gf_file_read(const char *path, int format, int file_real, const int32_t size[4], int real, int layout, void *U,
                 int on_device, void *stream);
int gf_file_write(const char *path, int format, int file_real, const int32_t size[4], int real, int layout,
                  const void *U, int on_device, const char *template_path, int sa_steps, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* GFIX_H */
