/*
 * jimwlk.h -- C ABI of libjimwlk, a B200 (sm_100a) JIMWLK Langevin engine.
 *
 * Two layers:
 *
 *  1. Call-for-call replacements of the reference solver's hot-path functions
 *     (ElsevierSoftwareX/SOFTX-D-21-00092: field.h, mpi_fftw_class.h,
 *     su3_matrix.h, config.h), operating on device-resident fields.  A port of
 *     main_optimized.cpp's evolution loop replaces each reference call with
 *     the jw_* call named beside it and gets the reference's results (FP64,
 *     same operation order, noise from a seeded counter-based stream instead
 *     of the reference's clock-seeded ranlux24).
 *
 *  2. The batched engine: many independent events of (possibly different)
 *     lattice sizes resident on one GPU, advanced by fused kernels -- noise
 *     generation, the V xi V^dagger rotation, both momentum-space convolutions
 *     (FFT -> kernel multiply -> inverse FFT) and the SU(3) update -- in FP64
 *     or mixed precision (FP32 transforms, FP64 exponentials and V), with the
 *     dipole correlator accumulated on the device.
 *
 * Conventions
 *  - Every function returns a jw_status (0 = JW_OK, negative = error).
 *  - Host field arrays use the reference's layout (field.h:73, 170-173):
 *    site-major, interleaved complex double, component k (row-major 3x3 index
 *    3*row+col for t = 9; k = 0 for t = 1) of site (x, y) at complex offset
 *    (x*Ny + y)*t + k.
 *  - Work is ordered on the context's / engine's CUDA stream.  Functions that
 *    copy to or from the host synchronise that stream; the others only
 *    enqueue.  jw_context_sync / jw_engine_sync wait for completion and
 *    return the first device-side error flagged since the previous sync
 *    (JW_ENOCONV when the QL eigensolver did not converge at some site,
 *    JW_ENAN for a non-finite result).
 *  - A context or engine may be used from one host thread at a time.
 *  - Lattices are square (Nx == Ny).  A context (the call-for-call and
 *    position layers) takes any side from 2 to 2048; the batched engine and
 *    the server take powers of two from 8 to 2048.
 */
#ifndef JIMWLK_H
#define JIMWLK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int jw_status;
#define JW_OK 0
#define JW_EINVAL (-1)       /* bad argument (size, enum, null pointer, mismatched fields) */
#define JW_ENOMEM (-2)       /* device or host allocation failed / footprint over budget */
#define JW_ECUDA (-3)        /* a CUDA runtime call failed */
#define JW_ENOCONV (-4)      /* eigensolver QL fallback did not converge at some site */
#define JW_ENAN (-5)         /* non-finite value produced */
#define JW_ETIMEOUT (-6)     /* a bounded wait ran out */
#define JW_EUNSUPPORTED (-7) /* option the reference does not define (e.g. HATTA in momentum space) */
#define JW_ENOTFOUND (-8)    /* unknown event / request id */
#define JW_EBUSY (-9)        /* resource in use */

const char* jw_status_string(jw_status s);

/* ------------------------------------------------------------------ config */
/* Enumerations with the reference's values (config.h:38-42). */
#define JW_POSITION_EVOLUTION 0
#define JW_MOMENTUM_EVOLUTION 1
#define JW_SQRT_COUPLING_CONSTANT 0
#define JW_NOISE_COUPLING_CONSTANT 1
#define JW_HATTA_COUPLING_CONSTANT 2
/* Fixed coupling (alpha_s folded into `step`): the reference's plain
 * generate_gaussian (field.h:2116) with the NOISE_COUPLING_CONSTANT kernel
 * factor 1 (field.h:2035-2036, 2049-2050).  main_optimized.cpp:243-247 pairs
 * NOISE with the site-indexed noise factor instead, so this value exists only
 * in this library. */
#define JW_FIXED_COUPLING_CONSTANT 3
#define JW_LINEAR_KERNEL 0
#define JW_SIN_KERNEL 1

/* class config (config.h:44-73); Nx, Ny are compile-time macros there
 * (config.h:31-32) and run-time fields here. */
typedef struct jw_config {
    int Nx, Ny;
    int stat;
    double mu;
    double mass;
    int elementaryWilsonLines;
    char file_name[64];
    int langevin_steps;
    int measurements;
    double step;
    int EvolutionChoice;
    int CouplingChoice;
    int KernelChoice;
    uint64_t seed; /* noise stream key (the reference seeds from the clock) */
} jw_config;

/* Defaults of config.h:60-73 with Nx = Ny = 64, seed = 1. */
jw_status jw_config_defaults(jw_config* cfg);
/* config::read_config_from_file (config.h:76-136): same line grammar; mu,
 * mass and step are parsed through float exactly as the reference does, so
 * the doubles match it bit for bit.  Unknown choice strings keep the
 * previous value, as in the reference. */
jw_status jw_config_read(jw_config* cfg, const char* path);

/* ------------------------------------------------------------------ context & fields */
typedef struct jw_context jw_context;
typedef struct jw_field jw_field;

/* Replaces the set-up of main_optimized.cpp:68-92 (mpi_class, momenta,
 * positions, fftw2D::init2D): binds device `device`, creates a stream and the
 * FFT twiddle tables for cfg->Nx.  Nx = Ny, any size from 2 to 2048 (the
 * reference plans FFTW for any size, mpi_fftw_class.h:165-186); sizes that
 * are not powers of two transform by the chirp-z form.  JW_EUNSUPPORTED
 * otherwise.  The batched engine and the server take powers of two only. */
jw_status jw_context_create(const jw_config* cfg, int device, jw_context** out);
/* Also releases every field still open in the context; those handles are
 * invalid afterwards. */
jw_status jw_context_destroy(jw_context* ctx);
jw_status jw_context_sync(jw_context* ctx);
/* The context's cudaStream_t, as void*. */
void* jw_context_stream(jw_context* ctx);

/* lfield<double,t>(Nxl, Nyl) (field.h:152-283): t = 1 or 9, zero-filled. */
jw_status jw_field_create(jw_context* ctx, int t, jw_field** out);
jw_status jw_field_destroy(jw_field* f);
/* Host <-> device in the reference layout (2*t*Nx*Ny doubles). */
jw_status jw_field_set(jw_field* f, const double* host);
jw_status jw_field_get(const jw_field* f, double* host);
/* lfield::operator= (field.h:301-318). */
jw_status jw_field_copy(jw_field* dst, const jw_field* src);
/* No counterpart in the reference (it has no checkpoints).  A field to and
 * from a file: a 16-byte header ("JWFIELD1", int32 N, int32 t) and then
 * 2*t*N*N native doubles in the reference layout.  Loading checks N and t. */
jw_status jw_field_save(const jw_field* f, const char* path);
jw_status jw_field_load(jw_field* f, const char* path);
/* lfield::setToUnit / setToZero (field.h:181-211). */
jw_status jw_field_set_unit(jw_field* f);
jw_status jw_field_set_zero(jw_field* f);

/* ------------------------------------------------------------------ reference hot-path calls */
/* fftw2D::execute2D(lfield*, dir) (mpi_fftw_class.h:191-315): in-place 2-D
 * DFT of every component, dir = 1 X->K (exp(-i...)), dir = 0 K->X, then
 * x 1/sqrt(Nx*Ny). */
jw_status jw_execute2D(jw_context* ctx, jw_field* f, int dir);

/* generate_gaussian (field.h:2116-2243) and, when with_coupling != 0,
 * generate_gaussian_with_noise_coupling_constant (field.h:2245-2365): 16 unit
 * normals per site from the stream of (ctx seed, step_index), embedded as
 * sum_a n_a lambda_a into xi_x and sum_a m_a lambda_a into xi_y. */
jw_status jw_generate_gaussian(jw_context* ctx, jw_field* xi_x, jw_field* xi_y, uint64_t step_index,
                               int with_coupling);

/* lfield::setMVModel (field.h:683-757): 8 normals per site from the MV stream
 * of (ctx seed, slice) times sigma = g*mu/sqrt(Ny_slices), embedded. */
jw_status jw_set_mv_model(jw_context* ctx, jw_field* f, int slice, double g, double mu, int ny_slices);
/* lfield::solvePoisson (field.h:867-877): f(k) *= -g / (-phat2(k) + mass^2). */
jw_status jw_solve_poisson(jw_context* ctx, jw_field* f, double mass, double g);
/* lfield::operator*= (field.h:337-365): V(x) <- V(x) exp(+i f(x)). */
jw_status jw_mul_exp(jw_context* ctx, jw_field* V, const jw_field* f);

/* prepare_A_local(out, xi_x, xi_y, momenta, mpi, Coupling, Kernel) (field.h:1998-2075). */
jw_status jw_prepare_A_local(jw_context* ctx, jw_field* out, const jw_field* xi_x, const jw_field* xi_y,
                             int coupling, int kernel);
/* uxiulocal (field.h:1892-1933): ux = V xi_x V^dagger, uy = V xi_y V^dagger. */
jw_status jw_uxiulocal(jw_context* ctx, jw_field* ux, jw_field* uy, const jw_field* V, const jw_field* xi_x,
                       const jw_field* xi_y);
/* update_uf (field.h:1966-1996): V <- exp(+i sqrt(step) B) V exp(-i sqrt(step) A). */
jw_status jw_update_uf(jw_context* ctx, jw_field* V, const jw_field* B, const jw_field* A, double step);

/* lfield::trace (field.h:1375-1432): corr(k) = tr(Vk Vk^dagger)/(Nx Ny)^2, corr t = 1. */
jw_status jw_trace(jw_context* ctx, const jw_field* Vk, jw_field* corr);
/* gfield::average_and_symmetrize (field.h:1460-1492). */
jw_status jw_average_and_symmetrize(jw_context* ctx, jw_field* corr);
/* No counterpart in the reference.  jw_average_and_symmetrize for callers
 * that cannot allocate device memory: jw_context_create allocates (a stream,
 * tables and the scratch plane this operation needs), which a program that
 * hands all device memory to its own pool allocator, or a time-critical loop
 * that cannot afford cudaMalloc/cudaFree, must avoid.  corr is the caller's
 * device array of N*N complex doubles (element (kx, ky) at complex offset
 * kx*N + ky), symmetrised in place on `stream` (a cudaStream_t, 0 = the
 * default stream).  The scratch plane is a fixed array inside the library,
 * 512*512 complex doubles (4 MiB) on every GPU that loads it, held until the
 * process exits; N > 512 returns JW_EINVAL.  All calls share that array and
 * each call overwrites what it reads, so calls that overlap on the GPU race
 * and must be ordered by the caller.  corr must be 16-byte aligned
 * (JW_EINVAL otherwise).  CUDA loads the library's device code lazily, so the
 * array is reserved on a device by the first call there, which also looks up
 * its device address with that device current (again after the device's
 * context was reset).  A caller whose pool allocator takes the device's free
 * memory first calls jw_average_and_symmetrize_noalloc(NULL, 0, NULL) with
 * the device current, before the pool reserves its memory: that set-up call
 * launches nothing.  Make the first call before any stream capture begins.
 * Calls no cudaMalloc or cudaFree. */
jw_status jw_average_and_symmetrize_noalloc(double* corr, int N, void* stream);
/* gfield::reduce(sum, err, mpi) (field.h:1521-1536): sum += corr, err += corr^2. */
jw_status jw_reduce(jw_context* ctx, const jw_field* corr, jw_field* sum, jw_field* err);
/* No counterpart in the reference, which writes C(k) only (print).  The
 * dipole of one symmetrised correlator corr (t = 1, after jw_trace and
 * jw_average_and_symmetrize): S(x, y) = (N^2/3) sum_k corr(k) exp(+2 pi i
 * k.(x, y)/N), i.e. (1/3N^2) sum_z tr V(z) V(z + (x, y))^dagger; its angular
 * average over bins b = floor(|r| + 1/2) <= N/2 of minimum-image distances;
 * and Q_s = sqrt(2)/r_s with S(r_s) = exp(-1/2), linear between the bins that
 * bracket it (0 if none).  S_xy (N*N doubles, x-major) and the bins
 * (nbins_cap >= N/2 + 1) are optional. */
jw_status jw_dipole(jw_context* ctx, const jw_field* corr, double* S_xy, double* S_bins, double* r_bins, int* counts,
                    int nbins_cap, int* nbins, double* Qs);
/* print(measurement, sum, err, momenta, x, mpi, fileroot) (field.h:2521-2547):
 * appends to <fileroot>_<Nx>_<Ny>_mpi1_r0.dat. */
jw_status jw_print(jw_context* ctx, int measurement, const jw_field* sum, const jw_field* err, double x,
                   const char* fileroot);

/* Whole-driver conveniences built from the calls above (main_optimized.cpp). */
/* :88, 178-191 -- MV initial condition into V with the config's mu, mass,
 * elementaryWilsonLines (g = 1, mu_MV = mu/Nx). */
jw_status jw_initial_condition(jw_context* ctx, jw_field* V);
/* :243-269, 304 -- n momentum-space Langevin steps with global step indices
 * step0 .. step0+n-1 and the config's coupling, kernel and step. */
jw_status jw_evolve_momentum(jw_context* ctx, jw_field* V, uint64_t step0, int n);

/* ------------------------------------------------------------------ position-space evolution */
/* The loop of main_optimized.cpp:287-300 over every site, i.e.
 * prepare_A_and_B_local(x, y, x_global, y_global, xi_x, xi_y, A, B, uf,
 * positions, rr, Coupling, Kernel) (field.h:2368-2519) for all (x, y):
 *   A(x) = sum_y [k_x(x-y) xi_x(y) + k_y(x-y) xi_y(y)]
 *   B(x) = sum_y V(y) [k_x(x-y) xi_x(y) + k_y(x-y) xi_y(y)] V(y)^dagger
 * with the real kernel k_i(d) = c(d) d_i / r2(d) of positions::set
 * (positions.h:105-150) for the SIN kernel or the wrapped distance for the
 * LINEAR kernel, zero where r2 <= 1e-8.  c = 1 for NOISE and FIXED coupling,
 * sqrt(4 pi / (9 log((lambda + 1.26 / (36 r2 / N^2)^5)^0.2))) for SQRT and,
 * at min(r2, rr), for HATTA (the reference leaves c uninitialised there;
 * this is the formula its comments describe).  Computed as circular
 * convolutions through the transform (exact up to rounding).  The inputs are
 * not modified. */
jw_status jw_prepare_A_and_B(jw_context* ctx, jw_field* A, jw_field* B, const jw_field* xi_x,
                             const jw_field* xi_y, const jw_field* V, int rr, int coupling, int kernel);

/* lfield::setCorrelationsForCouplingConstant(momenta) (field.h:1633-1651):
 * corr(k) = 4 pi / (9 log((lambda + (phat2(k) N^2 / 36)^5)^0.2)) / N, t = 1.
 * main_optimized.cpp:147-149 follows it with jw_execute2D(corr, 0). */
jw_status jw_set_correlations_for_coupling_constant(jw_context* ctx, jw_field* corr);

/* gmatrix<double> holding the Cholesky factor (matrix.h:151-200). */
typedef struct jw_cholesky jw_cholesky;
/* gmatrix::decompose(corr) (matrix.h:151-200): the complex-symmetric
 * Cholesky factor L (L L^T = S, no conjugation) of the site-site matrix
 * S(i, j) = corr(|x_i - x_j|, |y_i - y_j|) (non-periodic distances), with
 * (Nx Ny)^2 complex doubles on the device (68.7 GB at 256^2).  JW_ENOMEM when
 * the device cannot hold it. */
jw_status jw_cholesky_decompose(jw_context* ctx, const jw_field* corr, jw_cholesky** out);
jw_status jw_cholesky_destroy(jw_cholesky* L);
/* L to the host in the reference layout: row-major, element (i, j) at
 * complex offset i * Nx*Ny + j, zero above the diagonal. */
jw_status jw_cholesky_get(const jw_cholesky* L, double* host);
/* gfield::multiplyByCholesky(gmatrix) (field.h:1653-1689): xi <- L xi for
 * each of the t components. */
jw_status jw_multiply_by_cholesky(jw_context* ctx, jw_field* xi, const jw_cholesky* L);

/* gfield::reduce_hatta(sum, err, mpi, xr, yr) (field.h:1538-1564): adds
 * corr(xr, yr) to sum(xr, yr) and its square to err(xr, yr). */
jw_status jw_reduce_hatta(jw_context* ctx, const jw_field* corr, jw_field* sum, jw_field* err, int xr, int yr);

/* :232-304 for EvolutionChoice == POSITION_EVOLUTION -- n position-space
 * steps (step indices step0 .. step0+n-1) with the config's coupling, kernel
 * and step: plain generate_gaussian noise, for NOISE coupling multiplied by
 * the Cholesky factor L (required then, ignored otherwise), then
 * jw_prepare_A_and_B with `rr` and jw_update_uf.  FIXED coupling is the
 * NOISE kernel factor 1 without the Cholesky factor. */
jw_status jw_evolve_position(jw_context* ctx, jw_field* V, uint64_t step0, int n, int rr, const jw_cholesky* L);

/* ------------------------------------------------------------------ batched engine */
#define JW_PRECISION_FP64 0  /* FP64 everywhere */
#define JW_PRECISION_MIXED 1 /* FP32 noise/rotation/transforms, FP64 exponentials, V, reunitarisation, sums */

typedef struct jw_engine_options {
    int precision;        /* JW_PRECISION_* */
    int reunitarize;      /* project V back onto SU(3) after every step (FP64) */
    size_t max_bytes;     /* device-memory budget for events and workspaces; 0 = 90% of free */
    int max_batch;        /* events advanced per launch group (0 = all) */
    size_t max_batch_sites; /* and at most this many lattice sites per launch group (0 = no limit;
                               at least one event), which also bounds each size's workspace */
    int autotune;         /* 1: the first mixed-precision run of each lattice size times
                             every compiled column-tile width of the column pass on its own
                             workspace and keeps the fastest (jw_engine_tuning); results do
                             not depend on the choice.  2: the column transforms' radix
                             schedules compete as well (radix-2/4 pass first or last, for N
                             that has one); a schedule rounds differently, so results then
                             depend on the recorded choice.  0: the built-in default */
} jw_engine_options;

typedef struct jw_event_desc {
    int N;                /* lattice side */
    int ny_slices;        /* MV slices (elementaryWilsonLines) */
    double mu;            /* config mu (mu_MV = mu/N, g = 1) */
    double mass;          /* config mass (Poisson mass = mass * mu_MV) */
    double step;          /* Langevin step (config step) */
    int coupling;         /* JW_SQRT_, JW_NOISE_, JW_FIXED_ (and, in position space, JW_HATTA_) COUPLING_CONSTANT */
    int kernel;           /* JW_SIN_KERNEL; JW_LINEAR_KERNEL in position space only (in momentum
                             space its multiplier is not Hermitian-symmetric at the Nyquist
                             lines, which the engine's packed coefficients cannot represent:
                             JW_EUNSUPPORTED, use the call-for-call layer) */
    uint64_t seed;        /* noise stream key of this event */
    /* 0: momentum-space steps (main_optimized.cpp:249-269).  Nonzero:
     * position-space steps (:271-302, jw_prepare_A_and_B) with plain noise;
     * coupling SQRT, FIXED (factor 1) or HATTA at min(r^2, rr).  NOISE in
     * position space needs the Cholesky factor and is JW_EUNSUPPORTED here
     * (use jw_evolve_position). */
    int position_space;
    int rr;               /* Hatta distance squared (position space, HATTA) */
    uint64_t step0;       /* noise index of the event's first step (default 0) */
} jw_event_desc;

typedef struct jw_engine jw_engine;

jw_status jw_engine_create(const jw_engine_options* opt, int device, jw_engine** out);
jw_status jw_engine_destroy(jw_engine* e);
jw_status jw_engine_sync(jw_engine* e);
void* jw_engine_stream(jw_engine* e);
/* Device bytes an event of this description holds while resident. */
size_t jw_engine_event_bytes(const jw_engine* e, const jw_event_desc* d);
/* Admit an event (allocates its V and accumulators; V = 1). */
jw_status jw_engine_add_event(jw_engine* e, const jw_event_desc* d, int* event_id);
jw_status jw_engine_remove_event(jw_engine* e, int event_id);
/* MV initial condition for the listed events (main_optimized.cpp:178-191). */
jw_status jw_engine_init_mv(jw_engine* e, const int* ids, int n);
/* Host V in the reference layout. */
jw_status jw_engine_set_V(jw_engine* e, int event_id, const double* host);
jw_status jw_engine_get_V(jw_engine* e, int event_id, double* host);
/* Advance the listed events by nsteps Langevin steps each (main_optimized.cpp:234-304
 * per step).  Mixed precision runs the steps of each launch group as pass 1,
 * then nsteps - 1 times (pass 2, pass 3 fused with the next pass 1), then pass 2
 * and pass 3, with the repeated part replayed as a CUDA graph; any split of
 * the steps into calls gives the same lattices bit for bit.  Asynchronous on
 * the engine stream (jw_engine_sync reports device errors). */
jw_status jw_engine_step(jw_engine* e, const int* ids, int n, int nsteps);
/* Dipole measurement of the listed events: C(k) of main_optimized.cpp:321-334
 * accumulated (sum, sum of squares) into each event's FP64 accumulators. */
jw_status jw_engine_measure(jw_engine* e, const int* ids, int n);
/* Accumulated sum / err (N*N complex each, reference layout t = 1) and count. */
jw_status jw_engine_get_correlator(jw_engine* e, int event_id, double* sum, double* err, int* nmeas);
/* Reset an event's accumulators. */
jw_status jw_engine_reset_correlator(jw_engine* e, int event_id);
/* Reset the accumulators of n events (one synchronisation). */
jw_status jw_engine_reset_correlators(jw_engine* e, const int* ids, int n);
/* V of event dst <- V of event src (same N), on the device: e.g. the Hatta
 * branches' common start uftmp = uf (main_optimized.cpp:230). */
jw_status jw_engine_copy_V(jw_engine* e, int dst, int src);
/* No counterpart in the reference.  Checkpoint of one event: its descriptor,
 * next noise index, measurement count, V (reference layout) and FP64
 * accumulators, so that a loaded event continues bit for bit.  File: the
 * header ("JWEVENT1", jw_event_desc, uint64 step, int32 nmeas, int32 0), then
 * 18*N*N doubles of V and 4*N*N doubles of accumulators (sum, compensation,
 * err, compensation).  Loading adds a new event and returns its id. */
jw_status jw_engine_save_event(jw_engine* e, int event_id, const char* path);
jw_status jw_engine_load_event(jw_engine* e, const char* path, int* event_id);
/* An event's next noise index: step0 plus the steps taken so far. */
jw_status jw_engine_event_steps(jw_engine* e, int event_id, uint64_t* steps);
/* For each event ids[i], its accumulated symmetrised correlator at one
 * momentum (xr[i], yr[i]): sum[i] (real part) and err[i] (sum of squares),
 * i.e. what gfield::reduce_hatta (field.h:1538-1564) adds for a Hatta branch
 * measured once since its last reset. */
jw_status jw_engine_correlator_at(jw_engine* e, const int* ids, int n, const int* xr, const int* yr, double* sum,
                                  double* err);
/* Dipole in position space from the event's accumulated correlator (mean over
 * its measurements; the reference stops at C(k), field.h:2521-2547):
 * S(r) = (N^2/3) sum_k C(k) exp(+2 pi i k.r/N), optionally all N*N values
 * (S_xy, row-major displacement), the angular average over bins
 * b = floor(|r| + 1/2) <= N/2 (S_bins, r_bins = mean |r|, counts; nbins_cap >=
 * N/2 + 1), and Q_s = sqrt(2)/r_s with S(r_s) = exp(-1/2) (linear
 * interpolation between bins; 0 if S never falls below exp(-1/2)).  Any output
 * pointer may be null. */
jw_status jw_engine_dipole(jw_engine* e, int event_id, double* S_xy, double* S_bins, double* r_bins, int* counts,
                           int nbins_cap, int* nbins, double* Qs);
/* One ensemble measurement over the listed events (one lattice size): the
 * symmetrised correlators of main_optimized.cpp:321-334 summed over the events
 * as gfield::reduce sums them over stats (field.h:1521-1536), written to host
 * arrays sum and err (N*N complex each, reference layout t = 1).  The events'
 * own accumulators are not touched.  Page-locked arrays (cudaMallocHost,
 * cudaHostRegister) receive the result by direct device-to-host copies. */
jw_status jw_engine_measure_ensemble(jw_engine* e, const int* ids, int n, double* sum, double* err);
/* jw_engine_step(ids, nsteps) followed by jw_engine_measure_ensemble(ids):
 * the body of main_optimized.cpp's Langevin loop (evolution :234-304, then the
 * measurement :317-336) as one call, with the same results.  In mixed
 * precision the last step's third pass also row-transforms the new V for the
 * measurement, so V is not read again. */
jw_status jw_engine_step_measure_ensemble(jw_engine* e, const int* ids, int n, int nsteps, double* sum,
                                          double* err);
/* The column-tile width the autotuner chose for lattice size N (columns per
 * CTA of the mixed column pass), or 0 when it has not run for that size.
 * JW_ENOTFOUND if the engine holds no event of that size. */
jw_status jw_engine_tuning(jw_engine* e, int N, int* p2_cols);
/* Fix the column-tile width of size N's column pass (1, 2, 4 or 8 where it
 * fits; 24 = the persistent form with 8-column tiles that move through the
 * tensor memory accelerator, 64 <= N <= 512, and 20 its 4-column form at
 * N = 1024, 16 meaning whichever of the two N has; JW_EINVAL otherwise; 0 = the
 * built-in default), for example a width found once by the autotuner and kept;
 * the autotuner then skips that size.  Every such choice gives bit-identical
 * events.  Adding 32 to a choice selects the radix-first schedule of the column
 * transforms (N = 16, 32, 128, 256, 1024, 2048 only): its events are
 * bit-identical among its own widths, and differ from the default schedule's
 * by FP32 rounding. */
jw_status jw_engine_set_tuning(jw_engine* e, int N, int p2_cols);
/* nsteps Langevin steps of the listed events (one lattice size) with a CUDA
 * event around each kernel launch.  kernel_ms[4] receives the milliseconds
 * spent in each kernel kind and launches[4] its launch count: pass 1, pass 2,
 * pass 3, and pass 3 fused with the next step's pass 1 (mixed precision runs
 * nsteps steps as pass 1, nsteps - 1 times (pass 2, fused pass), pass 2,
 * pass 3); total_ms is the time from the first launch to the last. */
jw_status jw_engine_step_timed(jw_engine* e, const int* ids, int n, int nsteps, double* kernel_ms, int* launches,
                               double* total_ms);

/* ------------------------------------------------------------------ serving */
/* Continuous-batching evolution server over the engine.  A request is one
 * event: MV initial condition, `steps` Langevin steps, a final dipole
 * measurement returned as the angle-averaged S(r) and Q_s (jw_engine_dipole).
 * A worker thread owns the device: it admits queued requests first-fit by
 * device footprint (max_bytes), advances every resident event together each
 * tick (one launch group per lattice size, up to max_steps_per_tick steps),
 * and retires finished events, freeing memory for the queue.  Requests that
 * arrive while others run join at the next tick; an event's result does not
 * depend on what else is resident.  The functions are thread-safe. */
typedef struct jw_server_options {
    int precision;              /* JW_PRECISION_* */
    int reunitarize;
    size_t max_bytes;           /* device budget for resident events (0 = 90% of free) */
    int max_steps_per_tick;     /* steps per tick per launch group */
    int max_active;             /* resident events (0 = no limit beyond memory) */
    int fake_device;            /* 1: host-only stand-in backend (no GPU; scheduler tests) */
    double fake_ns_per_site_step;
    /* 0: every resident request advances at every tick.  Otherwise a tick
     * advances the resident requests with the least remaining work (sites x
     * (remaining steps + pending MV slices)) first, as many as fit in this
     * many lattice sites (at least one), and a request's MV initial condition
     * runs when it is first chosen: short requests finish early instead of
     * sharing every tick with long ones. */
    size_t tick_sites;
} jw_server_options;

typedef struct jw_request_desc {
    int N;                      /* lattice side, power of two 8..2048 */
    int ny_slices;              /* MV slices */
    double mu;                  /* config mu (mu_MV = mu/N) */
    double mass;                /* config mass */
    double step;                /* Langevin step */
    int coupling;               /* SQRT, NOISE or FIXED */
    int kernel;                 /* SIN */
    uint64_t seed;
    int steps;                  /* Langevin steps */
} jw_request_desc;

typedef struct jw_request_result {
    int status;                 /* JW_OK or the error that ended the request */
    int N, steps;
    double t_submit, t_admit, t_done;  /* seconds on the server's monotonic clock */
    double Qs;
    int nbins;                  /* N/2 + 1 */
} jw_request_result;

typedef struct jw_server_stats {
    int64_t submitted, completed, failed, queued;
    double site_steps;          /* Langevin site-steps executed */
    int max_active;             /* most events resident at once */
    double now;                 /* server clock, seconds */
    /* worker wall time, seconds, by phase: admission (device allocation),
     * MV initial conditions, Langevin ticks (launch to completion), retiring
     * (final measurement, S(r), release) */
    double t_admit, t_mv, t_step, t_retire;
} jw_server_stats;

typedef struct jw_server jw_server;
jw_status jw_server_create(const jw_server_options* opt, int device, jw_server** out);
/* Stops the worker; requests still queued or running are dropped. */
jw_status jw_server_destroy(jw_server* s);
/* JW_EUNSUPPORTED / JW_EINVAL for parameters the engine cannot run, JW_ENOMEM
 * for a request larger than the whole budget; otherwise queued. */
jw_status jw_server_submit(jw_server* s, const jw_request_desc* d, int64_t* request_id);
/* Waits up to timeout_s for the request; JW_ETIMEOUT if it has not finished.
 * On return the request is forgotten by the server.  S_bins/r_bins (may be
 * null) receive nbins values when nbins_cap >= N/2 + 1. */
jw_status jw_server_wait(jw_server* s, int64_t request_id, double timeout_s, jw_request_result* res,
                         double* S_bins, double* r_bins, int nbins_cap);
jw_status jw_server_get_stats(jw_server* s, jw_server_stats* st);
/* No counterpart in the reference.  Per-lattice-size totals of the server's
 * work so far, sizes in increasing order: site-steps advanced, device
 * milliseconds of the Langevin-step launches (CUDA events on the engine
 * stream around each size's launches of a tick) and of the MV initial
 * conditions, and the ticks that stepped the size.  Fills at most cap entries
 * of the (optional) arrays; *count receives the number of sizes. */
jw_status jw_server_size_stats(jw_server* s, int* N, double* site_steps, double* step_ms, double* mv_ms,
                               int64_t* ticks, int cap, int* count);

#ifdef __cplusplus
}
#endif

#endif
