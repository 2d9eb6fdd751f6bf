/*
 * libocto_b200 -- B200 (sm_100a) strong-strong PIC collision backend, C ABI.
 *
 * Drop-in boundary for Octopus.jl's
 *   collide!(solver::PICPoissonSolver, beam1::Beam, beam2::Beam, backend[, ctx]) -> Float64
 * (src/tasks/strongstrong/interface.jl:13-74, 508-509; CPU method pic_cpu.jl:1-32;
 * CUDA method pic_cuda.jl:94-143).  Plain pointers and sizes only: a Julia `ccall`,
 * a Python `ctypes` binding or C/C++ code can drive every entry point.
 *
 * Threading: one context per (task, collision label); a context is not re-entrant.
 * Independent contexts may run concurrently on different streams or devices.
 * Errors never cross the ABI as exceptions: every call returns an OCTO_* status and
 * octo_last_error() returns the message.
 */
#ifndef OCTO_B200_H
#define OCTO_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The Julia shim maps every non-OK code to ArgumentError with the
 * message, as the reference raises from interface.jl:541-599 (non-finite),
 * pic_cpu.jl:517-576 / 730-809 (unsupported option combinations) and
 * pic_cpu.jl:1663-1670 (degenerate extent). */
#define OCTO_OK 0
#define OCTO_ERR_NONFINITE 1   /* non-finite coordinate; report carries role, pair, turn, first index */
#define OCTO_ERR_UNSUPPORTED 2 /* an option combination this backend does not implement */
#define OCTO_ERR_EXTENT 3      /* zero-width transverse extent without min_transverse_extent */
#define OCTO_ERR_ARG 4         /* invalid argument (sizes, pointers, option values) */
#define OCTO_ERR_CUDA 5        /* CUDA runtime failure */
#define OCTO_ERR_TIMEOUT 6     /* a bounded device-side wait gave up */

/* Enumerations of the PICPoissonSolver symbols (interface.jl:1384-1411). */
#define OCTO_CIC 0
#define OCTO_TSC 1
#define OCTO_GREEN_INTEGRATED 0
#define OCTO_GREEN_STANDARD 1
#define OCTO_CACHE_NONE 0
#define OCTO_CACHE_SLICE_PAIR 1
#define OCTO_GRID_SLICE_PAIR 0
#define OCTO_GRID_SOURCE_SLICE 1    /* one union-sized mesh per source slice; pairs run in collision order */
#define OCTO_GRID_NODE 2
#define OCTO_SLICING_NORMAL_QUANTILE 0
#define OCTO_SLICING_SPECIFIED 1
#define OCTO_SLICING_EQUAL_AREA 2   /* LongitudinalSlicing()'s default (slicing.jl:104-156) */
#define OCTO_SLICING_EQUAL_COUNT 3  /* slicing.jl:330-365 */
#define OCTO_SLICING_EQUAL_WIDTH 4  /* also :equal_spaced (slicing.jl:367-388) */
#define OCTO_CENTER_CENTROID 0
#define OCTO_CENTER_MIDPOINT 1

/* One beam: structure-of-arrays device pointers (Phase6DRep, Beam.jl:45-55), caller-owned
 * and updated in place.  dtype 0 = float64. */
typedef struct {
    int64_t n;
    int32_t dtype;
    int32_t reserved;
    void *x, *px, *y, *py, *z, *pz;
} octo_beam;

/* BeamParams (Beam.jl:29-35). */
typedef struct {
    double charge, mc2, E0, r0, npart;
} octo_beam_params;

/* POD twin of PICPoissonSolver's fields (interface.jl:1350-1382) and of the two
 * LongitudinalSlicing configurations (interface.jl:762-831). */
typedef struct {
    int32_t nx, ny;                    /* grid */
    int32_t deposit_method;            /* OCTO_CIC / OCTO_TSC */
    int32_t lum_deposit_method;        /* -1 = inherit deposit_method */
    int32_t lum_nx, lum_ny;            /* luminosity_grid; 0 = inherit grid */
    int32_t green_type;                /* OCTO_GREEN_* */
    int32_t green_cache;               /* OCTO_CACHE_* */
    int32_t field_derivative;          /* 2 = :second, 4 = :fourth */
    int32_t slice_interpolation;       /* 0 = :linear, 1 = :quadratic */
    int32_t interaction_grid;          /* OCTO_GRID_* */
    int32_t grid_extent;               /* 0 = :extrema (the reference CUDA backend rejects :sigma) */
    double grid_extent_sigma;
    double min_extent_x, min_extent_y; /* min_transverse_extent */
    double grid_quantize;
    double green_min_ratio;            /* slice_pair_green_min_ratio */
    double green_growth;               /* slice_pair_green_growth */
    int32_t longitudinal_kick;
    int32_t slicing_method1, slicing_method2;   /* OCTO_SLICING_* */
    int32_t nslices1, nslices2;
    int32_t center_position1, center_position2; /* OCTO_CENTER_* */
    const double *positions1, *positions2;      /* :specified internal positions (nslices-1 each) */
    int32_t has_kbb1, has_kbb2, has_lum_scale;
    double kbb1, kbb2, lum_scale;
    int32_t precision;                 /* 0 = FP64 plain form, 1 = FP32 precision form (float32 beams) */
    /* GaussianPICPoissonSolver (gaussian_pic.jl:87-112): 1 = subtract the drifted reference Gaussian of
     * each source slice before the solve and add its Bassetti-Erskine kick back analytically; in both forms
     * (the precision form keeps the moments, the reference Gaussians and the add-back in FP64) */
    int32_t gaussian;
    double margin_sigma;               /* hybrid: Gaussian containment half-width in sigmas (default 5) */
    int32_t neutralize;                /* hybrid: rescale the subtracted Gaussian to the deposited charge */
    /* GaussianPoissonSolver, the soft-Gaussian strong-strong solver (src/tasks/strongstrong/gaussian.jl,
     * options interface.jl:949-1020): solver = OCTO_SOLVER_SOFT_GAUSSIAN runs it instead of the PIC solve
     * (the grid, deposit, Green and interaction-grid fields are then unused; kbb1/kbb2/lum_scale overrides,
     * the slicings and longitudinal_kick keep their meaning).  Float64 beams, or float32 beams with precision = 1
     * (stored in float, computed in FP64 as the reference promotes them). */
    int32_t solver;                    /* OCTO_SOLVER_PIC / OCTO_SOLVER_SOFT_GAUSSIAN */
    int32_t gaussian_when_luminosity;  /* 1 or 2: the beam whose slice is the Gaussian the luminosity samples */
    int32_t ignore_centroid1, ignore_centroid2;
    int32_t virtual_drift;             /* 0 = :hirata, 1 = :chromatic, 2 = :exact (strong_beam.jl:20-30, 517-606) */
    int32_t include_sigma_xy;          /* 1: the full (coupled) transverse slice covariance */
    double min_sigma;                  /* transverse RMS floor, finite and >= 0 */
    int32_t resolution1, resolution2;  /* LongitudinalSlicing resolution (:equal_area bins per slice); 0 = 100 */
    /* hybrid (gaussian = 1): |r_xy| of a drifted source slice above which the coupled (rotated) subtraction runs
     * (gaussian_pic.jl:94-110, 525-536); INFINITY (the reference's default) always subtracts the separable
     * Gaussian; must be >= 0.  Zero-initialised structs get 0: set INFINITY for the default. */
    double coupling_tol;
} octo_pic_options;
#define OCTO_SOLVER_PIC 0
#define OCTO_SOLVER_SOFT_GAUSSIAN 1

/* What a collide reports besides the luminosity. */
typedef struct {
    int32_t status;
    int32_t role;            /* 0 none, 1 source, 2 field, 3 beam (slicing), 4 node-mesh build,
                                5 :source_slice union box */
    int32_t pair_i, pair_j;  /* 1-based slice pair of the first failure */
    int32_t direction;       /* 1 or 2 */
    int32_t n_batches;       /* wavefronts executed */
    int64_t turn;
    int64_t first_index;     /* 1-based particle index (caller order) of the first non-finite coordinate */
    int64_t dropped;         /* particles outside their mesh (pic_cpu.jl:394-457) */
    int64_t green_hits, green_misses, green_rebuilds;  /* cumulative, as Contracts.jl:947-960 compares */
    int64_t kernel_launches; /* device kernels this call launched */
    int32_t replayed;        /* 1 when the collide ran as its captured graph (octo_set_collide_graph) */
    int32_t pad;
} octo_collide_report;

typedef struct octo_ctx octo_ctx;

/* Context holding device workspaces, the slice-pair Green cache (pic_cpu.jl:1729-1821)
 * and twiddle tables; the twin of task.runtime_cache (pic_cpu.jl:23-32, 499-515). */
octo_ctx *octo_create(int32_t device, const octo_pic_options *options);
void octo_destroy(octo_ctx *ctx);

/* collide! (pic_cpu.jl:82-275 / pic_cuda.jl:298-516): slices both beams, runs every slice pair
 * in collision-time wavefronts, kicks both beams in place and returns the luminosity
 * (NaN when compute_luminosity == 0, as for a skipped luminosity_schedule turn).
 * stream: a cudaStream_t or NULL for the legacy default stream. */
int32_t octo_pic_collide(octo_ctx *ctx, octo_beam *beam1, octo_beam *beam2, const octo_beam_params *p1,
                         const octo_beam_params *p2, int64_t turn, int32_t compute_luminosity,
                         double *luminosity, octo_collide_report *report, void *stream);

/* A batch of independent collides (one per context, e.g. the collision points of a lattice or the cases
 * of a parameter scan), each on its own stream: the slicing of every collide is enqueued first, then each
 * collide's schedule is built and its wavefronts enqueued while the earlier ones run, then all are
 * finished.  Same results as `count` octo_pic_collide calls (the reference runs its collision points
 * one after another in the turn loop, interface.jl:2499-2501).  status[k] receives each collide's
 * code; the return value is OCTO_OK or the first failing code.  Contexts must be distinct; streams
 * should be distinct for the collides to overlap.  luminosity, reports and status may be NULL. */
int32_t octo_pic_collide_batch(int32_t count, octo_ctx *const *ctx, octo_beam *const *beam1, octo_beam *const *beam2,
                               const octo_beam_params *const *p1, const octo_beam_params *const *p2, int64_t turn,
                               int32_t compute_luminosity, double *luminosity, octo_collide_report *reports,
                               int32_t *status, void *const *streams);

/* Launch-shape autotuner (no reference counterpart; the extras' tile autotuner): times `rounds` collides
 * of beam1/beam2 with each of four launch shapes -- charge-deposit blocks of at least one or two waves of
 * the GPU's SMs per wavefront, kick blocks sized to fill one or two times the resident block slots -- after
 * one untimed collide, and keeps the fastest shape for this context's later collides (*choice: 0..3).
 * The shape changes only the time, never a result: charge sums are exact integers and every particle's
 * kick is its own.  The collides update beam1 and beam2 in place, so pass scratch copies.  rounds: 1..16. */
int32_t octo_pic_autotune(octo_ctx *ctx, octo_beam *beam1, octo_beam *beam2, const octo_beam_params *p1,
                          const octo_beam_params *p2, int32_t rounds, int32_t *choice, void *stream);

/* Order of the particles inside each slice of a plain PIC context's working copy (no reference counterpart;
 * the reference keeps caller order, slicing.jl:431-521).  1 (default): grouped by transverse position (a 64 x 64
 * binning of each slice's box), so the kick's field gathers of a warp touch neighbouring cells; 0: caller order.
 * The plain PIC collide does not depend on this order -- charge and luminosity grids are exact int64 sums and
 * every kick is its own particle's -- so both give bit-identical results.  The Gaussian-subtracted hybrid and the
 * soft-Gaussian solver always keep caller order (their slice moments are ordered floating-point sums). */
int32_t octo_set_particle_order(octo_ctx *ctx, int32_t order);
/* Captured collide graphs, on by default for the plain PIC collide (no reference counterpart: the reference
 * schedules each collide on the host, pic_cpu.jl:82-275).  Once two consecutive collides of a context have the
 * same schedule -- slice counts and starts, collision order -- the next one captures its kernels into a CUDA
 * graph; later collides launch it behind a one-block device guard that checks the schedule and recomputes the
 * slice drifts, so a collide costs one host synchronisation instead of two and no schedule upload.  A collide
 * whose schedule differs, a changed beam address, interaction scale, launch shape or workspace falls back to
 * the ordinary path on the untouched beams.  Results are bit-identical either way.  enable: 1 (default) or 0;
 * setting it synchronises the device and drops the current graph. */
int32_t octo_set_collide_graph(octo_ctx *ctx, int32_t enable);
/* out = graphs captured, collides replayed, replays the guard declined, capture failures (two failures turn
 * the graphs off for the context). */
int32_t octo_collide_graph_stats(octo_ctx *ctx, int64_t out[4]);

/* Green-cache counters (the contract of Contracts.jl:947-960). */
int32_t octo_green_cache_stats(octo_ctx *ctx, int64_t *hits, int64_t *misses, int64_t *rebuilds);

/* Per-pair luminosity of the last collide in collision order: the sink of interface.jl:389-410,
 * compared by Contracts.jl:916-945.  Writes up to cap entries; returns the count. */
int64_t octo_pair_luminosity_trace(octo_ctx *ctx, int32_t *pair_i, int32_t *pair_j, double *lum, int64_t cap);

/* Linear 6D one-turn map (linear6d.jl:110-121), row-major 6x6, applied `turns` times in place. */
int32_t octo_linear6d(octo_ctx *ctx, octo_beam *beam, const double matrix[36], int32_t turns, void *stream);

/* Line tracking between collisions: a sequence of zero-length elements applied to every particle in one
 * fused pass (one read and one write of the six coordinates per particle and call), the twin of
 * track!(rep, elems, turns; context) with fusedTrack (src/track/phase6d_track.jl:25-35, 197-212;
 * src/track/fused_track.jl:53-77) for the elements the production strong-strong lines place around the
 * collision (examples/strong_strong_tracking.jl:206-262).  Element parameters (p[]) per kind: */
#define OCTO_ELEM_LINEAR6D 1             /* p[0..35] row-major 6x6 matrix (linear6d.jl:110-121) */
#define OCTO_ELEM_THIN_CRAB_CAVITY 2     /* p[0] frequency [Hz], finite and nonzero; harmonic h < nharm:
                                            p[1+h] strengthX, p[9+h] strengthY, p[17+h] phase [rad]
                                            (crab_cavity.jl:87-144) */
#define OCTO_ELEM_LORENTZ_BOOST 3        /* p[0] half crossing angle [rad] (lorentz_boost.jl:128-143) */
#define OCTO_ELEM_REV_LORENTZ_BOOST 4    /* p[0] half crossing angle [rad] (lorentz_boost.jl:148-161) */
#define OCTO_ELEM_CHROMATICITY_KICK 5    /* p[0..1] xi, p[2..3] beta, p[4..5] alpha, p[6..9] zeta,
                                            p[10..13] eta, p[14..17] R (chromaticity_kick.jl:74-136) */
#define OCTO_ELEM_LUMPED_RAD 6           /* p[0..2] damping_turns, p[3..5] beta, p[6..8] alpha,
                                            p[9..11] sigma (all >= 0 enables excitation, all < 0 disables it),
                                            p[12..15] zeta, p[16..19] eta, p[20..23] R; mode = OCTO_RAD_*,
                                            is_damping, is_excitation, rng_id (radiation.jl:83-232) */
#define OCTO_ELEM_CRAB_DISPERSION 7      /* p[0..3] zeta1..zeta4 (linear_maps.jl:125-132) */
#define OCTO_ELEM_MOMENTUM_DISPERSION 8  /* p[0..3] eta1..eta4 (linear_maps.jl:213-220) */
#define OCTO_ELEM_XY_COUPLING 9          /* p[0..3] r1..r4, 1 + r1 r4 - r2 r3 > 0; mode 0 identity, 1 A, 2 B
                                            (linear_maps.jl:296-310, 355-373) */
#define OCTO_RAD_RADIATION 0 /* Radiation6DMap: damping and excitation as flagged */
#define OCTO_RAD_DAMPING 1   /* Damping6DMap: damping only */
#define OCTO_RAD_DIFFUSION 2 /* Diffusion6DMap: excitation only */
#define OCTO_RNG_PHILOX 1    /* RNG_PHILOX (counter_rng.jl:10) */
#define OCTO_RNG_SPLITMIX 2  /* RNG_SPLITMIX (counter_rng.jl:13) */
#define OCTO_CRAB_MAX_HARMONICS 8
#define OCTO_LINE_MAX_ELEMENTS 32
typedef struct {
    int32_t kind;          /* OCTO_ELEM_* */
    int32_t nharm;         /* thin crab cavity: harmonic count N, 1..OCTO_CRAB_MAX_HARMONICS */
    int32_t mode;          /* lumped radiation: OCTO_RAD_*; xy coupling: 0, 1, 2 */
    int32_t is_damping;    /* lumped radiation flags */
    int32_t is_excitation;
    int32_t reserved;
    uint64_t rng_id;       /* lumped radiation counter-RNG stream id */
    double p[40];
} octo_element;
/* Applies elems[0..n_elems) to every particle of beam, `turns` times.  Turn t (0-based) of the call draws
 * the radiation noise of TrackingContext turn `turn + t` (seed, rng_method: OCTO_RNG_*), particle i
 * (0-based) as particle_id i + 1, so a run split into several calls is bit-identical to one call.
 * Parameters are validated as the reference's constructors do (OCTO_ERR_ARG with the message). */
int32_t octo_track_line(octo_ctx *ctx, octo_beam *beam, const octo_element *elems, int32_t n_elems, int64_t turn,
                        int32_t turns, uint64_t seed, int32_t rng_method, void *stream);

/* One moment row of a beam as MomentObserver records it (src/tasks/BeamObservers.jl:630-720, 1000-1060,
 * 1254-1271): row[0] = turn; row[1 + k] = moment k of powers[6k .. 6k+5] (exponents of x, px, y, py, z, pz),
 * the mean of its coordinate for order 1, else the central moment mean(prod (c_d - <c_d>)^p_d).  With
 * mask_lost != 0 (allow_lost_particles) only particles whose six coordinates are finite count, and a beam
 * without such particles gets NaN moments; otherwise a non-finite particle makes the row NaN.  `row` is a
 * DEVICE pointer (a slot of the caller's record buffer): the call never synchronises the host.  Up to
 * OCTO_MOMENTS_MAX moments, each order-1 moment at most once, exponents 0..32. */
#define OCTO_MOMENTS_MAX 256
int32_t octo_beam_moments(octo_ctx *ctx, const octo_beam *beam, const int32_t *powers, int32_t n_moments,
                          int32_t mask_lost, int64_t turn, double *row, void *stream);

/* Seeded Gaussian beam on the device as Beam(n, backend, Float64; beta, alpha, sigma, cutoff, rng_id)
 * builds it (Beam.jl:475-515; counter RNG counter_rng.jl:154-233).  Float64 beams only (dtype 0). */
int32_t octo_beam_gaussian(octo_ctx *ctx, octo_beam *beam, uint64_t seed, uint64_t rng_id, const double beta[3],
                           const double alpha[3], const double sigma[3], double cutoff, void *stream);

/* Charge-grid capture, a test hook for the bit-exact fixed-point claim (the reference's charge grid is the
 * one _pic_deposit_drifted_* fills, pic_cpu.jl:2015-2146; its CPU backend exposes it to its own tests only
 * through the solved fields).  octo_capture_charge_plane arms a copy of one field-solve plane of the next
 * collide on this context: slice pair (pair_i, pair_j) (1-based), direction 1 (beam-1 slice sources) or 2,
 * plane 0 = the sL deposit, 1 = the sR deposit, 2 = the third plane (:slice_pair quadratic: the midpoint;
 * :node with the longitudinal kick: sR on the L mesh).  The copy is taken right after the deposit, before the
 * solve consumes the grid.  octo_captured_charge_plane synchronises the device and returns the int64 grid
 * (nx*ny, x fastest: grid[(iy-1)*nx + (ix-1)] is 1-based node (ix, iy)), the mesh it was deposited on
 * (mesh = {x0, y0, width, height}), the field mesh of its interaction (field_mesh, may be NULL) and the
 * fixed-point scale (a tap is round(w * 2^fixed_bits)); it fails with OCTO_ERR_ARG when nothing was captured.
 * Capturing adds three device copies to that collide. */
int32_t octo_capture_charge_plane(octo_ctx *ctx, int32_t pair_i, int32_t pair_j, int32_t direction, int32_t plane);
int32_t octo_captured_charge_plane(octo_ctx *ctx, int64_t *grid, double mesh[4], double field_mesh[4],
                                   int32_t *fixed_bits);

/* BF16 GEMM on the tensor cores (tcgen05.mma with a TMEM accumulator), the contraction of the learned field
 * correction's convolutions; no reference counterpart.  out[z][m][n] = sum over split z of k of A[m][k] B[n][k]
 * (fp32, row stride ldc, split z at out + z*M*ldc), or with out_bf16 set (splits = 1):
 * out_bf16[m*ldo + n] = bf16(relu?(acc + bias[n])).  a_mode 0: A is a dense row-major bf16 matrix (lda, a
 * multiple of 8); a_mode 1: A is the implicit im2col of a 3x3, padding-1 convolution over the NHWC bf16 tensor
 * A[M/(H*W)][H][W][C] (C a multiple of 8, K = 9*C, k = (ky*3 + kx)*C + c).  B is row-major bf16 [N][ldb].
 * Device pointers, 16-byte aligned; K a multiple of 8.  Synchronises the stream; OCTO_ERR_TIMEOUT if a
 * bounded device wait gave up. */
typedef struct {
    int32_t M, N, K, a_mode, H, W, C, splits, relu, pad;
    const void *A;
    int64_t lda;
    const void *B;
    int64_t ldb;
    float *out;
    int64_t ldc;
    const float *bias;
    void *out_bf16;
    int64_t ldo;
} octo_gemm_desc;
int32_t octo_gemm_bf16(int32_t device, const octo_gemm_desc *desc, void *stream);

/* The learned field correction's network (no reference counterpart): a 4-level U-Net of 3x3 convolutions with
 * 32 base channels (641k parameters) whose convolutions run on the tensor cores (octo_gemm_bf16's kernel), with
 * its forward pass, backward pass and Adam update on the GPU.  Input: NHWC bf16 [batch][height][width][8];
 * output: fp32 [batch][height][width][2].  height and width multiples of 8 (>= 16); batch <= max_batch.
 * Parameters are an fp32 vector (per layer: weights [Cout][3][3][Cin], then bias [Cout]). */
typedef struct octo_cnn octo_cnn;
octo_cnn *octo_cnn_create(int32_t device, int32_t height, int32_t width, int32_t max_batch, uint64_t seed);
void octo_cnn_destroy(octo_cnn *net);
int64_t octo_cnn_num_params(const octo_cnn *net);
int32_t octo_cnn_get_params(octo_cnn *net, float *params, int64_t n);        /* host buffer of n floats */
int32_t octo_cnn_set_params(octo_cnn *net, const float *params, int64_t n);
/* input, output: device pointers; synchronises the stream. */
int32_t octo_cnn_forward(octo_cnn *net, const void *input, int32_t batch, float *output, void *stream);
/* One training step: forward, the mean-square loss of output channels 0..1 against target (fp32 [batch][h][w][2])
 * weighted per pixel by mask (fp32 [batch][h][w], NULL = 1) and normalised by the total weight, the gradients of
 * every parameter, and (update != 0) an Adam step of learning rate lr (beta 0.9 / 0.999, eps 1e-8).  loss and
 * grads (host, num_params floats) may be NULL.  Synchronises the stream. */
int32_t octo_cnn_train_step(octo_cnn *net, const void *input, const float *target, const float *mask, int32_t batch,
                            float lr, int32_t update, double *loss, float *grads, void *stream);

/* Attach the learned field correction to a coarse-grid PIC context -- the Gaussian-subtracted hybrid (options.gaussian
 * = 1, the correction of gaussian_pic.jl's coarse-grid solve) or the plain PIC solver -- with :slice_pair grids,
 * linear slice interpolation, the :integrated Green function and green_cache = :none (no reference counterpart).
 * Every field-solve plane of the context's
 * collides then gets the network's correction: its charge grid (grid units, the node charges over the plane total
 * times the node count, with log(hy/hx) as a second channel) goes through the network after the deposit, and
 * the output (dEx*hx, dEy*hy of a unit charge, times out_scale) is added to the plane's field cells after the
 * solve, except within `edge` nodes of the mesh border.  The largest correction of a plane is its error
 * estimate: octo_field_correction_report returns how many planes of the last collide exceeded `tolerance` (the
 * caller's signal to fall back to the plain solver).  net = NULL detaches.  The network's height x width must be
 * the grid's ny x nx and its max_batch at least the planes of a wavefront (4 per slice pair of the narrower
 * beam's slice count).  The context keeps a pointer: destroy the network after detaching it. */
int32_t octo_set_field_correction(octo_ctx *ctx, octo_cnn *net, float out_scale, float tolerance, int32_t edge);
int32_t octo_field_correction_report(octo_ctx *ctx, int32_t *planes_over_tolerance);

/* Message of the last failing call on this context (NUL-terminated, truncated to len). */
int32_t octo_last_error(octo_ctx *ctx, char *buf, int64_t len);

/* Per-phase device timing, the twin of the reference's pic_timing diagnostics
 * (StrongStrongDiagnostics, interface.jl:301-386; _CUDAPICTimingStats, pic_cuda.jl:552-700).
 * While enabled, CUDA events bracket each launch group; octo_timing_report returns the
 * accumulated device milliseconds, launch counts and algorithmic HBM bytes per phase
 * (bytes: kick 11 values, deposit 4, bounds 5, luminosity 4 per particle visit, FP64). */
#define OCTO_PHASE_SLICING 0
#define OCTO_PHASE_BOUNDS 1
#define OCTO_PHASE_PLAN 2
#define OCTO_PHASE_GREEN 3
#define OCTO_PHASE_LUMINOSITY 4
#define OCTO_PHASE_DEPOSIT 5
#define OCTO_PHASE_FFT 6
#define OCTO_PHASE_FIELD 7
#define OCTO_PHASE_KICK 8
#define OCTO_PHASE_UNSORT 9
#define OCTO_PHASE_NODE 10
#define OCTO_NPHASES 11
int32_t octo_set_timing(octo_ctx *ctx, int32_t enable); /* enabling also clears the accumulators */
/* Restrict the timing to the phases whose bit (1 << OCTO_PHASE_*) is set in mask (default: all).  Each
 * timed launch group records two events; timing one phase keeps that overhead off the others. */
int32_t octo_set_timing_phases(octo_ctx *ctx, uint32_t mask);
int32_t octo_timing_report(octo_ctx *ctx, double ms[OCTO_NPHASES], int64_t launches[OCTO_NPHASES],
                           double bytes[OCTO_NPHASES]);

/* Seeded Gaussian beam construction that allocates no device memory.
 *
 * This entry point has no counterpart in the reference.  It exists for callers that cannot call
 * cudaMalloc: hosts whose device memory is owned by a pool allocator (Julia's CUDA.jl pool or
 * PyTorch's caching allocator reserve the device up front, so an out-of-band allocation can fail
 * or fragment their pool), and long-running services that forbid allocation after start-up.
 * It needs no octo_ctx (creating one allocates).  Its reduction scratch lives in a fixed 32 KiB
 * static device array inside libocto_b200.so, which every GPU that loads the library holds until
 * process exit.  The limit that follows: n <= OCTO_NOALLOC_MAX_PARTICLES particles per call; larger
 * beams are rejected with OCTO_ERR_ARG and a message in err.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current; make that first call before any stream capture.  The address is cached per device
 * together with the device's current context: after a device reset (cudaDeviceReset, CUDA.jl's
 * device_reset!) the new context loads the library's module afresh, and the next call looks the address
 * up again, so it too belongs before any stream capture.  The call makes `device` current while it runs
 * and restores the calling thread's current context before it returns.  All calls share the one array,
 * so calls that overlap on the GPU (different streams, threads or processes sharing a context)
 * race: serialise them.  Float64 beams only (dtype 0).  The caller owns beam, and err (may be NULL)
 * receives a message on failure.
 * Output matches octo_beam_gaussian to rounding (its reduction uses a different block count). */
#define OCTO_NOALLOC_PARTICLES_PER_BLOCK 8192
#define OCTO_NOALLOC_MAX_BLOCKS 4094
#define OCTO_NOALLOC_MAX_PARTICLES (OCTO_NOALLOC_PARTICLES_PER_BLOCK * OCTO_NOALLOC_MAX_BLOCKS)
int32_t octo_beam_gaussian_noalloc(int32_t device, octo_beam *beam, uint64_t seed, uint64_t rng_id,
                                   const double beta[3], const double alpha[3], const double sigma[3],
                                   double cutoff, void *stream, char *err, int64_t err_len);

/* Host-side helpers shared with the slicing: the normal quantile sqrt(2)*erfinv(2s/ns - 1)
 * used for :normal_quantile boundaries (slicing.jl:420-429), and the library version. */
double octo_normal_quantile(int32_t s, int32_t ns);
double octo_erfinv(double x);
int32_t octo_version(void);

#ifdef __cplusplus
}
#endif
#endif
