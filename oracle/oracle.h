/*
 * FP64 CPU oracle for the strong-strong PIC collision -- TEST INFRASTRUCTURE.
 *
 * This library is a CPU restatement of the reference's CPU PIC path
 * (Octopus.jl `src/tasks/strongstrong/pic_cpu.jl`, `slicing.jl`,
 * `src/beam/Beam.jl`, `src/math/counter_rng.jl`, `src/elements/linear6d.jl`).
 * It exists only to check the CUDA path: tests, the smoke check and the CPU
 * baseline leg of the benchmark load it; the product library never does.
 *
 * Parity pins: Philox4x32-10 Random123 known-answer vectors
 * (counter_rng.jl:250-258), the integrated Green kernel's on-axis zeros
 * (test/runtests.jl:2576-2591), the quadratic-interpolation identities
 * (test/runtests.jl:9741-9776), the 4th-vs-2nd order Bassetti-Erskine field
 * test (test/runtests.jl:9628-9693) and the production golden luminosity
 * 1.0254361754701657e+30 (docs/history/cpu_benchmark_history.tsv:2).
 * Line elements: the reference's element tests (test/runtests.jl:188-240,
 * 341-508), symplecticity and the boost pair's Jacobian determinants, and the
 * crossing-angle luminosity anchor (validation/crossing_luminosity_anchor.jl).
 * Soft-Gaussian solver: the two-Gaussian luminosity, the point-charge far kick,
 * the rotated kick of a tilted Gaussian, agreement with the PIC solve on
 * Gaussian beams, and the two forms of the rotation term L/D.
 */
#ifndef OCTO_ORACLE_H
#define OCTO_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OO_OK = 0, OO_ERR_NONFINITE = 1, OO_ERR_UNSUPPORTED = 2, OO_ERR_EXTENT = 3, OO_ERR_ARG = 4 };

/* POD twin of PICPoissonSolver's fields (interface.jl:1350-1382). */
typedef struct {
    int32_t nx, ny;                    /* grid */
    int32_t deposit_method;            /* 0 = :CIC, 1 = :TSC */
    int32_t lum_deposit_method;        /* -1 inherit, 0 CIC, 1 TSC */
    int32_t lum_nx, lum_ny;            /* 0 = inherit grid */
    int32_t green_type;                /* 0 = :integrated, 1 = :standard */
    int32_t green_cache;               /* 0 = :none, 1 = :slice_pair */
    int32_t field_derivative;          /* 2 = :second, 4 = :fourth */
    int32_t slice_interpolation;       /* 0 = :linear, 1 = :quadratic */
    int32_t interaction_grid;          /* 0 = :slice_pair, 1 = :source_slice, 2 = :node */
    int32_t grid_extent;               /* 0 = :extrema, 1 = :sigma */
    double grid_extent_sigma;
    double min_extent_x, min_extent_y; /* min_transverse_extent */
    double grid_quantize;
    double green_min_ratio;            /* slice_pair_green_min_ratio */
    double green_growth;               /* slice_pair_green_growth */
    int32_t longitudinal_kick;
    int32_t slicing_method1, slicing_method2;  /* 0 = :normal_quantile, 1 = :specified, 2 = :equal_area,
                                                  3 = :equal_count, 4 = :equal_width */
    int32_t nslices1, nslices2;
    int32_t center_position1, center_position2; /* 0 = :centroid, 1 = :midpoint */
    const double *positions1, *positions2;      /* :specified internal positions (nslices-1) */
    int32_t has_kbb1, has_kbb2, has_lum_scale;
    double kbb1, kbb2, lum_scale;
    int32_t fixed_point_deposit;       /* 1: int64 fixed-point charge grid (see oo_fixed_scale_bits) */
    int32_t nthreads;                  /* OpenMP threads for the pair batches (results do not depend on it) */
    int32_t gaussian;                  /* 1: GaussianPICPoissonSolver (Gaussian-subtracted hybrid) */
    int32_t neutralize;                /* hybrid: rescale the subtracted Gaussian to the deposited charge */
    double margin_sigma;               /* hybrid: adaptive-box half-width in beam sigmas */
    int32_t resolution1, resolution2;  /* :equal_area histogram bins per slice (LongitudinalSlicing resolution) */
    double coupling_tol;               /* hybrid: |r_xy| above which the coupled (rotated) subtraction runs; inf = never */
} oo_options;

typedef struct { double charge, mc2, E0, r0, npart; } oo_beam_params;

/* Gaussian-subtracted hybrid pieces (gaussian_pic.jl, strong_beam.jl, SpecialMath.jl). */
void oo_faddeeva(double zr, double zi, double out[2]);
/* kick (Kx, Ky) and kbb-scaled potential Hessians (Hxx, Hyy) of a (sigx, sigy) Gaussian at (x, y) */
void oo_be_response(double kbb, double sigx, double sigy, double x, double y, double out[4]);
/* erf-integrated CIC (0) / TSC (1) node profile of a 1D Gaussian on nodes x0 + i h, i < n */
void oo_gaussian_profile(int32_t method, double x0, double h, double mu, double sigma, int32_t n, double *g);

/* Counter RNG and beam construction (counter_rng.jl, Beam.jl). */
void oo_philox4x32_block(const uint32_t c[4], const uint32_t k[2], uint32_t out[4]);
uint64_t oo_counter_uint64(uint64_t seed, uint64_t turn, uint64_t rng_id, uint64_t particle, uint64_t component);
double oo_normal(uint64_t seed, uint64_t turn, uint64_t rng_id, uint64_t particle, uint64_t component);
void oo_beam_gaussian(int64_t n, uint64_t seed, uint64_t rng_id, const double beta[3], const double alpha[3],
                      const double sigma[3], double cutoff, double *x, double *px, double *y, double *py,
                      double *z, double *pz);
double oo_erfinv(double x);

/* Building blocks exposed for the analytic pins. */
double oo_kernel_integral(double x, double y);
double oo_atan_ratio(double num, double den);
void oo_cic_weights(double u, int32_t n, int32_t *base, double w[2]);
void oo_tsc_weights(double u, int32_t n, int32_t *base, double w[3]);
void oo_green_table(int32_t green_type, double fx0, double fy0, double sx0, double sy0, double hx, double hy,
                    int32_t nx, int32_t ny, double *out /* (2nx)*(2ny) column-major */);
void oo_fft2(double *re, double *im, int32_t n1, int32_t n2, int32_t inverse);
void oo_field(const double *phi, int32_t nx, int32_t ny, double hx, double hy, int32_t fourth, double *Ex, double *Ey);
/* Fixed-point scale (bits) used for a plane with nsrc source particles. */
int32_t oo_fixed_scale_bits(int64_t nsrc);
/* Drifted deposit into a (2nx)*(2ny) column-major grid (only the nx*ny quadrant is written).
   fixed != 0 accumulates round(w * 2^bits) in int64 and writes the integer grid to qfix as well. */
void oo_deposit_drifted(int32_t method, const double *x, const double *px, const double *y, const double *py,
                        int64_t n, double s, double x0, double y0, double hx, double hy, int32_t nx, int32_t ny,
                        int32_t fixed, double *charge, int64_t *qfix);
/* One field solve (deposit -> FFT -> x G^ -> iFFT -> E) on grid (x0,y0,w,h) against the Green
   function of (source grid, field grid). Outputs nx*ny column-major phi, Ex, Ey. */
void oo_solve_field(const oo_options *opt, const double *x, const double *y, int64_t n, double sx0, double sy0,
                    double sw, double sh, double fx0, double fy0, double *phi, double *Ex, double *Ey);
void oo_interpolation_grids(const oo_options *opt, const double b[8], double out[8]);
/* _pic_interpolate_kick / _pic_interpolate_kick_quadratic on an nx*ny mesh (grid = x0, y0, w, h).
   quadratic = 0: two-node with zL = param, zR = 1 - zL ; 1: three-node at t = param.  out = Kx, Ky, Kz. */
void oo_interpolate(const oo_options *opt, const double grid[4], double x, double y, const double *phiL,
                    const double *ExL, const double *EyL, const double *phiM, const double *ExM, const double *EyM,
                    const double *phiR, const double *ExR, const double *EyR, int32_t quadratic, double param,
                    double out[3]);
/* _pic_luminosity! (pic_cpu.jl:2700-2736); q1, q2 receive the (lnx+1)*(lny+1) column-major deposits. */
double oo_luminosity(const oo_options *opt, const double *x1, const double *y1, int64_t n1, const double *x2,
                     const double *y2, int64_t n2, double klum, double *q1, double *q2);

/* Slicing (slicing.jl:51-75; methods as slicing_method1). Outputs: boundary[ns+1], center[ns], weight[ns],
   count[ns], order[n] (slice-major member lists: ascending particle index, rank order for :equal_count).
   resolution: :equal_area histogram bins per slice (<= 0: the default 100). */
int oo_slices(int32_t method, int32_t ns, int32_t center_position, const double *positions, const double *z,
              int64_t n, double *boundary, double *center, double *weight, int64_t *count, int64_t *order,
              int32_t resolution);
/* Julia's collect(range(start, stop; length = len)) for Float64 endpoints (the :equal_width boundaries). */
void oo_julia_range(double start, double stop, int64_t len, double *out);
/* Collision order + wavefront batches (slicing.jl:561-647). pairs[k] = (batch, i, j) 0-based in order
   of batches; returns the number of batches. */
int32_t oo_pair_batches(const double *c1, int32_t ns1, const double *c2, int32_t ns2, int32_t *batch_of,
                        int32_t *pi, int32_t *pj, int32_t *order_i, int32_t *order_j);

/* The :source_slice union box of one source slice (x, px, y, py) against a partner beam (x, px, y, py, z):
   out = source (xmin, xmax, ymin, ymax) then field (xmin, xmax, ymin, ymax); *valid = 0 when the partner has
   no finite z.  Returns OO_OK or the error code of a non-finite coordinate. */
int32_t oo_union_bounds(const double *src[4], int64_t ns, double center, const double *part[5], int64_t np,
                        double out[8], int32_t *valid);

/* A collide context keeps the slice-pair Green cache across calls, as task.runtime_cache does. */
void *oo_create(const oo_options *opt);
void oo_destroy(void *ctx);
int oo_collide(void *ctx, double *b1[6], int64_t n1, double *b2[6], int64_t n2, const oo_beam_params *p1,
               const oo_beam_params *p2, int32_t compute_luminosity, double *luminosity);
void oo_cache_stats(void *ctx, int64_t out[3]);
int64_t oo_dropped(void *ctx);
/* Per-pair luminosity of the last collide in collision order (i, j 1-based); returns count. */
int64_t oo_pair_trace(void *ctx, int32_t *pi, int32_t *pj, double *lum, int64_t cap);
const char *oo_last_error(void *ctx);
/* Capture one field-solve charge grid of the next collide (fixed_point_deposit on): pair (i, j), direction,
   plane 0 = sL, 1 = sR, 2 = the third (midpoint / :node Z).  oo_captured_plane writes the nx*ny int64 grid
   (x fastest), the mesh {x0, y0, width, height} and the fixed-point bits; nonzero when nothing was captured. */
void oo_capture_plane(void *ctx, int32_t i, int32_t j, int32_t dir, int32_t kind);
int32_t oo_captured_plane(void *ctx, int64_t *q, double mesh[4], int32_t *bits);
/* collide!(::GaussianPoissonSolver, ...) (src/tasks/strongstrong/gaussian.jl:7-185): the soft-Gaussian solver,
   include_sigma_xy: the coupled covariance; virtual_drift 0 :hirata, 1 :chromatic, 2 :exact; opt gives the slicings, kbb / luminosity-scale overrides and longitudinal_kick. */
int oo_gaussian_collide(const oo_options *opt, double min_sigma, int32_t gaussian_when_luminosity,
                        int32_t ignore_centroid1, int32_t ignore_centroid2, int32_t virtual_drift,
                        int32_t include_sigma_xy, double *b1[6], int64_t n1, double *b2[6], int64_t n2,
                        const oo_beam_params *p1, const oo_beam_params *p2, double *luminosity);
const char *oo_gaussian_last_error(void);
/* Rotation-term pins: out = Kx, Ky, H1, H2, L/D; the elliptic kick alone (s1 > s2). */
void oo_be_near_round_L(double kbb, double v, double eta, double x, double y, double out[5]);
void oo_be_principal_L(double kbb, double s1, double s2, double x, double y, double out[5]);
void oo_be_elliptic(double s1, double s2, double x, double y, double out[2]);
/* Line elements (the layout of octo_element in the product header; kinds 1..9: Linear6D, thin crab
   cavity, Lorentz boost, reverse boost, chromaticity kick, lumped radiation, crab dispersion, momentum
   dispersion, xy coupling).  oo_track_line applies elems to each particle `turns` times, turn t drawing
   the counter-RNG noise of turn `turn + t` (rng_method 1 Philox, 2 SplitMix), particle i as id i + 1
   (src/track/phase6d_track.jl:25-35 with fusedTrack, src/track/fused_track.jl:53-77). */
typedef struct {
    int32_t kind, nharm, mode, is_damping, is_excitation, reserved;
    uint64_t rng_id;
    double p[40];
} oo_element;
void oo_track_line(const oo_element *elems, int32_t n_elems, int64_t turn, int32_t turns, uint64_t seed,
                   int32_t rng_method, double *x, double *px, double *y, double *py, double *z, double *pz,
                   int64_t n);
/* octopus_normal (counter_rng.jl:168-176) for either method. */
double oo_octopus_normal(uint64_t seed, int32_t rng_method, uint64_t turn, uint64_t rng_id, uint64_t particle,
                         uint64_t component);
/* Linear 6D one-turn map (linear6d.jl:110-121) with a row-major 6x6 matrix. */
void oo_linear6d(const double m[36], double *x, double *px, double *y, double *py, double *z, double *pz, int64_t n);
void oo_linear6d_matrix(const double beta[3], const double alpha[3], const double tune[3], double m[36]);

#ifdef __cplusplus
}
#endif
#endif
