/*
 * ffa_cuda.h -- C ABI of libffa_cuda.so, the sm_100a tracking hot path.
 *
 * PyFFA (the reference) is pure Python + Numba and exposes no FFI; its
 * hot-path boundary is the Python call interface of the tracking loop.
 * Each entry point below replaces one group of those calls (cited per
 * function, paths relative to the reference project).
 *
 * Conventions
 *  - Every pointer named "device" is caller-owned device memory (typically a
 *    torch tensor's data_ptr()).  Objects created here (field maps, space-charge
 *    plans) own only their packed tables and scratch.
 *  - Every call returns an int error code (FFA_OK = 0).  Argument errors are
 *    reported before any work is enqueued.
 *  - Calls are stream-ordered on the cudaStream_t passed as `stream` (NULL =
 *    legacy default stream), never synchronise implicitly, and are not
 *    thread-safe per object.  Kernels never trap: problems are counted in the
 *    caller's device status words (ffa_status_index).
 *  - Particle state is structure-of-arrays, float64, with the reference's
 *    meaning per array (src/FFAG_Bunch.py:23-74 column map).  An empty bunch
 *    (n = 0) is valid with NULL columns: the calls do nothing (a space-charge
 *    update then reports a degenerate grid).
 */
#ifndef FFA_CUDA_H
#define FFA_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFA_ABI_VERSION 1

#define FFA_MAX_POLY 16
#define FFA_MAX_SEG 16
#define FFA_MAX_GAPS 8
#define FFA_MAX_ORDER 4
#define FFA_MAX_HARMONICS 16

enum ffa_error {
    FFA_OK = 0,
    FFA_ERR_INVALID = 1,     /* bad argument (null pointer, size, flag) */
    FFA_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    FFA_ERR_NOMEM = 3,       /* device allocation failed */
    FFA_ERR_UNSUPPORTED = 4  /* valid but not built (e.g. order > FFA_MAX_ORDER) */
};

/* ffa_push flags */
enum ffa_push_flags {
    FFA_BORIS = 0,                /* relativistic Boris (solver_type 1) */
    FFA_RK4 = 1,                  /* 4th-order Runge-Kutta (solver_type 0) */
    FFA_FP64 = 0,                 /* all arithmetic in float64 */
    FFA_FP32C = 2,                /* Boris and RK4: float32 field exponentials and map lookup, float64
                                     push / RK4 stages */
    FFA_RF_PHYSICAL_SUM = 4,      /* sum every RF gap (reference: last gap wins) */
    FFA_FP32 = 8,                 /* Boris: float32 field and push, r / fi / z / RF phase accumulated in
                                     float64 (no space charge, no field-error harmonics) */
    /* Launch shape of the Boris pushers, bits 8-11 (0: the default shape).
     * Bits 8-9: threads per block 32 << v (32, 64, 128, 256).  Bits 10-11:
     * register cap per thread 80, 72, 64, 56; caps below 80 are built for the
     * FFA_FP32C pusher without space charge or field-error harmonics (else
     * FFA_ERR_UNSUPPORTED).  The
     * shape sets how many warps are resident per SM, not the arithmetic: the
     * results are the same for every shape.  RK4 takes the default only. */
    FFA_SHAPE_TB_SHIFT = 8,
    FFA_SHAPE_NREG_SHIFT = 10,
    FFA_SHAPE_MASK = 0xF00
};

/* Device status words, int64 each, accumulated with atomics. */
enum ffa_status_index {
    FFA_STATUS_LOST = 0,          /* particles lost at the aperture */
    FFA_STATUS_NAN = 1,           /* non-finite coordinates seen after a push */
    FFA_STATUS_OUT_OF_MAP = 2,    /* high-order map lookups clamped at the edge */
    FFA_STATUS_SC_DEGENERATE = 3, /* space-charge updates with an empty grid */
    FFA_STATUS_WORDS = 8
};

/* Mid-plane field: analytic orders 0/1 (src/FFAG_Field.py:1333-1426) and the
 * z-Taylor maps of orders 1..max_order (src/FFAG_MathTools.py:1139-1188). */
typedef struct ffa_field_desc {
    int32_t nsectors;
    int32_t n_spoly;              /* s(r) coefficients, highest degree first */
    int32_t n_spolyp;             /* s'(r) coefficients */
    int32_t n_convex;             /* flutter segments */
    int32_t max_order;            /* 0..FFA_MAX_ORDER */
    int32_t pad0;
    double B0, k;                 /* B0 * r^k */
    double spoly[FFA_MAX_POLY];
    double spolyp[FFA_MAX_POLY];
    double convex[FFA_MAX_SEG * 5];  /* x0, x1, W0, y01, y02 (rad) */
    double r_min, r_step;
    int64_t r_size;
    double fi_min, fi_step;
    int64_t fi_size;
    /* device, float64, shape (max_order+1, r_size, fi_size), row-major;
     * order 0 is not read */
    const double *bz_stack;
    const double *bfi_stack;
    const double *br_stack;
} ffa_field_desc;

/* RF gaps.  Fixed rectangles (spiral_nodes == NULL; FFAG_EField_new,
 * src/FFAG_Field.py:167-306, emap_kernel src/FFAG_Utils.py:984-1036): the
 * last gap's rectangle decides (or every gap's, FFA_RF_PHYSICAL_SUM), field
 * acc * (cos, sin)(theta_n - fi).
 * Spiral gaps (spiral_nodes != NULL; FFAG_EField_spiral, src/FFAG_Field.py:
 * 379-550, interpolate_spiral_emap_unique_gap_kernel src/FFAG_MathTools.py:
 * 1042-1114): one (r, phi) map of Er, Ez / z and Ephi shared by the gaps,
 * each gap placed at gap_azimuth[g].  For g = 0, 1, ... the local azimuth
 * phi = d + k 2 pi, d = fi - gap_azimuth[g], k = rint((phi_c - d) / 2 pi),
 * phi_c the middle of the phi axis; the first g with phi on the axis
 * [phi0, phi0 + dphi (nphi - 1)] is the particle's gap (none: no field).
 * Bilinear interpolation at (r, phi) with floor indices clamped to
 * [0, n - 2] and weights from the unclamped offsets (linear extrapolation
 * outside the r axis), field acc * (Er, Ez/z * z, Ephi) * sin(RF phase +
 * rf_shift[g]).  physical_sum does not apply (one gap per point). */
typedef struct ffa_rf_desc {
    int32_t enable;               /* Emap EnableFlag */
    int32_t ngaps;                /* 1..FFA_MAX_GAPS */
    int32_t pad0, pad1;
    double poly_x[FFA_MAX_GAPS][4];
    double poly_y[FFA_MAX_GAPS][4];
    double box[FFA_MAX_GAPS][4];  /* x_min, x_max, y_min, y_max */
    double theta_n[FFA_MAX_GAPS]; /* gap azimuth + pi/2 */
    double rf_shift[FFA_MAX_GAPS];
    /* spiral gaps */
    const double *spiral_nodes;   /* device, nr * nphi nodes of 4 doubles (Er, Ez/z, Ephi, 0), phi fastest */
    int32_t spiral_nr, spiral_nphi;   /* >= 2 each */
    double spiral_r0, spiral_dr;      /* r axis [m] */
    double spiral_phi0, spiral_dphi;  /* phi axis [rad], relative to the gap azimuth */
    double gap_azimuth[FFA_MAX_GAPS]; /* rad */
} ffa_rf_desc;

typedef struct ffa_aperture {
    int32_t enable;
    int32_t pad0;
    double rmin, rmax, zmin, zmax;
} ffa_aperture;

typedef struct ffa_consts {
    double q, c, m0, E0;          /* C, m/s, kg, J */
} ffa_consts;

/* Particle state (device SoA).  f5 is dfi/dt for Boris, Etot [J] for RK4.
 * inj/surv are 0/1 bytes (cols 7/8).  inj_step[i] is the absolute step index
 * at which particle i is injected (-1: never), precomputed by the host from
 * the reference's InjectParticles rule (src/FFAG_Bunch.py:265-303).
 * The e_pre / e_pp arrays and the sc_pre / sc_pp masks hold the two most
 * recent space-charge endpoints used by the per-step linear extrapolation
 * (src/FFAG_track.py:449-478); they may be NULL when sc_step == 0. */
typedef struct ffa_state_soa {
    double *r, *vr, *z, *vz, *fi, *f5, *rf;
    double *esc_r, *esc_z, *esc_fi;
    uint8_t *inj, *surv;
    const int32_t *inj_step;
    double *e_pre_r, *e_pre_z, *e_pre_fi;
    double *e_pp_r, *e_pp_z, *e_pp_fi;
    uint8_t *sc_pre, *sc_pp;
    /* Optional (NULL: identity): thread t of a push launch advances particle
     * order[t], a permutation of 0 .. n-1.  Every particle's arithmetic is
     * the same in any order; an order in which the 32 particles of a warp
     * are close in (r, vr, azimuth, energy) lets their z-Taylor node loads
     * share cache lines. */
    const int32_t *order;
} ffa_state_soa;

/* Per-step host-precomputed scalars (device arrays indexed by absolute step).
 * Boris: drf[s] = f_rf(t_s) * pi * 2 * dt, acc[s] = V0(t_s) / gap_width.
 * RK4:   drf[4s+k], acc[4s+k] for the stage times t, t+h/2, t+h/2, t+h, with
 *        drf the phase rate f_rf * pi * 2. */
typedef struct ffa_step_table {
    const double *drf;
    const double *acc;
    int64_t nsteps;               /* entries (Boris) or stage quadruples (RK4) */
} ffa_step_table;

/* Azimuth-crossing capture (PositionDumpBunch, src/FFAG_dump.py:789-1130;
 * detect_azimuth_crossing, src/FFAG_MathTools.py:1633-1695).  During a push,
 * every particle whose survival flag is 1 at the start of a step (after that
 * step's injection) and whose azimuth mod 2 pi passes one of the targets
 * within the step appends one record of FFA_CROSSING_RECORD doubles:
 *   [0] target index, [1] particle index, [2] absolute step,
 *   [3] interpolation ratio of the target within the step,
 *   [4..10]  pre-step  r, vr, z, vz, fi, f5, RF phase,
 *   [11..17] post-step r, vr, z, vz, fi, f5, RF phase,
 *   [18] post-step survival flag, [19] injection flag,
 *   [20..22] the space-charge field the step used (Esc r, z, fi).
 * Records come in no particular order.  `count` (device int64) is advanced
 * atomically; records past `capacity` are counted but not written.
 *
 * One-turn-map sums instead of records (fit_sums != NULL; one target): the
 * closed-orbit and tune fits of many instances (groups of particles, one
 * energy each) need, per instance and transverse plane, only the normal
 * equations of the least-squares map x' = M x + b between a particle's
 * successive crossings (the reference fits that map one trajectory at a
 * time: FFAG_SearchSEO / GetQrQz, src/FFAG_track.py:1142-1371).  At each
 * crossing the kernel interpolates the step as a cubic Hermite curve in
 * Cartesian coordinates rotated by the target (positions and velocities at
 * both ends, the crossing time by three Newton steps from the linear
 * estimate, velocities linear in time) to s = (r, vr, z, vz) at the target,
 * forms u = (s - fit_centre[k]) * fit_scale[k] for the particle's instance
 * k = fit_instance[i], and, when fit_has[i] is set, adds with float64
 * atomics to fit_sums[k * FFA_FIT_SUMS + 12 p + j], plane p (0: r, vr;
 * 1: z, vz), f = (w_p0, w_p1, 1) of the previous crossing w = fit_last[i]:
 *   j = 0..5:  f0 f0, f0 f1, f0, f1 f1, f1, 1     (f f^T, upper triangle)
 *   j = 6..11: u_p0 f0, u_p0 f1, u_p0, u_p1 f0, u_p1 f1, u_p1   (u' f^T)
 * and adds 1 to fit_sums[k * FFA_FIT_SUMS + 24] for every crossing; then
 * fit_last[i] = u, fit_has[i] = 1.  Memory is O(instances + particles),
 * whatever the number of turns; buf, capacity and count are not used.  The
 * sums depend on the order of the atomics at the rounding level. */
#define FFA_CROSSING_RECORD 23
#define FFA_MAX_CROSSING_TARGETS 8
#define FFA_FIT_SUMS 25
typedef struct ffa_crossing {
    int32_t ntargets;             /* 1 .. FFA_MAX_CROSSING_TARGETS */
    int32_t pad;
    double target[FFA_MAX_CROSSING_TARGETS];  /* rad, each in [0, 2 pi) */
    double *buf;                  /* device, capacity * FFA_CROSSING_RECORD */
    int64_t capacity;
    int64_t *count;               /* device */
    const int32_t *fit_instance;  /* device, n; NULL unless fit_sums */
    const double *fit_centre;     /* device, (instances, 4) */
    const double *fit_scale;      /* device, (instances, 4) */
    double *fit_last;             /* device, (n, 4) */
    uint8_t *fit_has;             /* device, n */
    double *fit_sums;             /* device, (instances, FFA_FIT_SUMS); NULL: records */
} ffa_crossing;

/* ffa_push with azimuth-crossing capture (all three pushers).  Replaces the
 * per-step PositionDumpBunch.check_and_dump of the step loop
 * (src/FFAG_dump.py:1098-1130, called from src/FFAG_track.py:297-579). */
int ffa_push_crossing(const struct ffa_fieldmap *fm, const ffa_rf_desc *rf, const ffa_aperture *ap,
                      const ffa_consts *cs, const ffa_step_table *tab, ffa_state_soa *st,
                      int64_t n, int64_t step0, int32_t nsteps, double dt, int32_t sc_step,
                      int32_t flags, void *stream, int64_t *status, const ffa_crossing *xing);

typedef struct ffa_fieldmap ffa_fieldmap;

/* Packs the z-Taylor stacks into the interleaved node layout the push kernels
 * read (float64 and float32 copies).  Replaces FFAG_Bfield_analytical map
 * loading (src/FFAG_Field.py:636-711). */
int ffa_fieldmap_create(const ffa_field_desc *desc, void *stream, ffa_fieldmap **out);
int ffa_fieldmap_destroy(ffa_fieldmap *fm);

/* Field-error harmonics of a field map: every pusher then adds
 * Bz += sum_k amp[k] cos(m[k] fi + phase[k]) over the k with
 * rmin[k] <= r <= rmax[k] (fi the unwrapped azimuth; Br, Bfi unchanged) after
 * the mid-plane map.  Replaces FFAG_BField_Error + AddBHarmonics_to_Bmap_njit
 * (src/FFAG_Field.py:947-1042, bharmonics_kernel_1d :1541-1587) as called by
 * Boris_solve (src/FFAG_track.py:1007) and FunctionForAccelerationBunch_dt
 * (:1782).  Host arrays of n <= FFA_MAX_HARMONICS values (amp in tesla, phase
 * in rad, m an integer), copied to a small device table (allocated on the
 * first call, synchronous copy); n = 0 removes them.  The closed-orbit tracks
 * (ffa_theta_track) do not take them.  Takes effect for later pushes. */
int ffa_fieldmap_set_harmonics(ffa_fieldmap *fm, int32_t n, const double *m, const double *amp,
                               const double *phase, const double *rmin, const double *rmax);

/* Applies the injection of absolute step `step` (flags only).
 * Replaces FFAG_Bunch.InjectParticles (src/FFAG_Bunch.py:265-303). */
int ffa_inject(ffa_state_soa *st, int64_t n, int64_t step, void *stream);

/* Advances n particles by nsteps fixed steps starting at absolute step
 * step0: per step injection, space-charge extrapolation (sc_step > 0), field
 * evaluation and the Boris or RK4 update, fused in one launch with the state
 * held in registers.  Replaces one iteration of the step loop of
 * rk4_solve_dt_bunch3_withSC_boris / _withSC per step
 * (src/FFAG_track.py:297-579, 65-294): Boris_solve (:948-1049) or
 * rk4_step_malloc + RK4_Post_Step_njit (:51-61, src/FFAG_MathTools.py:2269).
 * status: device int64[FFA_STATUS_WORDS]. */
int ffa_push(const ffa_fieldmap *fm, const ffa_rf_desc *rf, const ffa_aperture *ap,
             const ffa_consts *cs, const ffa_step_table *tab, ffa_state_soa *st,
             int64_t n, int64_t step0, int32_t nsteps, double dt, int32_t sc_step,
             int32_t flags, void *stream, int64_t *status);

/* Resident blocks per SM and threads per block of the push kernel that
 * ffa_push / ffa_push_crossing (crossing != 0) would launch for `flags` and
 * a field map of `max_order`, without space charge (the runtime's occupancy
 * calculator; needs a device).  For the launch-shape autotuner's report.
 * No counterpart in the reference, whose Numba kernels have no launch shape. */
int ffa_push_occupancy(int32_t flags, int32_t max_order, int32_t crossing, int32_t *blocks_per_sm,
                       int32_t *threads_per_block);

/* Converts between the reference's N x 16 row-major matrix (device) and the
 * SoA state.  soa_to_aos writes cols 0-5 and 7-12 and leaves 6, 13-15.
 * Replaces the LocalBunch column views used throughout src/FFAG_track.py. */
int ffa_aos_to_soa(const double *aos, int64_t n, ffa_state_soa *st, void *stream);
int ffa_soa_to_aos(const ffa_state_soa *st, int64_t n, double *aos, void *stream);

/* Sum of fi over the particles whose fi is not NaN, written to *out (device
 * double), and their count to *count (device int64); the host divides.
 * Replaces the mean in the stop test of src/FFAG_track.py:559-577. */
int ffa_mean_fi(const ffa_state_soa *st, int64_t n, double *out, int64_t *count, void *stream);

/* ------------------------------------------------------- space charge */

/* 2.5D slice-by-slice space charge (src/FFAG_Bunch.py:1157-1352). */
typedef struct ffa_sc_desc {
    int32_t ns, nx, nz;           /* slices, transverse grid */
    int32_t hockney;              /* 0: periodic kernel (reference); 1: open boundary */
    int32_t boris;                /* 1: gamma from |v|; 0: gamma = Etot / E0 */
    int32_t pad0;
    int64_t n_max;                /* particle capacity of the scratch */
    double sigma_ratio;           /* grid half-width in rms sizes */
    double q_macro;               /* marcosize * q [C] */
    double speed_c, E0_rest_MeV, E0_J;
    /* closed-orbit tables (device, float64): r0 and pr0 of shape (nE, nfi),
     * perimeter (nE); Ek axis [MeV] and fi axis [rad] uniform */
    int64_t nE, nfi;
    double Ek0, dEk, fi0, dfi;
    const double *seo_Ek;         /* device, nE (for the perimeter interpolation) */
    const double *seo_r;
    const double *seo_pr;
    const double *seo_perimeter;
} ffa_sc_desc;

/* Diagnostics of the last update (device struct written by ffa_sc_step). */
typedef struct ffa_sc_diag {
    double fi_s, fi_e, slice_step, mean_gamma_m1;
    double mean_x, mean_z, sigma_x, sigma_z;
    double xmin, xmax, zmin, zmax, dx, dz;
    double bunch_length, q_density;
    int64_t count, degenerate;
} ffa_sc_diag;

typedef struct ffa_sc_plan ffa_sc_plan;

/* Plan of ffa_sc_step for one bunch capacity and grid: owns the device
 * scratch.  Replaces the grid and FFT set-up of the step loop
 * (pyfftw plans and buffers, src/FFAG_track.py:319-328). */
int ffa_sc_plan_create(const ffa_sc_desc *desc, void *stream, ffa_sc_plan **out);
int ffa_sc_plan_destroy(ffa_sc_plan *plan);

/* One space-charge update over the particles with surv != 0: coordinates,
 * slice arc and moments, CIC deposit, Poisson solve per slice, field and
 * gather into esc_*.  Replaces Build_2_5D_SliceGrid_sbs
 * (src/FFAG_Bunch.py:1157-1352) and the endpoint roll of src/FFAG_track.py:341-400.  When `roll` is
 * nonzero the extrapolation endpoints are rolled afterwards as the step loop
 * does (first != 0 at step 0).  diag: device ffa_sc_diag or NULL. */
int ffa_sc_step(ffa_sc_plan *plan, ffa_state_soa *st, int64_t n, int32_t roll, int32_t first,
                void *stream, int64_t *status, ffa_sc_diag *diag);

/* Space-charge update that allocates nothing.  No counterpart in the
 * reference (its space charge runs on host memory); it exists for callers
 * that cannot allocate device memory while running -- host codes that
 * reserve their whole device budget at start-up, or tracking loops embedded
 * in a control system where an allocation could fail or stall the device.
 * Same inputs, outputs and results as ffa_sc_plan_create + ffa_sc_step, but
 * all scratch lives in one fixed device array compiled into the library
 * (about 30 MB, held by every device that loads the library until exit).
 * Limits: n <= FFA_SC_STATIC_MAX_PARTICLES (else FFA_ERR_INVALID);
 * ns * nz * nx <= FFA_SC_STATIC_MAX_CELLS, nx, nz <= 128, periodic boundary
 * (else FFA_ERR_UNSUPPORTED).  Every call on a device shares the array and
 * finds the previous call's contents there (the charge accumulator is
 * cleared each call, the FFT twiddles are formed inside the kernels); calls
 * that overlap on the GPU race and must be serialised by the caller.  Each
 * call looks up the array's address on the current device
 * (cudaGetSymbolAddress, which allocates nothing). */
#define FFA_SC_STATIC_MAX_PARTICLES 524288
#define FFA_SC_STATIC_MAX_CELLS 524288
int ffa_sc_step_static(const ffa_sc_desc *desc, ffa_state_soa *st, int64_t n, int32_t roll, int32_t first,
                       void *stream, int64_t *status, ffa_sc_diag *diag);

/* Device views of the plan's last charge, potential and field cubes
 * (float32, (ns, nz, nx)), and of the per-particle slice / cell indices
 * (int32 slice, int64 cell = (s*nz + iz)*nx + ix, -1 when not deposited):
 * the rho / phi / Ex / Ez grids Build_2_5D_SliceGrid_sbs returns
 * (src/FFAG_Bunch.py:1346-1352). */
int ffa_sc_buffers(const ffa_sc_plan *plan, const float **rho, const float **phi,
                   const float **ex, const float **ez, const int32_t **slice_idx,
                   const int64_t **cell_idx);

/* ------------------------------------------------------ bunch generation
 * One sub-bunch of GenerateInitDistributionDtInjNew
 * (src/FFAG_Distribution.py:1152-1345) written on the device: n rows of the
 * reference's p-format matrix (r, pr, z, pz, fi, Ek [MeV], inj_t [ns],
 * flags 0, RF phase 0, space-charge fields 0, Bunch_ID, Local_ID, Global_ID),
 * drawn from the distribution shapes of src/FFAG_Distribution.py:76-1149
 * through the Twiss transformation of TwissContainer (:16-73).  Random
 * numbers: Philox4x32-10, counter (particle id0 + i, draw group, sub_bunch)
 * under the key `seed`, so the rows do not depend on the launch or on how a
 * bunch is split over calls.  `twiss` holds (alpha, beta, emittance) of the
 * horizontal, vertical and longitudinal planes as the reference's
 * generator receives them; each shape applies its own emittance factor
 * (KV2D 4x, water-bag 2D 6x, KV1D 2x, water-bag 1D 4x).  Rejection shapes
 * (Gauss with a cut-off, hollow water-bag 2D) try FFA_BUNCH_MAX_ATTEMPTS
 * times; particles that never pass keep the last draw and are counted in
 * *rejected (device, may be NULL). */
#define FFA_BUNCH_MAX_ATTEMPTS 64
enum ffa_dist_type {
    FFA_DIST_GAUSS = 0,
    FFA_DIST_KV = 1,
    FFA_DIST_WATERBAG = 2,
    FFA_DIST_HOLLOW_WATERBAG = 3,
    FFA_DIST_UNIFORM_GAUSS = 4     /* longitudinal only: t uniform, dE normal */
};
typedef struct ffa_bunch_desc {
    int64_t n;                    /* rows */
    int64_t id0;                  /* Local_ID / Global_ID of the first row */
    uint64_t seed;
    int64_t sub_bunch;            /* painting index (Bunch_ID's stream) */
    int32_t transverse, longitudinal;
    double cut_off;               /* Gauss cut-off in rms units, <= 0: none */
    double twiss[3][3];           /* (alpha, beta, emittance) of x, z, longitudinal */
    double uniform_length;        /* FFA_DIST_UNIFORM_GAUSS: t span [ns] */
    double uniform_sigma;         /* FFA_DIST_UNIFORM_GAUSS: rms of dE [MeV] */
    double centre[6];             /* added: r, pr, z, pz, Ek, inj_t */
    double fi;                    /* injection azimuth [rad] */
    double bunch_id;
    double *out;                  /* device, n x 16 */
} ffa_bunch_desc;

int ffa_bunch_sample(const ffa_bunch_desc *desc, unsigned long long *rejected, void *stream);

/* ------------------------------------------------------ closed-orbit tracks
 * Tracks of the closed-orbit search (FunctionForSEO through rk4_solve /
 * rk4_solve_vect, src/FFAG_track.py:582-640 and 1698-1740): m trajectories
 * (r, pr, z, pz) at fixed momentum P with the azimuth as independent variable,
 * from 0 over n_points - 1 RK4 steps of h = t_end / (n_points - 1) through
 * the analytic field of `fm` (the mid-plane field and its z-linear terms; the
 * z-Taylor tables are not used).  Stage azimuths of step i: i h (time_mode 0,
 * rk4_solve) or the running sum of h (time_mode 1, rk4_solve_vect). */
typedef struct ffa_theta_track_desc {
    int64_t m;                    /* trajectories */
    int32_t n_points;             /* azimuth points, >= 2 */
    int32_t time_mode;            /* 0: i h, 1: running sum */
    int32_t traj_cols;            /* 2: r, pr; 7: r, pr, z, pz, Bz, Br, Bfi (field at that point) */
    int32_t pad;
    double t_end;                 /* rad */
    double q;                     /* charge [C] */
    const double *x0;             /* device [m][5]: r, pr, z, pz, P */
    double *x1;                   /* device [m][4]: r, pr, z, pz at t_end */
    double *traj;                 /* device [m][n_points][traj_cols] at every point, or NULL */
} ffa_theta_track_desc;

/* Runs the m tracks in one launch (one thread each); replaces the per-orbit
 * rk4_solve / rk4_solve_vect calls of FFAG_SearchSEO (src/FFAG_track.py:1245-1371). */
int ffa_theta_track(const struct ffa_fieldmap *fm, const ffa_theta_track_desc *desc, void *stream);

/* ---------------------------------------------------------- map generation
 * z-Taylor coefficient tables of a scaling map, B0(r, th) = a r^k G(th - s(r))
 * (Generate_Bmaps / Generate_Bmaps_MultiProcess, src/FFAG_HighOrder.py:828-998;
 * main_Bmap, examples/main_Bmap.py:17-75).  Every table entry is a linear
 * combination of the flutter derivatives G^(p) on the theta grid, rolled by
 * the row's integer spiral shift (shift_function, src/FFAG_HighOrder.py:393-398):
 *   T[c][n][i][j] = sum_p weights[c][n][i][p] * G^(p)[(j - shift[i]) mod n_theta] / mean(G)
 * with c = 0 Bz, 1 Br, 2 Bfi.  The host forms the weights from the Laplacian
 * term algebra (r-only factors); the library computes the flutter derivatives
 * (sigmoid-derivative polynomials, src/FFAG_HighOrder.py:212-350), their
 * sector mean, and the tables. */
#define FFA_MAPGEN_MAX_DERIV 16
typedef struct ffa_mapgen_desc {
    int32_t n_seg;                /* flutter magnets, <= FFA_MAX_SEG */
    int32_t n_deriv;              /* G derivatives 0 .. n_deriv-1, <= FFA_MAPGEN_MAX_DERIV */
    int32_t n_orders;             /* Taylor orders 0 .. n_orders-1 */
    int32_t pad;
    int64_t n_r, n_theta;
    double seg_x0[FFA_MAX_SEG], seg_x1[FFA_MAX_SEG];   /* rad */
    double seg_k[FFA_MAX_SEG];    /* 16 / W0 */
    double seg_y[FFA_MAX_SEG];    /* signed amplitude */
    /* device [n_seg][2][n_deriv][n_deriv + 1]: coefficients, highest power
     * first, of the i-th sigmoid derivative as a polynomial in the sigmoid,
     * for steepness +k (entry / 0) and -k (exit / 1); row i uses i + 2 of them */
    const double *sig_poly;
    const double *theta;          /* device [n_theta] */
    const double *weights;        /* device [3][n_orders][n_r][n_deriv] */
    const int32_t *shift;         /* device [n_r] */
    double *gder;                 /* device scratch [n_deriv][n_theta] */
    double *gmean;                /* device scratch [1]: sector mean of G */
    double *bz, *br, *bfi;        /* device [n_orders][n_r][n_theta] */
} ffa_mapgen_desc;

/* Fills bz, br, bfi; replaces Generate_Bmaps (src/FFAG_HighOrder.py:828-998). */
int ffa_mapgen(const ffa_mapgen_desc *desc, void *stream);

/* ------------------------------------------------------ learned sector map
 * A residual network for the one-sector transfer map in normalised
 * coordinates s = (u, pu, v, pv, e, 0):
 *   y = s + s Ws + bs + q(s) Wq + f(s),  f = L4 . SiLU . L3 . SiLU . L2 . SiLU . L1,
 * with q(s) the 15 products s_i s_j (i <= j < 5, ordered (0,0), (0,1) .. (0,4),
 * (1,1) .. (4,4)): a second-order skip connection around a network of widths
 * 6 -> 256 -> 256 -> 256 -> 6, L(h) = h W + b.  The reference has no
 * counterpart; the map it learns is one sector of the azimuth-domain tracker
 * (ffa_theta_track), which follows FunctionForSEO (src/FFAG_track.py:1597-1640).
 *
 * Parameters: one float32 block of FFA_MLP_PARAMS values, row-major (n_in,
 * n_out) matrices with padded shapes:
 *   W1 [16][256] (rows 6..15 zero), b1 [256], W2 [256][256], b2 [256],
 *   W3 [256][256], b3 [256], W4 [256][8] (columns 6, 7 zero), b4 [8],
 *   Ws [8][8] (6 x 6 used), bs [8], Wq [16][8] (15 x 6 used).
 * Hidden-layer products run on the tensor cores with bfloat16 operands and
 * float32 accumulation; the skip connection and the state stay float32.
 * Samples and states: float32 [n][8], columns 6, 7 ignored. */
#define FFA_MLP_HIDDEN 256
#define FFA_MLP_PARAMS 138192
#define FFA_MLP_WPACK_BYTES 278528   /* bfloat16 copies of W1..W4 for inference */
#define FFA_MLP_SPLIT_WORK 1048576    /* floats of split-K partial products in the training work area */

/* One optimiser step (no counterpart in the reference, whose tracker has no
 * learned map): forward, mean-squared error over the first n_fit
 * outputs, backward into `grads` (every parameter, same layout), then Adam
 * on the entries whose `mask` byte is non-zero (mask NULL: all) when lr > 0.
 * `step` is the 1-based Adam step (bias correction).  `work` holds
 * 8 * batch * 256 + 24 * batch + FFA_MLP_SPLIT_WORK floats; `loss_part` 148 doubles whose sum is
 * the batch's summed squared error (before the step). */
typedef struct ffa_mlp_train_desc {
    int64_t batch;
    int32_t n_fit;                /* 1..6 */
    int32_t step;
    float lr, beta1, beta2, eps;
    float *params, *grads, *adam_m, *adam_v;
    const uint8_t *mask;
    const float *x, *target;      /* device [batch][8] */
    float *work;
    double *loss_part;
    /* Optional device schedule (both or neither): the step takes its
     * learning rate from lr_table[*counter] and is Adam step *counter + 1
     * (bias corrections formed on the device), then increments *counter;
     * lr and step above are then ignored and the update always runs.  With
     * nothing read from the host per step, the call can be captured once in
     * a CUDA graph and replayed. */
    const float *lr_table;
    int32_t *counter;
} ffa_mlp_train_desc;

int ffa_mlp_train_step(const ffa_mlp_train_desc *desc, void *stream);

/* No counterpart in the reference (part of the learned map's training).
 * C[M][N] = op(A) op(B) (+ bias[N]) in bfloat16 x bfloat16 -> float32 on
 * the tensor cores; op(A)[m][k] = A[m lda + k] (transA 0) or A[k lda + m],
 * op(B)[k][n] = B[k ldb + n] (transB 0) or B[n ldb + k].  The training step's
 * building block, exported for tests. */
int ffa_mlp_gemm(const float *A, int lda, int transA, const float *B, int ldb, int transB, float *C, int ldc,
                 int M, int N, int K, const float *bias, void *stream);

/* Tensor-core GEMM tiles (ffa_mlp_gemm, ffa_mlp_train_step) whose bounded
 * pipeline waits ran out since the last call (their output tiles hold NaN);
 * reads and clears the device counter, synchronising the device.  No
 * counterpart in the reference (its training path does not exist; the
 * learned map is new). */
int ffa_mlp_gemm_timeouts(int32_t *count);

/* No counterpart in the reference (learned map).
 * Inference weights: the bfloat16 packing of a parameter block into `wpack`
 * (FFA_MLP_WPACK_BYTES, 16-byte aligned).  Call again after the parameters
 * change. */
int ffa_mlp_pack(const float *params, void *wpack, void *stream);

/* No counterpart in the reference (learned map; it stands in for the
 * per-sector steps of the tracking loop, src/FFAG_track.py:297-579).
 * Applies the map n_apply times to each state in place (tcgen05 tensor
 * cores, one CTA per SM).  A state takes a map only while it is inside the
 * training domain, u^2 + pu^2 <= radius2, v^2 + pv^2 <= radius2 and
 * |e| <= 1 (radius2 <= 0: no check); the first state outside it is kept, and
 * applied[i] (when not NULL) is the number of maps state i took.  The
 * kernel's internal pipeline waits are bounded (2 s): if one runs out, the
 * kernel stops, leaves the states it had not finished unchanged and sets
 * *error to 1 (when not NULL). */
typedef struct ffa_mlp_infer_desc {
    int64_t n;
    int32_t n_apply;
    float radius2;
    const float *params;
    const void *wpack;
    float *state;                 /* device [n][8], 16-byte aligned */
    int32_t *applied;             /* device [n] or NULL */
    int32_t *error;               /* device word or NULL */
} ffa_mlp_infer_desc;

int ffa_mlp_infer(const ffa_mlp_infer_desc *desc, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FFA_CUDA_H */
