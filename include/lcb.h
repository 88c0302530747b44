/*
 * lcb.h -- C ABI of liblcb.so, the B200 (sm_100a) kernels of the quasistatic
 * 3D xi step of lcodePy.
 *
 * Conventions
 *  - Every pointer argument is a device pointer unless stated otherwise.
 *    All arrays are C-ordered (row-major); grids are N x N with the flat
 *    index  y + N * x  (x = first axis), as in the reference
 *    (lcode/plasma3d/weights.py:180).  Plasma particle arrays of all sorts
 *    are concatenated: sort s occupies [s * n_per_sort, (s+1) * n_per_sort).
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *  - Every call is asynchronous on `stream` and returns LCB_OK or an error
 *    code; lcb_last_error() gives a message for the calling thread.
 *  - `err` (may be NULL) is a device int32 that kernels OR error bits into
 *    (LCB_DEVERR_*).  The host reads it at its own sync points.
 *  - The library allocates no device memory: scratch is passed in by the
 *    caller, with its size given by the matching *_workspace_bytes query.
 *
 * Reference interfaces replaced (paths relative to the lcodePy project root)
 * are cited beside each entry point.
 */
#ifndef LCB_H
#define LCB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LCB_OK 0
#define LCB_ERR_INVALID 1   /* bad argument (size, pointer, alignment) */
#define LCB_ERR_CUDA 2      /* a CUDA runtime call failed */
#define LCB_ERR_DEVICE 3    /* a device error word was found set */

/* Device error bits. */
#define LCB_DEVERR_PLASMA_STENCIL 1  /* plasma stencil left the grid (NaN or runaway) */
#define LCB_DEVERR_BEAM_STENCIL 2    /* beam stencil left the N*N array */
#define LCB_DEVERR_CAPACITY 4        /* a device-side buffer would overflow */
#define LCB_DEVERR_FIXED_RANGE 8     /* a deposit contribution near the fixed-point range */

/* Precision modes for the field solver and deposition. */
#define LCB_PREC_FP64 0   /* FP64 everywhere: the reference's arithmetic */
#define LCB_PREC_MIXED 1  /* fixed-point deposition, FP32 transforms; FP64 particles */

const char *lcb_last_error(void);
int lcb_version(void);
/* Number of kernel launches issued by this library since load (all threads). */
int64_t lcb_launch_count(void);

/* ---------------------------------------------------------------------
 * Plasma particles
 * ------------------------------------------------------------------- */

/* Copy prev -> full and free-stream the offsets:
 *   full = prev;  where m != 0:  x_offt += px / (gamma m - pz) * xi_step.
 * Replaces move_particles_wo_fields, lcode/plasma3d/move.py:331-349
 * (the copy) with the kernel move_wo_fields_cupy, move.py:292-313.
 * prev and full may alias (then it is the in-place kernel alone). */
int lcb_plasma_move_wo_fields(int64_t n, double xi_step, const double *m,
                              const double *x_offt_prev, const double *y_offt_prev,
                              const double *px_prev, const double *py_prev,
                              const double *pz_prev, const double *q_prev,
                              double *x_offt_full, double *y_offt_full,
                              double *px_full, double *py_full, double *pz_full,
                              double *q_full, void *stream);

/* Fused midpoint field gather and momentum/position update with reflection
 * at +-boundary and absorption (q_full := 0).  Fields are N x N planes.
 * Replaces move_smart_cupy, lcode/plasma3d/move.py:169-289, driven by
 * move_particles_smart, move.py:351-381. */
int lcb_plasma_move_smart(int64_t n, double xi_step, double boundary, double h,
                          int grid_steps, const double *Ex, const double *Ey,
                          const double *Ez, const double *Bx, const double *By,
                          const double *Bz, const double *x_init,
                          const double *y_init, const double *x_offt_prev,
                          const double *y_offt_prev, const double *px_prev,
                          const double *py_prev, const double *pz_prev,
                          const double *m, double *q_full, double *x_offt_full,
                          double *y_offt_full, double *px_full, double *py_full,
                          double *pz_full, int *err, void *stream);

/* Charge and current deposition of all sorts.  Outputs ro, jx, jy, jz are
 * (2, N, N) planes (plane s = sort s), zeroed here first.  When ro_initial
 * is not NULL (background ions) plane 1 of ro is set to it afterwards.
 * precision LCB_PREC_MIXED accumulates 64-bit fixed-point sums (resolution
 * 2^-32, exact and order independent) and converts them to FP64.
 * Replaces compute_rhoj, lcode/plasma3d/rhoj.py:11-20, with deposit_plasma,
 * weights.py:249-285, and its kernel deposit_plasma_cupy, weights.py:151-190. */
int lcb_plasma_deposit(int64_t n_per_sort, int n_sorts, int grid_steps,
                       double h, int particles_side, int precision,
                       const double *x_init, const double *y_init,
                       const double *x_offt, const double *y_offt,
                       const double *px, const double *py, const double *pz,
                       const double *q, const double *m, const double *ro_initial,
                       double *ro, double *jx, double *jy, double *jz,
                       void *workspace, size_t workspace_bytes, int *err,
                       void *stream);
size_t lcb_plasma_deposit_workspace_bytes(int grid_steps, int precision);

/* Plasma particle arrays of all sorts (concatenated). */
typedef struct lcb_plasma_particles {
    double *x_init, *y_init, *x_offt, *y_offt, *px, *py, *pz, *q, *m;
} lcb_plasma_particles;

typedef struct lcb_move_deposit_args {
    int64_t n_per_sort;
    int n_sorts, particles_side, grid_steps, precision;
    int first;               /* 1: first stage of an xi step (full estimated here) */
    int lattice_fineness;    /* particles per cell along an axis (window size hint) */
    double xi_step, boundary, h;
    const double *fields[6]; /* Ex Ey Ez Bx By Bz used for the midpoint gather */
    lcb_plasma_particles prev, full;  /* full.{x_offt,y_offt,px,py,pz,q} written */
    const double *ro_initial;         /* background ions, or NULL */
    double *ro, *jx, *jy, *jz;        /* (2, N, N) outputs, zeroed here */
    void *workspace;                  /* lcb_plasma_deposit_workspace_bytes */
    size_t workspace_bytes;
    int *err;
} lcb_move_deposit_args;

/* One predictor-corrector stage fused: move_smart on every particle and the
 * deposition of its new state, and for the first stage of an xi step the
 * free-streaming estimate before them.  The results equal
 * lcb_plasma_move_wo_fields (first stage) + lcb_plasma_move_smart +
 * lcb_plasma_deposit.  Replaces, for one stage of
 * Plane2d3vPlasmaSolver.step_dxi (lcode/plasma3d/solver.py:29-76), the calls
 * move_particles_wo_fields / move_particles / compute_rhoj. */
int lcb_plasma_move_deposit(const lcb_move_deposit_args *a, void *stream);

/* ---------------------------------------------------------------------
 * Field solver
 * ------------------------------------------------------------------- */

/* Constant operators of the field solver, built once per grid on the device
 * by lcb_field_operators_build into a caller buffer of
 * lcb_field_operators_bytes(N, precision) bytes (256-byte aligned): the
 * even/odd halves of the DST-I matrix 2 sin(pi (j+1)(k+1)/(N-1)) (order N-2)
 * and of the DCT-I matrix c_j cos(pi j k/(N-1)) (order N), and the
 * reference's Dirichlet, mixed (and its transpose) and Neumann solver
 * matrices (lcode/plasma3d/initialization.py:15-67), in FP64, or in FP32
 * for LCB_PREC_MIXED.  subtraction_coeff is the Helmholtz shift of the mixed
 * matrix ('field-solver-subtraction-coefficient' after the 3D adjustment). */
size_t lcb_field_operators_bytes(int grid_steps, int precision);
int lcb_field_operators_build(int grid_steps, double h, double subtraction_coeff,
                              int precision, void *operators, size_t bytes,
                              void *stream);

/* Seven N x N planes in the order Ex, Ey, Ez, Bx, By, Bz, Phi. */
typedef struct lcb_fields {
    double *f[7];
} lcb_fields;

/* Currents: four (n_planes, N, N) arrays ro, jx, jy, jz. */
typedef struct lcb_currents {
    const double *ro, *jx, *jy, *jz;
    int n_planes;
} lcb_currents;

typedef struct lcb_compute_fields_args {
    int grid_steps;
    double h, xi_step, subtraction_coeff;
    int precision;
    const void *operators;   /* from lcb_field_operators_build (same N, h,
                                coefficient and precision) */
    lcb_fields fields;       /* Ex, Ey, Bx, By read (Helmholtz term) */
    lcb_fields fields_prev;  /* read */
    lcb_currents currents_prev, currents_full;
    const double *rho_beam_full, *rho_beam_prev; /* N x N */
    double rho_beam_divisor;  /* beam planes are divided by this (h^2 or 1) */
    lcb_fields out_full;      /* written; any plane may be NULL (skipped) */
    lcb_fields out_half;      /* written; any plane may be NULL */
    void *workspace;
    size_t workspace_bytes;
} lcb_compute_fields_args;

/* Replaces compute_fields, lcode/plasma3d/fields.py:276-322 (with
 * calculate_Ex_Ey_Bx_By :176-230, calculate_Ez :112-139, calculate_Bz
 * :233-266, calculate_Phi :142-159 and the GPU transforms :36-107): every
 * DST-I / DCT-I / mixed transform is a dense batched matrix product.
 * Phi is skipped when both its out_full and out_half planes are NULL.
 * The transforms run on one of two tensor-core wave kernels (one CTA per
 * output tile, or a persistent warp-specialised one); the first call for a
 * (device, grid_steps, precision) that is not under stream capture times
 * both on the caller's stream and keeps the faster (it computes the same
 * outputs several times and synchronises the stream once).
 * LCB_WAVE_KERNEL=tiled or =persistent in the environment fixes the choice. */
int lcb_compute_fields(const lcb_compute_fields_args *a, void *stream);
size_t lcb_compute_fields_workspace_bytes(int grid_steps, int precision);

/* The wave kernel chosen for (grid_steps, precision) on the current device:
 * 1 one CTA per tile, 2 persistent, 0 not measured yet.  No counterpart in
 * the reference (reporting only). */
int lcb_wave_kernel_choice(int grid_steps, int precision);

/* Allocation-free compute_fields.  No counterpart in the reference: it exists
 * for callers that cannot allocate device memory themselves -- a host code
 * that only receives device pointers from another framework's memory pool,
 * or a language binding with no route to a CUDA allocator -- and so cannot
 * provide the workspace lcb_compute_fields asks for.
 *
 * Same arguments and results as lcb_compute_fields, except that a->workspace
 * and a->workspace_bytes are ignored: the scratch is a file-scope device
 * array of LCB_NOALLOC_FIELDS_SCRATCH_BYTES bytes inside liblcb.so, held on
 * every GPU that loads the library until the process exits.  Grids whose
 * scratch need (lcb_compute_fields_workspace_bytes) exceeds it are rejected
 * with LCB_ERR_INVALID; every odd grid_steps up to 283 fits in
 * LCB_PREC_FP64 and up to 427 in LCB_PREC_MIXED.  Nothing is allocated or
 * freed.
 *
 * The first call on a device looks up the array's device address there
 * (cudaGetSymbolAddress, with that device current); make that first call
 * before any stream capture.  All calls share the one array and find the
 * previous call's contents in it; the solver clears what must start at zero
 * itself.  Calls that overlap on the GPU (e.g. on two streams at once) race
 * on the array and give wrong results: serialise them. */
#define LCB_NOALLOC_FIELDS_SCRATCH_BYTES ((size_t)16 << 20)
int lcb_compute_fields_noalloc(const lcb_compute_fields_args *a, void *stream);

/* ---------------------------------------------------------------------
 * Beam
 * ------------------------------------------------------------------- */

/* Beam density: 25-point transverse x linear-in-xi deposit of a layer into
 * the carried plane ro0 (weight xi_loc) and the next plane ro1 (1 - xi_loc),
 * xi_loc = (-xi_step * layer_idx - xi) / xi_step.  Accumulates (no zeroing).
 * Replaces deposit_beam, lcode/beam3d/weights.py:152-163, and its kernel
 * deposit_beam_cupy, weights.py:108-138. */
int lcb_beam_deposit(int64_t n, int grid_steps, double h, double xi_step,
                     int64_t layer_idx, const double *x, const double *y,
                     const double *xi, const double *q_norm, double *ro0,
                     double *ro1, int *err, void *stream);

/* Substep sizes for the first n_fresh particles of a layer:
 *   d = 1, halved while d > sqrt(sqrt(1/q_m^2 + pz^2) / substep_energy);
 *   dt = d * time_step; remaining_steps = (int64)(1 / d).
 * Replaces start_moving_layer with calculate_substepping_step,
 * lcode/beam3d/beam_calculator.py:28-46,97-114. */
int lcb_beam_substepping(int64_t n_fresh, const double *q_m, const double *pz,
                         double substep_energy, double time_step, double *dt,
                         int64_t *remaining_steps, void *stream);

/* Substepped Higuera-Cary push of a layer between plane k (fields_k,
 * = previous xi step) and plane k+1 (fields_k1, = new xi step).  Writes
 * flags[i] = 1 lost | 2 moved | 4 fell.
 * Replaces move_beam_layer, lcode/beam3d/beam_calculator.py:116-134, with
 * the kernel move_beam_cupy, lcode/beam3d/move.py:132-276. */
int lcb_beam_move(int64_t n, double xi_step, double r_max,
                  int64_t beam_layer_idx, double h, int grid_steps,
                  const double *q_m, const double *dt,
                  const lcb_fields *fields_k, const lcb_fields *fields_k1,
                  int64_t *remaining_steps, int64_t *id, double *x, double *y,
                  double *xi, double *px, double *py, double *pz,
                  uint8_t *flags, int *err, void *stream);

/* Beam particles as SoA arrays (lcode/beam3d/data.py:21-60): xi x y px py pz
 * q_m q_norm (FP64), id (int64), dt (FP64), remaining_steps (int64). */
typedef struct lcb_beam_soa {
    double *xi, *x, *y, *px, *py, *pz, *q_m, *q_norm;
    int64_t *id;
    double *dt;
    int64_t *remaining_steps;
} lcb_beam_soa;

typedef struct lcb_beam_step_args {
    int grid_steps;
    double h, xi_step, r_max, substep_energy, time_step;
    int64_t layer_idx;                 /* plasma layer i just computed: the push
                                          moves layer i-1 between planes i-1, i */
    int64_t layout_idx;                /* layer deposited into ro0 / ro1 */
    lcb_beam_soa source;               /* beam sorted by xi, descending */
    int64_t layout_begin, layout_end;  /* slice of source deposited (layer layout_idx) */
    int64_t move_begin, move_end;      /* slice of source pushed (layer i-1, fresh) */
    lcb_beam_soa fell_in;              /* particles that fell from the last push */
    const int64_t *fell_in_count;      /* device */
    lcb_beam_soa fell_out;             /* written: particles falling now */
    int64_t *fell_out_count;           /* device, overwritten */
    int64_t fell_capacity;
    lcb_beam_soa drain;                /* moved particles are appended */
    int64_t *drain_count;              /* device, advanced */
    int64_t drain_capacity;
    lcb_beam_soa lost;                 /* lost particles appended; all NULL: dropped */
    int64_t *lost_count;               /* device, advanced (may be NULL if dropped) */
    int64_t lost_capacity;
    lcb_beam_soa stage;                /* scratch, >= fresh + fell particles */
    uint8_t *stage_flags;
    int64_t stage_capacity;
    double *ro0, *ro1;                 /* beam density: this step's and the next
                                          (ro1 is cleared first: N*N doubles) */
    const lcb_fields *fields_k, *fields_k1;  /* previous and new plasma fields */
    int *err;
} lcb_beam_step_args;

/* One xi step of the beam with every count kept on the device: push layer
 * i-1 (fresh particles get their substep sizes first) followed by the
 * particles that fell from the previous push, compact in order: moved ->
 * drain, fell -> fell_out, lost -> lost; then deposit the layout layer into
 * ro0 and ro1, ro1 having been cleared by the push's grid (with three
 * rotating planes it last held the density that the plasma step of layer i
 * has just read).  The deposit only reads the source, so a caller may lay
 * out layer i+1 right after the plasma step of layer i.  Replaces the per-layer
 * body of PusherAndSolver3D.step_dt for a non-rigid beam,
 * lcode/push_solvers/push_solver.py:237-261 (layout_beam_layer,
 * move_beam_layer, create_next_layer, push_beam_layer). */
int lcb_beam_step(const lcb_beam_step_args *a, void *stream);

/* ---------------------------------------------------------------------
 * Capturable xi steps (batched and served simulations)
 * ------------------------------------------------------------------- */

/* Rigid Gaussian driver of the benchmark configurations evaluated on the
 * device for xi step first_layer + *counter (device int64):
 *   rho = amplitude exp(-r^2 / (2 sigma_r^2)) (1 + cos(sqrt(pi/2) xi)) / 2
 * for -xi_len <= xi <= 0, else 0, on the reference's meshgrid
 * (beam_calculator.py:158-170); rho_prev is the previous step's plane (zeros
 * for the first).  Replaces the per-step host call of the driver function in
 * RigidBeamCalculator.layout_beam_layer (beam_calculator.py:166-170) for this
 * family of drivers, so a captured graph needs no host input. */
int lcb_rigid_gaussian(int grid_steps, double h, double xi_step, double amplitude,
                       double sigma_r, double xi_len, int64_t first_layer,
                       const int64_t *counter, double *rho_full, double *rho_prev,
                       void *stream);

/* history[*counter] = plane[N/2][N/2] (the on-axis value), then *counter += 1.
 * The device-side form of the per-step on-axis Ez record
 * (push_solver.py:272-278). */
int lcb_record_axis(const double *plane, int grid_steps, int64_t *counter,
                    double *history, int64_t capacity, void *stream);

/* ---------------------------------------------------------------------
 * Declustering noise filter of the plasma electrons
 * (lcode/plasma3d/noise_filter.py:82-239; applied after the last move of an
 * xi step, lcode/plasma3d/solver.py:68-72).  n is the electrons' lattice
 * side; every array is n x n FP64, C order.
 * ------------------------------------------------------------------- */

/* dx_inhom, dy_inhom = the mean over the two lattice directions of the
 * offsets' inhomogeneity (a point minus the mean of its neighbours,
 * one-sided second differences at the ends, 0 where a stencil offset is
 * exactly 0): noise_filter.py:52-73, 123-124. */
int lcb_declustering_inhomogeneity(int n, const double *x_offt, const double *y_offt,
                                   double *dx_inhom, double *dy_inhom, void *stream);

typedef struct lcb_declustering_args {
    int n;
    double xi_step;
    double force;                      /* declustering-force */
    double damping;                    /* damping-declustering */
    double limit;                      /* declustering-limit */
    const double *dx_inhom, *dy_inhom;         /* lcb_declustering_inhomogeneity */
    const double *dx_average, *dy_average;     /* their Gaussian averages */
    const double *dx_chaotic_prev, *dy_chaotic_prev;  /* previous xi step's */
    double *px, *py;                   /* updated in place */
    double *dx_chaotic, *dy_chaotic;   /* written (not the previous arrays) */
} lcb_declustering_args;

/* Chaotic displacement = inhomogeneity - average; limiter 1 - d^2/limit^2
 * (0 beyond limit); restoring force -force * chaotic * limiter; momentum
 * kicks to each point and its lattice neighbours and damping of the change
 * of the chaotic displacement (noise_filter.py:164-232). */
int lcb_declustering_apply(const lcb_declustering_args *a, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* LCB_H */
