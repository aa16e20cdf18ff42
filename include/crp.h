/* crp.h — C ABI of the B200 implementation of CUDA-RP's simulation path:
 * staggered-grid FDTD of the bubbly mixture (velocity, split-field pressure,
 * mixture density, PML), per-bubble Rayleigh–Plesset integration, and the
 * two-way bubble/grid coupling with its Picard sub-loop.
 *
 * Plain C types only.  Every function returns a crp_status; nothing exits the
 * process or throws across this boundary.  A crp_sim owns all of its device
 * memory and its CUDA stream; host buffers passed in are owned by the caller.
 * One crp_sim per host thread at a time (handles are independent of each
 * other; there is no process-global state).  A crp_sim lives on the device that
 * was current at crp_create; its entry points make that device current while
 * they run and restore the caller's device, so any host thread may drive it.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   crp_config / crp_config_parse_file  <- Boost program_options keys and
 *                                           config-file parsing, src/bubbles.cpp:61-195
 *   crp_create                          <- initialize_variables + initialize_CUDA_variables
 *                                           + the init kernels, src/bubble_CUDA.cu:93-188,
 *                                           479-521, 1231-1520
 *   crp_step                            <- one pass of the main loop of solve_bubbles,
 *                                           src/bubble_CUDA.cu:203-285
 *   crp_read_field / crp_read_bubbles   <- the device-to-host copies before a save,
 *                                           src/bubble_CUDA.cu:360-392
 *   crp_write_rawdata                   <- save_ascii, src/output_styles.cpp:139-341
 *   crp_destroy                         <- destroy_CUDA_variables, src/bubble_CUDA.cu:1523-1623
 *   solve_bubbles (inc/bubble_CUDA.h:235) as a whole is crp_create + crp_step
 *   loop + crp_read_* + crp_destroy, driven by the `bubbles` program.
 */
#ifndef CRP_H_
#define CRP_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum crp_status {
  CRP_OK = 0,
  CRP_ERR_INVALID = 1,      /* bad argument or configuration value */
  CRP_ERR_UNSUPPORTED = 2,  /* configuration outside what this library implements */
  CRP_ERR_CUDA = 3,         /* a CUDA runtime call failed; see crp_last_error */
  CRP_ERR_ALLOC = 4,        /* device or host allocation failed */
  CRP_ERR_RP_STEPS = 5,     /* a bubble exceeded the Rayleigh–Plesset sub-step cap */
  CRP_ERR_PICARD = 6,       /* the Picard sub-loop exceeded its iteration cap */
  CRP_ERR_NONFINITE = 7,    /* a NaN/Inf was found in the state */
  CRP_ERR_IO = 8,           /* file could not be read or written */
  CRP_ERR_PARSE = 9,        /* configuration file syntax or value error */
  CRP_ERR_NO_DEVICE = 10,   /* no usable CUDA device */
  CRP_ERR_TOO_LARGE = 11    /* input larger than a fixed-size buffer of this library */
} crp_status;

/* Arithmetic of the grid fields. */
typedef enum crp_precision {
  CRP_PREC_FP64 = 0,   /* all state and arithmetic in FP64 (the reference's precision) */
  CRP_PREC_MIXED = 1   /* velocity and pressure stored as an FP32 value plus an FP32
                          compensation term (FP64 arithmetic); void fraction stored in
                          FP32 (FP64 sums); bubble thermal model in FP32 while
                          |R/R0 - 1| <= 1e-3, FP64 otherwise; radius update FP64 */
} crp_precision;

/* Every key of the reference configuration (src/bubbles.cpp:76-132) plus the
 * extension keys of the [ext] section.  crp_config_defaults fills the
 * reference's defaults (zero where the reference has none). */
typedef struct crp_config {
  /* [grid] */
  int32_t grid_x, grid_y;            /* cells */
  double grid_lx, grid_ly;           /* m */
  /* [pml] */
  int32_t pml_x0, pml_x1, pml_y0, pml_y1;
  int32_t pml_grid_number;
  double pml_sigma;
  int32_t pml_order;
  /* [simulation] */
  double sim_cfl;
  double sim_dt0;
  int32_t sim_n_step_max;
  double sim_t_step_max;
  int32_t sim_save_interval;
  int32_t sim_order;                 /* FDTD order (2 is the only order the kernels use) */
  int32_t sim_smooth_delta_band;
  /* [transducer] */
  double tr_amp, tr_freq, tr_focal_dist;
  int32_t tr_pid, tr_pid_start_step;
  double tr_init_control;
  int32_t tr_pid_iterate;
  double tr_box_size;
  int32_t tr_cylindrical;
  int32_t tr_on_wave, tr_off_wave;
  int32_t tr_plane_v, tr_plane_p;    /* keys transducer.transducer_v / transducer_p */
  int32_t tr_focused_v, tr_focused_p;
  /* [bubbles] */
  int32_t bub_enable;
  double bub_fg0, bub_R0, bub_P0, bub_T0, bub_gamma;
  double bub_sigma, bub_mu, bub_rho, bub_K0;
  /* [debug] (also selects which rawdata files are written) */
  int32_t dbg_display;
  int32_t dbg_fg, dbg_T, dbg_p, dbg_v, dbg_bubbles;
  /* generic options that may also appear in the file */
  int32_t opt_ascii, opt_sph;
  /* [ext] — extensions, all off by default so reference configs behave as before */
  double ext_rho_inf;        /* liquid density, default 1000 (hard-coded in the reference) */
  double ext_c_inf;          /* sound speed, default 1500 (hard-coded in the reference) */
  double ext_p_inf;          /* mixture reference pressure for the Picard residual, default 1e5 */
  int32_t ext_source_row;    /* 0: source on the y=0 ghost row only without a y0 PML (reference);
                                j>0: source forced on row j (p0 for *_p sources, vy for *_v) */
  double ext_ramp_cycles;    /* cosine ramp-up/down length of each burst in cycles (0 = off) */
  int32_t ext_precision;     /* crp_precision */
  int32_t ext_picard_cap;    /* Picard iteration cap per step (reference: none), default 1000 */
  int32_t ext_rp_step_cap;   /* RP sub-step cap per bubble per call, default 1000000 */
  int32_t ext_bubble_count;  /* >0: seed this many bubbles instead of the per-cell lattice */
  uint64_t ext_bubble_seed;
  double ext_r0_sigma_ln;    /* lognormal sigma of seeded R0 (median bubbles.R0) */
  int32_t ext_cloud_shape;   /* 0 cylinder (r <= cloud_r, |z - focus| <= cloud_h/2), 1 sphere, 2 gaussian */
  double ext_cloud_r, ext_cloud_h;
  double ext_n_b;            /* weight n_B of each seeded bubble, default 1 */
  double ext_picard_tol;     /* Picard residual threshold, max|dp0|/P_inf; 0 selects the reference's
                                1e-7 (FP64) or 1e-5 (mixed: FP32 storage has a higher noise floor) */
  int32_t ext_graphs;        /* 1: steps after the first run as CUDA graphs with the Picard loop
                                decided on the device (one read-back per crp_step call); 0 (default):
                                every step driven from the host.  Graphs save about 10 us per step on
                                small grids; on 1024 x 2048 and with many concurrent simulations the
                                host-driven steps measured faster */
  int32_t ext_elements;      /* >0: the pressure source's aperture is split into this many elements
                                (equal bands of distance from the focus axis; rings about the axis
                                in the axisymmetric geometry), each with an amplitude factor and a
                                phase offset (crp_set_source_elements; default 1 and 0, which leave
                                the source unchanged) */
  int32_t ext_rp_scheme;     /* crp_rp_scheme: integrator of the bubble radius (default: the
                                reference's three-level variable step) */
  double ext_rp_tol;         /* CRP_RP_RK45: relative error tolerance per step (0: 1e-6) */
  /* 3-D Cartesian grid (no counterpart in the reference, which is 2-D): with
     ext_grid_z > 0 the grid is grid_x x grid_y x ext_grid_z cells of
     lx/x x ly/y x lz/z, planar (transducer.cylindrical off), with a PML on all
     six faces (pml.x0..y1 and ext.pml_z0/z1 must all be on), bubbles in 3-D,
     and the hemispherical array below as its source. */
  int32_t ext_grid_z;
  double ext_grid_lz;
  int32_t ext_pml_z0, ext_pml_z1;
  int32_t ext_array_elements;  /* elements of the hemispherical bowl (3-D source) */
  double ext_array_radius;     /* [m] bowl radius about the grid's centre; opens towards +z */
  double ext_array_focus_dx;   /* [m] focus offset from the centre along x (the bowl's phases focus there) */
  uint64_t ext_array_seed;     /* seed of the phases when ext_array_phases = 1 */
  int32_t ext_array_phases;    /* 0: focusing phases omega |x_e - focus| / c; 1: seeded, uniform in [0, 2 pi) */
  int32_t ext_rp_reuse;        /* 1 (default): a Picard iteration after a step's first re-solves only
                                  the bubbles whose gathered liquid pressure changed (bit pattern) since
                                  the last solve and keeps the others' results, which are bit for bit
                                  what a re-solve returns; 0: every bubble every iteration, as the
                                  reference (src/bubble_CUDA.cu:239-276) */
} crp_config;

/* Integrator of the bubble radius and gas pressure over one mixture step. */
typedef enum crp_rp_scheme {
  CRP_RP_REF = 0,   /* the reference's three-level variable-step scheme with its
                       semi-implicit gas-pressure update (inc/bubble_CUDA_kernel.cuh:227-260,
                       326-340, 506-539): step limits 1.01 dt, dt0, 1 % radius change,
                       0.1 R / sqrt|R''| */
  CRP_RP_RK45 = 1   /* Dormand-Prince 5(4) with embedded error control on (R, R', PG),
                       the gas pressure from the continuous form of the same thermal
                       model; each mixture step ends exactly on the step's end.  In the
                       mixed path the thermal model runs in FP32 only near equilibrium
                       (|R / R0 - 1| <= 1e-3); in the stiff phase (R / R0 < 0.3 or
                       |R'| > 0.1 c_inf) and elsewhere all of it is FP64 */
} crp_rp_scheme;

/* Dense host layouts of the readable fields, in the reference's index order:
 * row-major, x fastest, widths and heights from crp_dims. */
typedef enum crp_field {
  CRP_FIELD_P0 = 0,    /* i1m x j1m, pressure p0 = px + py with boundary values */
  CRP_FIELD_PX = 1,    /* i1m x j1m, split pressure components */
  CRP_FIELD_PY = 2,
  CRP_FIELD_PNX = 3,   /* i1m x j1m, previous-step split pressure */
  CRP_FIELD_PNY = 4,
  CRP_FIELD_VX = 5,    /* i2n x j2m */
  CRP_FIELD_VY = 6,    /* i2m x j2n */
  CRP_FIELD_FG = 7,    /* i2m x j2m, void fraction */
  CRP_FIELD_FGN = 8,   /* i2m x j2m, previous step */
  CRP_FIELD_FGM = 9,   /* i2m x j2m, two steps back */
  CRP_FIELD_RHO_M = 10, /* i1m x j1m, mixture density as the next velocity update sees it */
  CRP_FIELD_T = 11,     /* i2m x j2m, mixture temperature rise over T_inf (debug.T = 1 only) */
  /* 3-D grids: cell fields are (Z+2) planes of (Y+2) x (X+2), x fastest; vx is
     (Z+2) x (Y+2) x (X+3), vy (Z+2) x (Y+3) x (X+2), vz (Z+3) x (Y+2) x (X+2). */
  CRP_FIELD_VZ = 12,    /* 3-D only */
  CRP_FIELD_PZ = 13     /* 3-D only: the z split component of the pressure */
} crp_field;

typedef enum crp_bubble_field {
  CRP_BUB_X = 0, CRP_BUB_Y = 1, CRP_BUB_R_T = 2, CRP_BUB_R_P = 3, CRP_BUB_R_N = 4,
  CRP_BUB_D1R = 5, CRP_BUB_PG = 6, CRP_BUB_PL_P = 7, CRP_BUB_PL_N = 8, CRP_BUB_PL_M = 9,
  CRP_BUB_DT = 10, CRP_BUB_RE = 11, CRP_BUB_Q_B = 12, CRP_BUB_N_B = 13, CRP_BUB_R0 = 14,
  CRP_BUB_VX = 15, CRP_BUB_VY = 16,
  CRP_BUB_IBM_X = 17, CRP_BUB_IBM_Y = 18, CRP_BUB_IBN_X = 19, CRP_BUB_IBN_Y = 20,
  CRP_BUB_SUBSTEPS = 21, /* RP sub-steps of the bubble's last radius solve */
  CRP_BUB_Z = 22, CRP_BUB_VZ = 23, CRP_BUB_IBM_Z = 24, CRP_BUB_IBN_Z = 25  /* 3-D only */
} crp_bubble_field;

typedef struct crp_dims {
  int32_t i1m, j1m, i2m, j2m, i2n, j2n;
  int32_t num_bubbles;
  double dx, dy, dt;
} crp_dims;

/* crp_dims of a 3-D grid: cells per axis with ghost layers (X+2, Y+2, Z+2),
 * the bubble count, the spacings, the step, and the cells of the bowl source. */
typedef struct crp_dims3 {
  int32_t nx, ny, nz;
  int32_t num_bubbles;
  double dx, dy, dz, dt;
  int32_t source_cells;
} crp_dims3;

typedef struct crp_stats {
  int64_t steps;               /* mixture steps taken */
  double time;                 /* simulated time (compensated sum) */
  int64_t picard_total;        /* Picard sub-iterations summed over all steps */
  int32_t picard_last;         /* sub-iterations of the last step */
  int32_t picard_max;
  int64_t rp_substeps_max;     /* largest RP sub-step count of one bubble in one call */
  double residual_last;        /* last max|dp0| / P_inf */
  int64_t kernel_launches;     /* CUDA kernels launched by this handle */
  int64_t fdtd_launches, rp_launches, couple_launches;
  /* Device time per kernel class, accumulated while profiling is on
   * (crp_set_profiling): the fused FDTD kernel, the RP kernel, the coupling
   * gather + pressure kernel, and everything else (ghosts, motion, binning). */
  double ms_fdtd, ms_rp, ms_couple, ms_other;
  /* Steps whose Picard loop the mixed path ended on stagnation: the residual
   * stopped falling (less than halved by an iteration, from the third on)
   * while below CRP_MIXED_STALL_RESIDUAL.  Always 0 in the FP64 path. */
  int64_t picard_stalls;
  /* Bubble radius solves that a Picard iteration kept from the previous one
   * (ext.rp_reuse: the bubble's gathered liquid pressure was unchanged),
   * summed over all steps.  The oracle re-solves every bubble (always 0). */
  int64_t rp_reused;
} crp_stats;

/* Residual (max |dp0| / P_inf) below which the mixed path accepts a stagnating
 * Picard loop.  FP32 storage of the void fraction puts a floor of about 1e-6
 * under the residual, and a loop can settle into a short cycle above it. */
#define CRP_MIXED_STALL_RESIDUAL 1.0e-3

/* Explicit bubble population: n bubbles with position (x, y), equilibrium
 * radius R0 and weight n_B.  Replaces the per-cell lattice of the reference
 * (src/bubble_CUDA.cu:811-839) when passed to crp_create. */
typedef struct crp_bubbles_in {
  int32_t n;
  const double* x;
  const double* y;
  const double* r0;
  const double* n_b;
  const double* z;  /* 3-D grids only (NULL otherwise) */
} crp_bubbles_in;

typedef struct crp_sim crp_sim;

/* Reference defaults for every key (src/bubbles.cpp:97-132); [ext] defaults. */
crp_status crp_config_defaults(crp_config* cfg);

/* Parse a reference configuration file (INI: `[section]`, `key = value`, `#`
 * comments; unknown keys ignored as the reference does) on top of *cfg. */
crp_status crp_config_parse_file(const char* path, crp_config* cfg, char* err, size_t err_len);
crp_status crp_config_parse_string(const char* text, crp_config* cfg, char* err, size_t err_len);

/* Seeded bubble population of the [ext] keys (ext_bubble_count > 0): positions
 * uniform in the cloud around the focal point, R0 lognormal with median
 * bubbles.R0 and sigma ext_r0_sigma_ln, weight ext_n_b.  Host only; fills
 * caller arrays of length ext_bubble_count from a Philox-4x32-10 stream keyed
 * by ext_bubble_seed. */
crp_status crp_seed_bubbles(const crp_config* cfg, double* x, double* y, double* r0, double* n_b);

/* The same for a 3-D grid (ext_grid_z > 0): positions around the bowl's focus
 * (the grid's centre plus ext_array_focus_dx along x) in a cylinder along z
 * (radius cloud_r about the focus line, length cloud_h), a ball of radius
 * cloud_r, or a Gaussian cloud of standard deviation cloud_r per axis. */
crp_status crp_seed_bubbles3(const crp_config* cfg, double* x, double* y, double* z, double* r0, double* n_b);

/* Build the simulation on the current CUDA device.  bubbles may be NULL (the
 * reference's lattice seeding, or ext seeding when ext_bubble_count > 0).
 * stream may be NULL (a stream is created) or a cudaStream_t to run on. */
crp_status crp_create(const crp_config* cfg, const crp_bubbles_in* bubbles, void* stream, crp_sim** out);

/* Advance n mixture time steps.  Blocks until they are done.  Without bubbles
 * (and without the temperature branch or profiling) the steps after the first
 * are queued back to back and their state is checked once, after the last: a
 * non-finite pressure is then reported (CRP_ERR_NONFINITE) at the end of the
 * call, with the step count including every queued step. */
crp_status crp_step(crp_sim* sim, int32_t n);

crp_status crp_get_dims(const crp_sim* sim, crp_dims* dims);
/* Dimensions of a 3-D simulation (CRP_ERR_INVALID for a 2-D one). */
crp_status crp_get_dims3(const crp_sim* sim, crp_dims3* dims);
crp_status crp_get_stats(const crp_sim* sim, crp_stats* stats);

/* Copy one field into a dense host array (layout above). */
crp_status crp_read_field(crp_sim* sim, crp_field field, double* host);

/* Copy one per-bubble quantity into host[num_bubbles]. */
crp_status crp_read_bubbles(crp_sim* sim, crp_bubble_field what, double* host);

/* Write the reference's plain-text rawdata files for the current step into
 * dir (created if missing, never cleared): fg/p0/vx/vy_step_%05d.txt and
 * bubble_radii_/bubble_PG_%05d.txt as selected by the debug keys. */
crp_status crp_write_rawdata(crp_sim* sim, const char* dir);

/* Write the reference's binary SPH files for the current step into dir
 * (save_sph, src/output_styles.cpp:36-137; record layout of SphData::SaveSph,
 * src/SphDataType.cpp:142-192): fg/p0/T_step_%05d.sph as selected by the
 * debug keys; updates the same min/max as crp_write_rawdata. */
crp_status crp_write_sph(crp_sim* sim, const char* dir);

/* Running min/max of the f_g and p0 values written by crp_write_rawdata so far
 * (what save_ascii accumulates for *_minmax.txt, src/output_styles.cpp:200-224). */
crp_status crp_minmax(const crp_sim* sim, double* fg_min, double* fg_max, double* p0_min, double* p0_max);
/* The same for the T values written (T_minmax.txt, src/bubbles.cpp:273-279). */
crp_status crp_minmax_T(const crp_sim* sim, double* T_min, double* T_max);

/* Record CUDA events around every kernel launch (on the simulation's stream)
 * and accumulate device time per kernel class into crp_stats. */
crp_status crp_set_profiling(crp_sim* sim, int32_t enable);

/* Device stream the simulation runs on (a cudaStream_t). */
void* crp_stream(crp_sim* sim);

/* Void fraction of a bubble population, computed without allocating anything.
 *
 * No counterpart in the reference, which only forms the void fraction inside a
 * simulation (calculate_void_fraction, src/bubble_CUDA.cu:1198-1218).  It is for
 * callers that may not allocate device memory when they need the result: loops
 * where cudaMalloc/cudaFree would synchronise the device, and programs whose
 * own pool owns the GPU's memory.
 *
 * Inputs are device arrays of n bubbles: x, y (m), r (radius, m), n_b (bubbles
 * per point).  Output f_g is a dense device array of (grid_y + 2) x (grid_x + 2)
 * doubles, row j at f_g + j * (grid_x + 2), i and j from 0: the same values and
 * summation order crp_create forms for its initial void fraction from x, y, R0
 * and n_B (smooth delta of band 2 only; other bands give CRP_ERR_UNSUPPORTED).
 * Kernels are queued on stream (a cudaStream_t, NULL for the default stream);
 * the call does not wait for them.
 *
 * Scratch space is one static device array of CRP_NOALLOC_SCRATCH_BYTES per
 * GPU, shared by all calls: calls whose kernels overlap on a GPU race on it and
 * must be ordered (one stream, or events).  crp_void_fraction_noalloc_scratch
 * gives the bytes a call needs; a call that needs more returns
 * CRP_ERR_TOO_LARGE and queues nothing (SIZE_MAX from the size query means the
 * grid alone is too large).  The first call on each device looks up the array's
 * device address (cudaGetSymbolAddress, with that device current): make it
 * before any stream capture.  The address is cached for the process: after
 * cudaDeviceReset on a device, do not call this entry point there again.  A
 * failing call's message is crp_last_error(NULL) on the calling thread. */
#define CRP_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)
size_t crp_void_fraction_noalloc_scratch(int32_t grid_x, int32_t grid_y, int32_t n);
crp_status crp_void_fraction_noalloc(const crp_config* cfg, int32_t n, const double* x, const double* y,
                                     const double* r, const double* n_b, double* f_g, void* stream);

/* Focal tracker and PID focus control (src/bubble_CUDA.cu:123-153, 310-352;
 * inc/bubble_CUDA_kernel.cuh:117-129, 1132-1184).  They run with the
 * temperature branch (debug.T = 1, or transducer.pid = 1, which turns the
 * branch on).  After every step the focal depth is tracked from the step's
 * temperature increment dT: the reference's reduction functors are missing
 * from its source tree, so the depth is defined here as the mean of the
 * cell-centre depths (j - 1/2) dy over the interior cells weighted by
 * max(dT - max(dT) / 2, 0) (0 while max(dT) <= 1e-30 K: increments of
 * rounding size define no focus).  It passes through the
 * reference's fourth-order Butterworth low-pass.  With transducer.pid, after
 * step pid_start_step the PID of focal_PID moves the focus the source aims at
 * (clamped to [focal depth, LY]).
 * crp_focus_history copies the tracked depths (which = 0, the reference's
 * focalpoint[].y, starting with 0) or the control depths (which = 1, its
 * control[].y, starting with the initial focus) and returns how many there are
 * (at most capacity are copied).  crp_get/set_focus_state carry the control
 * point, the PID accumulators and the filter state from one simulation to the
 * next (transducer.pid_iterate passes); set it before the first step. */
typedef struct crp_focus_state {
  double control_x, control_y;        /* focus the source aims at (focal_point_c) */
  double err_total_x, err_total_y;    /* PID accumulated error */
  double d_err_x, d_err_y;            /* PID last derivative term */
  double filter_in[5], filter_out[5]; /* Butterworth filter history */
} crp_focus_state;
int64_t crp_focus_history(const crp_sim* sim, int32_t which, double* out, int64_t capacity);
crp_status crp_get_focus_state(const crp_sim* sim, crp_focus_state* state);
crp_status crp_set_focus_state(crp_sim* sim, const crp_focus_state* state);

/* Main loop with saves (src/bubble_CUDA.cu:203-438): step while
 * (n_steps != 0 && steps < n_steps) || (t_max != 0 && time < t_max); after
 * every save_interval-th step write rawdata to dir (if not NULL) and call
 * progress (if not NULL).  With n_steps = t_max = 0 the limits come from cfg
 * (sim_n_step_max, sim_t_step_max); cfg may be NULL otherwise.  Steps already
 * taken count towards the limits. */
typedef struct crp_output_plan {
  int64_t n_steps;
  double t_max;
  int32_t save_interval;
  const char* dir;
  int32_t sph;  /* nonzero: write SPH files instead of text rawdata (the reference's -s) */
  void (*progress)(int64_t step, double time, void* user);
  void* user;
} crp_output_plan;
crp_status crp_run(crp_sim* sim, const crp_output_plan* plan, const crp_config* cfg);

/* State snapshots (no reference counterpart: the reference keeps no
 * checkpoints).  crp_save_state copies every device array of the simulation
 * (fields, void-fraction ring, bubbles, bins, source elements, device scalars:
 * crp_state_bytes bytes) into a device blob on the simulation's GPU, and keeps
 * the host-side step state (time, buffer phases, statistics, coupling boxes,
 * focal history) beside it.  *state == NULL allocates a snapshot; an existing
 * one, taken from this simulation, is overwritten.  crp_load_state puts a
 * snapshot back into the simulation it was taken from (or one created from the
 * same configuration and bubbles on the same GPU): the run then continues bit
 * for bit as it did after the save.  The counters of work done (launch counts,
 * profiling times) are not rewound.  Both calls wait for the copy. */
typedef struct crp_state crp_state;
size_t crp_state_bytes(const crp_sim* sim);
crp_status crp_save_state(crp_sim* sim, crp_state** state);
crp_status crp_load_state(crp_sim* sim, const crp_state* state);
void crp_state_free(crp_state* state);

/* Launch shapes (no reference counterpart), chosen by crp_batch_tune or set
 * directly; results are bit for bit the same under every setting.
 * fdtd_rows: rows per chunk of the 2-D FDTD strip kernel, 4, 8 (default) or 16
 * (the 3-D path accepts the value and ignores it).  rp_blocks: blocks of the
 * persistent radius kernel (0, the default: one lane per bubble up to the
 * occupancy limit, rp_blocks_max, which crp_get_tuning reports; larger
 * values are clamped to it). */
typedef struct crp_tuning {
  int32_t fdtd_rows;
  int32_t rp_blocks;
  int32_t rp_blocks_max; /* output of crp_get_tuning; ignored by crp_set_tuning */
} crp_tuning;
crp_status crp_get_tuning(const crp_sim* sim, crp_tuning* tuning);
crp_status crp_set_tuning(crp_sim* sim, const crp_tuning* tuning);

/* Batched sweep: count independent simulations (cfgs[k], bubbles[k] or NULL /
 * n = 0 for the configuration's own seeding), each with its own stream, run
 * concurrently.  Replaces re-running `bubbles` over a list of configuration
 * files (scripts/executor.sh:28-47).  crp_batch_run advances simulation k by
 * steps[k] mixture steps, largest cells x steps first; per_sim (may be NULL)
 * receives each status and the first non-OK status in index order is
 * returned.  threads > 0: a pool of that many host threads, each driving its
 * simulations' steps and Picard loops; threads = 0: the batch's tuning
 * (crp_batch_set_tuning / crp_batch_tune; by default a pool of up to 32
 * threads).  The simulations are crp_sim handles (crp_batch_sim) for reading
 * fields, stats and rawdata. */
typedef struct crp_batch crp_batch;
crp_status crp_batch_create(int32_t count, const crp_config* cfgs, const crp_bubbles_in* bubbles, crp_batch** out);
crp_status crp_batch_run(crp_batch* batch, const int32_t* steps, int32_t threads, crp_status* per_sim);
int32_t crp_batch_count(const crp_batch* batch);
crp_sim* crp_batch_sim(crp_batch* batch, int32_t k);
void crp_batch_destroy(crp_batch* batch);

/* How crp_batch_run drives a batch (threads = 0).
 * CRP_BATCH_THREADS: host threads, each running its simulations' steps with
 * the host-driven Picard loop.  CRP_BATCH_GRAPHS: one host thread queues every
 * simulation's steps as CUDA graphs with the Picard loop decided on the device
 * (ext.graphs) on each simulation's stream, then waits for all; simulations
 * that cannot run as graphs (3-D grids, no bubbles, the first step, debug.T)
 * run those steps on a host thread meanwhile.  fdtd_rows and
 * rp_bubbles_per_lane are applied to every simulation: the radius kernel gets
 * ceil(n_bubbles / (128 rp_bubbles_per_lane)) blocks (at most its occupancy
 * limit; 1 is the default grid).  ms_per_step: the wall-clock time per batch
 * step crp_batch_tune measured for this setting (0 when not measured). */
typedef enum crp_batch_mode { CRP_BATCH_THREADS = 0, CRP_BATCH_GRAPHS = 1 } crp_batch_mode;
typedef struct crp_batch_tuning {
  int32_t mode;
  int32_t threads;              /* CRP_BATCH_THREADS: pool size (0: min(count, 32)) */
  int32_t blocking;             /* CRP_BATCH_THREADS: 1 = the host threads block on events inside a
                                   step instead of spinning (for more threads than host cores) */
  int32_t fdtd_rows;            /* 4, 8 or 16 */
  int32_t rp_bubbles_per_lane;  /* >= 1 */
  double ms_per_step;
} crp_batch_tuning;
crp_status crp_batch_get_tuning(const crp_batch* batch, crp_batch_tuning* tuning);
crp_status crp_batch_set_tuning(crp_batch* batch, const crp_batch_tuning* tuning);
/* The autotuner: times trial_steps batch steps (after 2 untimed ones) under
 * each candidate setting, searched one parameter at a time from the defaults
 * (mode; threads min(count, 32), count or 16, spinning or blocking; fdtd_rows
 * 4, 8, 16; rp_bubbles_per_lane 1, 4, 16), restoring every simulation's state
 * (crp_save_state / crp_load_state) after each trial, and applies the
 * fastest.  The batch's
 * simulations end where they started.  n_tried (may be NULL) receives the
 * number of settings timed; tried (may be NULL, capacity entries) their
 * timings. */
crp_status crp_batch_tune(crp_batch* batch, int32_t trial_steps, crp_batch_tuning* best,
                          crp_batch_tuning* tried, int32_t capacity, int32_t* n_tried);

/* Phased-array source and its adjoint.  Neither has a counterpart in the
 * reference (its source is one focused aperture, src/bubble_CUDA.cu:542-551,
 * inc/bubble_CUDA_kernel.cuh:883-926); they extend the same source.
 *
 * crp_set_source_elements: amplitude factors amp[e] and phase offsets phase[e]
 * (radians, added to the burst's sine) of the cfg.ext_elements elements; n must
 * equal cfg.ext_elements.  Element e covers the source cells whose distance from
 * the focus axis is in [e, e+1) r_ap / n, r_ap the largest such distance among
 * the source's cells.
 *
 * crp_adjoint: advances the simulation obj->steps mixture steps (as crp_step)
 * and returns J = sum over those steps of dt * sum over the cells within
 * obj->focal_radius of the focus of w p0^2 (w the cell volume: 2 pi r dx dy in
 * the axisymmetric geometry, dx dy otherwise; source-row cells excluded), and
 * its gradient with respect to the elements' amplitudes and phases, the state
 * at the call held fixed.  The gradient comes from a hand-written discrete
 * adjoint of the FDTD/PML step run backwards over the recorded focal pressure
 * (the step is linear without bubbles, so no other forward state is needed).
 * Supported: bubbles off, pressure sources (plane or focused), any PML faces;
 * otherwise CRP_ERR_UNSUPPORTED (the temperature branch, when on, runs with the
 * forward steps; it does not act on the pressure).  grad_amp and
 * grad_phase receive cfg.ext_elements values each (either may be NULL).
 * On a 3-D grid (ext.grid_z > 0, bubbles off) the focus is the point the
 * bowl's phases aim at, w = dx dy dz (the bowl's source cells excluded), and
 * the parameters are the ext.array_elements elements' amplitude factors and
 * phases (crp_set_source_elements sets them; the phases are absolute there,
 * the focusing delays included).  The call's device workspace (the adjoint
 * fields and the focal record) stays allocated for the next call and is
 * released by crp_destroy. */
typedef struct crp_objective {
  int32_t steps;        /* mixture steps to run and differentiate over */
  double focal_radius;  /* [m] radius of the focal region around the source's focus */
} crp_objective;
crp_status crp_set_source_elements(crp_sim* sim, int32_t n, const double* amp, const double* phase);
crp_status crp_adjoint(crp_sim* sim, const crp_objective* obj, double* J, double* grad_amp, double* grad_phase);

/* Message of the handle's last failed call; with sim == NULL, of the calling
 * thread's last failed call that takes no handle (crp_void_fraction_noalloc). */
const char* crp_last_error(const crp_sim* sim);
const char* crp_status_string(crp_status s);
void crp_destroy(crp_sim* sim);

#ifdef __cplusplus
}
#endif
#endif /* CRP_H_ */
