/* CPU oracle for the CUDA-RP simulation path — TEST INFRASTRUCTURE ONLY.
 *
 * An FP64 host restatement of the reference's initialisers, kernels and main
 * loop (src/bubble_CUDA.cu, inc/bubble_CUDA_kernel.cuh, inc/complex.cuh,
 * inc/double_vector_math.cuh), used by the tests to check the CUDA path and by
 * bench.py as the timed CPU baseline.  The product never links or calls it.
 *
 * Parity pin: the initialisers and bubble-physics functions are compared
 * bit-for-bit with the reference's own code compiled on the host
 * (oracle/_ref/libcrp_ref.so), and whole runs are compared with the reference's
 * own kernels run on the GPU (golden fixtures under tests/golden/).
 *
 * Layout: the reference's dense arrays, row-major with x fastest, widths
 * i1m/i2m/i2n and heights j1m/j2m/j2n (crp_dims), indexed by the reference's
 * logical (i, j) ranges.
 */
#ifndef CRP_ORACLE_H_
#define CRP_ORACLE_H_
#include "crp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct crpo_sim crpo_sim;

/* Same meaning as crp_create; bubbles == NULL selects the reference lattice. */
crp_status crpo_create(const crp_config* cfg, const crp_bubbles_in* bubbles, crpo_sim** out);
crp_status crpo_step(crpo_sim* sim, int32_t n);
/* Same meaning as crp_set_source_elements. */
crp_status crpo_set_source_elements(crpo_sim* sim, int32_t n, const double* amp, const double* phase);
crp_status crpo_get_dims(const crpo_sim* sim, crp_dims* dims);
crp_status crpo_get_stats(const crpo_sim* sim, crp_stats* stats);
crp_status crpo_read_field(crpo_sim* sim, crp_field field, double* host);
int64_t crpo_focus_history(const crpo_sim* sim, int32_t which, double* out, int64_t capacity);
crp_status crpo_read_bubbles(crpo_sim* sim, crp_bubble_field what, double* host);
/* Number of OpenMP threads the oracle uses (0 = library default). */
void crpo_set_threads(int32_t n);
int32_t crpo_get_threads(void);
void crpo_destroy(crpo_sim* sim);

/* Workload inputs built without the product library (oracle/workload.cpp):
 * the reference's configuration defaults and config-file grammar, and the
 * seeded [ext] bubble population; same meaning as crp_config_defaults,
 * crp_config_parse_file and crp_seed_bubbles. */
crp_status crpo_config_defaults(crp_config* cfg);
crp_status crpo_config_parse_file(const char* path, crp_config* cfg, char* err, size_t err_len);
crp_status crpo_seed_bubbles(const crp_config* cfg, double* x, double* y, double* r0, double* n_b);
crp_status crpo_seed_bubbles3(const crp_config* cfg, double* x, double* y, double* z, double* r0, double* n_b);
/* One Philox-4x32-10 block (key seed, counter, stream word), as the seeding draws. */
void crpo_philox_block(uint64_t seed, uint64_t counter, uint32_t stream, uint32_t out[4]);

/* The 3-D Cartesian extension (ext_grid_z > 0; oracle/oracle3d.inc states its
 * discretisation).  Dense layouts as crp_read_field documents for 3-D grids. */
typedef struct crpo3_sim crpo3_sim;
crp_status crpo3_create(const crp_config* cfg, const crp_bubbles_in* bubbles, crpo3_sim** out);
crp_status crpo3_step(crpo3_sim* sim, int32_t n);
crp_status crpo3_set_source_elements(crpo3_sim* sim, int32_t n, const double* amp, const double* phase);
crp_status crpo3_get_stats(const crpo3_sim* sim, crp_stats* stats);
int32_t crpo3_num_bubbles(const crpo3_sim* sim);
int32_t crpo3_num_source_cells(const crpo3_sim* sim);
crp_status crpo3_read_field(crpo3_sim* sim, crp_field field, double* host);
crp_status crpo3_read_bubbles(crpo3_sim* sim, crp_bubble_field what, double* host);
void crpo3_destroy(crpo3_sim* sim);

/* Bubble physics on single inputs, for comparison with the reference's
 * functions (inc/bubble_CUDA_kernel.cuh:227-340).  bp = (R0, PG0, PL0, T0, gam,
 * sig, mu, rho, K0, dt0). */
void crpo_rp_step(const double* bp, double* state /* Rt,Rp,Rn,d1R,dt,remain */, double PG, double PL);
double crpo_omega_n(const double* bp, double PG, double R, double* alpha /* re, im */);
void crpo_upsilon_lp(double are, double aim, double gam, double R, double* out /* U re,im, Lp re,im */);
double crpo_solve_pg(const double* bp, double PGn, double Rp, double Rn, double omega_N, double dt,
                     double lp_re, double lp_im);
/* One bubble from rest at R_init advanced nsteps mixture steps (length dt_mix)
 * in a liquid held at P0 + dpl, with the sub-stepping and thermal gas model of
 * the radius kernel.  R_out/PG_out get R_t and PG after each step.  Returns the
 * total number of sub-steps (-1 if it exceeded 1e8). */
int64_t crpo_bubble_history(const double* bp, double R_init, double dt_mix, double dpl, int32_t nsteps, double* R_out,
                            double* PG_out);
/* One bubble from rest at R_init driven by a liquid pressure P0 + p_amp
 * sin(omega_drive t) for nsteps mixture steps of dt_mix, with the reference's
 * sub-step scheme (scheme 0, its step limits divided by param >= 1) or the
 * rk45 scheme (scheme 1, rtol = param).  R_out/PG_out get R_t and PG after each
 * step.  Returns the total number of steps (-1 on failure). */
int64_t crpo_bubble_drive(const double* bp, double R_init, double dt_mix, double p_amp, double omega_drive,
                          int32_t nsteps, int32_t scheme, double param, double* R_out, double* PG_out);
/* Derived scalars in the order of crp_ref_host_scalars (oracle/ref_harness.inc). */
void crpo_host_scalars(const crp_config* cfg, double* out);
/* PML profiles and cylindrical metrics: mx[i1m], my[j1m], nx[i2n], ny[j2n], xu[i2n], rxp[i2m]. */
crp_status crpo_host_sigma(const crp_config* cfg, double* mx, double* my, double* nx, double* ny,
                           double* xu, double* rxp);

#ifdef __cplusplus
}
#endif
#endif
