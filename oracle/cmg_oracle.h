/*
 * cmg_oracle.h -- CPU oracle for the octree multigrid-preconditioned CG
 * pressure-Poisson solve of Cirrus-amg.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: a plain-C restatement of
 * the reference algorithm that the CUDA product is compared against.  It is
 * loaded only by the test-suite, by the smoke check and by the CPU-baseline
 * leg of the benchmark.  Nothing in the product links it or calls it.
 *
 * Each function cites the reference file:line it restates (paths relative
 * to the Cirrus-amg project root).
 *
 * Parity pin: the reference ships no golden vectors for this path
 * (tests/SolverTests.cu prints, it does not store).  The oracle is pinned by
 * (1) the reference's own known-answer tests restated in tests/ (analytic
 * Laplacian truncation error, -lap == div grad, Neumann/Dirichlet recovery,
 * divergence-free velocity after projection), and (2) the FP64 CSR assembly
 * of the same operator solved independently.  The reference's CUDA solver
 * cannot be run against it: on the adaptive sphere grid it stops on its own
 * device assertion (src/AMGSolver.cu:873), so it is not run at all.
 */
#ifndef CMG_ORACLE_H
#define CMG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* tile types (HATileInfo.h:10) and cell types (PoissonTile.h:7) */
#define OG_LEAF 1
#define OG_NONLEAF 2
#define OG_GHOST 4
#define OG_DIRICHLET 1
#define OG_INTERIOR 2
#define OG_NEUMANN 4

/* built-in refinement / cell-type cases */
#define OG_CASE_UNIFORM 0       /* TestGrids.cuh:33  */
#define OG_CASE_CENTER_POINT 1  /* TestGrids.cuh:43  */
#define OG_CASE_SPHERE_EMPTY 2  /* TestGrids.cuh:58  */
#define OG_CASE_SPHERE_SOLID 3  /* TestGrids.cuh:75  */
#define OG_CASE_STAR_EMPTY 4    /* TestGrids.cuh:95  */
#define OG_CASE_STAR_SOLID 5    /* TestGrids.cuh:118 */
#define OG_CASE_SHELL 6         /* sphere shell bands (adaptive sphere workload) */
#define OG_CASE_MULTI_SPHERE 7  /* several spheres, one refinement band */

typedef struct og_grid og_grid;

og_grid* og_grid_new(float h0, int num_levels);
void og_grid_free(og_grid* g);
int og_set_tile(og_grid* g, int level, int i, int j, int k, int type);
int og_rebuild(og_grid* g);
int og_refine_case(og_grid* g, int case_id, const double* params, int nparams);
typedef int (*og_target_fn)(void* user, int level, int i, int j, int k);
int og_refine_fn(og_grid* g, og_target_fn fn, void* user);
int og_num_tiles(const og_grid* g);
int og_max_level(const og_grid* g);
void og_get_tiles(const og_grid* g, int* level, int* ijk, uint8_t* type);
void og_get_tables(const og_grid* g, int* nbr, int* parent, int* child);

int og_alloc_channels(og_grid* g, int nch);
float* og_channel(og_grid* g, int ch);
uint8_t* og_cell_types(og_grid* g);
void og_set_leaf_cell_types_case(og_grid* g, int case_id, const double* params, int nparams);

void og_coarsen_types_and_coeffs(og_grid* g, int coeff_ch, float R);
void og_cutcell_sphere_coeffs(og_grid* g, int coeff_ch, float R, int nspheres, const float* spheres);
void og_prepare_system(og_grid* g, int coeff_ch, float R);

void og_full_neg_lap_leafs(og_grid* g, int x_ch, int coeff_ch, int ax_ch);
void og_gauss_seidel(og_grid* g, int iters, int order, int level, int x_ch, int coeff_ch, int rhs_ch, double omega);
void og_residual_restrict(og_grid* g, int level, int x_ch, int coeff_ch, int rhs_ch, float R_restrict);
void og_fas_save(og_grid* g, int level, int x_ch, int coeff_ch, int rhs_ch, int x0_ch);
void og_fas_prolong(og_grid* g, int level, int x_ch, int x0_ch, float P);
void og_fas_mu_cycle(og_grid* g, int mu, int x_ch, int rhs_ch, int x0_ch, int coeff_ch, int level_iters, int coarsest_iters, double omega, float R_restrict, float P);
/* AMGSolver::VCycle / muCycle (correction schemes for rhs f) and FASFCycle */
void og_vcycle(og_grid* g, int x_ch, int f_ch, int rhs_ch, int coeff_ch, int level_iters, int coarsest_iters, double omega, float R_restrict, float P);
void og_mu_cycle(og_grid* g, int repeat_times, int x_ch, int f_ch, int rhs_ch, int coeff_ch, int level_iters, int coarsest_iters, double omega,
                 float R_restrict, float P);
void og_fas_f_cycle(og_grid* g, int mu, int x_ch, int rhs_ch, int x0_ch, int coeff_ch, int level_iters, int coarsest_iters, double omega,
                    float R_restrict, float P);
double og_dot(og_grid* g, int a_ch, int b_ch);
int og_amg_solve(og_grid* g, int coeff_ch, double omega, int mu, float R_restrict, float P, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride, int pure_neumann, double* rel_res);

void og_face_velocity_fourier(og_grid* g, int u_ch, int nmodes, const double* k, const double* amp, const double* phase);
void og_divergence(og_grid* g, int u_ch, int coeff_ch, int out_ch);
void og_add_gradient_to_face(og_grid* g, int x_ch, int coeff_ch, int u_ch);

/* geometric multigrid preconditioners (GMGSolver.cu, CMGSolver.cu) */
#define OG_GMG 1
#define OG_CMG 2
void og_calc_cell_types_from_leafs(og_grid* g);
void og_geo_full_neg_lap(og_grid* g, int kind, int x_ch, int ax_ch);
void og_geo_gauss_seidel(og_grid* g, int kind, int iters, int order, int level, int x_ch, int rhs_ch);
void og_geo_vcycle(og_grid* g, int kind, int x_ch, int f_ch, int rhs_ch, int level_iters, int coarsest_iters, float one_over_alpha, float P);
int og_geo_solve(og_grid* g, int kind, float one_over_alpha, float P, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride, int pure_neumann, double* rel_res);

/* stand-alone iterative solvers of the reference's test harness */
int og_fas_mu_cycle_solve(og_grid* g, int coeff_ch, int repeat_times, double omega, float R_restrict, float P, int max_iters, double tol, int level_iters, int coarsest_iters, double* rel_res);
int og_gmg_damped_jacobi_solve(og_grid* g, int max_iters, double tol, float omega, double* rel_res);

/* FP64 CSR assembly of the leaf operator (unknowns = INTERIOR cells of LEAF tiles) */
int og_assemble_count(og_grid* g, int coeff_ch, int* n_rows, long long* nnz);
int og_assemble(og_grid* g, int coeff_ch, long long* rowptr, int* col, double* val, int* row_tile, int* row_cell);
int og_csr_solve(int n, const long long* rowptr, const int* col, const double* val, const double* b, double* x, double tol, int max_iters, int method, int* iters_out, double* rel_out);
int og_csr_matvec(int n, const long long* rowptr, const int* col, const double* val, const double* x, double* y);

/* pieces exported so that tests can compare them with the reference's own
 * host-compiled functions (oracle/_ref, built by oracle/build_ref.py) */
float og_frac_inside(float a, float b);
void og_face_fluid_ratio(const float* phi4, int n, float* out);
void og_cell_corner_inside_count(const float* nodes729, float iso, int* out512);
int og_case_target_at(float h0, int case_id, const double* params, int nparams, int level, int i, int j, int k);
void og_case_types_at(float h0, int case_id, int level, int i, int j, int k, uint8_t* out512);
/* 1: coarsen off-diagonals under the reference's cell-type mask applied to the
 * types the grid holds at that point (NONLEAF types included); 0 (default):
 * the mask is open */
void og_set_reference_mask(og_grid* g, int on);
/* 1: the mixed-precision cycle -- x and rhs of levels >= 3 held in BF16 (every write there
 * rounded to BF16; the finest right-hand side read through its BF16 copy) */
void og_set_x_bf16(og_grid* g, int on);

#ifdef __cplusplus
}
#endif
#endif
