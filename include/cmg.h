/*
 * cmg.h -- C ABI of the B200 octree multigrid pressure-Poisson solver.
 *
 * Plain pointers, sizes and status codes only; no C++ or torch types cross
 * this boundary.  Each entry point names the Cirrus-amg interface it stands
 * in for (file:line relative to that project's root).  Every function
 * returns CMG_OK (0) or a CMG_ERR_* code; cmg_last_error() gives the
 * message of the last failure on the calling thread.
 *
 * Object model (the reference's, re-laid-out for the GPU):
 *   cmg_grid   <-> HADeviceGrid<PoissonTile<float,15>> (src/HAGrid.h:357):
 *                  an octree of 8^3-cell tiles, LEAF / NONLEAF / GHOST tiles
 *                  per level, num_channels float channels per cell and one
 *                  uint8 cell type per cell.  On the device every channel is
 *                  a plane of num_tiles*512 floats, tile-major, cell index
 *                  i*64 + j*8 + k inside a tile (src/HAAccessor.h:32).  Tiles
 *                  are ordered by (level, tile type, Morton code).
 *   cmg_amg_solver <-> AMGSolver (src/AMGSolver.h:19-75).
 *
 * Channel conventions of the solve follow PoissonTile (src/PoissonTile.h:13-18):
 * x = 0, b = r = 1 (overwritten by the residual), p = 2, Ap = 3, z = 4.
 */
#ifndef CMG_H
#define CMG_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* tile types (src/HATileInfo.h:10) */
#define CMG_LEAF 1
#define CMG_NONLEAF 2
#define CMG_GHOST 4
/* cell types (src/PoissonTile.h:7) */
#define CMG_DIRICHLET 1
#define CMG_INTERIOR 2
#define CMG_NEUMANN 4

/* status codes */
#define CMG_OK 0
#define CMG_ERR_INVALID 1    /* bad argument (channel, level, pointer, size) */
#define CMG_ERR_CUDA 2       /* a CUDA call failed; see cmg_last_error() */
#define CMG_ERR_STATE 3      /* call order: e.g. solve before prepare */
#define CMG_ERR_TOPOLOGY 4   /* octree not 2:1 face-balanced where the operator needs it */
#define CMG_ERR_NONFINITE 5  /* a NaN/Inf reached a reduction */

/* built-in refinement targets (tests/TestGrids.cuh:33-142 and the
 * adaptive-sphere workloads); params[0] = min level, params[1] = max level. */
#define CMG_CASE_UNIFORM 0
#define CMG_CASE_CENTER_POINT 1
#define CMG_CASE_SPHERE_EMPTY 2
#define CMG_CASE_SPHERE_SOLID 3
#define CMG_CASE_STAR_EMPTY 4
#define CMG_CASE_STAR_SOLID 5
#define CMG_CASE_SHELL 6        /* + mid level, centre xyz, radius, fine band, mid band */
#define CMG_CASE_MULTI_SPHERE 7 /* + band, count, then (x, y, z, r) per sphere */

typedef struct cmg_grid cmg_grid;
typedef struct cmg_amg_solver cmg_amg_solver;

/* Refinement target of a tile: the level it should reach (the device lambda
 * passed to HADeviceGrid::iterativeRefine, src/HAGrid.h:1173). */
typedef int (*cmg_level_target_fn)(void* user, int level, int i, int j, int k);

const char* cmg_last_error(void);
int cmg_version(void);
/* Self-check of the division the Gauss-Seidel sweeps use (one double multiply
 * by a double reciprocal of the divisor, rounded to float; the reciprocal either
 * correctly rounded or refined by Newton steps) against the IEEE float
 * division, on n pseudo-random pairs from `seed`.  mismatches
 * receives the number of results that differ in any bit; first_pair (may be
 * NULL) the bit patterns of the first differing (a, d).  No counterpart in the
 * reference, which divides directly (src/AMGSolver.cu:868-875). */
int cmg_check_division(long long n, unsigned long long seed, long long* mismatches, unsigned int* first_pair);

/* ---- grid: HADeviceGrid ------------------------------------------------ */
/* HADeviceGrid(h0, levels_log2_hash) (src/HAGrid.h:416); num_levels = number
 * of hash levels there, num_channels = PoissonTile NUMCHNLS (15). */
int cmg_grid_create(float h0, int num_levels, int num_channels, cmg_grid** out);
int cmg_grid_destroy(cmg_grid* g);
/* setTileHost (src/HAGrid.h:526): add a tile or change its type. */
int cmg_grid_set_tile(cmg_grid* g, int level, int i, int j, int k, int tile_type);
/* rebuild (src/HAGrid.h:892): spawn GHOST tiles, order tiles, upload tables.
 * Channel data and cell types of tiles that survive are kept; a LEAF or NONLEAF tile
 * made by refinement takes them from its parent, cell by cell (PoissonTile::childTile,
 * src/PoissonTile.h:151, as refineStep does, src/HAGrid.h:1140-1160); a new GHOST tile
 * starts at zero.  The copy runs on the device. */
int cmg_grid_rebuild(cmg_grid* g);
/* iterativeRefine (src/HAGrid.h:1173) with a host callback or a built-in case. */
int cmg_grid_iterative_refine(cmg_grid* g, cmg_level_target_fn fn, void* user, int* steps);
int cmg_grid_refine_case(cmg_grid* g, int case_id, const double* params, int nparams, int* steps);
/* The same refinement as cmg_grid_refine_case, then the ghost layer, the canonical tile
 * order and the index tables, all built in device memory on the grid's stream: a tile pool
 * with an atomic counter, an open-addressing hash of tile keys, two kernels per level for
 * refineStep's flags and the new tiles (src/HAGrid.h:1088-1170; the reference does that
 * part on the host), one for spawnGhostTiles (:856-889) and a radix sort for the order.
 * The result equals cmg_grid_refine_case's tile for tile.  Cases 0-3, 6 and 7; the star
 * cases (4, 5), whose targets use transcendental functions, are refined on the host. */
int cmg_grid_refine_case_device(cmg_grid* g, int case_id, const double* params, int nparams, int* steps);
/* numTotalTiles / mMaxLevel (src/HAGrid.h:504, 366) */
int cmg_grid_info(cmg_grid* g, int* num_tiles, int* max_level, int* num_leaf_tiles);
/* tile list in device order: level[n], ijk[3n], type[n] (host buffers) */
int cmg_grid_tiles(cmg_grid* g, int* level, int* ijk, uint8_t* type);
/* device tables: nb[8n] (-x,-y,-z,+x,+y,+z, parent, -1), child[8n] (dx*4+dy*2+dz) */
int cmg_grid_tables(cmg_grid* g, int* nb, int* child);
/* device pointers of channel planes / the cell-type plane (num_tiles*512 each) */
int cmg_grid_channel_ptr(cmg_grid* g, int ch, float** dev_ptr);
int cmg_grid_cell_type_ptr(cmg_grid* g, uint8_t** dev_ptr);
/* host <-> device copies of a whole channel plane or the cell types */
int cmg_grid_upload_channel(cmg_grid* g, int ch, const float* host, size_t count);
int cmg_grid_download_channel(cmg_grid* g, int ch, float* host, size_t count);
int cmg_grid_upload_cell_types(cmg_grid* g, const uint8_t* host, size_t count);
int cmg_grid_download_cell_types(cmg_grid* g, uint8_t* host, size_t count);
int cmg_grid_fill_channel(cmg_grid* g, int ch, float value);
/* device-to-device copy of a whole channel plane (Copy over all tiles and
 * cells, src/PoissonGrid.cu:87, without the cell-type mask) */
int cmg_grid_copy_channel(cmg_grid* g, int src_ch, int dst_ch);
/* CreateTestGrid cell types of LEAF tiles (tests/TestGrids.cuh:161-167) */
/* CalcCellTypesFromLeafs (src/PoissonGrid.cu:923-977): NONLEAF cell types from their
 * LEAF/NONLEAF children, finest level first (DIRICHLET before INTERIOR before
 * NEUMANN), then GHOST cell types from their parents.  Needed before a GMG or CMG
 * solve; AMG sets its own types in cmg_amg_prepare_types_and_coeffs. */
int cmg_grid_calc_cell_types_from_leafs(cmg_grid* g);
/* HADeviceGrid::loadBinaryBlob / dumpBinaryBlob (src/HAGrid.h:687-853): the 'HAGR'
 * version-1 grid blob with raw PoissonTile<float,15> records (44880 bytes each).
 * Loading rebuilds the octree from the LEAF and NONLEAF records (GHOST tiles are
 * spawned again and must match the blob's), copies the cell values of the first
 * min(num_channels, 15) channels and the cell types of every record, and zeroes any
 * further channels.  Dumping writes every tile with min(num_channels, 15) channels;
 * with buf == NULL it only reports the size. */
int cmg_grid_load_hagr(const uint8_t* blob, size_t size, int num_channels, cmg_grid** out);
/* The record layout this library reads and writes, for a binding that checks it against
 * its own build of the reference structs: out[0..13] = header bytes (sizeof of the local
 * Header struct of HADeviceGrid::dumpBinaryBlob, src/HAGrid.h:699-708), the offsets of its
 * eight fields (magic, version, num_levels, max_level, tile_size, coord_size, h0,
 * tile_count), sizeof(Coord), sizeof(PoissonTile<float,15>), offsetof its mCellType,
 * its channel count and channel stride in floats (src/PoissonTile.h:28-39).  Returns the
 * number of entries (14); with out == NULL only that. */
int cmg_ref_record_layout(long long* out, int n);
/* A view of the reference's own device tiles, for a caller that keeps its HADeviceGrid
 * (src/HAGrid.h:357-406): every tile is a PoissonTile<float,15> in device memory
 * (src/PoissonTile.h:34-39: float mData[15][736], cell values in the first 512 of each
 * channel; uint8 mCellType[512] at byte 44352; 44880 bytes), reached through the device
 * pointer of its HATileInfo.  tile_ptrs (host array) holds, for each tile of g in the order
 * of cmg_grid_tiles, the device address of the reference tile with the same level and
 * coordinate; tile_bytes must be 44880.  Gather copies channels [first_ch, first_ch+num_ch)
 * (and, with with_types, the cell types) from those tiles into g; scatter writes the
 * channels of g back into them.  Both run on the device on g's stream and leave every
 * other byte of the tiles untouched; only the pointer list crosses from the host. */
int cmg_grid_gather_device_tiles(cmg_grid* g, const void* const* tile_ptrs, size_t tile_bytes, int first_ch, int num_ch, int with_types);
int cmg_grid_scatter_device_tiles(cmg_grid* g, const void* const* tile_ptrs, size_t tile_bytes, int first_ch, int num_ch);
int cmg_grid_dump_hagr(cmg_grid* g, uint8_t* buf, size_t capacity, size_t* size);
int cmg_grid_set_leaf_cell_types_case(cmg_grid* g, int case_id, const double* params, int nparams);
/* stream used by every later call on this grid (NULL = legacy default) */
int cmg_grid_set_stream(cmg_grid* g, void* cuda_stream);
int cmg_grid_synchronize(cmg_grid* g);

/* ---- operator set-up: AMGSolver.cu / MeshCutCell.cu ------------------- */
/* CoarsenTypesAndAMGCoeffs (src/AMGSolver.cu:256-318), the body of
 * AMGSolver::prepareTypesAndCoeffs (src/AMGSolver.cu:1394). */
int cmg_amg_prepare_types_and_coeffs(cmg_grid* g, int coeff_ch, float R_matrix);
/* PrepareLaplacianSystemFromLeafAndGhostCellTypesAndFaceCoeffs (src/AMGSolver.cu:89) */
int cmg_amg_prepare_system(cmg_grid* g, int coeff_ch, float R_matrix);
/* CreateAMGLaplacianSystemWithSolidCutOnNodeSDF (cirrus_cutcell/MeshCutCell.cu:416)
 * with the node SDF of a union of spheres (x, y, z, r per sphere). */
int cmg_amg_cutcell_sphere_coeffs(cmg_grid* g, int coeff_ch, float R_matrix, int nspheres, const float* spheres);
/* face velocity u = sum_m amp_m sin(2 pi k_m . x + phase_m) on LEAF faces (k[3m], amp[3m], phase[m]) */
int cmg_amg_face_velocity_fourier(cmg_grid* g, int u_ch, int nmodes, const double* k, const double* amp, const double* phase);
/* AMGVolumeWeightedDivergenceOnLeafs (src/AMGSolver.cu:790) */
int cmg_amg_divergence(cmg_grid* g, int u_ch, int coeff_ch, int out_ch);
/* AMGVolumeWeightedDivergenceWithoutCoeffOnLeafs (src/AMGSolver.cu:750), the form the
 * reference's projection step calls (cirrus_cutcell/FluidEuler.cu:698, 723): faces
 * weighted by h*h instead of the coefficients. */
int cmg_amg_divergence_without_coeff(cmg_grid* g, int u_ch, int out_ch);
/* AMGAddGradientToFace (src/AMGSolver.cu:680): u += grad x on faces with a
 * positive fluid ratio, LEAF and GHOST tiles (GHOST x is first set from the parents) */
int cmg_amg_add_gradient_to_face(cmg_grid* g, int x_ch, int coeff_ch, int u_ch);
/* AMGFullNegativeLaplacianOnLeafs (src/AMGSolver.cu:589): Ax on LEAF tiles */
int cmg_amg_full_neg_lap(cmg_grid* g, int x_ch, int coeff_ch, int ax_ch);
/* Dot over LEAF tiles (src/PoissonGrid.cu:203) */
int cmg_amg_dot(cmg_grid* g, int a_ch, int b_ch, double* out);
/* The same dot product as cmg_amg_dot (equal bit for bit), for callers that may not
 * allocate at the call: it allocates no memory.  Its scratch is a fixed 128 KB array in
 * the library's static device memory, so it serves grids of at most 16384 LEAF tiles
 * (larger grids: CMG_ERR_INVALID) and needs the grid's device copy to be current
 * already (CMG_ERR_STATE otherwise).  It runs on the grid's device.  Calls that overlap
 * in time share that scratch and race; each call clears it first, so only the
 * overlapping calls are affected, and one that finds no result reports CMG_ERR_CUDA.
 * The first call on a device looks up the scratch address (not refreshed after a
 * cudaDeviceReset).  No counterpart in the reference. */
int cmg_amg_dot_noalloc(cmg_grid* g, int a_ch, int b_ch, double* out);

/* ---- solver: AMGSolver ------------------------------------------------- */
/* AMGSolver(coeff_channel, R_matrix, R_restrict, P) (src/AMGSolver.h:31);
 * omega = 1.5, mu = 2 as there (src/AMGSolver.h:28-29). */
int cmg_amg_solver_create(int coeff_ch, float R_matrix, float R_restrict, float P, cmg_amg_solver** out);
int cmg_amg_solver_destroy(cmg_amg_solver* s);
/* public fields omega / mu_cycle_repeat_times (src/AMGSolver.h:28-29); omega is held as a
 * float, as the reference's field is (T omega), so the Gauss-Seidel update
 * x + delta * omega rounds exactly as the reference's does */
int cmg_amg_solver_set_smoother(cmg_amg_solver* s, double omega, int mu);
/* One smoother setting for the autotuner.  finest_iters: sweeps per visit (before and after
 * the coarse correction alike) on the finest level, levels >= 3; -1: level_iters, which is
 * the reference's cycle. */
typedef struct cmg_tune_candidate {
    double omega;
    int mu, level_iters, coarsest_iters, finest_iters;
} cmg_tune_candidate;
/* Autotuner (no counterpart in the reference): solves the grid's current rhs (channel 1)
 * under each of n candidate settings to tol, `repeats` timed solves each after one untimed
 * solve (a candidate whose first solve is slower than 1.5x the best so far, or does not
 * converge, is not timed further; its ms[i] is that first solve's), and keeps the fastest
 * setting that converges, except that among the settings within 3 % of the fastest time
 * the one with the fewest iterations wins, and among those the one whose last iteration
 * reached the smallest relative residual: ms[i] (-1: did not converge),
 * iters[i], *best (-1: none).  The
 * solver takes the best candidate's omega, mu and finest_iters; pass its
 * level_iters and coarsest_iters to cmg_amg_solve.  Channel 1 is restored, channel 0 holds
 * the last solution.  Tune on a right-hand side other than the ones to be timed. */
int cmg_amg_solver_autotune(cmg_amg_solver* s, cmg_grid* g, int n, const cmg_tune_candidate* candidates, int max_iters, double tol,
                            int repeats, float* ms, int* iters, int* best);
/* Sweeps per visit on the finest level (levels >= 3), the same before and after the coarse
 * correction so that the preconditioner stays symmetric; -1 (default): level_iters, as the
 * reference does on every level.  No counterpart in the reference. */
int cmg_amg_solver_set_finest_iters(cmg_amg_solver* s, int finest_iters);
/* True-residual replacement, the mixed-precision solve's safeguard: every `every` PCG
 * iterations (0, the default: never) the recurrence residual is replaced by b - A x computed
 * on the device with the stencil summed in double, from a copy of b the solve keeps.  The
 * reference has no counterpart: its residual is the recurrence's, and its only other
 * residual is the FP64 dot of it (src/AMGSolver.cu:1487-1499).  `count` receives the
 * replacements the last solve made. */
int cmg_amg_solver_set_residual_replacement(cmg_amg_solver* s, int every);
int cmg_amg_solver_residual_replacements(cmg_amg_solver* s, int* count);
/* Direct coarsest solve (mixed-precision mode; no counterpart in the reference, which runs
 * coarsest_iters Gauss-Seidel sweeps on level 0, src/AMGSolver.cu:1260-1264): with on != 0,
 * whenever levels 0-2 are complete (the cluster step runs them), level 0 is solved exactly,
 * x0 = A0^-1 b0 in double.  A0 is the 8^3 root operator on its INTERIOR cells; its inverse
 * is formed from an FP64 Cholesky factor on the host when the operator changes, and applied
 * on the device.  Other octrees keep the sweeps. */
int cmg_amg_solver_set_coarsest_direct(cmg_amg_solver* s, int on);
/* BF16 storage of the preconditioner's grids (mixed-precision mode; no counterpart in the
 * reference): with on != 0, x, rhs and the saved FAS x of levels >= 3 live in BF16 planes
 * and every sweep, restriction, FAS update and prolongation there reads and writes BF16,
 * computing in FP32; levels 0-2 and the outer PCG stay FP32.  The right-hand side enters
 * rounded to BF16 and z leaves widened from it.  Needs the pipelined smoother (the default
 * launch mode) and is ignored by the learned solve. */
int cmg_amg_solver_set_cycle_bf16(cmg_amg_solver* s, int on);
/* Launch flags (default CMG_LAUNCH_GRAPH).
 * GRAPH: the solve runs as one CUDA graph with a device-side while loop;
 * without it the same kernels are launched one by one with the loop test on
 * the host (for profilers that do not enter conditional graph nodes).
 * PERSISTENT: each visit of multigrid level 2 or 3 runs as one cooperative
 * kernel with grid barriers; without it, one kernel per phase.
 * NO_CLUSTER: when levels 0-2 are complete grids, each visit of level 2 (with
 * its recursion through levels 1 and 0) normally runs as one launch of an
 * 9-CTA thread-block cluster; this flag launches those phases separately.
 * NO_PIPELINE: the smoothing sweeps of the cycle normally run as a persistent
 * kernel that loads the next tile while it computes one; this flag uses one
 * block per tile instead.
 * None has a counterpart in the reference, which launches every phase from
 * the host. */
#define CMG_LAUNCH_GRAPH 1
#define CMG_LAUNCH_PERSISTENT 2
#define CMG_LAUNCH_NO_CLUSTER 4
#define CMG_LAUNCH_NO_PIPELINE 8
int cmg_amg_solver_set_launch_mode(cmg_amg_solver* s, int flags);
/* Mixed-precision preconditioner (no counterpart in the reference, which is FP32
 * throughout): the smoothing sweeps of the mu-cycle on levels 3 and finer read the
 * operator planes (diagonal and face coefficients) from a BF16 or FP16 copy made once
 * per solve, widening every value to float; x, b, residuals, restriction, the coarse
 * levels and the PCG iteration stay FP32 with FP64 dot products.  Default FP32, which
 * is the reference's arithmetic. */
#define CMG_STORAGE_FP32 0
#define CMG_STORAGE_BF16 1
#define CMG_STORAGE_FP16 2
int cmg_amg_solver_set_storage(cmg_amg_solver* s, int storage);
/* Learned finest-level smoother (no counterpart in the reference).  A per-tile 3-D conv
 * net on BF16 tensor cores, hidden = 8 or 16 (conv3x3x3 8->H, ReLU, H->H, ReLU, H->1) or
 * 32 (conv 8->32, ReLU, four residual blocks x = relu(x + conv(relu(conv(x))))) at 32
 * channels, conv 32->1; tcgen05 MMAs with TMEM accumulators for inference and training), adds
 * (S/D) f(rho/S, INTERIOR, DIRICHLET, diag/D) to z on the finest level's LEAF tiles after
 * each mu-cycle, rho = r - A z being the residual the cycle leaves (S: its RMS on the
 * tile, D: the tile's largest diagonal).  The solve then runs flexible CG (Polak-Ribiere
 * beta), judges the result by the true residual |b - A x| / |b| and falls back to the
 * plain solve when that exceeds 10 tol, the solve does not converge, or its residual stalls
 * (its norm falls by less than 2x over 4 iterations).
 * Samples are tiles of 512 cells (cell i*64 + j*8 + k): rho, the diagonal of A (the
 * coefficient channel coeff+3), cell types and the target error d = A^-1 rho.
 * The net keeps its parameters, Adam state and samples on the device; training runs
 * the forward and backward kernels on the GPU. */
typedef struct cmg_learned cmg_learned;
int cmg_learned_create(int hidden, unsigned long long seed, cmg_learned** out);
int cmg_learned_destroy(cmg_learned* net);
int cmg_learned_num_params(cmg_learned* net, int* n);
/* fp32 parameters: W1[H][27][8], b1[H], W2[H][27][H], b2[H], W3[27][H]; tap = dx*9+dy*3+dz.
 * hidden = 32: W0[32][27][8], b0[32], per block k = 0..3 Wa[32][27][32], ba[32], Wb[32][27][32],
 * bb[32], then Wo[27][32] (229,248 in all) */
int cmg_learned_get_params(cmg_learned* net, float* host, int n);
int cmg_learned_set_params(cmg_learned* net, const float* host, int n); /* also resets Adam */
/* training/evaluation tiles: rho, diag, types, target [n][512]; optional (NULL: absent, the
 * inputs read 0): faces [n][3][512], the -x/-y/-z face coefficients of each cell; halo
 * [n][768], the residual across the tile's six faces (value of face r, side s, cell (a, b) at
 * r*128 + s*64 + a*8 + b, then the same layout of 1/0 flags for cells that exist and are
 * INTERIOR).  In the solve the net reads both from the grid itself. */
int cmg_learned_set_samples(cmg_learned* net, int n, const float* rho, const float* diag, const uint8_t* types, const float* target,
                            const float* faces, const float* halo);
/* correction (S/D) f on INTERIOR cells (0 elsewhere) of samples first..first+n-1 */
int cmg_learned_forward(cmg_learned* net, int first, int n, float* out);
/* The net on the grid itself, as the learned solve applies it: on the LEAF tiles of `level`,
 * rho = channel r_ch - channel az_ch (az_ch < 0: r_ch holds rho), the face coefficients from
 * coeff_ch..coeff_ch+2 and the diagonal from coeff_ch+3, the halo from same-level LEAF
 * neighbours; out_ch += the correction (= with overwrite) on INTERIOR cells. */
int cmg_learned_apply_grid(cmg_learned* net, cmg_grid* g, int level, int r_ch, int az_ch, int coeff_ch, int out_ch, int overwrite);
/* inference kernel of every net in the process: 0 (default) mma.sync, 1 tcgen05.mma with
 * TMEM accumulators; both compute the same network (FP32 accumulation, BF16 operands).  With
 * 8 output channels the tcgen05 MMAs are M = 64, N = 8 and measured slower than mma.sync. */
int cmg_learned_set_inference(int kind);
/* training loss per tile, e = f - target D/S on INTERIOR cells (0 elsewhere):
 * kind 0 (default) sum e^2; kind 1 (energy) e^T L e, L the tile's 7-point Laplacian
 * (6 on the diagonal, -1 per neighbour inside the tile), which weighs rough errors as PCG does */
int cmg_learned_set_loss(cmg_learned* net, int kind);
/* mean loss (sum of tile losses) / (n 512) over samples first..first+n-1 and its gradient */
int cmg_learned_gradient(cmg_learned* net, int first, int n, double* loss, float* grad);
/* Adam (beta 0.9/0.999) over shuffled batches; epoch_loss[e] (may be NULL) */
int cmg_learned_train(cmg_learned* net, int epochs, int batch, float lr, unsigned long long seed, float* epoch_loss);
/* use the net's current parameters as the solver's finest-level smoother (NULL: plain) */
int cmg_amg_solver_set_learned(cmg_amg_solver* s, cmg_learned* net);
/* of the last cmg_amg_solve with a learned smoother: true relative residual, whether it
 * fell back to the plain solve, and the learned attempt's iterations */
int cmg_amg_solver_learned_status(cmg_amg_solver* s, double* true_rel, int* fell_back, int* learned_iters);

/* ---- geometric multigrid preconditioners ---------------------------------
 * GMGSolver(one_over_alpha, prolong_coeff) (src/GMGSolver.h:21) and
 * CMGSolver(one_over_alpha, prolong_coeff) (src/CMGSolver.h:21): the same
 * solver handle type, solved with cmg_amg_solve (GMGSolver::solve,
 * src/GMGSolver.cu:472-607; CMGSolver::solve, src/CMGSolver.cu:466-601: PCG
 * preconditioned by one V-cycle, channels as for AMG).  They use no coefficient
 * channels: the operator comes from tile and cell types.  The reference's tests
 * construct both with (1, 1) (tests/SolverTests.cu:1055,1077). */
int cmg_gmg_solver_create(float one_over_alpha, float prolong_coeff, cmg_amg_solver** out);
int cmg_cmg_solver_create(float one_over_alpha, float prolong_coeff, cmg_amg_solver** out);
/* GMGSolver::VCycle / CMGSolver::VCycle (src/GMGSolver.cu:324, src/CMGSolver.cu:377):
 * x_ch <- V-cycle applied to f_ch, rhs_ch used as the cycle's right-hand-side scratch */
int cmg_mg_vcycle(cmg_amg_solver* s, cmg_grid* g, int x_ch, int f_ch, int rhs_ch, int level_iters, int coarsest_iters);
/* GaussSeidelGMG / GaussSeidelCMG (src/GMGSolver.cu:217, src/CMGSolver.cu:271) */
int cmg_mg_gauss_seidel(cmg_amg_solver* s, cmg_grid* g, int iters, int order, int level, int x_ch, int rhs_ch);
/* FullNegativeLaplacian / ConservativeFullNegativeLaplacian (src/GMGSolver.cu:167,
 * src/CMGSolver.cu:210); writes GHOST (and, for CMG, NONLEAF) values of x_ch */
int cmg_mg_full_neg_lap(cmg_amg_solver* s, cmg_grid* g, int x_ch, int ax_ch);

/* AMGSolver::FASMuCycleSolve (src/AMGSolver.cu:1311-1356): the FAS mu-cycle with
 * repeat_times recursions as a stand-alone iteration on x (channel 0) against b
 * (channel 1, kept), channel 2 as scratch.  iters is the index of the iteration at
 * which |b - A x| < tol |b| (max_iters if never), rel_res = |b - A x| / |b|.  The
 * reference's test harness uses it as "amg_vcycle" with AMGSolver(coeff, 0.5, 0.5, 1)
 * (tests/SolverTests.cu:1100-1112).  Synchronises the host once per iteration. */
int cmg_amg_fas_mu_cycle_solve(cmg_amg_solver* s, cmg_grid* g, int repeat_times, int verbose, int max_iters, double tol, int level_iters,
                               int coarsest_iters, int* iters, double* rel_res);
/* GMGSolver::dampedJacobiSolve (src/GMGSolver.cu:390-470), a GMG solver only: x (channel
 * 0) += omega r / D against b (channel 1), channels 2-3 as scratch; same result
 * convention as cmg_amg_fas_mu_cycle_solve ("gmg_jacobi", tests/SolverTests.cu:1063). */
int cmg_gmg_damped_jacobi_solve(cmg_amg_solver* s, cmg_grid* g, int verbose, int max_iters, double tol, float omega, int* iters, double* rel_res);
/* AMGSolver::solve (src/AMGSolver.cu:1399): solves -lap x = b, b read from
 * channel 1 and overwritten by the residual, x written to channel 0.
 * iters/rel_res are the reference's (num_iters, relative_residual), with
 * rel_res = -1 when sync_stride <= 0.  The PCG loop runs on the device as a
 * CUDA-graph while-loop; no host synchronisation happens inside it. */
int cmg_amg_solve(cmg_amg_solver* s, cmg_grid* g, int verbose, int max_iters, double relative_tolerance,
                  int level_iters, int coarsest_iters, int sync_stride, int is_pure_neumann,
                  int* iters, double* rel_res);
/* The same solve with host buffers: b (num_tiles*512 floats, device order)
 * is copied in, x copied out; the copies are part of the call. */
int cmg_amg_solve_host(cmg_amg_solver* s, cmg_grid* g, const float* b_host, float* x_host, size_t count,
                       int max_iters, double relative_tolerance, int level_iters, int coarsest_iters,
                       int sync_stride, int is_pure_neumann, int* iters, double* rel_res);
/* A batch of n independent solves, each AMGSolver::solve (src/AMGSolver.h:62) on its own
 * grid with its own solver object; the reference has no batched call, its callers loop
 * over solve().  Every solve is enqueued first, on its grid's stream (cmg_grid_set_stream),
 * so solves on distinct streams run concurrently; then the call waits for all of them.
 * b_host and x_host are NULL (b and x in channels 1 and 0 on the device) or arrays of n
 * host pointers (num_tiles*512 floats each, pinned for the copies to overlap): b is copied
 * in and x copied out as in cmg_amg_solve_host, inside the call.  solvers and grids must
 * each be n distinct objects.  iters, rel_res and ms (device time of each solve from CUDA
 * events on its stream; may be NULL) receive n values. */
int cmg_amg_solve_batch(cmg_amg_solver* const* solvers, cmg_grid* const* grids, int n,
                        const float* const* b_host, float* const* x_host,
                        int max_iters, double relative_tolerance, int level_iters, int coarsest_iters,
                        int sync_stride, int is_pure_neumann, int* iters, double* rel_res, float* ms);
/* ---- many octrees in ONE persistent launch ----
 * n independent solves, each AMGSolver::solve (src/AMGSolver.h:62) of grid i with the
 * settings of solver i (omega, mu, coefficient channel, finest-level sweeps), run by one
 * cooperative kernel launch captured in a CUDA graph.  The resident blocks form groups of
 * `group_blocks` blocks; each group takes the next octree from a device work queue (the
 * largest mu-cycle work first), runs its whole PCG solve, and takes the next.  Results are
 * cmg_amg_solve's bit for bit.  The reference has no batched call: its callers loop over
 * solve() (cirrus_cutcell/FluidEuler.cu:702-707).
 * Grids must be n distinct built grids on the current device; a solver may serve several
 * grids.  Solvers must be AMG solvers with FP32 storage and none of the learned,
 * residual-replacement, BF16-cycle or direct-coarsest options (CMG_ERR_INVALID otherwise).
 * The batch keeps the pointers: solvers and grids must outlive it, and a grid rebuilt
 * since the last call is picked up by the next call. */
typedef struct cmg_batch cmg_batch;
int cmg_batch_create(cmg_amg_solver* const* solvers, cmg_grid* const* grids, int n, cmg_batch** out);
int cmg_batch_destroy(cmg_batch* b);
/* The schedule: blocks of `slots` 128-thread slots (4, the default, 6 or 8; more slots hide
 * more memory latency, fewer leave each thread more registers), groups of `group_blocks`
 * blocks (0, the default: the resident blocks spread over the octrees) that take octrees
 * from the shared queue, largest first.  split > 0: each
 * octree that would not end within split x (total work / resident blocks) in such a group
 * gets a group of its own sized for that budget (work: each octree's block-time measured by
 * the last cmg_batch_autotune, else an estimate from its tiles per level); 0: no such groups. */
int cmg_batch_set_schedule(cmg_batch* b, int slots, int group_blocks, double split);
/* the plan the next solve uses: slots, small groups' blocks, groups, dedicated groups, resident blocks */
int cmg_batch_schedule(cmg_batch* b, int* slots, int* group_blocks, int* groups, int* dedicated, int* resident_blocks);
/* b_host / x_host: NULL (b and x in channels 1 and 0 on the device) or n host pointers
 * (num_tiles*512 floats each, pinned for full-speed copies), copied in and out inside the
 * call.  iters, rel_res (n values, required) as cmg_amg_solve gives them; instance_ms
 * (n values, may be NULL): each octree's solve time inside the launch (device clock);
 * batch_ms (may be NULL): the launch's time (CUDA events). */
int cmg_batch_solve(cmg_batch* b, const float* const* b_host, float* const* x_host, int max_iters, double relative_tolerance,
                    int level_iters, int coarsest_iters, int sync_stride, int is_pure_neumann, int* iters, double* rel_res,
                    float* instance_ms, float* batch_ms);
/* The schedule autotuner: one calibration run measures each octree's block-time; then the
 * batch (convergence test every iteration) is timed under each candidate schedule
 * (slots[i], group_blocks[i], split[i]; slots may be NULL: the current, split may be NULL:
 * all 0), best of `repeats` runs after one
 * untimed run, each run from the right-hand sides the grids hold on entry (restored at the
 * end); keeps the fastest candidate whose solves all converge.  ms[i] = its time (-1: did
 * not converge), *best = its index (-1: none). */
int cmg_batch_autotune(cmg_batch* b, const int* slots, const int* group_blocks, const double* split, int ncand, int max_iters,
                       double relative_tolerance, int level_iters, int coarsest_iters, int repeats, float* ms, int* best);
/* GaussSeidelAMG (src/AMGSolver.cu:887) on one level */
int cmg_amg_gauss_seidel(cmg_amg_solver* s, cmg_grid* g, int iters, int order, int level, int x_ch, int rhs_ch);
/* The same sweeps as the multigrid cycle runs them (the pipelined persistent kernel):
 * x must hold 0 on every cell that is not INTERIOR, which the cycle keeps true and
 * GaussSeidelAMG then preserves.  Results equal cmg_amg_gauss_seidel's on such x. */
int cmg_amg_gauss_seidel_masked(cmg_amg_solver* s, cmg_grid* g, int iters, int order, int level, int x_ch, int rhs_ch);
/* AMGSolver::FASMuCycle (src/AMGSolver.cu:1279) */
int cmg_amg_fas_mu_cycle(cmg_amg_solver* s, cmg_grid* g, int x_ch, int rhs_ch, int x0_ch, int level_iters, int coarsest_iters);
/* The cycles nothing in the reference's solve calls, on the grid's stream:
 * AMGSolver::VCycle (src/AMGSolver.cu:1060): a correction-scheme V-cycle from x = 0 (every
 * tile) with right-hand side f (f_ch, read only) copied into rhs_ch (0 on GHOST tiles);
 * AMGSolver::muCycle (src/AMGSolver.cu:1151): its mu-cycle, repeat_times visits of each
 * coarser level, the LEAF tiles of a coarser level solving for f minus the flux from their
 * NONLEAF neighbours (muCycleStep, :1130); AMGSolver::FASFCycle (src/AMGSolver.cu:1358): the
 * rhs restricted to every level, the coarsest level smoothed, then prolongation and one
 * FASMuCycleStep per level from coarse to fine (x0_ch: the saved x).  Channels must be
 * distinct. */
int cmg_amg_vcycle(cmg_amg_solver* s, cmg_grid* g, int x_ch, int f_ch, int rhs_ch, int level_iters, int coarsest_iters);
int cmg_amg_mu_cycle(cmg_amg_solver* s, cmg_grid* g, int repeat_times, int x_ch, int f_ch, int rhs_ch, int level_iters, int coarsest_iters);
int cmg_amg_fas_f_cycle(cmg_amg_solver* s, cmg_grid* g, int x_ch, int rhs_ch, int x0_ch, int level_iters, int coarsest_iters);
/* Process-wide: launch the pipelined smoothing and restriction passes as programmatic
 * dependent launches of the kernel before them (1, the default), so that each pass's blocks
 * start as the previous kernel drains and copy their first tile's operator planes meanwhile;
 * 0: ordinary launches.  Results are the same bits either way.  Applies to solves whose CUDA
 * graph is built afterwards. */
int cmg_set_dependent_launch(int on);
/* device time of the last cmg_amg_solve, milliseconds (CUDA events) */
int cmg_amg_last_solve_ms(cmg_amg_solver* s, float* ms);
/* number of this library's kernels the last cmg_amg_solve executed (counted
 * from the kernel nodes of its graph times the loop trips); no counterpart in
 * the reference, which launches each kernel from the host */
int cmg_amg_last_solve_launches(cmg_amg_solver* s, long long* launches);

#ifdef __cplusplus
}
#endif
#endif
