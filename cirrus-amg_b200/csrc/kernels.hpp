// Host launchers of the device kernels (kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "device.cuh"

namespace cmg {

// device-resident scalars of one PCG solve (the reference keeps them in a
// thrust::device_vector<double>(7), src/AMGSolver.h:309-318)
struct PcgScalars {
    double gamma, gamma_old, beta, alpha, pAp, rr, rr0, thr, tol;
    double mean, count;
    int iter, done, converged, nonfinite;
    int replaced;  // true-residual replacements made by the solve
    int max_iters, sync_stride;
    unsigned int counter[8];
    // stall test of the learned solve (window 0: off): the solve stops, not converged, when the
    // residual norm has fallen by less than 2x over the last `stall_window` iterations
    double rr_hist[4];
    int stall_window, stalled;
};

struct ReduceScratch {
    double* partial;  // one double per tile (LEAF tiles at most)
    double* partial2;
    PcgScalars* s;
};

// --- geometric multigrid (geo_mg.cu): GMGSolver / CMGSolver ---
enum SolverKind : int { kAMG = 0, kGMG = 1, kCMG = 2 };
// operator on tiles t0..t0+nt whose type (NONLEAF counted as LEAF when sl_is_level) is in `types`
void launch_geo_lap(int kind, const DevGrid& g, int t0, int nt, const float* X, float* AX, bool sl_is_level, int types, cudaStream_t st,
                    bool diag = false);
void launch_leaf_residual(const DevGrid& g, const int* leaf, int nleaf, const float* B, float* R, bool interior_only, cudaStream_t st);
void launch_jacobi_update(const DevGrid& g, const int* leaf, int nleaf, float* X, const float* R, const float* D, float omega, cudaStream_t st);
void launch_geo_gs(int kind, const DevGrid& g, int t0, int nt, float* X, const float* B, int color, cudaStream_t st);
void launch_geo_restrict(int kind, const DevGrid& g, int t0, int nt, const float* X, float* RHS, float one_over_alpha, cudaStream_t st);
void launch_geo_prolong(const DevGrid& g, int t0, int nt, float* X, float P, cudaStream_t st);
void launch_geo_vinit(const DevGrid& g, float* X, float* RHS, const float* F, cudaStream_t st);
// CalcCellTypesFromLeafs step 1 on the NONLEAF tiles in t0..t0+nt (one level per launch, finest first)
void launch_types_from_children(const DevGrid& g, int t0, int nt, cudaStream_t st);
// cell_mask: the cell types whose values count (AccumulateToParentsOneStepKernel's cell_types)
void launch_accumulate_cells(const DevGrid& g, int t0, int nt, int types, const float* SRC, float* DST, float coeff, bool additive,
                             cudaStream_t st, int cell_mask = dInterior | dDirichlet | dNeumann);

// --- multigrid ---
// persistent, software-pipelined colour pass for the multigrid cycle (gs_pipe.cu); needs the
// x plane masked to INTERIOR cells.  gs_pipe_init: resident blocks on the device (0: unusable).
int gs_pipe_init();
// 1 if a pipelined sweep gave up waiting for its bulk copies since the last call (then cleared)
int gs_pipe_take_error();
// launch the pipelined passes as programmatic dependents of the previous kernel (default on)
void gs_pipe_set_dependent_launch(bool on);
bool gs_pipe_dependent_launch();
// Storage of the operator planes the pipelined smoother reads: the float channels, or a
// BF16 / FP16 copy (coeff16: four planes of num_tiles*512 elements, made by launch_coeff16).
constexpr int kStorageFP32 = 0, kStorageBF16 = 1, kStorageFP16 = 2;
void launch_gs_pipe(const DevGrid& g, int t0, int nt, void* X, const void* B, bool x16, int coeff_ch, int color, double omega,
                    cudaStream_t st, int storage, const void* coeff16);
size_t coeff16_bytes(const DevGrid& g);
// learned finest-level smoother: per-tile conv net, hidden width H = 8 or 16 (learned.cu), or
// H = 32, the residual net of four blocks of two 32-channel convs (learned_deep.cu)
int net_params(int H);      // fp32 parameters
int net_pack_elems(int H);  // bf16 elements of the packed operands
int net_bias_elems(int H);  // fp32 elements of the bias vector the kernels read
size_t net_train_scratch_bytes(int H, int nb);  // device scratch a training launch of nb samples needs
int net_train_rows(int H, int nb);              // gradient rows it writes (summed by launch_net_reduce_adam)
bool net_init();
void net_set_inference_kind(int kind);  // 0: mma.sync (default), 1: tcgen05
int net_inference_kind();
int net_take_tc_error();  // 1 if a tcgen05 launch (any inference, the residual net's training) timed out waiting (then cleared)
void launch_net_pack(int H, const float* params, void* pack, float* bias, cudaStream_t st);
// Optional inputs of the net beyond rho, the cell types and the diagonal: the -x/-y/-z face
// coefficients (face a of tile t at faces + a*fstride + t*ftile), and the residual's 1-cell
// halo, either stored per sample (halo: [768] per sample, 6 faces x 64 values then 6 x 64
// flags, face r*128 + side*64 + a*8 + b) or read on the grid from same-level LEAF neighbours
// through the face-neighbour table (nbx, with rho = r - az there).
struct NetExtra {
    const float* faces = nullptr;
    size_t fstride = 0, ftile = 0;
    const float* halo = nullptr;
    const int* nbx = nullptr;
};
// samples s < ns are tiles (idx ? idx[s] : t0 + s) of the planes; rho = r - az (az may be null);
// out[t] += (S/D) f (or = with overwrite) on INTERIOR cells
void launch_net_forward(int H, const float* r, const float* az, const float* diag, const uint8_t* types, const int* idx, int t0, int ns,
                        const void* pack, const float* bias, float* out, bool overwrite, cudaStream_t st, const NetExtra& ex = NetExtra{});
void launch_net_train(int H, const float* rho, const float* diag, const uint8_t* types, const float* target, const int* idx, int nb,
                      const void* pack, const float* bias, float* grad, float* loss, int loss_kind, cudaStream_t st,
                      const NetExtra& ex = NetExtra{}, void* scratch = nullptr);
// the residual net (learned_deep.cu), dispatched to by the net_* / launch_net_* functions for H = 32
int deep_params();
int deep_pack_elems();
int deep_bias_elems();
size_t deep_scratch_bytes();
int deep_train_blocks(int nb);
bool deep_init();
int deep_take_error();
void launch_deep_pack(const float* params, void* pack, float* bias, cudaStream_t st);
void launch_deep_forward(const float* r, const float* az, const float* diag, const uint8_t* types, const int* idx, int t0, int ns,
                         const void* pack, const float* bias, float* out, bool overwrite, cudaStream_t st, const NetExtra& ex);
void launch_deep_train(const float* rho, const float* diag, const uint8_t* types, const float* target, const int* idx, int nb,
                       const void* pack, const float* bias, float* grad, float* loss, int loss_kind, cudaStream_t st, const NetExtra& ex,
                       void* scratch);
void launch_net_reduce_adam(const float* grad, int nb, int np, float scale, float* gout, float* p, float* m, float* v, float lr, int step,
                            bool update, cudaStream_t st);
// flexible-CG beta (Polak-Ribiere): gamma = r.z, beta = -alpha (Ap.z) / gamma_old
void launch_dot_flex(const DevGrid& g, const int* leaf, int nleaf, const float* R, const float* Z, const float* AP, ReduceScratch rs,
                     cudaStream_t st);
// ResidualAndRestrictAMG128Kernel on tiles t0..t0+nt-1 with the same prefetching pipeline
// (x masked to INTERIOR cells, as inside the cycle); equals launch_restrict bit for bit.
// residual and restriction of the tiles t0..t0+nt into their parents: x and b of the tiles in
// float or BF16 (x16), the parents' x and rhs planes Xp/RHSp in float or BF16 (p16)
void launch_restrict_pipe(const DevGrid& g, int t0, int nt, const void* X, const void* B, bool x16, void* Xp, void* RHSp, bool p16,
                          int coeff_ch, float Rr, cudaStream_t st);
// the mixed-precision cycle's BF16 levels: FAS update of NONLEAF tiles (rhs += A x, x0 = x),
// prolongation from a parent level in BF16 (p16) or float, and the conversions of the
// finest right-hand side and result on the given LEAF tiles
void launch_fas_pipe_x16(const DevGrid& g, int t0, int nt, const void* X, void* RHS, void* X0, int coeff_ch, cudaStream_t st);
void launch_prolong_x16(const DevGrid& g, int t0, int nt, void* X, const void* Xc, const void* X0c, bool p16, float P, cudaStream_t st);
void launch_leaf_to_bf16(const int* leaf, int nleaf, const float* R, void* R16, cudaStream_t st);
void launch_leaf_from_bf16(const int* leaf, int nleaf, const void* X16, float* Z, cudaStream_t st);
void launch_coeff16(const DevGrid& g, int coeff_ch, int storage, void* out, cudaStream_t st);
void launch_gs(const DevGrid& g, int t0, int nt, float* X, const float* B, int coeff_ch, int color, double omega, cudaStream_t st);
void launch_restrict(const DevGrid& g, int t0, int nt, float* X, float* RHS, int coeff_ch, float R_restrict, cudaStream_t st);
void launch_fas_save(const DevGrid& g, int t0, int nt, const float* X, float* RHS, float* X0, int coeff_ch, cudaStream_t st);
void launch_prolong(const DevGrid& g, int t0, int nt, float* X, const float* X0, float P, cudaStream_t st);
// the correction-scheme cycles (AMGSolver::VCycle / muCycle) and FASFCycle: x = 0 and rhs = f
// (0 on GHOST tiles) on every tile; prolongation x += P x_parent (GHOST: x = x_parent) on the
// tiles t0..t0+nt of one level; rhs = f - (terms from NONLEAF neighbour tiles) on LEAF tiles
void launch_cycle_init(const DevGrid& g, float* X, float* RHS, const float* F, cudaStream_t st);
void launch_prolong_add(const DevGrid& g, int t0, int nt, float* X, float P, cudaStream_t st);
void launch_deduct_flux(const DevGrid& g, int t0, int nt, const float* X, const float* F, float* RHS, int coeff_ch, cudaStream_t st);
// Whole FASMuCycleStep of level `top` (0 or 1) in one thread block, the
// root and its eight children resident in shared memory as dense grids.
void launch_coarse_step(const DevGrid& g, int top, float* X, float* RHS, float* X0, int coeff_ch, int mu, int level_iters,
                        int coarsest_iters, double omega, float R_restrict, float P, cudaStream_t st);
size_t coarse_step_smem_bytes();
// FASMuCycleStep of level 2 with its recursion through levels 1 and 0 in one
// launch of a 9-CTA cluster (coarse_cluster.cu).  Requires levels 0-2 to be
// complete grids: the root, its 8 children and their 64 children, no GHOST tile.
// tile1: the 8 level-1 tiles in root child order; tile2: the 64 level-2 tiles
// indexed by (i >> 3) * 16 + (j >> 3) * 4 + (k >> 3) of their cells in the 32^3
// grid.  pack: cluster_pack_bytes() of device memory filled by launch_cluster_pack
// from the current coefficients and cell types (once per solve).  fas2: do
// FASSaveSolutionAndUpdateSource on level 2 first (all 64 tiles NONLEAF).
cudaError_t launch_cluster_step(const DevGrid& g, const int* tile1, const int* tile2, const void* pack, float* X, float* RHS, float* X0,
                                int coeff_ch, int mu, int level_iters, int coarsest_iters, double omega, float R_restrict, float P,
                                bool fas2, cudaStream_t st, const double* root_inv = nullptr);
// root_inv (optional): the coarsest level solved exactly as x0 = A0^-1 b0 in double instead of
// by Gauss-Seidel sweeps; [j][t] = (A0^-1)[cluster_thread_cell(j)][cluster_thread_cell(t)],
// 512 x 512 doubles, zero rows and columns for cells that are not INTERIOR
int cluster_thread_cell(int t);  // root cell owned by thread t of the coarse CTA
void launch_cluster_pack(const DevGrid& g, const int* tile1, const int* tile2, int coeff_ch, void* pack, cudaStream_t st);
size_t cluster_pack_bytes();
bool cluster_step_supported();  // the current device can co-schedule the 9-CTA cluster
// FASMuCycleStep of level `top` (2 or 3) with all its recursions in one
// cooperative launch of `nblocks` co-resident blocks; bar = 3 zeroed words
// (barrier count, generation, error flag).  Level ranges indexed by level 0..3.
cudaError_t launch_persist_step(const DevGrid& g, int top, const int* lb, const int* ab, const int* le, const int* nlb, float* X, float* RHS,
                                float* X0, int coeff_ch, int mu, int level_iters, int coarsest_iters, double omega, float R_restrict,
                                float P, unsigned int* bar, int nblocks, cudaStream_t st);
int persist_blocks();  // co-resident blocks of the persistent kernel on the current device

// --- many octrees solved by one persistent launch (batch_persist.cu) ---
// One instance: its octree, level ranges, the mu-cycle settings of its solver, and its
// own scratch.  Planes of the solve: x 0, r 1, p 2, Ap 3, z 4 (the cycle's x); the cycle's
// rhs and saved x live in planes 1 and 3 on NONLEAF tiles, as in the single solve.
constexpr int kBatchMaxLevels = 16;
struct BatchInst {
    DevGrid g;
    const int* leaf;
    int nleaf, top;  // LEAF tile list; finest level
    int lb[kBatchMaxLevels], ab[kBatchMaxLevels], le[kBatchMaxLevels], nlb[kBatchMaxLevels];
    int coeff_ch, mu, finest_iters, exact;  // exact: relaxation form (relax_mode of omega)
    float om, Rr, P;
    double omega;
    double* partial;  // 4 * nleaf doubles: two buffers of (per-tile sums, per-tile counts), used in turn
    PcgScalars* s;     // final scalars, read by the host
    unsigned long long* clock;  // [4]: start and end of this instance's solve (globaltimer, ns), blocks and group that ran it
};
// A group of blocks: blocks [first, first + size) solve the instances order[sbegin..send)
// first, one after another, then take instances from the shared queue order[dyn_begin..n)
struct BatchGroup {
    int first, size, sbegin, send;
};
struct BatchArgs {
    const BatchInst* inst;
    const int* order;              // queue position -> instance
    const BatchGroup* groups;      // ngroups entries
    const int* block_group;        // block -> its group
    int n, ngroups, dyn_begin;
    int max_iters, sync_stride, pure_neumann, level_iters, coarsest_iters;
    double tol;
    unsigned int* ctl;  // batch_ctl_words(groups) zeroed words: queue head, error flag, per-group barrier
};
size_t batch_ctl_words(int groups);
// blocks of `slots` 128-thread slots (4, 6 or 8): co-resident blocks on the current device
bool batch_slots_supported(int slots);
int batch_resident_blocks(int slots);
size_t batch_smem_bytes(int slots);
cudaError_t launch_batch_solve(const BatchArgs& A, int nblocks, int slots, cudaStream_t st);

// --- PCG on LEAF tiles (tile list) ---
enum DotMode : int { kDotStore = 0, kDotRR0 = 1, kDotGammaInit = 2, kDotBeta = 3, kDotAlpha = 4 };
void launch_leaf_apply(const DevGrid& g, const int* leaf, int nleaf, const float* P, float* AP, int coeff_ch, bool fuse_alpha,
                       ReduceScratch rs, cudaStream_t st);
// r = b - A x (stencil in double) on the LEAF tiles when the solve's iteration count is a
// positive multiple of `every`; a no-op launch on the other iterations
void launch_true_residual(const DevGrid& g, const int* leaf, int nleaf, const float* X, const float* B, float* R, int coeff_ch,
                          PcgScalars* s, int every, cudaStream_t st);
void launch_xr_update(const DevGrid& g, const int* leaf, int nleaf, float* X, float* R, const float* P, const float* AP,
                      ReduceScratch rs, cudaGraphConditionalHandle loop_h, cudaGraphConditionalHandle body_h, bool use_handles,
                      cudaStream_t st);
void launch_dot(const DevGrid& g, const int* leaf, int nleaf, const float* A, const float* B, int mode, double* out,
                ReduceScratch rs, cudaStream_t st);
void launch_p_update(const DevGrid& g, const int* leaf, int nleaf, float* P, const float* Z, ReduceScratch rs, cudaStream_t st);
void launch_leaf_fill(const DevGrid& g, const int* leaf, int nleaf, float* X, float value, cudaStream_t st);
void launch_leaf_copy(const DevGrid& g, const int* leaf, int nleaf, float* dst, const float* src, cudaStream_t st);
void launch_recenter(const DevGrid& g, const int* leaf, int nleaf, float* R, ReduceScratch rs, cudaStream_t st);
void launch_loop_gate(ReduceScratch rs, cudaGraphConditionalHandle loop_h, bool use_handle, cudaStream_t st);
void init_kernel_attributes();
void note_kernel_launch();        // counts one launch made outside kernels.cu
long long kernel_launch_count();
// dot product over the LEAF tiles with scratch in a fixed static device array
// (dot_noalloc.cu); cudaErrorInvalidValue if nleaf exceeds dot_noalloc_max_leaf_tiles()
cudaError_t dot_noalloc(int device, const int* leaf, int nleaf, const float* A, const float* B, double* out_host, cudaStream_t st);
int dot_noalloc_max_leaf_tiles();
// div_by_recip against the IEEE division on n pseudo-random pairs; 0 or 2 (CUDA error)
int check_division(long long n, unsigned long long seed, long long* mismatches, unsigned int* first_pair);  // kernels enqueued (or captured) by this library so far

// --- operator set-up and right-hand side ---
void launch_ghost_types(const DevGrid& g, int t0, int nt, cudaStream_t st);
void launch_face_coeffs(const DevGrid& g, int t0, int nt, int coeff_ch, int nspheres, const float* spheres_dev, cudaStream_t st);
void launch_cutcell_neumann(const DevGrid& g, const int* leaf, int nleaf, int nspheres, const float* spheres_dev, cudaStream_t st);
void launch_coarsen_offdiag(const DevGrid& g, int t0, int nt, int coeff_ch, float R, cudaStream_t st);
void launch_diag(const DevGrid& g, int t0, int nt, int coeff_ch, float R, cudaStream_t st);
void launch_face_velocity(const DevGrid& g, const int* leaf, int nleaf, int u_ch, int nmodes, const double* modes_dev, cudaStream_t st);
void launch_propagate_ghost(const DevGrid& g, int t0, int nt, int ch, cudaStream_t st);
void launch_accumulate_faces(const DevGrid& g, const int* leaf, int nleaf, int u_ch, cudaStream_t st);
void launch_divergence(const DevGrid& g, const int* leaf, int nleaf, int u_ch, int coeff_ch, int out_ch, cudaStream_t st);
void launch_gradient(const DevGrid& g, const float* X, int coeff_ch, int u_ch, cudaStream_t st);
// channel data and cell types of a new tile order: from the old tile src_of_new[t].x, s =
// src_of_new[t].y levels up (0: the same tile; -1 in .x: zero); meta: the new tiles' meta
// channels [first, first+num) (and the cell types) of the reference's device tiles
// (PoissonTile<float,15>) to and from the planes; ptrs: a device array of g.n tile addresses
constexpr size_t kRefTileBytes = 44880;
void launch_gather_tiles(const DevGrid& g, const void* const* ptrs, int first, int num, bool types, cudaStream_t st);
void launch_scatter_tiles(const DevGrid& g, void* const* ptrs, int first, int num, cudaStream_t st);
void launch_remap(const float* src, float* dst, const int2* src_of_new, const int4* meta, int n_new, int nch, int n_old, cudaStream_t st);
void launch_remap_types(const uint8_t* src, uint8_t* dst, const int2* src_of_new, const int4* meta, int n_new, cudaStream_t st);
void launch_fill(float* p, size_t n, float v, cudaStream_t st);
void launch_count_bad_diag(const DevGrid& g, int t0, int nt, int coeff_ch, int* out, cudaStream_t st);

}  // namespace cmg
