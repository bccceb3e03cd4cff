// Host objects behind the C ABI: the device octree (cmg_grid) and the AMG
// solver (cmg_amg_solver).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "kernels.hpp"
#include "topology.hpp"
#include "topo_device.hpp"

namespace cmg {

void set_error(const std::string& msg);
const char* last_error();

// Device octree: HADeviceGrid's role (src/HAGrid.h:357).
struct Grid {
    Topology topo;
    int nch;
    cudaStream_t stream = nullptr;

    int n = 0;  // tiles on the device
    bool built = false;                   // host topology ordered and tabled
    unsigned long long host_version = 0;  // bumps on every rebuild
    unsigned long long dev_version = 0;   // host_version the device copy matches
    std::vector<unsigned long long> dev_keys;
    std::vector<int> dev_types;  // tile types of the device copy, in its order
    float* chan = nullptr;
    uint8_t* ctype = nullptr;
    int4* meta = nullptr;
    int* nb = nullptr;
    int* child = nullptr;
    int* nbx = nullptr;  // packed face neighbours, see DevGrid::nbx
    int* leaf = nullptr;
    int nleaf = 0;
    unsigned long long version = 0;
    float* spheres = nullptr;  // device scratch for set-up calls
    double* modes = nullptr;
    void** tile_ptrs = nullptr;  // device copy of a caller's tile address list (reference tiles)
    int tile_ptrs_cap = 0;
    double* dot_out = nullptr;
    DeviceTopoBuilder* topo_builder = nullptr;  // device octree builder (refine_case_device)
    int device = -1;  // the CUDA device the device copy lives on (current at its first allocation)

    Grid(float h0, int num_levels, int num_channels) : topo(h0, num_levels), nch(num_channels) {}
    ~Grid();
    int rebuild();        // host: ghosts, order, tables
    // the built-in refinement case built on the device (cases 0-3, 6, 7; the others on the host)
    int refine_case_device(int case_id, const double* params, int nparams, int* steps);
    int ensure_device();  // device: storage and tables of the current topology
    DevGrid dev() const {
        DevGrid d;
        d.n = n;
        d.nch = nch;
        d.h0 = topo.h0();
        d.chan = chan;
        d.ctype = ctype;
        d.meta = meta;
        d.nb = nb;
        d.child = child;
        d.nbx = nbx;
        return d;
    }
    float* plane(int c) const { return chan + (size_t)c * (size_t)n * kCells; }
    int max_level() const { return topo.max_level(); }
    int level_begin(int l) const { return topo.level_begin[l]; }
    int level_end(int l) const { return topo.level_end[l]; }
    int nonleaf_begin(int l) const { return topo.nonleaf_begin[l]; }
    int ghost_begin(int l) const { return topo.ghost_begin[l]; }
};

struct MuArgs {
    float* X;
    float* RHS;
    float* X0;
    // the mixed-precision cycle: x, rhs and saved x of levels >= 3 in BF16 planes (null: float)
    void* X16 = nullptr;
    void* RHS16 = nullptr;
    void* X016 = nullptr;
    int coeff_ch, mu, level_iters, coarsest_iters;
    int finest_level = -1, finest_iters = -1;  // sweeps on the finest level when >= 0 (levels >= 3)
    double omega;
    float Rr, P;
};

struct Net;

struct TuneCandidate {
    double omega;
    int mu, level_iters, coarsest_iters, finest_iters;
};

// AMGSolver (src/AMGSolver.h:19-75)
struct Solver {
    int coeff_ch;
    float R_matrix, R_restrict, P;
    double omega = 1.5;
    int mu = 2;
    int finest_iters = -1;  // sweeps on the finest level (-1: level_iters, as the reference)

    double* partial = nullptr;
    double* partial2 = nullptr;
    int partial_cap = 0;
    PcgScalars* s = nullptr;
    PcgScalars* h_s = nullptr;  // pinned mirror
    cudaStream_t cap_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.0f;
    bool conditional_ok = true;

    struct Key {
        const Grid* g;
        unsigned long long version;
        int level_iters, coarsest_iters, pure_neumann, mu, sync;
        double omega;
        bool operator<(const Key& o) const {
            return std::tie(g, version, level_iters, coarsest_iters, pure_neumann, mu, sync, omega) <
                   std::tie(o.g, o.version, o.level_iters, o.coarsest_iters, o.pure_neumann, o.mu, o.sync, o.omega);
        }
    };
    struct Plan {
        cudaGraphExec_t exec;
        int k_pre, k_body, k_if;  // kernel nodes before the loop, per iteration, in the per-iteration IF body
    };
    std::map<Key, Plan> graphs;
    static constexpr size_t kMaxCachedGraphs = 64;
    long long last_launches = 0;

    Solver(int c, float rm, float rr, float p) : coeff_ch(c), R_matrix(rm), R_restrict(rr), P(p) {}
    // GMGSolver(one_over_alpha, prolong_coeff) / CMGSolver(...) (src/GMGSolver.h:21, src/CMGSolver.h:21)
    Solver(int kind_, float one_over_alpha, float prolong) : coeff_ch(0), R_matrix(1), R_restrict(one_over_alpha), P(prolong), kind(kind_) {}
    int kind = kAMG;
    void enqueue_geo_full_neg_lap(Grid& G, float* X, float* AX, cudaStream_t st) const;
    void enqueue_geo_gs(Grid& G, int level, int iters, int order, float* X, const float* RHS, cudaStream_t st) const;
    void enqueue_geo_vcycle(Grid& G, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters, cudaStream_t st) const;
    void enqueue_geo_full_neg_lap_diag(Grid& G, float* X, float* D, cudaStream_t st) const;
    // AMGSolver::FASMuCycleSolve and GMGSolver::dampedJacobiSolve: host-driven iterations
    int fas_mu_cycle_solve(Grid& G, int repeat_times, int max_iters, double tol, int level_iters, int coarsest_iters, int* iters, double* rel);
    int damped_jacobi_solve(Grid& G, int max_iters, double tol, float omega, int* iters, double* rel);
    int host_dot(Grid& G, const int* list, int nlist, const float* A, const float* B, double* out);
    // z = M r with the solver's preconditioner (AMG: FAS mu-cycle; GMG/CMG: V-cycle), channel 3 as scratch
    void enqueue_precond(Grid& G, const Key& k, cudaStream_t st) const;
    ~Solver();
    int init();
    int ensure_scratch(int nleaf);
    ReduceScratch scratch() const { return ReduceScratch{partial, partial2, s}; }
    MuArgs mu_args(Grid& G, int x_ch, int rhs_ch, int x0_ch, int level_iters, int coarsest_iters) const;
    // pipelined: the x plane is known to be masked to INTERIOR cells (inside the cycle)
    void enqueue_gs(Grid& G, int level, int iters, int order, float* X, const float* RHS, cudaStream_t st, bool pipelined = false,
                    void* X16 = nullptr, const void* RHS16 = nullptr) const;
    void enqueue_mu_step(Grid& G, int level, const MuArgs& A, cudaStream_t st, bool fas2 = false) const;
    void enqueue_mu_cycle(Grid& G, const MuArgs& A, cudaStream_t st) const;
    // AMGSolver::VCycle (src/AMGSolver.cu:1060-1128) and muCycle (:1151-1174): correction
    // schemes from x = 0 with right-hand side f (channel F, read only) and working rhs RHS
    void enqueue_vcycle_cs(Grid& G, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters, cudaStream_t st) const;
    void enqueue_mu_cycle_cs(Grid& G, int repeat_times, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters,
                             cudaStream_t st) const;
    void enqueue_mu_step_cs(Grid& G, int level, int repeat_times, float* X, const float* F, float* RHS, int level_iters,
                            int coarsest_iters, cudaStream_t st) const;
    // AMGSolver::FASFCycle (src/AMGSolver.cu:1358-1387): the rhs restricted to every level, the
    // coarsest level smoothed, then prolongation and one FASMuCycleStep per level, coarse to fine
    void enqueue_fas_f_cycle(Grid& G, const MuArgs& A, cudaStream_t st) const;
    bool use_graph = true;    // false: launch kernel by kernel from the host (profiling)
    bool use_persist = false;  // levels 2-3 in one cooperative kernel per visit
    bool use_cluster = true;   // levels 0-2 in one cluster launch per visit of level 2
    bool cluster_ok = false;   // the device can run that cluster
    bool use_pipe = true;      // pipelined smoothing kernel inside the cycle
    bool pipe_ok = false;      // the device can run it
    void* cluster_pack = nullptr;  // packed static operands of levels 0-2 (launch_cluster_pack)
    // storage of the operator planes the pipelined smoother reads (kStorageFP32/BF16/FP16);
    // 16-bit modes read coeff16, a copy made once per solve or cycle by enqueue_operand_pack
    int storage = kStorageFP32;
    // learned finest-level smoother (a copy of a Net's packed operands); H = 0: none
    struct LearnedOps {
        int H = 0;
        bool enabled = false;
        void* pack = nullptr;
        float* bias = nullptr;
    } lnet;
    bool learned_suspended = false;  // the plain fallback solve of a learned solve
    float* aux = nullptr;            // plane-sized scratch of the learned solve
    float* bsave = nullptr;          // its right-hand side, kept for the true-residual judge
    size_t aux_cap = 0;
    double last_true_rel = -1.0;
    int last_fallback = 0, last_learned_iters = 0;
    bool learned_active() const { return lnet.enabled && kind == kAMG && !learned_suspended; }
    int set_learned(const Net* net);
    // a learned solve stops as stalled (and the plain solve takes over) when its residual norm
    // has fallen by less than 2x over this many iterations
    static constexpr int kLearnedStallWindow = 4;
    // a learned solve passes when its true relative residual is at most this many times tol:
    // the FP32 operator apply itself leaves the plain solve of the adaptive sphere octree at
    // 3.5 tol, so a tighter bound would reject sound solves
    static constexpr double kLearnedJudgeSlack = 10.0;
    int ensure_aux(const Grid& G);
    // FP64 true-residual replacement every `replace_every` PCG iterations (0: off, the
    // reference's recurrence); bkeep holds the solve's right-hand side for it
    int replace_every = 0;
    float* bkeep = nullptr;
    size_t bkeep_cap = 0;
    int last_replaced = 0;
    int ensure_bkeep(const Grid& G);
    bool replacing() const { return replace_every > 0 && kind == kAMG; }
    // BF16 storage of the cycle's x and rhs on levels >= 3 (mixed-precision mode); three
    // BF16 planes (x, rhs, saved x) of the grid's size
    bool cycle_bf16 = false;
    void* x16 = nullptr;
    size_t x16_cap = 0;
    int ensure_x16(const Grid& G);
    bool cycle16_active(const Grid& G) const;
    // direct coarsest solve inside the cluster step (mixed-precision mode): the inverse of
    // the 8^3 root operator in double, from an FP64 Cholesky factor formed on the host
    // whenever the root's operator changes; null or off: the reference's sweeps
    bool coarsest_direct = false;
    double* root_inv = nullptr;
    std::vector<float> root_ops;  // the root operator the inverse was formed from
    int prepare_root_inverse(Grid& G);
    void* coeff16 = nullptr;
    size_t coeff16_cap = 0;
    int ensure_coeff16(const Grid& G);
    // once per solve or cycle: the cluster step's packed operands and the 16-bit operator copy
    void enqueue_operand_pack(Grid& G, cudaStream_t st) const;
    bool cluster_active(const Grid& G) const;
    void enqueue_cluster_pack(Grid& G, cudaStream_t st) const;
    int persist_nblocks = 0;
    unsigned int* bar = nullptr;  // grid-barrier words of the persistent kernel
    unsigned int* h_bar = nullptr;
    void enqueue_pre(Grid& G, const Key& k, cudaGraphConditionalHandle loop_h, bool graph, cudaStream_t st) const;
    void enqueue_body(Grid& G, cudaGraphConditionalHandle loop_h, cudaGraphConditionalHandle body_h, bool graph, cudaStream_t st) const;
    void enqueue_tail(Grid& G, const Key& k, cudaStream_t st) const;
    int build_graph(Grid& G, const Key& k, Plan* out);
    int solve(Grid& G, bool verbose, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride,
              bool pure_neumann, int* iters, double* rel);
    // Autotuner: times solves of the grid's current rhs (channel 1) under each candidate
    // (omega, mu, level_iters, coarsest_iters), keeps the fastest that converges and sets its
    // omega and mu on the solver.  ms[i] = best of `repeats` timed solves (-1: not converged).
    int autotune(Grid& G, int n, const TuneCandidate* c, int max_iters, double tol, int repeats, float* ms, int* iters, int* best);
    // solve() in two halves, for batches of independent solves: solve_begin enqueues the whole
    // solve and the read-back of its scalars on the grid's stream and returns; solve_finish
    // waits for that stream and computes (iters, rel) as solve() does
    int solve_begin(Grid& G, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride, bool pure_neumann);
    int solve_finish(bool verbose, int* iters, double* rel);
    struct Pending {
        bool active = false;
        cudaStream_t stream = nullptr;
        int sync_stride = 0;
        Plan plan{};
        long long stream_launches = -1;
    } pending;
};

// The learned finest-level smoother's network (learned.cu) with its parameters, Adam state
// and training samples on the device.
struct Net {
    int H = 0, np = 0;
    float* p = nullptr;  // fp32 parameters
    float* m = nullptr;  // Adam moments
    float* v = nullptr;
    int adam_step = 0;
    int loss_kind = 0;     // 0: squared error; 1: energy (tile Laplacian-weighted)
    void* pack = nullptr;  // bf16 operands made from p
    float* bias = nullptr;
    int ns = 0;  // training samples: tiles of 512 cells
    float* rho = nullptr;
    float* diag = nullptr;
    uint8_t* types = nullptr;
    float* target = nullptr;
    float* grad = nullptr;  // per batch slot (the residual net: per training block)
    float* loss = nullptr;  // per sample
    float* gsum = nullptr;
    int* idx = nullptr;
    int batch_cap = 0;
    void* scratch = nullptr;  // the residual net's per-block training scratch
    cudaStream_t st = nullptr;
    ~Net();
    int init(int hidden, unsigned long long seed);
    int set_params(const float* host);
    int get_params(float* host);
    // faces: [n][3][512] -x/-y/-z face coefficients, halo: [n][768] (NetExtra's layout); either may be null
    float* faces = nullptr;
    float* halo = nullptr;
    int set_samples(int n, const float* rho, const float* diag, const uint8_t* types, const float* target, const float* faces_h = nullptr,
                    const float* halo_h = nullptr);
    NetExtra extra(int first) const;
    int forward(int first, int n, float* out_host);
    int gradient(int first, int n, double* loss_out, float* grad_host);
    int train(int epochs, int batch, float lr, unsigned long long seed, float* epoch_loss);
    int ensure_batch(int nb);
};

// Many octrees solved by one persistent cooperative launch inside a CUDA graph
// (batch_persist.cu).  Each instance is a grid with the AMG solver whose settings (omega,
// mu, coefficient channel, finest-level sweeps) it is solved with; the solver objects only
// carry settings here, the batch owns all scratch.
// The schedule: groups of `group_blocks` blocks take octrees from a shared queue, largest
// first.  With split > 0 the octrees too large for such a group get a group of their own,
// sized so that it ends in about split x (total work / resident blocks); the work of each
// octree is its measured block-time from the last autotune, else a cycle-work estimate.
struct Batch {
    std::vector<Solver*> solvers;
    std::vector<Grid*> grids;
    int device = 0;
    int slots = 4;         // 128-thread slots per block: 4, 6 or 8
    int group_blocks = 0;  // 0: automatic (the resident blocks spread over the instances)
    double split = 0.0;
    int last_plan_gs = 0;
    std::vector<double> weight;  // block-ms per instance, measured by autotune (empty: estimate)
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    BatchInst* d_inst = nullptr;
    BatchInst* h_inst = nullptr;  // pinned
    int* d_order = nullptr;
    int* h_order = nullptr;  // pinned
    BatchGroup* d_groups = nullptr;
    BatchGroup* h_groups = nullptr;  // pinned
    int* d_block_group = nullptr;
    int* h_block_group = nullptr;  // pinned
    unsigned int* d_ctl = nullptr;
    unsigned int* h_ctl = nullptr;  // pinned: the error word read back
    size_t ctl_words = 0;
    double* d_part = nullptr;
    size_t part_cap = 0;  // doubles
    PcgScalars* d_s = nullptr;
    PcgScalars* h_s = nullptr;  // pinned
    unsigned long long* d_clock = nullptr;
    unsigned long long* h_clock = nullptr;  // pinned, 4 per instance
    cudaGraphExec_t exec = nullptr;
    struct GraphKey {
        int slots, nblocks, ngroups, dyn_begin, max_iters, sync_stride, pure_neumann, level_iters, coarsest_iters;
        double tol;
        bool operator==(const GraphKey& o) const {
            return std::tie(slots, nblocks, ngroups, dyn_begin, max_iters, sync_stride, pure_neumann, level_iters, coarsest_iters, tol) ==
                   std::tie(o.slots, o.nblocks, o.ngroups, o.dyn_begin, o.max_iters, o.sync_stride, o.pure_neumann, o.level_iters,
                            o.coarsest_iters, o.tol);
        }
    } key{};
    float last_ms = 0.0f;
    int last_nblocks = 0, last_groups = 0, last_dedicated = 0;
    ~Batch();
    int init(Solver* const* s, Grid* const* g, int n);
    // the plan a run uses: groups (h_groups, h_block_group), queue order (h_order), the first
    // shared-queue position; returns the blocks launched (0: none resident)
    int plan(const std::vector<double>& w, int* ngroups, int* dyn_begin, int* dedicated);
    // the plan a run would use: slots per block, small groups' size, groups, dedicated groups,
    // resident blocks
    int schedule(int* ns, int* G, int* groups, int* dedicated, int* resident);
    int run(const float* const* b_host, float* const* x_host, int max_iters, double tol, int level_iters, int coarsest_iters,
            int sync_stride, bool pure_neumann, int* iters, double* rel, float* instance_ms);
    // One calibration run measures each octree's block-time; then the batch is timed under
    // each candidate schedule (slots[i], group_blocks[i], split[i]), best of `repeats` runs after one
    // untimed run, every run from the right-hand sides the grids held on entry (restored
    // afterwards); the fastest whose solves all converge is kept.
    int autotune(const int* slots_c, const int* cand, const double* split_c, int ncand, int max_iters, double tol, int level_iters,
                 int coarsest_iters, int sync_stride, int repeats, float* ms, int* best);
};

int check_cuda(cudaError_t e, const char* what);
int validate_solver_topology(const Grid& G);

}  // namespace cmg
