// Device octree and AMG solver (see cmg_impl.hpp).
#include "cmg_impl.hpp"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <unordered_map>

namespace cmg {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
const char* last_error() { return g_err.c_str(); }

int check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return 0;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return 2;
}
#define CK(call)                                      \
    do {                                              \
        int _rc = check_cuda((call), #call);          \
        if (_rc) return _rc;                          \
    } while (0)

template <class T>
static void dfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// The channel planes and cell types of grids come from a stream-ordered pool per device
// that keeps freed memory: an octree rebuilt for every position of a moving obstacle (a
// new grid or a new topology each time) reuses the same few hundred MB instead of
// mapping fresh memory each time.
static cudaError_t plane_pool(int dev, cudaMemPool_t* out) {
    static std::mutex m;
    static std::unordered_map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(m);
    auto it = pools.find(dev);
    if (it != pools.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    unsigned long long keep = ~0ull;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
    pools.emplace(dev, pool);
    *out = pool;
    return cudaSuccess;
}
cudaError_t pool_malloc(void** p, size_t bytes, int dev, cudaStream_t st) {
    cudaMemPool_t pool;
    cudaError_t e = plane_pool(dev, &pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}
void pool_release(void* p, cudaStream_t st) {
    if (p) cudaFreeAsync(p, st);
}
template <class T>
static cudaError_t pool_alloc(T** p, size_t bytes, int dev, cudaStream_t st) {
    cudaMemPool_t pool;
    cudaError_t e = plane_pool(dev, &pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync((void**)p, bytes, pool, st);
}
template <class T>
static void pool_free(T*& p, cudaStream_t st) {
    pool_release((void*)p, st);
    p = nullptr;
}

static int plane_class_tiles(int n) {
    if (n <= 64) return n;
    int p = 64;
    while (p * 2 <= n) p *= 2;
    const int q = p / 16;
    return (n + q - 1) / q * q;
}

Grid::~Grid() {
    // cudaFree synchronised the device here before the planes came from a pool; keep that,
    // so that no work of the grid's stream still reads them, then free on the legacy stream
    // (the caller's stream may be gone by now)
    if (chan || ctype || meta) cudaDeviceSynchronize();
    pool_free(chan, nullptr);
    pool_free(ctype, nullptr);
    pool_free(meta, nullptr);
    pool_free(nb, nullptr);
    pool_free(child, nullptr);
    pool_free(nbx, nullptr);
    pool_free(leaf, nullptr);
    dfree(spheres);
    dfree(modes);
    dfree(dot_out);
    dfree(tile_ptrs);
    delete topo_builder;
}

static unsigned long long tile_key(const TileRec& r) {
    return ((unsigned long long)(r.level & 0xff) << 56) | ((unsigned long long)((r.c[0] + 4) & 0x3ffff) << 36) |
           ((unsigned long long)((r.c[1] + 4) & 0x3ffff) << 18) | (unsigned long long)((r.c[2] + 4) & 0x3ffff);
}

// HADeviceGrid::rebuild (src/HAGrid.h:892): spawn ghosts, put the tiles in
// device order and build the tables (host side only).
int Grid::rebuild() {
    topo.spawn_ghosts();
    topo.canonicalize();
    built = true;
    ++host_version;
    return 0;
}

int Grid::refine_case_device(int case_id, const double* params, int nparams, int* steps) {
    if (!device_case_supported(case_id)) {
        const float h0 = topo.h0();
        std::vector<double> prm(params, params + nparams);
        const int st = topo.iterative_refine([&](int level, int i, int j, int k) {
            const int c[3] = {i, j, k};
            return case_target(case_id, prm.data(), (int)prm.size(), h0, level, c);
        });
        if (steps) *steps = st;
        return rebuild();
    }
    if (!topo_builder) topo_builder = new DeviceTopoBuilder();
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) {
        set_error("refine_case_device: no CUDA device");
        return 2;
    }
    topo_builder->dev = device;
    const int rc = device_refine_case(*topo_builder, topo, case_id, params, nparams, stream, steps);
    if (rc == 1) {
        set_error("refine_case_device: bad parameters");
        return 1;
    }
    if (rc) {
        set_error("refine_case_device: CUDA error in the device octree builder");
        return 2;
    }
    built = true;
    ++host_version;
    return 0;
}

// syncHostAndDevice (src/HAGrid.h:653): allocate the channel planes of the
// current topology and upload its tables.  Tiles that already had device
// storage keep their channel values and cell types; new tiles start at zero.
int Grid::ensure_device() {
    if (!built) {
        set_error("grid not built: call rebuild or refine first");
        return 3;
    }
    if (dev_version == host_version && n > 0) return 0;
    const int n_old = n;
    const int n_new = topo.size();
    std::unordered_map<unsigned long long, int> old_index;
    old_index.reserve(2 * dev_keys.size() + 1);
    for (int t = 0; t < (int)dev_keys.size(); ++t) old_index.emplace(dev_keys[t], t);
    // where each tile's data comes from (src/HAGrid.h:1140-1160, PoissonTile.h:151-172):
    // a tile that survives keeps its own (a LEAF that became NONLEAF included); a LEAF or
    // NONLEAF tile made by refinement -- new, or a GHOST it replaced -- starts from its
    // nearest surviving LEAF/NONLEAF ancestor, s levels up, each cell taking the value and
    // type of the ancestor cell that contains it (childTile applied s times); a new GHOST
    // tile starts at zero
    std::vector<int2> src_of_new(n_new);
    std::vector<unsigned long long> keys(n_new);
    for (int t = 0; t < n_new; ++t) {
        const TileRec& r = topo.tiles()[t];
        keys[t] = tile_key(r);
        auto it = old_index.find(keys[t]);
        src_of_new[t] = make_int2(-1, 0);
        if (it != old_index.end() && (dev_types[it->second] != kGhost || r.type == kGhost)) {
            src_of_new[t] = make_int2(it->second, 0);
        } else if (r.type != kGhost) {
            for (int sh = 1; sh <= r.level; ++sh) {
                const TileRec a{r.level - sh, {r.c[0] >> sh, r.c[1] >> sh, r.c[2] >> sh}, 0};
                auto ia = old_index.find(tile_key(a));
                if (ia != old_index.end() && dev_types[ia->second] != kGhost) {
                    src_of_new[t] = make_int2(ia->second, sh);
                    break;
                }
            }
        }
    }
    std::vector<int4> hm(n_new);
    for (int t = 0; t < n_new; ++t) {
        const TileRec& r = topo.tiles()[t];
        hm[t] = make_int4(r.level | (r.type << 8), r.c[0], r.c[1], r.c[2]);
    }

    float* chan_new = nullptr;
    uint8_t* ct_new = nullptr;
    const size_t cells = (size_t)n_new * kCells;
    // the allocations are rounded up to a size class (a sixteenth of the power of two at or
    // below the tile count, at most 6 % more): octrees of nearly the same size, rebuilt one
    // after another, then ask the pool for the same sizes and take back the same blocks
    const size_t cap_cells = (size_t)plane_class_tiles(n_new) * kCells;
    if (device < 0) CK(cudaGetDevice(&device));
    CK(pool_alloc(&chan_new, sizeof(float) * cap_cells * nch + 16, device, stream));
    CK(pool_alloc(&ct_new, cap_cells + 16, device, stream));
    // the tables come from the pool too, and the copies are stream-ordered (a pageable
    // source is staged before cudaMemcpyAsync returns)
    int2* d_map = nullptr;
    int4* d_meta = nullptr;
    CK(pool_alloc(&d_map, sizeof(int2) * (n_new + 1), device, stream));
    CK(pool_alloc(&d_meta, sizeof(int4) * (n_new + 1), device, stream));
    CK(cudaMemcpyAsync(d_map, src_of_new.data(), sizeof(int2) * n_new, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(d_meta, hm.data(), sizeof(int4) * n_new, cudaMemcpyHostToDevice, stream));
    if (n_old > 0) {
        launch_remap(chan, chan_new, d_map, d_meta, n_new, nch, n_old, stream);
        launch_remap_types(ctype, ct_new, d_map, d_meta, n_new, stream);
    } else {
        CK(cudaMemsetAsync(chan_new, 0, sizeof(float) * cells * nch, stream));
        CK(cudaMemsetAsync(ct_new, 0, cells, stream));
    }
    CK(cudaStreamSynchronize(stream));
    CK(cudaGetLastError());
    pool_free(d_map, stream);
    // the old planes and tables may still be read by work on other streams (a solver's, a
    // net's): wait for the device, as cudaFree did, before they go back to the pool
    if (chan || meta) CK(cudaDeviceSynchronize());
    pool_free(chan, stream);
    pool_free(ctype, stream);
    chan = chan_new;
    ctype = ct_new;

    std::vector<int> hx((size_t)8 * n_new, 0);
    for (int t = 0; t < n_new; ++t)
        for (int f = 0; f < 6; ++f) {
            const int q = topo.nb[8 * t + f];
            if (q >= 0) hx[8 * t + f] = ((q + 1) << 3) | topo.tiles()[q].type;
        }
    pool_free(meta, stream);
    meta = d_meta;
    pool_free(nb, stream);
    pool_free(child, stream);
    pool_free(nbx, stream);
    pool_free(leaf, stream);
    CK(pool_alloc(&nbx, sizeof(int) * 8 * (n_new + 1), device, stream));
    CK(cudaMemcpyAsync(nbx, hx.data(), sizeof(int) * 8 * n_new, cudaMemcpyHostToDevice, stream));
    CK(pool_alloc(&nb, sizeof(int) * 8 * (n_new + 1), device, stream));
    CK(pool_alloc(&child, sizeof(int) * 8 * (n_new + 1), device, stream));
    CK(pool_alloc(&leaf, sizeof(int) * (topo.leaf_list.size() + 1), device, stream));
    CK(cudaMemcpyAsync(nb, topo.nb.data(), sizeof(int) * 8 * n_new, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(child, topo.child.data(), sizeof(int) * 8 * n_new, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(leaf, topo.leaf_list.data(), sizeof(int) * topo.leaf_list.size(), cudaMemcpyHostToDevice, stream));
    // callers read the tables on other streams or from the host right after this
    CK(cudaStreamSynchronize(stream));
    n = n_new;
    nleaf = (int)topo.leaf_list.size();
    dev_keys.swap(keys);
    dev_types.resize(n_new);
    for (int t = 0; t < n_new; ++t) dev_types[t] = topo.tiles()[t].type;
    dev_version = host_version;
    // process-wide unique: a solver's cached graphs are keyed by (grid address, version), and a
    // grid created after another was destroyed may reuse its address
    static std::atomic<unsigned long long> next_version{0};
    version = ++next_version;
    return 0;
}

// The stencil kernels rely on three properties of a tree built by
// refineStep + spawnGhostTiles; a grid assembled by hand is checked here.
//  1. every GHOST tile has a LEAF parent tile;
//  2. where a LEAF tile touches a same-level NONLEAF tile, the NONLEAF cells on
//     that face have LEAF children (the reference reads them after a one-step
//     children-to-parent average, src/AMGSolver.cu:607);
//  3. levels 0 and 1 hold no GHOST tiles (they run in the coarse kernel).
int validate_solver_topology(const Grid& G) {
    const auto& T = G.topo.tiles();
    for (int t = 0; t < G.n; ++t) {
        const TileRec& r = T[t];
        if (r.type == kGhost) {
            const int p = G.topo.nb[8 * t + 6];
            if (p < 0 || !(T[p].type & kLeaf)) {
                set_error("GHOST tile without a LEAF parent");
                return 4;
            }
            if (r.level <= 1) {
                set_error("GHOST tile on level 0 or 1");
                return 4;
            }
        }
        if (r.type != kLeaf) continue;
        for (int a = 0; a < 6; ++a) {
            const int q = G.topo.nb[8 * t + a];
            if (q < 0 || T[q].type != kNonLeaf) continue;
            const int axis = a % 3, plus = a / 3;
            for (int ci = 0; ci < 8; ++ci) {
                const int bit = axis == 0 ? (ci >> 2) : axis == 1 ? ((ci >> 1) & 1) : (ci & 1);
                if (bit != (plus ? 0 : 1)) continue;  // children on the shared face
                const int c = G.topo.child[8 * q + ci];
                if (c < 0 || T[c].type != kLeaf) {
                    set_error("octree is not 2:1 face-balanced next to a LEAF tile");
                    return 4;
                }
            }
        }
    }
    return 0;
}

Solver::~Solver() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
    dfree(partial);
    dfree(partial2);
    dfree(s);
    if (cluster_pack) cudaFree(cluster_pack);
    dfree(coeff16);
    dfree(lnet.pack);
    dfree(lnet.bias);
    dfree(aux);
    dfree(bsave);
    dfree(bkeep);
    dfree(root_inv);
    dfree(x16);
    if (h_s) cudaFreeHost(h_s);
    if (h_bar) cudaFreeHost(h_bar);
    dfree(bar);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
}

int Solver::init() {
    CK(cudaMalloc(&s, sizeof(PcgScalars)));
    CK(cudaMemset(s, 0, sizeof(PcgScalars)));
    CK(cudaMallocHost(&h_s, sizeof(PcgScalars)));
    std::memset(h_s, 0, sizeof(PcgScalars));
    CK(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    CK(cudaMalloc(&bar, sizeof(unsigned int) * 4));
    CK(cudaMemset(bar, 0, sizeof(unsigned int) * 4));
    CK(cudaMallocHost(&h_bar, sizeof(unsigned int) * 4));
    init_kernel_attributes();
    persist_nblocks = persist_blocks();
    if (persist_nblocks <= 0) use_persist = false;
    cluster_ok = cluster_step_supported();
    pipe_ok = gs_pipe_init() > 0;
    if (cluster_ok) CK(cudaMalloc(&cluster_pack, cluster_pack_bytes()));
    return check_cuda(cudaGetLastError(), "kernel attributes");
}

int Solver::ensure_scratch(int nl) {
    if (nl <= partial_cap) return 0;
    dfree(partial);
    dfree(partial2);
    CK(cudaMalloc(&partial, sizeof(double) * (nl + 1)));
    CK(cudaMalloc(&partial2, sizeof(double) * (nl + 1)));
    partial_cap = nl;
    // captured graphs hold the old scratch pointers
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
    graphs.clear();
    return 0;
}

MuArgs Solver::mu_args(Grid& G, int x_ch, int rhs_ch, int x0_ch, int level_iters, int coarsest_iters) const {
    MuArgs A;
    A.X = G.plane(x_ch);
    A.RHS = G.plane(rhs_ch);
    A.X0 = G.plane(x0_ch);
    A.coeff_ch = coeff_ch;
    A.mu = mu;
    A.level_iters = level_iters;
    A.coarsest_iters = coarsest_iters;
    A.finest_level = G.max_level();
    A.finest_iters = finest_iters;
    A.omega = omega;
    A.Rr = R_restrict;
    A.P = P;
    return A;
}

// GaussSeidelAMG (src/AMGSolver.cu:887-894) on the LEAF and NONLEAF tiles of one level
void Solver::enqueue_gs(Grid& G, int level, int iters, int order, float* X, const float* RHS, cudaStream_t st, bool pipelined,
                        void* X16, const void* RHS16) const {
    const DevGrid d = G.dev();
    const int t0 = G.level_begin(level), nt = G.ghost_begin(level) - t0;
    const bool pipe = pipelined && use_pipe && pipe_ok;
    for (int it = 0; it < iters; ++it)
        for (int h = 0; h < 2; ++h) {
            const int color = h ? 1 - order : order;
            const int stg = kind == kAMG ? storage : kStorageFP32;
            if (X16) launch_gs_pipe(d, t0, nt, X16, RHS16, true, coeff_ch, color, omega, st, stg, coeff16);
            else if (pipe) launch_gs_pipe(d, t0, nt, X, RHS, false, coeff_ch, color, omega, st, stg, coeff16);
            else launch_gs(d, t0, nt, X, RHS, coeff_ch, color, omega, st);
        }
}

// Levels 0-2 are complete 8^3, 16^3 and 32^3 grids: a NONLEAF root, eight
// NONLEAF children and 64 grandchildren, none of them GHOST.
static bool coarse_levels_complete(const Grid& G) {
    if (G.max_level() < 2) return false;
    for (int l = 0; l <= 1; ++l)
        if (G.level_end(l) - G.level_begin(l) != (l ? 8 : 1) || G.nonleaf_begin(l) != G.level_begin(l) || G.ghost_begin(l) != G.level_end(l))
            return false;
    return G.ghost_begin(2) - G.level_begin(2) == 64 && G.level_end(2) == G.ghost_begin(2);
}

// the 8 level-1 tiles (root child order) and the 64 level-2 tiles by 4x4x4 tile position
static void coarse_tiles(const Grid& G, int* tile1, int* tile2) {
    const std::vector<int>& ch = G.topo.child;
    for (int c = 0; c < 8; ++c) tile1[c] = ch[c];  // the root is tile 0
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b)
            for (int c = 0; c < 4; ++c)
                tile2[a * 16 + b * 4 + c] = ch[8 * tile1[((a >> 1) << 2) | ((b >> 1) << 1) | (c >> 1)] + (((a & 1) << 2) | ((b & 1) << 1) | (c & 1))];
}

bool Solver::cluster_active(const Grid& G) const { return use_cluster && cluster_ok && coarse_levels_complete(G); }

// pack the static operands of levels 0-2 for the cluster step (coefficients and
// cell types are fixed for the duration of a solve)
void Solver::enqueue_cluster_pack(Grid& G, cudaStream_t st) const {
    if (!cluster_active(G)) return;
    int tile1[8], tile2[64];
    coarse_tiles(G, tile1, tile2);
    launch_cluster_pack(G.dev(), tile1, tile2, coeff_ch, cluster_pack, st);
}

// The solver keeps its own copy of the net's packed operands.  Graphs captured with the
// learned smoother read that copy, so a later set_learned with the same width only
// refreshes its contents; a new width reallocates it and drops the captured graphs.
int Solver::set_learned(const Net* net) {
    if (!net) {
        lnet.enabled = false;
        return 0;
    }
    if (!lnet.pack || lnet.H != net->H) {
        dfree(lnet.pack);
        dfree(lnet.bias);
        lnet.H = 0;
        CK(cudaMalloc(&lnet.pack, sizeof(uint16_t) * (size_t)net_pack_elems(net->H)));
        CK(cudaMalloc(&lnet.bias, sizeof(float) * net_bias_elems(net->H)));
        lnet.H = net->H;
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
        graphs.clear();
    }
    CK(cudaStreamSynchronize(net->st));
    CK(cudaMemcpy(lnet.pack, net->pack, sizeof(uint16_t) * (size_t)net_pack_elems(net->H), cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(lnet.bias, net->bias, sizeof(float) * net_bias_elems(net->H), cudaMemcpyDeviceToDevice));
    lnet.enabled = true;
    return 0;
}

int Solver::ensure_aux(const Grid& G) {
    const size_t need = (size_t)G.n * kCells;
    if (aux_cap >= need) return 0;
    dfree(aux);
    dfree(bsave);
    aux = bsave = nullptr;
    aux_cap = 0;
    CK(cudaMalloc(&aux, sizeof(float) * need));
    CK(cudaMalloc(&bsave, sizeof(float) * need));
    aux_cap = need;
    // captured graphs hold the old pointer
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
    graphs.clear();
    return 0;
}

int Solver::ensure_x16(const Grid& G) {
    const size_t need = (size_t)G.n * kCells;
    if (x16_cap >= need) return 0;
    dfree(x16);
    x16 = nullptr;
    x16_cap = 0;
    CK(cudaMalloc(&x16, 3 * 2 * need));
    x16_cap = need;
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);  // captured graphs hold the old pointer
    graphs.clear();
    return 0;
}
bool Solver::cycle16_active(const Grid& G) const {
    return cycle_bf16 && kind == kAMG && use_pipe && pipe_ok && !use_persist && !learned_active() && G.max_level() >= 3;
}

int Solver::ensure_bkeep(const Grid& G) {
    const size_t need = (size_t)G.n * kCells;
    if (bkeep_cap >= need) return 0;
    dfree(bkeep);
    bkeep = nullptr;
    bkeep_cap = 0;
    CK(cudaMalloc(&bkeep, sizeof(float) * need));
    bkeep_cap = need;
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);  // captured graphs hold the old pointer
    graphs.clear();
    return 0;
}

// The coarsest operator (the root tile, level 0: no neighbours, so every face outside it
// is a Dirichlet face with x = 0) on its INTERIOR cells, A[v][v] = diagonal and A[v][u] =
// the face coefficient between u and v, factorised A = L L^T in double and inverted as
// L^-T L^-1; the inverse goes to the device in the coarse CTA's thread order.  Rebuilt only
// when the root's operator changed since the last solve.
int Solver::prepare_root_inverse(Grid& G) {
    std::vector<float> ops((size_t)5 * kCells);
    for (int a = 0; a < 4; ++a)
        CK(cudaMemcpyAsync(&ops[(size_t)a * kCells], G.plane(coeff_ch + a), sizeof(float) * kCells, cudaMemcpyDeviceToHost, G.stream));
    std::vector<uint8_t> ty(kCells);
    CK(cudaMemcpyAsync(ty.data(), G.ctype, kCells, cudaMemcpyDeviceToHost, G.stream));
    CK(cudaStreamSynchronize(G.stream));
    for (int v = 0; v < kCells; ++v) ops[(size_t)4 * kCells + v] = (float)ty[v];
    if (root_inv && ops == root_ops) return 0;
    std::vector<int> idx(kCells, -1), cell;
    for (int v = 0; v < kCells; ++v)
        if (ty[v] == kInterior) {
            idx[v] = (int)cell.size();
            cell.push_back(v);
        }
    const int m = (int)cell.size();
    std::vector<double> A((size_t)m * m, 0.0);
    for (int r = 0; r < m; ++r) {
        const int v = cell[r];
        A[(size_t)r * m + r] = ops[(size_t)3 * kCells + v];
        const int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
        for (int a = 0; a < 3; ++a) {
            const int stride = a == 0 ? 64 : a == 1 ? 8 : 1;
            if (l[a] > 0 && idx[v - stride] >= 0) A[(size_t)r * m + idx[v - stride]] = ops[(size_t)a * kCells + v];               // -face of v
            if (l[a] < 7 && idx[v + stride] >= 0) A[(size_t)r * m + idx[v + stride]] = ops[(size_t)a * kCells + v + stride];  // -face of the upper cell
        }
    }
    // A = L L^T (lower triangle of A, in place)
    for (int j = 0; j < m; ++j) {
        double d = A[(size_t)j * m + j];
        for (int k = 0; k < j; ++k) d -= A[(size_t)j * m + k] * A[(size_t)j * m + k];
        if (!(d > 0.0)) {
            set_error("coarsest direct solve: the root operator is not positive definite");
            return 5;
        }
        const double ljj = std::sqrt(d);
        A[(size_t)j * m + j] = ljj;
        for (int i = j + 1; i < m; ++i) {
            double sum = A[(size_t)i * m + j];
            for (int k = 0; k < j; ++k) sum -= A[(size_t)i * m + k] * A[(size_t)j * m + k];
            A[(size_t)i * m + j] = sum / ljj;
        }
    }
    // W = L^-1 (lower triangular), then A^-1 = W^T W
    std::vector<double> W((size_t)m * m, 0.0);
    for (int c = 0; c < m; ++c)
        for (int i = c; i < m; ++i) {
            double sum = i == c ? 1.0 : 0.0;
            for (int k = c; k < i; ++k) sum -= A[(size_t)i * m + k] * W[(size_t)k * m + c];
            W[(size_t)i * m + c] = sum / A[(size_t)i * m + i];
        }
    std::vector<double> inv((size_t)m * m, 0.0);
    for (int r = 0; r < m; ++r)
        for (int c = 0; c <= r; ++c) {
            double sum = 0.0;
            for (int k = r; k < m; ++k) sum += W[(size_t)k * m + r] * W[(size_t)k * m + c];
            inv[(size_t)r * m + c] = inv[(size_t)c * m + r] = sum;
        }
    std::vector<double> M((size_t)kCells * kCells, 0.0);
    for (int j = 0; j < kCells; ++j) {
        const int rj = idx[cluster_thread_cell(j)];
        if (rj < 0) continue;
        for (int t = 0; t < kCells; ++t) {
            const int rt = idx[cluster_thread_cell(t)];
            if (rt >= 0) M[(size_t)j * kCells + t] = inv[(size_t)rj * m + rt];
        }
    }
    if (!root_inv) {
        CK(cudaMalloc(&root_inv, sizeof(double) * M.size()));
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);  // captured graphs hold the old pointer
        graphs.clear();
    }
    CK(cudaMemcpy(root_inv, M.data(), sizeof(double) * M.size(), cudaMemcpyHostToDevice));
    root_ops.swap(ops);
    return 0;
}

int Solver::ensure_coeff16(const Grid& G) {
    if (storage == kStorageFP32 || kind != kAMG) return 0;
    const size_t need = coeff16_bytes(G.dev());
    if (need <= coeff16_cap) return 0;
    dfree(coeff16);
    coeff16 = nullptr;
    coeff16_cap = 0;
    CK(cudaMalloc(&coeff16, need));
    coeff16_cap = need;
    // captured graphs hold the old pointer
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
    graphs.clear();
    return 0;
}

void Solver::enqueue_operand_pack(Grid& G, cudaStream_t st) const {
    if (kind != kAMG) return;
    enqueue_cluster_pack(G, st);
    if (storage != kStorageFP32) launch_coeff16(G.dev(), coeff_ch, storage, coeff16, st);
}

// AMGSolver::FASMuCycleStep (src/AMGSolver.cu:1257-1277).  A visit of level 2
// runs as one cluster launch when levels 0-2 are complete; otherwise levels 0
// and 1 run as a single coarse-kernel launch.
void Solver::enqueue_mu_step(Grid& G, int l, const MuArgs& A, cudaStream_t st, bool fas2) const {
    const DevGrid d = G.dev();
    if (l == 2 && cluster_active(G)) {
        int tile1[8], tile2[64];
        coarse_tiles(G, tile1, tile2);
        launch_cluster_step(d, tile1, tile2, cluster_pack, A.X, A.RHS, A.X0, A.coeff_ch, A.mu, A.level_iters, A.coarsest_iters, A.omega, A.Rr,
                            A.P, fas2, st, coarsest_direct ? root_inv : nullptr);
        return;
    }
    if (l <= 1) {
        launch_coarse_step(d, l, A.X, A.RHS, A.X0, A.coeff_ch, A.mu,
                           A.level_iters, A.coarsest_iters, A.omega, A.Rr, A.P, st);
        return;
    }
    if (use_persist && l <= 3) {
        int lb[4], ab[4], le[4], nlb[4];
        for (int q = 0; q < 4; ++q) {
            const bool has = q <= G.max_level();
            lb[q] = has ? G.level_begin(q) : 0;
            ab[q] = has ? G.ghost_begin(q) : 0;
            le[q] = has ? G.level_end(q) : 0;
            nlb[q] = has ? G.nonleaf_begin(q) : 0;
        }
        launch_persist_step(d, l, lb, ab, le, nlb, A.X, A.RHS, A.X0, A.coeff_ch, A.mu, A.level_iters, A.coarsest_iters, A.omega, A.Rr, A.P,
                            bar, persist_nblocks, st);
        return;
    }
    const int li = (l == A.finest_level && A.finest_iters >= 0) ? A.finest_iters : A.level_iters;
    if (A.X16 && l >= 3) {
        // the mixed-precision cycle's BF16 levels; level 2 and below stay float
        const bool p16 = l - 1 >= 3;
        void* Xp = p16 ? A.X16 : (void*)A.X;
        void* Rp = p16 ? A.RHS16 : (void*)A.RHS;
        void* X0p = p16 ? A.X016 : (void*)A.X0;
        enqueue_gs(G, l, li, 0, A.X, A.RHS, st, true, A.X16, A.RHS16);
        launch_restrict_pipe(d, G.level_begin(l), G.ghost_begin(l) - G.level_begin(l), A.X16, A.RHS16, true, Xp, Rp, p16, A.coeff_ch, A.Rr,
                             st);
        const bool fold = l - 1 == 2 && A.mu > 0 && cluster_active(G) && G.nonleaf_begin(2) == G.level_begin(2);
        const int nb0 = G.nonleaf_begin(l - 1), nbn = G.ghost_begin(l - 1) - nb0;
        if (p16) launch_fas_pipe_x16(d, nb0, nbn, A.X16, A.RHS16, A.X016, A.coeff_ch, st);
        else if (!fold) launch_fas_save(d, nb0, nbn, A.X, A.RHS, A.X0, A.coeff_ch, st);
        for (int r = 0; r < A.mu; ++r) enqueue_mu_step(G, l - 1, A, st, fold && r == 0);
        launch_prolong_x16(d, G.level_begin(l), G.level_end(l) - G.level_begin(l), A.X16, Xp, X0p, p16, A.P, st);
        enqueue_gs(G, l, li, 1, A.X, A.RHS, st, true, A.X16, A.RHS16);
        return;
    }
    enqueue_gs(G, l, li, 0, A.X, A.RHS, st, true);
    if (use_pipe && pipe_ok)
        launch_restrict_pipe(d, G.level_begin(l), G.ghost_begin(l) - G.level_begin(l), A.X, A.RHS, false, A.X, A.RHS, false, A.coeff_ch,
                             A.Rr, st);
    else
        launch_restrict(d, G.level_begin(l), G.ghost_begin(l) - G.level_begin(l), A.X, A.RHS, A.coeff_ch, A.Rr, st);
    // the first cluster launch of level 2 does level 2's FAS update itself when every level-2 tile is NONLEAF
    const bool fold = l - 1 == 2 && A.mu > 0 && cluster_active(G) && G.nonleaf_begin(2) == G.level_begin(2);
    if (!fold) launch_fas_save(d, G.nonleaf_begin(l - 1), G.ghost_begin(l - 1) - G.nonleaf_begin(l - 1), A.X, A.RHS, A.X0, A.coeff_ch, st);
    for (int r = 0; r < A.mu; ++r) enqueue_mu_step(G, l - 1, A, st, fold && r == 0);
    launch_prolong(d, G.level_begin(l), G.level_end(l) - G.level_begin(l), A.X, A.X0, A.P, st);
    enqueue_gs(G, l, li, 1, A.X, A.RHS, st, true);
}

// GaussSeidelGMG / GaussSeidelCMG (src/GMGSolver.cu:217-223, src/CMGSolver.cu:271-276)
void Solver::enqueue_geo_gs(Grid& G, int level, int iters, int order, float* X, const float* RHS, cudaStream_t st) const {
    const DevGrid d = G.dev();
    const int t0 = G.level_begin(level), nt = G.ghost_begin(level) - t0;
    for (int it = 0; it < iters; ++it) {
        launch_geo_gs(kind, d, t0, nt, X, RHS, order, st);
        launch_geo_gs(kind, d, t0, nt, X, RHS, 1 - order, st);
    }
}

// GMGSolver::VCycle (src/GMGSolver.cu:324-388), CMGSolver::VCycle (src/CMGSolver.cu:377-416).
// GMG restricts from and prolongs into the GHOST tiles of a level as well; CMG does not.
void Solver::enqueue_geo_vcycle(Grid& G, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters, cudaStream_t st) const {
    const DevGrid d = G.dev();
    launch_geo_vinit(d, X, RHS, F, st);
    const int top = G.max_level();
    for (int i = top; i > 0; --i) {
        enqueue_geo_gs(G, i, level_iters, 0, X, RHS, st);
        const int t0 = G.level_begin(i), t1 = kind == kGMG ? G.level_end(i) : G.ghost_begin(i);
        launch_geo_restrict(kind, d, t0, t1 - t0, X, RHS, R_restrict, st);
    }
    enqueue_geo_gs(G, 0, coarsest_iters / 2, 0, X, RHS, st);
    enqueue_geo_gs(G, 0, coarsest_iters / 2, 1, X, RHS, st);
    for (int i = 1; i <= top; ++i) {
        const int t0 = G.level_begin(i), t1 = kind == kGMG ? G.level_end(i) : G.ghost_begin(i);
        launch_geo_prolong(d, t0, t1 - t0, X, P, st);
        enqueue_geo_gs(G, i, level_iters, 1, X, RHS, st);
    }
}

// FullNegativeLaplacian (src/GMGSolver.cu:167-171): GHOST x from the parents, the operator
// on LEAF and GHOST tiles, GHOST results added into their LEAF parents.
// ConservativeFullNegativeLaplacian (src/CMGSolver.cu:210-222): GHOST x from the parents,
// NONLEAF x as the mean of the LEAF children, the operator on LEAF tiles.
void Solver::enqueue_geo_full_neg_lap(Grid& G, float* X, float* AX, cudaStream_t st) const {
    const DevGrid d = G.dev();
    const int ch = (int)((X - G.chan) / ((size_t)G.n * kCells));
    launch_propagate_ghost(d, 0, G.n, ch, st);
    if (kind == kCMG) launch_accumulate_cells(d, 0, G.n, dLeaf, X, X, 0.125f, false, st);
    launch_geo_lap(kind, d, 0, G.n, X, AX, false, kind == kGMG ? (dLeaf | dGhost) : dLeaf, st);
    if (kind == kGMG) launch_accumulate_cells(d, 0, G.n, dGhost, AX, AX, 1.0f, true, st);
}

// FullNegativeLaplacian with calc_diag (src/GMGSolver.cu:167-171): the diagonal, GHOST
// diagonals added into their LEAF parents (x's GHOST values are refreshed as a side effect)
void Solver::enqueue_geo_full_neg_lap_diag(Grid& G, float* X, float* D, cudaStream_t st) const {
    const DevGrid d = G.dev();
    const int ch = (int)((X - G.chan) / ((size_t)G.n * kCells));
    launch_propagate_ghost(d, 0, G.n, ch, st);
    launch_geo_lap(kind, d, 0, G.n, X, D, false, dLeaf | dGhost, st, true);
    launch_accumulate_cells(d, 0, G.n, dGhost, D, D, 1.0f, true, st);
}

// dot product over a device tile list, read back to the host
int Solver::host_dot(Grid& G, const int* list, int nlist, const float* A, const float* B, double* out) {
    if (int rc = ensure_scratch(nlist)) return rc;
    if (!G.dot_out) CK(cudaMalloc(&G.dot_out, sizeof(double)));
    launch_dot(G.dev(), list, nlist, A, B, kDotStore, G.dot_out, scratch(), G.stream);
    CK(cudaMemcpyAsync(out, G.dot_out, sizeof(double), cudaMemcpyDeviceToHost, G.stream));
    CK(cudaStreamSynchronize(G.stream));
    return 0;
}

// AMGSolver::FASMuCycleSolve (src/AMGSolver.cu:1311-1356): mu-cycles on x (channel 0) against
// b (channel 1), channel 2 as the FAS x0 and then r = b - A x; returns the index of the
// iteration at which |r| < tol |b| (or max_iters) and |r| / |b|
int Solver::fas_mu_cycle_solve(Grid& G, int repeat_times, int max_iters, double tol, int level_iters, int coarsest_iters, int* iters, double* rel) {
    if (int rc = validate_solver_topology(G)) return rc;
    if (int rc = ensure_coeff16(G)) return rc;
    const DevGrid d = G.dev();
    cudaStream_t st = G.stream;
    enqueue_operand_pack(G, st);
    launch_fill(G.plane(0), (size_t)G.n * kCells, 0.0f, st);
    double bb = 0;
    if (int rc = host_dot(G, G.leaf, G.nleaf, G.plane(1), G.plane(1), &bb)) return rc;
    const double rhs_norm = std::sqrt(bb);
    const double thr = std::max(tol * rhs_norm, DBL_MIN);
    MuArgs A = mu_args(G, 0, 1, 2, level_iters, coarsest_iters);
    A.mu = repeat_times;
    double res = rhs_norm;
    int i = 0;
    for (; i < max_iters; ++i) {
        enqueue_mu_step(G, G.max_level(), A, st);
        // AMGFullNegativeLaplacianOnLeafs with its side effects on x: GHOST and NONLEAF values
        launch_propagate_ghost(d, 0, G.n, 0, st);
        launch_accumulate_cells(d, 0, G.n, dLeaf, G.plane(0), G.plane(0), 0.125f, false, st);
        launch_leaf_apply(d, G.leaf, G.nleaf, G.plane(0), G.plane(2), coeff_ch, false, scratch(), st);
        launch_leaf_residual(d, G.leaf, G.nleaf, G.plane(1), G.plane(2), false, st);
        double rr = 0;
        if (int rc = host_dot(G, G.leaf, G.nleaf, G.plane(2), G.plane(2), &rr)) return rc;
        res = std::sqrt(rr);
        if (res < thr) break;
    }
    *iters = i;
    *rel = res / rhs_norm;
    return 0;
}

// GMGSolver::dampedJacobiSolve (src/GMGSolver.cu:390-470): channels x 0, b 1, r 2, D 3
int Solver::damped_jacobi_solve(Grid& G, int max_iters, double tol, float omega, int* iters, double* rel) {
    if (int rc = validate_solver_topology(G)) return rc;
    const DevGrid d = G.dev();
    cudaStream_t st = G.stream;
    launch_fill(G.plane(0), (size_t)G.n * kCells, 0.0f, st);
    // |b| over every tile (LEAF | NONLEAF | GHOST, src/GMGSolver.cu:407)
    std::vector<int> all(G.n);
    for (int t = 0; t < G.n; ++t) all[t] = t;
    int* dall = nullptr;
    CK(cudaMalloc(&dall, sizeof(int) * G.n));
    int rc = 0;
    double bb = 0, res = 0, rhs_norm = 0, thr = 0;
    int i = 0;
    if (cudaMemcpyAsync(dall, all.data(), sizeof(int) * G.n, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = 2;
    if (!rc) rc = host_dot(G, dall, G.n, G.plane(1), G.plane(1), &bb);
    cudaFree(dall);
    if (rc) return rc;
    rhs_norm = std::sqrt(bb);
    thr = std::max(tol * rhs_norm, DBL_MIN);
    res = rhs_norm;
    for (; i < max_iters; ++i) {
        enqueue_geo_full_neg_lap(G, G.plane(0), G.plane(2), st);
        launch_leaf_residual(d, G.leaf, G.nleaf, G.plane(1), G.plane(2), true, st);
        double rr = 0;
        if (int e = host_dot(G, G.leaf, G.nleaf, G.plane(2), G.plane(2), &rr)) return e;
        res = std::sqrt(rr);
        if (res < thr) break;
        enqueue_geo_full_neg_lap_diag(G, G.plane(0), G.plane(3), st);
        launch_jacobi_update(d, G.leaf, G.nleaf, G.plane(0), G.plane(2), G.plane(3), omega, st);
    }
    *iters = i;
    *rel = res / rhs_norm;
    return 0;
}

void Solver::enqueue_precond(Grid& G, const Key& k, cudaStream_t st) const {
    if (kind != kAMG) {
        enqueue_geo_vcycle(G, G.plane(4), G.plane(1), G.plane(3), k.level_iters, k.coarsest_iters, st);
    } else if (cycle16_active(G)) {
        // x, rhs and saved x of levels >= 3 in BF16: the right-hand side goes in on the LEAF
        // tiles of those levels, the cycle runs, z comes back out there
        MuArgs A = mu_args(G, 4, 1, 3, k.level_iters, k.coarsest_iters);
        const size_t plane = (size_t)G.n * kCells;
        A.X16 = x16;
        A.RHS16 = static_cast<unsigned short*>(x16) + plane;
        A.X016 = static_cast<unsigned short*>(x16) + 2 * plane;
        int first = 0;  // LEAF tiles of levels 0-2 lead the leaf list
        for (int l = 0; l < 3; ++l) first += G.nonleaf_begin(l) - G.level_begin(l);
        launch_fill(A.X, plane, 0.0f, st);
        cudaMemsetAsync(A.X16, 0, 2 * plane, st);
        launch_leaf_to_bf16(G.leaf + first, G.nleaf - first, A.RHS, A.RHS16, st);
        enqueue_mu_step(G, G.max_level(), A, st);
        launch_leaf_from_bf16(G.leaf + first, G.nleaf - first, A.X16, A.X, st);
    } else if (!learned_active()) {
        enqueue_mu_cycle(G, mu_args(G, 4, 1, 3, k.level_iters, k.coarsest_iters), st);
    } else {
        // learned: the cycle saves its FAS x0 in aux so that Ap (channel 3) survives for the
        // flexible beta; then rho = r - A z on the finest LEAF tiles and z += net(rho) there
        MuArgs A = mu_args(G, 4, 1, 3, k.level_iters, k.coarsest_iters);
        A.X0 = aux;
        enqueue_mu_cycle(G, A, st);
        const int L = G.max_level(), t0 = G.level_begin(L), nf = G.nonleaf_begin(L) - t0;
        launch_leaf_apply(G.dev(), G.leaf + (G.nleaf - nf), nf, G.plane(4), aux, coeff_ch, false, scratch(), st);
        // the net also sees each cell's face coefficients and the residual across the tile's faces
        NetExtra ex;
        ex.faces = G.plane(coeff_ch);
        ex.fstride = (size_t)G.n * kCells;
        ex.ftile = kCells;
        ex.nbx = G.nbx;
        launch_net_forward(lnet.H, G.plane(1), aux, G.plane(coeff_ch + 3), G.ctype, nullptr, t0, nf, lnet.pack, lnet.bias, G.plane(4), false,
                           st, ex);
    }
}

// AMGSolver::FASMuCycle (src/AMGSolver.cu:1279-1292): zero x everywhere, then the top step
void Solver::enqueue_mu_cycle(Grid& G, const MuArgs& A, cudaStream_t st) const {
    launch_fill(A.X, (size_t)G.n * kCells, 0.0f, st);
    enqueue_mu_step(G, G.max_level(), A, st);
}

// AMGSolver::VCycle (src/AMGSolver.cu:1060-1128): downstroke of pre-smoothing and
// restriction (the coarse x becomes the mean of the fine x), the coarsest level, then
// prolongation x += P x_coarse and post-smoothing, coarse to fine
void Solver::enqueue_vcycle_cs(Grid& G, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters, cudaStream_t st) const {
    const DevGrid d = G.dev();
    launch_cycle_init(d, X, RHS, F, st);
    for (int l = G.max_level(); l > 0; --l) {
        enqueue_gs(G, l, level_iters, 0, X, RHS, st);
        launch_restrict(d, G.level_begin(l), G.ghost_begin(l) - G.level_begin(l), X, RHS, coeff_ch, R_restrict, st);
    }
    enqueue_gs(G, 0, coarsest_iters / 2, 0, X, RHS, st);
    enqueue_gs(G, 0, coarsest_iters / 2, 1, X, RHS, st);
    for (int l = 1; l <= G.max_level(); ++l) {
        launch_prolong_add(d, G.level_begin(l), G.level_end(l) - G.level_begin(l), X, P, st);
        enqueue_gs(G, l, level_iters, 1, X, RHS, st);
    }
}
// AMGSolver::muCycleStep (src/AMGSolver.cu:1130-1149): below the pre-smoothing and the
// restriction, the LEAF tiles of the coarser level take rhs = f minus the flux from their
// NONLEAF neighbours and the NONLEAF tiles start from x = 0
void Solver::enqueue_mu_step_cs(Grid& G, int l, int repeat_times, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters,
                                cudaStream_t st) const {
    const DevGrid d = G.dev();
    if (l == 0) {
        enqueue_gs(G, 0, coarsest_iters / 2, 0, X, RHS, st);
        enqueue_gs(G, 0, coarsest_iters / 2, 1, X, RHS, st);
        return;
    }
    enqueue_gs(G, l, level_iters, 0, X, RHS, st);
    launch_restrict(d, G.level_begin(l), G.ghost_begin(l) - G.level_begin(l), X, RHS, coeff_ch, R_restrict, st);
    launch_deduct_flux(d, G.level_begin(l - 1), G.nonleaf_begin(l - 1) - G.level_begin(l - 1), X, F, RHS, coeff_ch, st);
    const int nb0 = G.nonleaf_begin(l - 1), nbn = G.ghost_begin(l - 1) - nb0;
    if (nbn > 0) launch_fill(X + (size_t)nb0 * kCells, (size_t)nbn * kCells, 0.0f, st);
    for (int r = 0; r < repeat_times; ++r) enqueue_mu_step_cs(G, l - 1, repeat_times, X, F, RHS, level_iters, coarsest_iters, st);
    launch_prolong_add(d, G.level_begin(l), G.level_end(l) - G.level_begin(l), X, P, st);
    enqueue_gs(G, l, level_iters, 1, X, RHS, st);
}
// AMGSolver::muCycle (src/AMGSolver.cu:1151-1174)
void Solver::enqueue_mu_cycle_cs(Grid& G, int repeat_times, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters,
                                 cudaStream_t st) const {
    launch_cycle_init(G.dev(), X, RHS, F, st);
    enqueue_mu_step_cs(G, G.max_level(), repeat_times, X, F, RHS, level_iters, coarsest_iters, st);
}
// AMGSolver::FASFCycle (src/AMGSolver.cu:1358-1387); the rhs goes down by
// RestrictSourceToCoarse (:1295-1307): R times the sum of the 8 children's INTERIOR values
void Solver::enqueue_fas_f_cycle(Grid& G, const MuArgs& A, cudaStream_t st) const {
    const DevGrid d = G.dev();
    launch_fill(A.X, (size_t)G.n * kCells, 0.0f, st);
    for (int l = G.max_level(); l > 0; --l)
        launch_accumulate_cells(d, G.level_begin(l), G.ghost_begin(l) - G.level_begin(l), dLeaf | dNonLeaf, A.RHS, A.RHS, A.Rr, false, st,
                                dInterior);
    enqueue_gs(G, 0, A.coarsest_iters / 2, 0, A.X, A.RHS, st);
    enqueue_gs(G, 0, A.coarsest_iters / 2, 1, A.X, A.RHS, st);
    for (int l = 1; l <= G.max_level(); ++l) {
        launch_prolong_add(d, G.level_begin(l), G.level_end(l) - G.level_begin(l), A.X, A.P, st);
        enqueue_mu_step(G, l, A, st);
    }
}

static int capture_tail(cudaStream_t st, std::vector<cudaGraphNode_t>& tail) {
    cudaStreamCaptureStatus stt;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(st, &stt, nullptr, nullptr, &deps, &nd));
    tail.assign(deps, deps + nd);
    return 0;
}

// The whole of AMGSolver::solve (src/AMGSolver.cu:1399-1549) as one graph:
//   x = 0; rr0 = r.r; [recenter]; z = M r; p = z; gamma = z.r; gate
//   WHILE (not done):  Ap = A p (+ alpha);  x, r update (+ r.r, convergence)
//                      IF (not done): [recenter]; z = M r; beta; p = z + beta p
// x = 0; rr0 = r.r; [recenter]; z = M r; p = z; gamma = z.r; loop gate (src/AMGSolver.cu:1405-1442)
void Solver::enqueue_pre(Grid& G, const Key& k, cudaGraphConditionalHandle loop_h, bool graph, cudaStream_t st) const {
    const DevGrid d = G.dev();
    const ReduceScratch rs = scratch();
    enqueue_operand_pack(G, st);
    launch_leaf_fill(d, G.leaf, G.nleaf, G.plane(0), 0.0f, st);
    if (replacing()) launch_leaf_copy(d, G.leaf, G.nleaf, bkeep, G.plane(1), st);
    if (k.sync > 0) launch_dot(d, G.leaf, G.nleaf, G.plane(1), G.plane(1), kDotRR0, nullptr, rs, st);
    if (k.pure_neumann) launch_recenter(d, G.leaf, G.nleaf, G.plane(1), rs, st);
    enqueue_precond(G, k, st);
    launch_leaf_copy(d, G.leaf, G.nleaf, G.plane(2), G.plane(4), st);
    launch_dot(d, G.leaf, G.nleaf, G.plane(4), G.plane(1), kDotGammaInit, nullptr, rs, st);
    launch_loop_gate(rs, loop_h, graph, st);
}
// Ap = A p with alpha; x += alpha p, r -= alpha Ap with r.r and the convergence test (src/AMGSolver.cu:1449-1499)
void Solver::enqueue_body(Grid& G, cudaGraphConditionalHandle loop_h, cudaGraphConditionalHandle body_h, bool graph, cudaStream_t st) const {
    const DevGrid d = G.dev();
    const ReduceScratch rs = scratch();
    if (kind == kAMG) {
        launch_leaf_apply(d, G.leaf, G.nleaf, G.plane(2), G.plane(3), coeff_ch, true, rs, st);
    } else {
        enqueue_geo_full_neg_lap(G, G.plane(2), G.plane(3), st);
        launch_dot(d, G.leaf, G.nleaf, G.plane(2), G.plane(3), kDotAlpha, nullptr, rs, st);
    }
    launch_xr_update(d, G.leaf, G.nleaf, G.plane(0), G.plane(1), G.plane(2), G.plane(3), rs, loop_h, body_h, graph, st);
}
// [recenter]; z = M r; gamma_old, gamma, beta; p = z + beta p (src/AMGSolver.cu:1500-1536)
void Solver::enqueue_tail(Grid& G, const Key& k, cudaStream_t st) const {
    const DevGrid d = G.dev();
    const ReduceScratch rs = scratch();
    if (replacing()) launch_true_residual(d, G.leaf, G.nleaf, G.plane(0), bkeep, G.plane(1), coeff_ch, s, replace_every, st);
    if (k.pure_neumann) launch_recenter(d, G.leaf, G.nleaf, G.plane(1), rs, st);
    enqueue_precond(G, k, st);
    if (learned_active()) launch_dot_flex(d, G.leaf, G.nleaf, G.plane(1), G.plane(4), G.plane(3), rs, st);
    else launch_dot(d, G.leaf, G.nleaf, G.plane(1), G.plane(4), kDotBeta, nullptr, rs, st);
    launch_p_update(d, G.leaf, G.nleaf, G.plane(2), G.plane(4), rs, st);
}

int Solver::build_graph(Grid& G, const Key& k, Plan* out) {
    cudaStream_t cs = cap_stream;
    const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;

    cudaGraph_t top;
    CK(cudaGraphCreate(&top, 0));
    cudaGraphConditionalHandle loop_h = 0, body_h = 0;
    CK(cudaGraphConditionalHandleCreate(&loop_h, top, 1, cudaGraphCondAssignDefault));

    const long long c0 = kernel_launch_count();
    CK(cudaStreamBeginCaptureToGraph(cs, top, nullptr, nullptr, 0, mode));
    enqueue_pre(G, k, loop_h, true, cs);
    std::vector<cudaGraphNode_t> tail;
    if (int rc = capture_tail(cs, tail)) return rc;
    CK(cudaStreamEndCapture(cs, &top));

    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = loop_h;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    CK(cudaGraphAddNode(&wnode, top, tail.data(), tail.size(), &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    CK(cudaGraphConditionalHandleCreate(&body_h, body, 0, cudaGraphCondAssignDefault));

    const long long c1 = kernel_launch_count();
    CK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, mode));
    enqueue_body(G, loop_h, body_h, true, cs);
    if (int rc = capture_tail(cs, tail)) return rc;
    CK(cudaStreamEndCapture(cs, &body));

    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = body_h;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode;
    CK(cudaGraphAddNode(&inode, body, tail.data(), tail.size(), &ip));
    cudaGraph_t ibody = ip.conditional.phGraph_out[0];

    const long long c2 = kernel_launch_count();
    CK(cudaStreamBeginCaptureToGraph(cs, ibody, nullptr, nullptr, 0, mode));
    enqueue_tail(G, k, cs);
    CK(cudaStreamEndCapture(cs, &ibody));

    out->k_pre = (int)(c1 - c0);
    out->k_body = (int)(c2 - c1);
    out->k_if = (int)(kernel_launch_count() - c2);
    CK(cudaGraphInstantiate(&out->exec, top, 0));
    cudaGraphDestroy(top);
    return 0;
}

int Solver::solve_begin(Grid& G, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride, bool pure_neumann) {
    pending = Pending{};
    if (G.n == 0 || G.nleaf == 0) {
        set_error("solve: grid has no LEAF tiles (rebuild first)");
        return 3;
    }
    if (G.nch < 5 || (kind == kAMG && (coeff_ch < 5 || coeff_ch + 4 > G.nch))) {
        set_error(kind == kAMG ? "solve: needs channels 0..4 and coefficient channels coeff..coeff+3 (coeff >= 5)"
                               : "solve: needs channels 0..4");
        return 1;
    }
    if (max_iters < 0 || level_iters < 0 || coarsest_iters < 0 || mu < 0) {
        set_error("solve: negative iteration count");
        return 1;
    }
    if (int rc = validate_solver_topology(G)) return rc;
    if (int rc = ensure_scratch(G.nleaf)) return rc;
    if (int rc = ensure_coeff16(G)) return rc;
    if (learned_active()) {
        if (int rc = ensure_aux(G)) return rc;
    }
    if (replacing()) {
        if (int rc = ensure_bkeep(G)) return rc;
    }
    if (cycle16_active(G)) {
        if (int rc = ensure_x16(G)) return rc;
    }
    if (coarsest_direct && kind == kAMG && cluster_active(G)) {
        if (int rc = prepare_root_inverse(G)) return rc;
    }
    Key k{&G, G.version, level_iters, coarsest_iters, pure_neumann ? 1 : 0, mu,
          (sync_stride > 0 ? 1 : 0) | (use_persist ? 2 : 0) | (use_cluster ? 4 : 0) | (use_pipe ? 8 : 0) | (storage << 4) |
              (learned_active() ? 256 : 0) | ((finest_iters + 1) << 10) | ((replacing() ? replace_every : 0) << 20) |
              (coarsest_direct ? (1 << 30) : 0) | (cycle16_active(G) ? (1 << 9) : 0),
          omega};
    Plan plan{};
    if (use_graph) {
        auto it = graphs.find(k);
        if (it == graphs.end() && graphs.size() >= kMaxCachedGraphs) {
            // graphs of grids that no longer exist never match again: drop the cache when it grows
            for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
            graphs.clear();
        }
        if (it == graphs.end()) {
            if (int rc = build_graph(G, k, &plan)) return rc;
            graphs[k] = plan;
        } else {
            plan = it->second;
        }
    }
    std::memset(h_s, 0, sizeof(PcgScalars));
    h_s->max_iters = max_iters;
    // the learned solve falls back to the plain one when its residual stalls
    h_s->stall_window = learned_active() ? kLearnedStallWindow : 0;
    h_s->sync_stride = sync_stride;
    h_s->thr = -1.0;
    h_s->tol = tol;  // the gate kernel turns it into max(tol^2 rr0, DBL_MIN)
    cudaStream_t st = G.stream;
    CK(cudaMemcpyAsync(s, h_s, sizeof(PcgScalars), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(ev0, st));
    long long stream_launches = -1;
    if (use_graph) {
        CK(cudaGraphLaunch(plan.exec, st));
    } else {
        // the same kernels launched one by one, the loop test read back on the
        // host after every update (for profilers that do not enter graphs)
        const long long c0 = kernel_launch_count();
        enqueue_pre(G, k, 0, false, st);
        for (;;) {
            CK(cudaMemcpyAsync(&h_s->done, &s->done, sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (h_s->done) break;
            enqueue_body(G, 0, 0, false, st);
            CK(cudaMemcpyAsync(&h_s->done, &s->done, sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (h_s->done) break;
            enqueue_tail(G, k, st);
        }
        stream_launches = kernel_launch_count() - c0;
    }
    CK(cudaEventRecord(ev1, st));
    CK(cudaMemcpyAsync(h_s, s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h_bar, bar, sizeof(unsigned int) * 4, cudaMemcpyDeviceToHost, st));
    pending.active = true;
    pending.stream = st;
    pending.sync_stride = sync_stride;
    pending.plan = plan;
    pending.stream_launches = stream_launches;
    return 0;
}

// iterations and relative residual of a finished solve, from its final scalars: with no
// convergence test (sync_stride 0) the residual is unknown (-1); b = 0 ends at once
static void pcg_outcome(const PcgScalars& r, int sync_stride, int* iters, double* rel) {
    int n_it = r.iter;
    double rel_res;
    if (sync_stride > 0) {
        if (r.rr0 == 0.0) {
            n_it = 0;
            rel_res = 0.0;
        } else if (n_it == 0) {
            rel_res = 1.0;
        } else {
            rel_res = std::sqrt(r.rr / r.rr0);
        }
    } else {
        rel_res = -1.0;
    }
    *iters = n_it;
    *rel = rel_res;
}

int Solver::solve_finish(bool verbose, int* iters, double* rel) {
    if (!pending.active) {
        set_error("solve: no solve in flight on this solver");
        return 3;
    }
    pending.active = false;
    const cudaStream_t st = pending.stream;
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    cudaEventElapsedTime(&last_ms, ev0, ev1);
    const PcgScalars& r = *h_s;
    last_replaced = r.replaced;
    int n_it = 0;
    double rel_res = 0.0;
    pcg_outcome(r, pending.sync_stride, &n_it, &rel_res);
    if (iters) *iters = n_it;
    if (rel) *rel = rel_res;
    // the IF body runs on every iteration except the one that ends the loop
    const Plan& plan = pending.plan;
    last_launches = use_graph ? plan.k_pre + (long long)r.iter * plan.k_body + (long long)(r.iter > 0 ? r.iter - 1 : 0) * plan.k_if
                              : pending.stream_launches;
    if (verbose) std::printf("cmg AMG-PCG: %d iterations, relative residual %.6e, %.3f ms\n", n_it, rel_res, last_ms);
    if (h_bar[2]) {
        cudaMemsetAsync(bar, 0, sizeof(unsigned int) * 4, st);
        set_error("solve: grid barrier of the persistent multigrid kernel timed out");
        return 2;
    }
    if (gs_pipe_take_error()) {
        set_error("solve: a smoothing sweep timed out waiting for its tile copies");
        return 2;
    }
    if (r.nonfinite) {
        set_error("solve: non-finite value in a PCG reduction");
        return 5;
    }
    return 0;
}

int Solver::solve(Grid& G, bool verbose, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride, bool pure_neumann,
                  int* iters, double* rel) {
    const bool learned = learned_active() && G.n > 0 && G.nleaf > 0;
    last_fallback = 0;
    last_true_rel = -1.0;
    if (learned) {
        if (int rc = ensure_aux(G)) return rc;
        CK(cudaMemcpyAsync(bsave, G.plane(1), sizeof(float) * (size_t)G.n * kCells, cudaMemcpyDeviceToDevice, G.stream));
    }
    if (int rc = solve_begin(G, max_iters, tol, level_iters, coarsest_iters, sync_stride, pure_neumann)) return rc;
    int it = 0;
    double rr = 0.0;
    const int rc = solve_finish(verbose, &it, &rr);
    const bool converged = h_s->converged != 0 || h_s->rr0 == 0.0;
    if (learned) {
        // the true residual judges the learned solve: |b - A x| / |b| on LEAF tiles
        const DevGrid d = G.dev();
        launch_leaf_apply(d, G.leaf, G.nleaf, G.plane(0), aux, coeff_ch, false, scratch(), G.stream);
        launch_leaf_residual(d, G.leaf, G.nleaf, bsave, aux, true, G.stream);
        double res = 0.0, bb = h_s->rr0;  // rr0 = b.b on LEAF tiles when the solve tracks the residual
        const bool have_bb = sync_stride > 0 && !pure_neumann;
        if (int e = host_dot(G, G.leaf, G.nleaf, aux, aux, &res)) return e;
        if (!have_bb) {
            if (int e = host_dot(G, G.leaf, G.nleaf, bsave, bsave, &bb)) return e;
        }
        last_true_rel = bb > 0.0 ? std::sqrt(res / bb) : 0.0;
        last_learned_iters = it;
        const bool tc_ok = net_take_tc_error() == 0;
        const bool judged_ok = rc == 0 && tc_ok && std::isfinite(last_true_rel) &&
                               (sync_stride <= 0 || (converged && last_true_rel <= kLearnedJudgeSlack * tol));
        if (!judged_ok && rc != 2) {
            // plain fallback from the saved right-hand side
            const float saved_ms = last_ms;
            CK(cudaMemcpyAsync(G.plane(1), bsave, sizeof(float) * (size_t)G.n * kCells, cudaMemcpyDeviceToDevice, G.stream));
            learned_suspended = true;
            int prc = solve_begin(G, max_iters, tol, level_iters, coarsest_iters, sync_stride, pure_neumann);
            if (prc == 0) prc = solve_finish(verbose, &it, &rr);
            learned_suspended = false;
            last_fallback = 1;
            last_ms += saved_ms;
            if (iters) *iters = it;
            if (rel) *rel = rr;
            return prc;
        }
    }
    if (iters) *iters = it;
    if (rel) *rel = rr;
    return rc;
}

constexpr float kTuneTie = 0.03f;

int Solver::autotune(Grid& G, int n, const TuneCandidate* c, int max_iters, double tol, int repeats, float* ms, int* iters, int* best) {
    *best = -1;
    if (int rc = ensure_aux(G)) return rc;  // bsave keeps the rhs between the timed solves
    const size_t bytes = sizeof(float) * (size_t)G.n * kCells;
    CK(cudaMemcpyAsync(bsave, G.plane(1), bytes, cudaMemcpyDeviceToDevice, G.stream));
    const double omega0 = omega;
    const int mu0 = mu, fi0 = finest_iters;
    auto restore = [&]() { omega = omega0, mu = mu0, finest_iters = fi0; };
    float best_ms = 0.0f;
    std::vector<double> rel_end(n, 0.0);
    for (int i = 0; i < n; ++i) {
        omega = c[i].omega;
        mu = c[i].mu;
        finest_iters = c[i].finest_iters;
        float tmin = -1.0f;
        bool ok = true;
        int it = 0;
        double rel_last = 0.0;
        for (int r = 0; r <= repeats; ++r) {  // the first solve builds the graph and is not counted
            CK(cudaMemcpyAsync(G.plane(1), bsave, bytes, cudaMemcpyDeviceToDevice, G.stream));
            if (int rc = solve_begin(G, max_iters, tol, c[i].level_iters, c[i].coarsest_iters, 1, false)) {
                restore();
                return rc;
            }
            double rel = 0.0;
            const int rc = solve_finish(false, &it, &rel);
            rel_last = rel;
            if (rc == 5) ok = false;  // non-finite: this setting diverges
            else if (rc) {
                restore();
                return rc;
            }
            if (!(h_s->converged || h_s->rr0 == 0.0)) ok = false;
            if (r > 0 && (tmin < 0.0f || last_ms < tmin)) tmin = last_ms;
            // a candidate whose first solve is already far slower than the best is not timed further
            if (r == 0 && (!ok || (*best >= 0 && last_ms > 1.5f * best_ms))) {
                if (ok) tmin = last_ms;
                break;
            }
        }
        ms[i] = ok ? tmin : -1.0f;
        iters[i] = it;
        rel_end[i] = rel_last;
        if (ok && (*best < 0 || tmin < best_ms)) {
            *best = i;
            best_ms = tmin;
        }
    }
    // near-ties (within kTuneTie of the fastest) go to the candidate with the fewest
    // iterations, then to the one whose last iteration reached the smallest residual:
    // timing noise then does not decide between settings of nearly equal cost, and the
    // cycle that converges fastest carries over best to other right-hand sides and octrees
    if (*best >= 0) {
        int pick = *best;
        for (int i = 0; i < n; ++i) {
            if (ms[i] < 0.0f || ms[i] > (1.0f + kTuneTie) * best_ms) continue;
            if (iters[i] < iters[pick] || (iters[i] == iters[pick] && rel_end[i] < rel_end[pick])) pick = i;
        }
        *best = pick;
    }
    CK(cudaMemcpyAsync(G.plane(1), bsave, bytes, cudaMemcpyDeviceToDevice, G.stream));
    CK(cudaStreamSynchronize(G.stream));
    restore();
    if (*best >= 0) {
        omega = c[*best].omega;
        mu = c[*best].mu;
        finest_iters = c[*best].finest_iters;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Batch: many octrees in one persistent launch inside a CUDA graph
// ---------------------------------------------------------------------------
Batch::~Batch() {
    if (st) cudaStreamSynchronize(st);
    if (exec) cudaGraphExecDestroy(exec);
    dfree(d_inst);
    dfree(d_order);
    dfree(d_groups);
    dfree(d_block_group);
    dfree(d_ctl);
    dfree(d_part);
    dfree(d_s);
    dfree(d_clock);
    for (void* p : {(void*)h_inst, (void*)h_order, (void*)h_groups, (void*)h_block_group, (void*)h_ctl, (void*)h_s, (void*)h_clock})
        if (p) cudaFreeHost(p);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (st) cudaStreamDestroy(st);
}

int Batch::init(Solver* const* s, Grid* const* g, int n) {
    solvers.assign(s, s + n);
    grids.assign(g, g + n);
    CK(cudaGetDevice(&device));
    int resident = 0;
    for (int ns : {4, 6, 8}) resident = std::max(resident, batch_resident_blocks(ns));
    if (resident <= 0) {
        set_error("batch: the persistent batched kernel cannot be resident on this device");
        return 2;
    }
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    const size_t m = (size_t)std::max(n, 1);
    CK(cudaMalloc(&d_inst, sizeof(BatchInst) * m));
    CK(cudaMallocHost(&h_inst, sizeof(BatchInst) * m));
    CK(cudaMalloc(&d_order, sizeof(int) * m));
    CK(cudaMallocHost(&h_order, sizeof(int) * m));
    CK(cudaMalloc(&d_groups, sizeof(BatchGroup) * resident));
    CK(cudaMallocHost(&h_groups, sizeof(BatchGroup) * resident));
    CK(cudaMalloc(&d_block_group, sizeof(int) * resident));
    CK(cudaMallocHost(&h_block_group, sizeof(int) * resident));
    CK(cudaMalloc(&d_s, sizeof(PcgScalars) * m));
    CK(cudaMallocHost(&h_s, sizeof(PcgScalars) * m));
    CK(cudaMalloc(&d_clock, sizeof(unsigned long long) * 4 * m));
    CK(cudaMallocHost(&h_clock, sizeof(unsigned long long) * 4 * m));
    ctl_words = batch_ctl_words(resident);
    CK(cudaMalloc(&d_ctl, sizeof(unsigned int) * ctl_words));
    CK(cudaMemset(d_ctl, 0, sizeof(unsigned int) * ctl_words));
    CK(cudaMallocHost(&h_ctl, sizeof(unsigned int) * 2));
    return 0;
}

// estimated work of one cycle per instance: each level's tiles (plus a fixed cost per step)
// times its visits per cycle, mu^(top - l)
static std::vector<double> batch_work_estimate(const Batch& B) {
    std::vector<double> w(B.grids.size());
    for (size_t i = 0; i < w.size(); ++i) {
        const Grid& G = *B.grids[i];
        const int mu = std::max(B.solvers[i]->mu, 1);
        double wk = 0.0, visits = 1.0;
        for (int l = G.max_level(); l >= 0; --l, visits *= mu) wk += visits * (G.level_end(l) - G.level_begin(l) + 16);
        w[i] = wk;
    }
    return w;
}

int Batch::schedule(int* ns, int* G, int* groups, int* dedicated, int* resident) {
    const int n = (int)grids.size();
    int ng = 0, dyn = 0, ded = 0;
    const int nb = plan(weight.size() == (size_t)n ? weight : batch_work_estimate(*this), &ng, &dyn, &ded);
    *ns = slots;
    *G = last_plan_gs;
    *groups = ng;
    *dedicated = ded;
    *resident = batch_resident_blocks(slots);
    if (nb <= 0) {
        set_error("batch: no resident blocks for the persistent batched kernel");
        return 2;
    }
    return 0;
}

int Batch::plan(const std::vector<double>& w, int* ngroups, int* dyn_begin, int* dedicated) {
    const int R = batch_resident_blocks(slots);
    const int n = (int)grids.size();
    *ngroups = *dyn_begin = *dedicated = 0;
    if (R <= 0 || n == 0) return 0;
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return w[a] > w[b]; });
    const int gs = std::min(R, group_blocks > 0 ? group_blocks : std::max(1, R / n));
    last_plan_gs = gs;
    int used = 0, ng = 0, nbig = 0;
    if (split > 0.0) {
        // octrees that would not end within the budget in a small group get a group of their own
        double total = 0.0;
        for (double v : w) total += v;
        const double T = split * total / R;
        for (int k = 0; k < n; ++k) {
            const int i = idx[k];
            const int need = std::min((int)std::ceil(w[i] / T), R - used - gs);  // keep one small group
            if (need <= gs) break;
            h_groups[ng] = BatchGroup{used, need, nbig, nbig + 1};
            h_order[nbig] = i;
            for (int b = used; b < used + need; ++b) h_block_group[b] = ng;
            used += need;
            ++ng;
            ++nbig;
        }
    }
    for (int k = nbig; k < n; ++k) h_order[k] = idx[k];
    // the remaining blocks as small groups on the shared queue (never more groups than octrees)
    const int small = std::min((R - used) / gs, std::max(n - nbig, 0));
    for (int q = 0; q < small; ++q) {
        h_groups[ng] = BatchGroup{used, gs, 0, 0};
        for (int b = used; b < used + gs; ++b) h_block_group[b] = ng;
        used += gs;
        ++ng;
    }
    *ngroups = ng;
    *dyn_begin = nbig;
    *dedicated = nbig;
    return used;
}

int Batch::run(const float* const* b_host, float* const* x_host, int max_iters, double tol, int level_iters, int coarsest_iters,
               int sync_stride, bool pure_neumann, int* iters, double* rel, float* instance_ms) {
    const int n = (int)grids.size();
    if (n == 0) return 0;
    if (max_iters < 0 || level_iters < 0 || coarsest_iters < 0) {
        set_error("batch: negative iteration count");
        return 1;
    }
    int cur = 0;
    CK(cudaGetDevice(&cur));
    if (cur != device) {
        set_error("batch: the current device is not the one the batch was created on");
        return 3;
    }
    // every instance: an AMG solver in the reference's FP32 form, a built grid on this device
    size_t need = 0;
    for (int i = 0; i < n; ++i) {
        const Solver& S = *solvers[i];
        Grid& G = *grids[i];
        if (S.kind != kAMG || S.storage != kStorageFP32 || S.lnet.enabled || S.replace_every > 0 || S.cycle_bf16 || S.coarsest_direct ||
            S.mu < 0) {
            set_error("batch: every solver must be an AMG solver with FP32 storage and no learned, replacement, BF16-cycle or "
                      "direct-coarsest option");
            return 1;
        }
        if (G.n == 0 || G.nleaf == 0) {
            set_error("batch: a grid has no LEAF tiles (rebuild first)");
            return 3;
        }
        if (G.nch < 5 || S.coeff_ch < 5 || S.coeff_ch + 4 > G.nch) {
            set_error("batch: needs channels 0..4 and coefficient channels coeff..coeff+3 (coeff >= 5)");
            return 1;
        }
        if (G.device != device) {
            set_error("batch: a grid lives on another device");
            return 3;
        }
        if (G.max_level() >= kBatchMaxLevels) {
            set_error("batch: octree deeper than the batched kernel supports");
            return 1;
        }
        if (int rc = validate_solver_topology(G)) return rc;
        need += 4 * (size_t)G.nleaf;
    }
    if (need > part_cap) {
        CK(cudaStreamSynchronize(st));
        dfree(d_part);
        CK(cudaMalloc(&d_part, sizeof(double) * need));
        part_cap = need;
    }
    int ngroups = 0, dyn_begin = 0, dedicated = 0;
    const int nblocks = plan(weight.size() == (size_t)n ? weight : batch_work_estimate(*this), &ngroups, &dyn_begin, &dedicated);
    if (nblocks <= 0) {
        set_error("batch: no resident blocks for the persistent batched kernel");
        return 2;
    }
    // instance table
    size_t off = 0;
    for (int i = 0; i < n; ++i) {
        const Solver& S = *solvers[i];
        Grid& G = *grids[i];
        BatchInst& I = h_inst[i];
        std::memset(&I, 0, sizeof(I));
        I.g = G.dev();
        I.leaf = G.leaf;
        I.nleaf = G.nleaf;
        I.top = G.max_level();
        for (int l = 0; l <= I.top; ++l) {
            I.lb[l] = G.level_begin(l);
            I.ab[l] = G.ghost_begin(l);
            I.le[l] = G.level_end(l);
            I.nlb[l] = G.nonleaf_begin(l);
        }
        I.coeff_ch = S.coeff_ch;
        I.mu = S.mu;
        I.finest_iters = S.finest_iters;
        I.exact = relax_mode(S.omega);
        I.om = (float)S.omega;
        I.omega = S.omega;
        I.Rr = S.R_restrict;
        I.P = S.P;
        I.partial = d_part + off;
        off += 4 * (size_t)G.nleaf;
        I.s = d_s + i;
        I.clock = d_clock + 4 * i;
    }
    // the grids' own streams may still carry uploads
    std::vector<cudaStream_t> seen;
    for (Grid* g : grids)
        if (std::find(seen.begin(), seen.end(), g->stream) == seen.end()) {
            seen.push_back(g->stream);
            CK(cudaStreamSynchronize(g->stream));
        }
    CK(cudaMemcpyAsync(d_inst, h_inst, sizeof(BatchInst) * n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_order, h_order, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_groups, h_groups, sizeof(BatchGroup) * ngroups, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_block_group, h_block_group, sizeof(int) * nblocks, cudaMemcpyHostToDevice, st));
    if (b_host)
        for (int i = 0; i < n; ++i)
            CK(cudaMemcpyAsync(grids[i]->plane(1), b_host[i], sizeof(float) * (size_t)grids[i]->n * kCells, cudaMemcpyHostToDevice, st));
    const GraphKey k{slots, nblocks, ngroups, dyn_begin, max_iters, sync_stride, pure_neumann ? 1 : 0, level_iters, coarsest_iters, tol};
    if (!exec || !(k == key)) {
        if (exec) {
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
        BatchArgs A;
        A.inst = d_inst;
        A.order = d_order;
        A.groups = d_groups;
        A.block_group = d_block_group;
        A.n = n;
        A.ngroups = ngroups;
        A.dyn_begin = dyn_begin;
        A.max_iters = max_iters;
        A.sync_stride = sync_stride;
        A.pure_neumann = pure_neumann ? 1 : 0;
        A.level_iters = level_iters;
        A.coarsest_iters = coarsest_iters;
        A.tol = tol;
        A.ctl = d_ctl;
        cudaStream_t cs = nullptr;
        CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaMemsetAsync(d_ctl, 0, sizeof(unsigned int) * ctl_words, cs);
            const cudaError_t le = launch_batch_solve(A, nblocks, slots, cs);
            e = cudaStreamEndCapture(cs, &graph);
            if (le != cudaSuccess) e = le;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) {
            exec = nullptr;
            return check_cuda(e, "batch: capture of the persistent launch");
        }
        key = k;
    }
    CK(cudaEventRecord(ev0, st));
    CK(cudaGraphLaunch(exec, st));
    CK(cudaEventRecord(ev1, st));
    if (x_host)
        for (int i = 0; i < n; ++i)
            CK(cudaMemcpyAsync(x_host[i], grids[i]->plane(0), sizeof(float) * (size_t)grids[i]->n * kCells, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h_s, d_s, sizeof(PcgScalars) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h_clock, d_clock, sizeof(unsigned long long) * 4 * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(unsigned int) * 2, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    cudaEventElapsedTime(&last_ms, ev0, ev1);
    last_nblocks = nblocks;
    last_groups = ngroups;
    last_dedicated = dedicated;
    if (h_ctl[1]) {
        set_error("batch: a group barrier of the persistent batched kernel timed out");
        return 2;
    }
    int rc = 0;
    for (int i = 0; i < n; ++i) {
        int it = 0;
        double rr = 0.0;
        pcg_outcome(h_s[i], sync_stride, &it, &rr);
        if (iters) iters[i] = it;
        if (rel) rel[i] = rr;
        if (instance_ms) instance_ms[i] = (float)((double)(h_clock[4 * i + 1] - h_clock[4 * i]) * 1e-6);
        if (h_s[i].nonfinite && rc == 0) {
            set_error("batch: non-finite value in a PCG reduction of instance " + std::to_string(i));
            rc = 5;
        }
    }
    return rc;
}

int Batch::autotune(const int* slots_c, const int* cand, const double* split_c, int ncand, int max_iters, double tol, int level_iters,
                    int coarsest_iters, int sync_stride, int repeats, float* ms, int* best) {
    *best = -1;
    const int n = (int)grids.size();
    if (n == 0) return 0;
    // the right-hand sides the grids hold now, restored before every run and at the end
    size_t total = 0;
    for (Grid* g : grids) total += (size_t)g->n * kCells;
    float* keep = nullptr;
    CK(cudaMalloc(&keep, sizeof(float) * total));
    auto copy_all = [&](bool save) -> int {
        size_t o = 0;
        for (Grid* g : grids) {
            const size_t c = (size_t)g->n * kCells;
            CK(cudaMemcpyAsync(save ? keep + o : g->plane(1), save ? g->plane(1) : keep + o, sizeof(float) * c, cudaMemcpyDeviceToDevice,
                               st));
            o += c;
        }
        return 0;
    };
    for (Grid* g : grids) CK(cudaStreamSynchronize(g->stream));
    int rc = copy_all(true);
    const int g0 = group_blocks, ns0 = slots;
    const double s0 = split;
    std::vector<int> it(n);
    std::vector<double> rr(n);
    std::vector<float> ims(n);
    // calibration: every octree's block-time (solve time x blocks of its group)
    if (rc == 0) rc = copy_all(false);
    if (rc == 0) {
        const int e = run(nullptr, nullptr, max_iters, tol, level_iters, coarsest_iters, sync_stride, false, it.data(), rr.data(), ims.data());
        if (e && e != 5) rc = e;
        if (rc == 0) {
            std::vector<double> w(n);
            for (int i = 0; i < n; ++i) w[i] = (double)ims[i] * (double)h_clock[4 * i + 2];
            weight = w;
        }
    }
    float best_ms = 0.0f;
    for (int c = 0; c < ncand && rc == 0; ++c) {
        group_blocks = cand[c];
        split = split_c ? split_c[c] : 0.0;
        slots = slots_c ? slots_c[c] : ns0;
        float tmin = -1.0f;
        bool ok = true;
        for (int r = 0; r <= repeats && rc == 0; ++r) {  // the first run builds the graph and is not counted
            if ((rc = copy_all(false))) break;
            const int e = run(nullptr, nullptr, max_iters, tol, level_iters, coarsest_iters, sync_stride, false, it.data(), rr.data(), nullptr);
            if (e == 5) ok = false;
            else if (e) rc = e;
            for (int i = 0; i < n && sync_stride > 0; ++i)
                if (!(h_s[i].converged || h_s[i].rr0 == 0.0)) ok = false;
            if (r > 0 && (tmin < 0.0f || last_ms < tmin)) tmin = last_ms;
        }
        ms[c] = ok ? tmin : -1.0f;
        if (rc == 0 && ok && (*best < 0 || tmin < best_ms)) {
            *best = c;
            best_ms = tmin;
        }
    }
    if (rc == 0) rc = copy_all(false);
    cudaStreamSynchronize(st);
    cudaFree(keep);
    if (*best >= 0) {
        group_blocks = cand[*best];
        split = split_c ? split_c[*best] : 0.0;
        slots = slots_c ? slots_c[*best] : ns0;
    } else {
        group_blocks = g0;
        split = s0;
        slots = ns0;
    }
    return rc;
}

}  // namespace cmg
