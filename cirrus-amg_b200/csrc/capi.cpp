// extern "C" entry points declared in include/cmg.h.
#include "cmg.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "cmg_impl.hpp"

struct cmg_grid {
    cmg::Grid g;
    // reduction scratch of the stand-alone dot product, owned by (and freed with) the grid
    double* dot_partial = nullptr;
    cmg::PcgScalars* dot_s = nullptr;
    int dot_cap = 0;
    cmg_grid(float h0, int nl, int nc) : g(h0, nl, nc) {}
    ~cmg_grid() {
        if (dot_partial) cudaFree(dot_partial);
        if (dot_s) cudaFree(dot_s);
    }
};
struct cmg_learned {
    cmg::Net n;
};
struct cmg_amg_solver {
    cmg::Solver s;
    cmg_amg_solver(int c, float rm, float rr, float p) : s(c, rm, rr, p) {}
    cmg_amg_solver(int kind, float one_over_alpha, float prolong) : s(kind, one_over_alpha, prolong) {}
};

namespace {

int fail(int code, const char* msg) {
    cmg::set_error(msg);
    return code;
}
#define GUARD_BEGIN try {
#define GUARD_END                                                   \
    }                                                               \
    catch (const std::bad_alloc&) { return fail(CMG_ERR_INVALID, "host allocation failed"); } \
    catch (const std::exception& e) { return fail(CMG_ERR_INVALID, e.what()); }
#define CKC(call)                                                    \
    do {                                                             \
        int _rc = cmg::check_cuda((call), #call);                    \
        if (_rc) return _rc;                                         \
    } while (0)

bool host_ready(cmg_grid* g) { return g && g->g.built && g->g.topo.size() > 0; }
// topology built and its device copy current (uploads it on first use)
bool grid_ready(cmg_grid* g) { return host_ready(g) && g->g.ensure_device() == 0; }
bool chan_ok(cmg_grid* g, int ch) { return ch >= 0 && ch < g->g.nch; }

int prepare_system(cmg::Grid& G, int coeff_ch, float R) {
    const cmg::DevGrid d = G.dev();
    for (int L = G.max_level(); L > 0; --L)
        cmg::launch_coarsen_offdiag(d, G.level_begin(L), G.level_end(L) - G.level_begin(L), coeff_ch, R, G.stream);
    for (int L = G.max_level(); L >= 0; --L) cmg::launch_diag(d, G.level_begin(L), G.level_end(L) - G.level_begin(L), coeff_ch, R, G.stream);
    return cmg::check_cuda(cudaGetLastError(), "prepare_system");
}

}  // namespace

extern "C" {

const char* cmg_last_error(void) { return cmg::last_error(); }
int cmg_version(void) { return 1; }
int cmg_check_division(long long n, unsigned long long seed, long long* mismatches, unsigned int* first_pair) {
    if (n < 0 || !mismatches) return fail(CMG_ERR_INVALID, "cmg_check_division: bad argument");
    if (cmg::check_division(n, seed, mismatches, first_pair)) return cmg::check_cuda(cudaGetLastError(), "check_division");
    return CMG_OK;
}

int cmg_grid_create(float h0, int num_levels, int num_channels, cmg_grid** out) {
    GUARD_BEGIN
    if (!out || !(h0 > 0) || num_levels < 1 || num_levels > 16 || num_channels < 1) return fail(CMG_ERR_INVALID, "cmg_grid_create: bad argument");
    *out = new cmg_grid(h0, num_levels, num_channels);
    return CMG_OK;
    GUARD_END
}
int cmg_grid_destroy(cmg_grid* g) {
    delete g;
    return CMG_OK;
}
int cmg_grid_set_tile(cmg_grid* g, int level, int i, int j, int k, int tile_type) {
    GUARD_BEGIN
    if (!g || (tile_type != CMG_LEAF && tile_type != CMG_NONLEAF && tile_type != CMG_GHOST)) return fail(CMG_ERR_INVALID, "cmg_grid_set_tile: bad type");
    if (g->g.topo.set(level, i, j, k, tile_type) < 0) return fail(CMG_ERR_INVALID, "cmg_grid_set_tile: level out of range");
    return CMG_OK;
    GUARD_END
}
int cmg_grid_rebuild(cmg_grid* g) {
    GUARD_BEGIN
    if (!g) return fail(CMG_ERR_INVALID, "null grid");
    return g->g.rebuild();
    GUARD_END
}
int cmg_grid_iterative_refine(cmg_grid* g, cmg_level_target_fn fn, void* user, int* steps) {
    GUARD_BEGIN
    if (!g || !fn) return fail(CMG_ERR_INVALID, "cmg_grid_iterative_refine: null argument");
    int st = g->g.topo.iterative_refine([&](int level, int i, int j, int k) { return fn(user, level, i, j, k); });
    if (steps) *steps = st;
    return g->g.rebuild();
    GUARD_END
}
int cmg_grid_refine_case(cmg_grid* g, int case_id, const double* params, int nparams, int* steps) {
    GUARD_BEGIN
    if (!g || !params || nparams < 2 || case_id < 0 || case_id > 7) return fail(CMG_ERR_INVALID, "cmg_grid_refine_case: bad argument");
    std::vector<double> prm(params, params + nparams);
    const float h0 = g->g.topo.h0();
    int st = g->g.topo.iterative_refine([&](int level, int i, int j, int k) {
        const int c[3] = {i, j, k};
        return cmg::case_target(case_id, prm.data(), (int)prm.size(), h0, level, c);
    });
    if (steps) *steps = st;
    return g->g.rebuild();
    GUARD_END
}
int cmg_grid_refine_case_device(cmg_grid* g, int case_id, const double* params, int nparams, int* steps) {
    GUARD_BEGIN
    if (!g || !params || nparams < 2 || nparams > cmg::kDevTopoMaxParams || case_id < 0 || case_id > 7)
        return fail(CMG_ERR_INVALID, "cmg_grid_refine_case_device: bad argument");
    return g->g.refine_case_device(case_id, params, nparams, steps);
    GUARD_END
}
int cmg_grid_info(cmg_grid* g, int* num_tiles, int* max_level, int* num_leaf_tiles) {
    if (!g) return fail(CMG_ERR_INVALID, "null grid");
    if (num_tiles) *num_tiles = g->g.built ? g->g.topo.size() : 0;
    if (max_level) *max_level = g->g.max_level();
    if (num_leaf_tiles) *num_leaf_tiles = g->g.built ? (int)g->g.topo.leaf_list.size() : 0;
    return CMG_OK;
}
int cmg_grid_tiles(cmg_grid* g, int* level, int* ijk, uint8_t* type) {
    if (!host_ready(g)) return fail(CMG_ERR_STATE, "cmg_grid_tiles: grid not built");
    const auto& T = g->g.topo.tiles();
    for (int t = 0; t < g->g.topo.size(); ++t) {
        if (level) level[t] = T[t].level;
        if (ijk)
            for (int d = 0; d < 3; ++d) ijk[3 * t + d] = T[t].c[d];
        if (type) type[t] = (uint8_t)T[t].type;
    }
    return CMG_OK;
}
int cmg_grid_tables(cmg_grid* g, int* nb, int* child) {
    if (!host_ready(g)) return fail(CMG_ERR_STATE, "cmg_grid_tables: grid not built");
    if (nb) std::memcpy(nb, g->g.topo.nb.data(), sizeof(int) * 8 * g->g.topo.size());
    if (child) std::memcpy(child, g->g.topo.child.data(), sizeof(int) * 8 * g->g.topo.size());
    return CMG_OK;
}
int cmg_grid_channel_ptr(cmg_grid* g, int ch, float** dev_ptr) {
    if (!grid_ready(g) || !dev_ptr) return fail(CMG_ERR_STATE, "cmg_grid_channel_ptr: grid not built");
    if (!chan_ok(g, ch)) return fail(CMG_ERR_INVALID, "channel out of range");
    *dev_ptr = g->g.plane(ch);
    return CMG_OK;
}
int cmg_grid_cell_type_ptr(cmg_grid* g, uint8_t** dev_ptr) {
    if (!grid_ready(g) || !dev_ptr) return fail(CMG_ERR_STATE, "cmg_grid_cell_type_ptr: grid not built");
    *dev_ptr = g->g.ctype;
    return CMG_OK;
}
int cmg_grid_upload_channel(cmg_grid* g, int ch, const float* host, size_t count) {
    if (!grid_ready(g) || !host) return fail(CMG_ERR_STATE, "cmg_grid_upload_channel: grid not built");
    if (!chan_ok(g, ch) || count != (size_t)g->g.n * 512) return fail(CMG_ERR_INVALID, "cmg_grid_upload_channel: bad channel or count");
    CKC(cudaMemcpyAsync(g->g.plane(ch), host, sizeof(float) * count, cudaMemcpyHostToDevice, g->g.stream));
    CKC(cudaStreamSynchronize(g->g.stream));
    return CMG_OK;
}
int cmg_grid_download_channel(cmg_grid* g, int ch, float* host, size_t count) {
    if (!grid_ready(g) || !host) return fail(CMG_ERR_STATE, "cmg_grid_download_channel: grid not built");
    if (!chan_ok(g, ch) || count != (size_t)g->g.n * 512) return fail(CMG_ERR_INVALID, "cmg_grid_download_channel: bad channel or count");
    CKC(cudaMemcpyAsync(host, g->g.plane(ch), sizeof(float) * count, cudaMemcpyDeviceToHost, g->g.stream));
    CKC(cudaStreamSynchronize(g->g.stream));
    return CMG_OK;
}
int cmg_grid_upload_cell_types(cmg_grid* g, const uint8_t* host, size_t count) {
    if (!grid_ready(g) || !host) return fail(CMG_ERR_STATE, "cmg_grid_upload_cell_types: grid not built");
    if (count != (size_t)g->g.n * 512) return fail(CMG_ERR_INVALID, "cmg_grid_upload_cell_types: bad count");
    CKC(cudaMemcpyAsync(g->g.ctype, host, count, cudaMemcpyHostToDevice, g->g.stream));
    CKC(cudaStreamSynchronize(g->g.stream));
    return CMG_OK;
}
int cmg_grid_download_cell_types(cmg_grid* g, uint8_t* host, size_t count) {
    if (!grid_ready(g) || !host) return fail(CMG_ERR_STATE, "cmg_grid_download_cell_types: grid not built");
    if (count != (size_t)g->g.n * 512) return fail(CMG_ERR_INVALID, "cmg_grid_download_cell_types: bad count");
    CKC(cudaMemcpyAsync(host, g->g.ctype, count, cudaMemcpyDeviceToHost, g->g.stream));
    CKC(cudaStreamSynchronize(g->g.stream));
    return CMG_OK;
}
// the caller's tile address list on the device (one upload per call)
static int upload_tile_ptrs(cmg_grid* g, const void* const* tile_ptrs, size_t tile_bytes, int first_ch, int num_ch, const char* who) {
    cmg::Grid& G = g->g;
    if (!tile_ptrs || tile_bytes != cmg::kRefTileBytes || first_ch < 0 || num_ch < 0 || first_ch + num_ch > std::min(G.nch, 15))
        return fail(CMG_ERR_INVALID, (std::string(who) + ": bad argument (tile_bytes must be 44880, channels within 0..14)").c_str());
    for (int t = 0; t < G.n; ++t)
        if (!tile_ptrs[t] || (reinterpret_cast<uintptr_t>(tile_ptrs[t]) & 15))
            return fail(CMG_ERR_INVALID, (std::string(who) + ": a tile address is null or not 16-byte aligned").c_str());
    if (G.n > G.tile_ptrs_cap) {
        if (G.tile_ptrs) cudaFree(G.tile_ptrs);
        G.tile_ptrs = nullptr;
        G.tile_ptrs_cap = 0;
        CKC(cudaMalloc(&G.tile_ptrs, sizeof(void*) * G.n));
        G.tile_ptrs_cap = G.n;
    }
    CKC(cudaMemcpyAsync(G.tile_ptrs, tile_ptrs, sizeof(void*) * G.n, cudaMemcpyHostToDevice, G.stream));
    return CMG_OK;
}
int cmg_grid_gather_device_tiles(cmg_grid* g, const void* const* tile_ptrs, size_t tile_bytes, int first_ch, int num_ch, int with_types) {
    GUARD_BEGIN
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "cmg_grid_gather_device_tiles: grid not built");
    if (int rc = upload_tile_ptrs(g, tile_ptrs, tile_bytes, first_ch, num_ch, "cmg_grid_gather_device_tiles")) return rc;
    cmg::launch_gather_tiles(g->g.dev(), g->g.tile_ptrs, first_ch, num_ch, with_types != 0, g->g.stream);
    CKC(cudaStreamSynchronize(g->g.stream));
    return cmg::check_cuda(cudaGetLastError(), "gather_device_tiles");
    GUARD_END
}
int cmg_grid_scatter_device_tiles(cmg_grid* g, const void* const* tile_ptrs, size_t tile_bytes, int first_ch, int num_ch) {
    GUARD_BEGIN
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "cmg_grid_scatter_device_tiles: grid not built");
    if (int rc = upload_tile_ptrs(g, tile_ptrs, tile_bytes, first_ch, num_ch, "cmg_grid_scatter_device_tiles")) return rc;
    cmg::launch_scatter_tiles(g->g.dev(), g->g.tile_ptrs, first_ch, num_ch, g->g.stream);
    CKC(cudaStreamSynchronize(g->g.stream));
    return cmg::check_cuda(cudaGetLastError(), "scatter_device_tiles");
    GUARD_END
}
int cmg_grid_fill_channel(cmg_grid* g, int ch, float value) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "cmg_grid_fill_channel: grid not built");
    if (!chan_ok(g, ch)) return fail(CMG_ERR_INVALID, "channel out of range");
    cmg::launch_fill(g->g.plane(ch), (size_t)g->g.n * 512, value, g->g.stream);
    return cmg::check_cuda(cudaGetLastError(), "fill");
}
int cmg_grid_copy_channel(cmg_grid* g, int src_ch, int dst_ch) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "cmg_grid_copy_channel: grid not built");
    if (!chan_ok(g, src_ch) || !chan_ok(g, dst_ch)) return fail(CMG_ERR_INVALID, "channel out of range");
    if (src_ch == dst_ch) return CMG_OK;
    CKC(cudaMemcpyAsync(g->g.plane(dst_ch), g->g.plane(src_ch), sizeof(float) * (size_t)g->g.n * 512, cudaMemcpyDeviceToDevice,
                        g->g.stream));
    return CMG_OK;
}
int cmg_grid_calc_cell_types_from_leafs(cmg_grid* g) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "cmg_grid_calc_cell_types_from_leafs: grid not built");
    cmg::Grid& G = g->g;
    const cmg::DevGrid d = G.dev();
    for (int L = G.max_level() - 1; L >= 0; --L)
        cmg::launch_types_from_children(d, G.nonleaf_begin(L), G.ghost_begin(L) - G.nonleaf_begin(L), G.stream);
    for (int L = 1; L <= G.max_level(); ++L) cmg::launch_ghost_types(d, G.ghost_begin(L), G.level_end(L) - G.ghost_begin(L), G.stream);
    return cmg::check_cuda(cudaGetLastError(), "calc_cell_types_from_leafs");
}
int cmg_grid_set_leaf_cell_types_case(cmg_grid* g, int case_id, const double* params, int nparams) {
    GUARD_BEGIN
    (void)params;
    (void)nparams;
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "grid not built");
    if (cmg::device_cell_types_supported(case_id)) {
        cmg::Grid& G = g->g;
        return cmg::check_cuda(cmg::device_leaf_cell_types(G.meta, G.ctype, G.leaf, G.nleaf, case_id, G.topo.h0(), G.stream),
                               "cmg_grid_set_leaf_cell_types_case");
    }
    const int n = g->g.n;
    std::vector<uint8_t> ty((size_t)n * 512);
    CKC(cudaMemcpy(ty.data(), g->g.ctype, ty.size(), cudaMemcpyDeviceToHost));
    const auto& T = g->g.topo.tiles();
    for (int t = 0; t < n; ++t) {
        if (T[t].type != cmg::kLeaf) continue;
        for (int v = 0; v < 512; ++v) ty[(size_t)t * 512 + v] = cmg::case_cell_type(case_id, g->g.topo.h0(), T[t].level, T[t].c, v);
    }
    CKC(cudaMemcpy(g->g.ctype, ty.data(), ty.size(), cudaMemcpyHostToDevice));
    return CMG_OK;
    GUARD_END
}
int cmg_grid_set_stream(cmg_grid* g, void* s) {
    if (!g) return fail(CMG_ERR_INVALID, "null grid");
    g->g.stream = (cudaStream_t)s;
    return CMG_OK;
}
int cmg_grid_synchronize(cmg_grid* g) {
    if (!g) return fail(CMG_ERR_INVALID, "null grid");
    CKC(cudaStreamSynchronize(g->g.stream));
    return cmg::check_cuda(cudaGetLastError(), "synchronize");
}

int cmg_amg_prepare_types_and_coeffs(cmg_grid* g, int coeff_ch, float R) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "grid not built");
    if (coeff_ch < 0 || coeff_ch + 4 > g->g.nch) return fail(CMG_ERR_INVALID, "coefficient channels out of range");
    const cmg::DevGrid d = g->g.dev();
    cmg::launch_ghost_types(d, 0, g->g.n, g->g.stream);
    cmg::launch_face_coeffs(d, 0, g->g.n, coeff_ch, 0, nullptr, g->g.stream);
    return prepare_system(g->g, coeff_ch, R);
}
int cmg_amg_prepare_system(cmg_grid* g, int coeff_ch, float R) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "grid not built");
    if (coeff_ch < 0 || coeff_ch + 4 > g->g.nch) return fail(CMG_ERR_INVALID, "coefficient channels out of range");
    return prepare_system(g->g, coeff_ch, R);
}
int cmg_amg_cutcell_sphere_coeffs(cmg_grid* g, int coeff_ch, float R, int nspheres, const float* spheres) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "grid not built");
    if (coeff_ch < 0 || coeff_ch + 4 > g->g.nch || nspheres < 1 || nspheres > 64 || !spheres)
        return fail(CMG_ERR_INVALID, "cmg_amg_cutcell_sphere_coeffs: bad argument");
    cmg::Grid& G = g->g;
    if (!G.spheres) CKC(cudaMalloc(&G.spheres, sizeof(float) * 4 * 64));
    CKC(cudaMemcpyAsync(G.spheres, spheres, sizeof(float) * 4 * nspheres, cudaMemcpyHostToDevice, G.stream));
    const cmg::DevGrid d = G.dev();
    cmg::launch_cutcell_neumann(d, G.leaf, G.nleaf, nspheres, G.spheres, G.stream);
    cmg::launch_ghost_types(d, 0, G.n, G.stream);
    cmg::launch_face_coeffs(d, 0, G.n, coeff_ch, nspheres, G.spheres, G.stream);
    int rc = prepare_system(G, coeff_ch, R);
    if (rc) return rc;
    CKC(cudaStreamSynchronize(G.stream));
    return CMG_OK;
}
int cmg_amg_face_velocity_fourier(cmg_grid* g, int u_ch, int nmodes, const double* k, const double* amp, const double* phase) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "grid not built");
    if (u_ch < 0 || u_ch + 3 > g->g.nch || nmodes < 1 || nmodes > 256 || !k || !amp || !phase)
        return fail(CMG_ERR_INVALID, "cmg_amg_face_velocity_fourier: bad argument");
    cmg::Grid& G = g->g;
    if (!G.modes) CKC(cudaMalloc(&G.modes, sizeof(double) * 7 * 256));
    CKC(cudaMemcpyAsync(G.modes, k, sizeof(double) * 3 * nmodes, cudaMemcpyHostToDevice, G.stream));
    CKC(cudaMemcpyAsync(G.modes + 3 * nmodes, amp, sizeof(double) * 3 * nmodes, cudaMemcpyHostToDevice, G.stream));
    CKC(cudaMemcpyAsync(G.modes + 6 * nmodes, phase, sizeof(double) * nmodes, cudaMemcpyHostToDevice, G.stream));
    cmg::launch_face_velocity(G.dev(), G.leaf, G.nleaf, u_ch, nmodes, G.modes, G.stream);
    CKC(cudaStreamSynchronize(G.stream));
    return cmg::check_cuda(cudaGetLastError(), "face velocity");
}
int cmg_amg_divergence(cmg_grid* g, int u_ch, int coeff_ch, int out_ch) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "grid not built");
    if (u_ch < 0 || u_ch + 3 > g->g.nch || coeff_ch < 0 || coeff_ch + 4 > g->g.nch || !chan_ok(g, out_ch))
        return fail(CMG_ERR_INVALID, "cmg_amg_divergence: channel out of range");
    cmg::Grid& G = g->g;
    const cmg::DevGrid d = G.dev();
    for (int a = 0; a < 3; ++a) cmg::launch_propagate_ghost(d, 0, G.n, u_ch + a, G.stream);
    cmg::launch_accumulate_faces(d, G.leaf, G.nleaf, u_ch, G.stream);
    cmg::launch_divergence(d, G.leaf, G.nleaf, u_ch, coeff_ch, out_ch, G.stream);
    return cmg::check_cuda(cudaGetLastError(), "divergence");
}
int cmg_amg_divergence_without_coeff(cmg_grid* g, int u_ch, int out_ch) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "grid not built");
    if (u_ch < 0 || u_ch + 3 > g->g.nch || !chan_ok(g, out_ch))
        return fail(CMG_ERR_INVALID, "cmg_amg_divergence_without_coeff: channel out of range");
    cmg::Grid& G = g->g;
    const cmg::DevGrid d = G.dev();
    for (int a = 0; a < 3; ++a) cmg::launch_propagate_ghost(d, 0, G.n, u_ch + a, G.stream);
    cmg::launch_accumulate_faces(d, G.leaf, G.nleaf, u_ch, G.stream);
    cmg::launch_divergence(d, G.leaf, G.nleaf, u_ch, -1, out_ch, G.stream);
    return cmg::check_cuda(cudaGetLastError(), "divergence_without_coeff");
}
int cmg_amg_add_gradient_to_face(cmg_grid* g, int x_ch, int coeff_ch, int u_ch) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "grid not built");
    if (!chan_ok(g, x_ch) || u_ch < 0 || u_ch + 3 > g->g.nch || coeff_ch < 0 || coeff_ch + 4 > g->g.nch)
        return fail(CMG_ERR_INVALID, "cmg_amg_add_gradient_to_face: channel out of range");
    cmg::Grid& G = g->g;
    cmg::launch_propagate_ghost(G.dev(), 0, G.n, x_ch, G.stream);
    cmg::launch_gradient(G.dev(), G.plane(x_ch), coeff_ch, u_ch, G.stream);
    return cmg::check_cuda(cudaGetLastError(), "add_gradient_to_face");
}
int cmg_amg_full_neg_lap(cmg_grid* g, int x_ch, int coeff_ch, int ax_ch) {
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "grid not built");
    if (!chan_ok(g, x_ch) || !chan_ok(g, ax_ch) || coeff_ch < 0 || coeff_ch + 4 > g->g.nch)
        return fail(CMG_ERR_INVALID, "cmg_amg_full_neg_lap: channel out of range");
    cmg::Grid& G = g->g;
    cmg::ReduceScratch rs{nullptr, nullptr, nullptr};
    cmg::launch_leaf_apply(G.dev(), G.leaf, G.nleaf, G.plane(x_ch), G.plane(ax_ch), coeff_ch, false, rs, G.stream);
    return cmg::check_cuda(cudaGetLastError(), "full_neg_lap");
}
int cmg_amg_dot(cmg_grid* g, int a_ch, int b_ch, double* out) {
    if (!grid_ready(g) || !out) return fail(CMG_ERR_STATE, "grid not built");
    if (!chan_ok(g, a_ch) || !chan_ok(g, b_ch)) return fail(CMG_ERR_INVALID, "cmg_amg_dot: channel out of range");
    cmg::Grid& G = g->g;
    if (g->dot_cap < G.nleaf) {
        if (g->dot_partial) cudaFree(g->dot_partial);
        g->dot_partial = nullptr;
        g->dot_cap = 0;
        CKC(cudaMalloc(&g->dot_partial, sizeof(double) * (G.nleaf + 1)));
        g->dot_cap = G.nleaf;
    }
    if (!g->dot_s) {
        CKC(cudaMalloc(&g->dot_s, sizeof(cmg::PcgScalars)));
        CKC(cudaMemset(g->dot_s, 0, sizeof(cmg::PcgScalars)));
    }
    if (!G.dot_out) CKC(cudaMalloc(&G.dot_out, sizeof(double)));
    cmg::launch_dot(G.dev(), G.leaf, G.nleaf, G.plane(a_ch), G.plane(b_ch), cmg::kDotStore, G.dot_out,
                    cmg::ReduceScratch{g->dot_partial, nullptr, g->dot_s}, G.stream);
    CKC(cudaMemcpyAsync(out, G.dot_out, sizeof(double), cudaMemcpyDeviceToHost, G.stream));
    CKC(cudaStreamSynchronize(G.stream));
    return CMG_OK;
}

int cmg_amg_dot_noalloc(cmg_grid* g, int a_ch, int b_ch, double* out) {
    if (!host_ready(g) || !out) return fail(CMG_ERR_STATE, "cmg_amg_dot_noalloc: grid not built or null result pointer");
    if (!chan_ok(g, a_ch) || !chan_ok(g, b_ch)) return fail(CMG_ERR_INVALID, "cmg_amg_dot_noalloc: channel out of range");
    cmg::Grid& G = g->g;
    const int nleaf = (int)G.topo.leaf_list.size();
    if (nleaf > cmg::dot_noalloc_max_leaf_tiles()) {
        return fail(CMG_ERR_INVALID, ("cmg_amg_dot_noalloc: " + std::to_string(nleaf) + " LEAF tiles exceed its fixed scratch of " +
                                      std::to_string(cmg::dot_noalloc_max_leaf_tiles()) + " tiles").c_str());
    }
    // uploading the topology would allocate: the device copy must already be current
    if (G.dev_version != G.host_version || G.n <= 0) return fail(CMG_ERR_STATE, "cmg_amg_dot_noalloc: the grid has no current device copy");
    return cmg::check_cuda(cmg::dot_noalloc(G.device, G.leaf, G.nleaf, G.plane(a_ch), G.plane(b_ch), out, G.stream), "cmg_amg_dot_noalloc");
}

int cmg_amg_solver_create(int coeff_ch, float R_matrix, float R_restrict, float P, cmg_amg_solver** out) {
    GUARD_BEGIN
    if (!out || coeff_ch < 0) return fail(CMG_ERR_INVALID, "cmg_amg_solver_create: bad argument");
    cmg_amg_solver* s = new cmg_amg_solver(coeff_ch, R_matrix, R_restrict, P);
    int rc = s->s.init();
    if (rc) {
        delete s;
        return rc;
    }
    *out = s;
    return CMG_OK;
    GUARD_END
}
int cmg_amg_solver_destroy(cmg_amg_solver* s) {
    delete s;
    return CMG_OK;
}
int cmg_amg_solver_set_smoother(cmg_amg_solver* s, double omega, int mu) {
    if (!s || mu < 0 || !(omega > 0)) return fail(CMG_ERR_INVALID, "cmg_amg_solver_set_smoother: bad argument");
    s->s.omega = (double)(float)omega;  // AMGSolver::omega is a float (src/AMGSolver.h:29)
    s->s.mu = mu;
    return CMG_OK;
}
int cmg_amg_solver_set_finest_iters(cmg_amg_solver* s, int finest_iters) {
    if (!s || finest_iters < -1) return fail(CMG_ERR_INVALID, "cmg_amg_solver_set_finest_iters: bad argument");
    s->s.finest_iters = finest_iters;
    return CMG_OK;
}
int cmg_amg_solver_set_residual_replacement(cmg_amg_solver* s, int every) {
    if (!s || every < 0 || every > 1000) return fail(CMG_ERR_INVALID, "cmg_amg_solver_set_residual_replacement: bad argument (0..1000)");
    s->s.replace_every = every;
    return CMG_OK;
}
int cmg_amg_solver_set_cycle_bf16(cmg_amg_solver* s, int on) {
    if (!s) return fail(CMG_ERR_INVALID, "cmg_amg_solver_set_cycle_bf16: null solver");
    s->s.cycle_bf16 = on != 0;
    return CMG_OK;
}
int cmg_amg_solver_set_coarsest_direct(cmg_amg_solver* s, int on) {
    if (!s) return fail(CMG_ERR_INVALID, "cmg_amg_solver_set_coarsest_direct: null solver");
    s->s.coarsest_direct = on != 0;
    return CMG_OK;
}
int cmg_amg_solver_residual_replacements(cmg_amg_solver* s, int* count) {
    if (!s || !count) return fail(CMG_ERR_INVALID, "cmg_amg_solver_residual_replacements: bad argument");
    *count = s->s.last_replaced;
    return CMG_OK;
}
int cmg_amg_solver_autotune(cmg_amg_solver* s, cmg_grid* g, int n, const cmg_tune_candidate* c, int max_iters, double tol, int repeats,
                            float* ms, int* iters, int* best) {
    GUARD_BEGIN
    if (!s || !g || n <= 0 || !c || !ms || !iters || !best || max_iters <= 0 || !(tol > 0.0) || repeats < 1)
        return fail(CMG_ERR_INVALID, "cmg_amg_solver_autotune: bad argument");
    std::vector<cmg::TuneCandidate> v(n);
    for (int i = 0; i < n; ++i) {
        if (!(c[i].omega > 0.0) || c[i].mu < 0 || c[i].level_iters < 0 || c[i].coarsest_iters < 0 || c[i].finest_iters < -1)
            return fail(CMG_ERR_INVALID, "cmg_amg_solver_autotune: bad candidate");
        v[i] = cmg::TuneCandidate{(double)(float)c[i].omega, c[i].mu, c[i].level_iters, c[i].coarsest_iters, c[i].finest_iters};
    }
    if (s->s.kind != cmg::kAMG) return fail(CMG_ERR_STATE, "cmg_amg_solver_autotune: not an AMG solver");
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "cmg_amg_solver_autotune: grid not built");
    return s->s.autotune(g->g, n, v.data(), max_iters, tol, repeats, ms, iters, best);
    GUARD_END
}
int cmg_amg_solver_set_launch_mode(cmg_amg_solver* s, int flags) {
    if (!s || (flags & ~15)) return fail(CMG_ERR_INVALID, "cmg_amg_solver_set_launch_mode: bad argument");
    s->s.use_graph = (flags & CMG_LAUNCH_GRAPH) != 0;
    s->s.use_cluster = (flags & CMG_LAUNCH_NO_CLUSTER) == 0;
    s->s.use_pipe = (flags & CMG_LAUNCH_NO_PIPELINE) == 0;
    s->s.use_persist = (flags & CMG_LAUNCH_PERSISTENT) != 0 && s->s.persist_nblocks > 0;
    return CMG_OK;
}
int cmg_amg_solver_set_storage(cmg_amg_solver* s, int storage) {
    if (!s || storage < CMG_STORAGE_FP32 || storage > CMG_STORAGE_FP16) return fail(CMG_ERR_INVALID, "cmg_amg_solver_set_storage: bad argument");
    if (s->s.kind != cmg::kAMG && storage != CMG_STORAGE_FP32)
        return fail(CMG_ERR_STATE, "cmg_amg_solver_set_storage: 16-bit operator storage is for AMG solvers");
    static_assert(CMG_STORAGE_BF16 == cmg::kStorageBF16 && CMG_STORAGE_FP16 == cmg::kStorageFP16, "storage codes");
    s->s.storage = storage;
    return CMG_OK;
}
int cmg_learned_create(int hidden, unsigned long long seed, cmg_learned** out) {
    GUARD_BEGIN
    if (!out || (hidden != 8 && hidden != 16 && hidden != 32))
        return fail(CMG_ERR_INVALID, "cmg_learned_create: hidden must be 8, 16 or 32");
    *out = nullptr;
    auto* n = new cmg_learned();
    if (int rc = n->n.init(hidden, seed)) {
        delete n;
        return rc;
    }
    *out = n;
    return 0;
    GUARD_END
}
int cmg_learned_destroy(cmg_learned* net) {
    delete net;
    return 0;
}
int cmg_learned_num_params(cmg_learned* net, int* n) {
    if (!net || !n) return fail(CMG_ERR_INVALID, "cmg_learned_num_params: null argument");
    *n = net->n.np;
    return 0;
}
int cmg_learned_get_params(cmg_learned* net, float* host, int n) {
    if (!net || !host || n != net->n.np) return fail(CMG_ERR_INVALID, "cmg_learned_get_params: bad argument");
    return net->n.get_params(host);
}
int cmg_learned_set_params(cmg_learned* net, const float* host, int n) {
    if (!net || !host || n != net->n.np) return fail(CMG_ERR_INVALID, "cmg_learned_set_params: bad argument");
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(host[i])) return fail(CMG_ERR_NONFINITE, "cmg_learned_set_params: non-finite parameter");
    return net->n.set_params(host);
}
int cmg_learned_set_samples(cmg_learned* net, int n, const float* rho, const float* diag, const uint8_t* types, const float* target,
                            const float* faces, const float* halo) {
    GUARD_BEGIN
    if (!net || n < 0 || (n > 0 && (!rho || !diag || !types))) return fail(CMG_ERR_INVALID, "cmg_learned_set_samples: bad argument");
    return net->n.set_samples(n, rho, diag, types, target, faces, halo);
    GUARD_END
}
int cmg_learned_forward(cmg_learned* net, int first, int n, float* out) {
    if (!net || !out || first < 0 || n <= 0 || first + n > net->n.ns) return fail(CMG_ERR_INVALID, "cmg_learned_forward: bad sample range");
    return net->n.forward(first, n, out);
}
int cmg_learned_apply_grid(cmg_learned* net, cmg_grid* g, int level, int r_ch, int az_ch, int coeff_ch, int out_ch, int overwrite) {
    GUARD_BEGIN
    if (!net || !grid_ready(g)) return fail(CMG_ERR_STATE, "cmg_learned_apply_grid: net or grid not ready");
    cmg::Grid& G = g->g;
    if (level < 0 || level > G.max_level() || !chan_ok(g, r_ch) || (az_ch >= 0 && !chan_ok(g, az_ch)) || !chan_ok(g, out_ch) ||
        coeff_ch < 0 || coeff_ch + 4 > G.nch || out_ch == r_ch || out_ch == az_ch)
        return fail(CMG_ERR_INVALID, "cmg_learned_apply_grid: bad argument");
    const int t0 = G.level_begin(level), nt = G.nonleaf_begin(level) - t0;
    cmg::NetExtra ex;
    ex.faces = G.plane(coeff_ch);
    ex.fstride = (size_t)G.n * 512;
    ex.ftile = 512;
    ex.nbx = G.nbx;
    cmg::launch_net_forward(net->n.H, G.plane(r_ch), az_ch >= 0 ? G.plane(az_ch) : nullptr, G.plane(coeff_ch + 3), G.ctype, nullptr, t0, nt,
                            net->n.pack, net->n.bias, G.plane(out_ch), overwrite != 0, G.stream, ex);
    CKC(cudaStreamSynchronize(G.stream));
    if (cmg::net_take_tc_error() == 1) return fail(CMG_ERR_CUDA, "cmg_learned_apply_grid: a tensor-core MMA did not complete in time");
    return cmg::check_cuda(cudaGetLastError(), "learned apply");
    GUARD_END
}
int cmg_learned_gradient(cmg_learned* net, int first, int n, double* loss, float* grad) {
    GUARD_BEGIN
    if (!net || first < 0 || n <= 0 || first + n > net->n.ns) return fail(CMG_ERR_INVALID, "cmg_learned_gradient: bad sample range");
    return net->n.gradient(first, n, loss, grad);
    GUARD_END
}
int cmg_learned_set_inference(int kind) {
    if (kind != 0 && kind != 1) return fail(CMG_ERR_INVALID, "cmg_learned_set_inference: kind must be 0 (mma.sync) or 1 (tcgen05)");
    cmg::net_set_inference_kind(kind);
    return 0;
}
int cmg_learned_set_loss(cmg_learned* net, int kind) {
    if (!net || (kind != 0 && kind != 1)) return fail(CMG_ERR_INVALID, "cmg_learned_set_loss: kind must be 0 or 1");
    net->n.loss_kind = kind;
    return 0;
}
int cmg_learned_train(cmg_learned* net, int epochs, int batch, float lr, unsigned long long seed, float* epoch_loss) {
    GUARD_BEGIN
    if (!net || epochs < 0 || batch <= 0 || !(lr > 0.0f)) return fail(CMG_ERR_INVALID, "cmg_learned_train: bad argument");
    if (net->n.ns <= 0) return fail(CMG_ERR_STATE, "cmg_learned_train: no samples");
    return net->n.train(epochs, batch, lr, seed, epoch_loss);
    GUARD_END
}
int cmg_amg_solver_set_learned(cmg_amg_solver* s, cmg_learned* net) {
    GUARD_BEGIN
    if (!s) return fail(CMG_ERR_INVALID, "cmg_amg_solver_set_learned: null solver");
    if (net && s->s.kind != cmg::kAMG) return fail(CMG_ERR_STATE, "cmg_amg_solver_set_learned: not an AMG solver");
    return s->s.set_learned(net ? &net->n : nullptr);
    GUARD_END
}
int cmg_amg_solver_learned_status(cmg_amg_solver* s, double* true_rel, int* fell_back, int* learned_iters) {
    if (!s) return fail(CMG_ERR_INVALID, "cmg_amg_solver_learned_status: null solver");
    if (true_rel) *true_rel = s->s.last_true_rel;
    if (fell_back) *fell_back = s->s.last_fallback;
    if (learned_iters) *learned_iters = s->s.last_learned_iters;
    return 0;
}
int cmg_amg_solve(cmg_amg_solver* s, cmg_grid* g, int verbose, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride,
                  int pure_neumann, int* iters, double* rel_res) {
    GUARD_BEGIN
    if (!s || !grid_ready(g)) return fail(CMG_ERR_STATE, "cmg_amg_solve: solver or grid not ready");
    return s->s.solve(g->g, verbose != 0, max_iters, tol, level_iters, coarsest_iters, sync_stride, pure_neumann != 0, iters, rel_res);
    GUARD_END
}
int cmg_amg_solve_host(cmg_amg_solver* s, cmg_grid* g, const float* b_host, float* x_host, size_t count, int max_iters, double tol,
                       int level_iters, int coarsest_iters, int sync_stride, int pure_neumann, int* iters, double* rel_res) {
    GUARD_BEGIN
    if (!s || !grid_ready(g) || !b_host || !x_host) return fail(CMG_ERR_STATE, "cmg_amg_solve_host: bad argument");
    cmg::Grid& G = g->g;
    if (count != (size_t)G.n * 512 || G.nch < 5) return fail(CMG_ERR_INVALID, "cmg_amg_solve_host: count must be num_tiles*512");
    CKC(cudaMemcpyAsync(G.plane(1), b_host, sizeof(float) * count, cudaMemcpyHostToDevice, G.stream));
    int rc = s->s.solve(G, false, max_iters, tol, level_iters, coarsest_iters, sync_stride, pure_neumann != 0, iters, rel_res);
    if (rc) return rc;
    CKC(cudaMemcpyAsync(x_host, G.plane(0), sizeof(float) * count, cudaMemcpyDeviceToHost, G.stream));
    CKC(cudaStreamSynchronize(G.stream));
    return CMG_OK;
    GUARD_END
}
int cmg_amg_solve_batch(cmg_amg_solver* const* solvers, cmg_grid* const* grids, int n, const float* const* b_host,
                        float* const* x_host, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride,
                        int pure_neumann, int* iters, double* rel_res, float* ms) {
    GUARD_BEGIN
    if (n < 0 || (n > 0 && (!solvers || !grids || !iters || !rel_res)) || (!b_host != !x_host))
        return fail(CMG_ERR_INVALID, "cmg_amg_solve_batch: bad argument");
    std::vector<const void*> seen_s, seen_g;
    for (int i = 0; i < n; ++i) {
        if (!solvers[i] || !grid_ready(grids[i])) return fail(CMG_ERR_STATE, "cmg_amg_solve_batch: solver or grid not ready");
        if (b_host && (!b_host[i] || !x_host[i])) return fail(CMG_ERR_INVALID, "cmg_amg_solve_batch: null host buffer");
        seen_s.push_back(solvers[i]);
        seen_g.push_back(grids[i]);
    }
    std::sort(seen_s.begin(), seen_s.end());
    std::sort(seen_g.begin(), seen_g.end());
    if (std::adjacent_find(seen_s.begin(), seen_s.end()) != seen_s.end() || std::adjacent_find(seen_g.begin(), seen_g.end()) != seen_g.end())
        return fail(CMG_ERR_INVALID, "cmg_amg_solve_batch: solvers and grids must be distinct objects");
    // enqueue every solve; on a failure, still wait for the ones already in flight
    int rc = CMG_OK, begun = 0;
    for (int i = 0; i < n && rc == CMG_OK; ++i) {
        cmg::Grid& G = grids[i]->g;
        if (b_host) {
            const cudaError_t e =
                cudaMemcpyAsync(G.plane(1), b_host[i], sizeof(float) * (size_t)G.n * 512, cudaMemcpyHostToDevice, G.stream);
            if (e != cudaSuccess) {
                rc = cmg::check_cuda(e, "solve_batch: copy of b");
                break;
            }
        }
        rc = solvers[i]->s.solve_begin(G, max_iters, tol, level_iters, coarsest_iters, sync_stride, pure_neumann != 0);
        if (rc != CMG_OK) break;
        ++begun;
        if (x_host) {
            const cudaError_t e =
                cudaMemcpyAsync(x_host[i], G.plane(0), sizeof(float) * (size_t)G.n * 512, cudaMemcpyDeviceToHost, G.stream);
            if (e != cudaSuccess) rc = cmg::check_cuda(e, "solve_batch: copy of x");
        }
    }
    std::string first_error = rc != CMG_OK ? cmg::last_error() : "";
    for (int i = 0; i < begun; ++i) {
        const int r = solvers[i]->s.solve_finish(false, &iters[i], &rel_res[i]);
        if (ms) ms[i] = solvers[i]->s.last_ms;
        if (r != CMG_OK && rc == CMG_OK) {
            rc = r;
            first_error = cmg::last_error();
        }
    }
    if (rc != CMG_OK) return fail(rc, first_error.c_str());
    return CMG_OK;
    GUARD_END
}
struct cmg_batch {
    cmg::Batch b;
};
int cmg_batch_create(cmg_amg_solver* const* solvers, cmg_grid* const* grids, int n, cmg_batch** out) {
    GUARD_BEGIN
    if (!out || n < 0 || (n > 0 && (!solvers || !grids))) return fail(CMG_ERR_INVALID, "cmg_batch_create: bad argument");
    std::vector<cmg::Solver*> sv(n);
    std::vector<cmg::Grid*> gv(n);
    std::vector<const void*> seen;
    for (int i = 0; i < n; ++i) {
        if (!solvers[i] || !grid_ready(grids[i])) return fail(CMG_ERR_STATE, "cmg_batch_create: solver or grid not ready");
        sv[i] = &solvers[i]->s;
        gv[i] = &grids[i]->g;
        seen.push_back(grids[i]);
    }
    std::sort(seen.begin(), seen.end());
    if (std::adjacent_find(seen.begin(), seen.end()) != seen.end())
        return fail(CMG_ERR_INVALID, "cmg_batch_create: grids must be distinct objects");
    cmg_batch* b = new cmg_batch();
    if (int rc = b->b.init(sv.data(), gv.data(), n)) {
        delete b;
        return rc;
    }
    *out = b;
    return CMG_OK;
    GUARD_END
}
int cmg_batch_destroy(cmg_batch* b) {
    delete b;
    return CMG_OK;
}
int cmg_batch_schedule(cmg_batch* b, int* slots, int* group_blocks, int* groups, int* dedicated, int* resident_blocks) {
    if (!b || !slots || !group_blocks || !groups || !dedicated || !resident_blocks)
        return fail(CMG_ERR_INVALID, "cmg_batch_schedule: bad argument");
    GUARD_BEGIN
    return b->b.schedule(slots, group_blocks, groups, dedicated, resident_blocks);
    GUARD_END
}
int cmg_batch_solve(cmg_batch* b, const float* const* b_host, float* const* x_host, int max_iters, double tol, int level_iters,
                    int coarsest_iters, int sync_stride, int pure_neumann, int* iters, double* rel_res, float* instance_ms, float* batch_ms) {
    GUARD_BEGIN
    const int n = b ? (int)b->b.grids.size() : 0;
    if (!b || (!b_host != !x_host) || (n > 0 && (!iters || !rel_res))) return fail(CMG_ERR_INVALID, "cmg_batch_solve: bad argument");
    if (b_host)
        for (int i = 0; i < n; ++i)
            if (!b_host[i] || !x_host[i]) return fail(CMG_ERR_INVALID, "cmg_batch_solve: null host buffer");
    for (cmg::Grid* g : b->b.grids)
        if (!g->built || g->ensure_device() != 0) return fail(CMG_ERR_STATE, "cmg_batch_solve: grid not built");
    const int rc = b->b.run(b_host, x_host, max_iters, tol, level_iters, coarsest_iters, sync_stride, pure_neumann != 0, iters, rel_res,
                            instance_ms);
    if (batch_ms) *batch_ms = b->b.last_ms;
    return rc;
    GUARD_END
}
int cmg_batch_set_schedule(cmg_batch* b, int slots, int group_blocks, double split) {
    if (!b || !cmg::batch_slots_supported(slots) || group_blocks < 0 || !(split >= 0.0))
        return fail(CMG_ERR_INVALID, "cmg_batch_set_schedule: bad argument");
    b->b.slots = slots;
    b->b.group_blocks = group_blocks;
    b->b.split = split;
    return CMG_OK;
}
int cmg_batch_autotune(cmg_batch* b, const int* slots, const int* group_blocks, const double* split, int ncand, int max_iters, double tol,
                       int level_iters, int coarsest_iters, int repeats, float* ms, int* best) {
    GUARD_BEGIN
    if (!b || !group_blocks || ncand <= 0 || !ms || !best || max_iters <= 0 || !(tol > 0.0) || repeats < 1)
        return fail(CMG_ERR_INVALID, "cmg_batch_autotune: bad argument");
    for (int i = 0; i < ncand; ++i)
        if (group_blocks[i] <= 0 || (split && !(split[i] >= 0.0)) || (slots && !cmg::batch_slots_supported(slots[i])))
            return fail(CMG_ERR_INVALID, "cmg_batch_autotune: bad candidate");
    for (cmg::Grid* g : b->b.grids)
        if (!g->built || g->ensure_device() != 0) return fail(CMG_ERR_STATE, "cmg_batch_autotune: grid not built");
    return b->b.autotune(slots, group_blocks, split, ncand, max_iters, tol, level_iters, coarsest_iters, 1, repeats, ms, best);
    GUARD_END
}
static int geo_create(int kind, float one_over_alpha, float prolong, cmg_amg_solver** out) {
    if (!out) return fail(CMG_ERR_INVALID, "solver create: null output");
    cmg_amg_solver* s = new cmg_amg_solver(kind, one_over_alpha, prolong);
    int rc = s->s.init();
    if (rc) {
        delete s;
        return rc;
    }
    *out = s;
    return CMG_OK;
}
int cmg_gmg_solver_create(float one_over_alpha, float prolong_coeff, cmg_amg_solver** out) {
    GUARD_BEGIN
    return geo_create(cmg::kGMG, one_over_alpha, prolong_coeff, out);
    GUARD_END
}
int cmg_cmg_solver_create(float one_over_alpha, float prolong_coeff, cmg_amg_solver** out) {
    GUARD_BEGIN
    return geo_create(cmg::kCMG, one_over_alpha, prolong_coeff, out);
    GUARD_END
}
int cmg_mg_vcycle(cmg_amg_solver* s, cmg_grid* g, int x_ch, int f_ch, int rhs_ch, int level_iters, int coarsest_iters) {
    if (!s || !grid_ready(g)) return fail(CMG_ERR_STATE, "solver or grid not ready");
    if (s->s.kind == cmg::kAMG) return fail(CMG_ERR_STATE, "cmg_mg_vcycle: the solver is an AMG solver (use cmg_amg_fas_mu_cycle)");
    if (!chan_ok(g, x_ch) || !chan_ok(g, f_ch) || !chan_ok(g, rhs_ch) || level_iters < 0 || coarsest_iters < 0)
        return fail(CMG_ERR_INVALID, "cmg_mg_vcycle: bad argument");
    if (int rc = cmg::validate_solver_topology(g->g)) return rc;
    s->s.enqueue_geo_vcycle(g->g, g->g.plane(x_ch), g->g.plane(f_ch), g->g.plane(rhs_ch), level_iters, coarsest_iters, g->g.stream);
    return cmg::check_cuda(cudaGetLastError(), "mg_vcycle");
}
int cmg_mg_gauss_seidel(cmg_amg_solver* s, cmg_grid* g, int iters, int order, int level, int x_ch, int rhs_ch) {
    if (!s || !grid_ready(g)) return fail(CMG_ERR_STATE, "solver or grid not ready");
    if (s->s.kind == cmg::kAMG) return fail(CMG_ERR_STATE, "cmg_mg_gauss_seidel: the solver is an AMG solver (use cmg_amg_gauss_seidel)");
    if (level < 0 || level > g->g.max_level() || !chan_ok(g, x_ch) || !chan_ok(g, rhs_ch) || (order != 0 && order != 1) || iters < 0)
        return fail(CMG_ERR_INVALID, "cmg_mg_gauss_seidel: bad argument");
    s->s.enqueue_geo_gs(g->g, level, iters, order, g->g.plane(x_ch), g->g.plane(rhs_ch), g->g.stream);
    return cmg::check_cuda(cudaGetLastError(), "mg_gauss_seidel");
}
int cmg_mg_full_neg_lap(cmg_amg_solver* s, cmg_grid* g, int x_ch, int ax_ch) {
    if (!s || !grid_ready(g)) return fail(CMG_ERR_STATE, "solver or grid not ready");
    if (s->s.kind == cmg::kAMG) return fail(CMG_ERR_STATE, "cmg_mg_full_neg_lap: the solver is an AMG solver (use cmg_amg_full_neg_lap)");
    if (!chan_ok(g, x_ch) || !chan_ok(g, ax_ch) || x_ch == ax_ch) return fail(CMG_ERR_INVALID, "cmg_mg_full_neg_lap: bad channels");
    s->s.enqueue_geo_full_neg_lap(g->g, g->g.plane(x_ch), g->g.plane(ax_ch), g->g.stream);
    return cmg::check_cuda(cudaGetLastError(), "mg_full_neg_lap");
}

int cmg_amg_fas_mu_cycle_solve(cmg_amg_solver* s, cmg_grid* g, int repeat_times, int verbose, int max_iters, double tol, int level_iters,
                               int coarsest_iters, int* iters, double* rel_res) {
    GUARD_BEGIN
    (void)verbose;
    if (!s || !grid_ready(g)) return fail(CMG_ERR_STATE, "solver or grid not ready");
    if (s->s.kind != cmg::kAMG) return fail(CMG_ERR_STATE, "cmg_amg_fas_mu_cycle_solve: not an AMG solver");
    if (!iters || !rel_res || repeat_times < 0 || max_iters < 0 || level_iters < 0 || coarsest_iters < 0 || g->g.nch < 3 ||
        s->s.coeff_ch + 4 > g->g.nch)
        return fail(CMG_ERR_INVALID, "cmg_amg_fas_mu_cycle_solve: bad argument");
    if (g->g.nleaf == 0) return fail(CMG_ERR_STATE, "cmg_amg_fas_mu_cycle_solve: no LEAF tiles");
    if (int rc = s->s.fas_mu_cycle_solve(g->g, repeat_times, max_iters, tol, level_iters, coarsest_iters, iters, rel_res)) return rc;
    return cmg::check_cuda(cudaGetLastError(), "fas_mu_cycle_solve");
    GUARD_END
}
int cmg_gmg_damped_jacobi_solve(cmg_amg_solver* s, cmg_grid* g, int verbose, int max_iters, double tol, float omega, int* iters, double* rel_res) {
    GUARD_BEGIN
    (void)verbose;
    if (!s || !grid_ready(g)) return fail(CMG_ERR_STATE, "solver or grid not ready");
    if (s->s.kind != cmg::kGMG) return fail(CMG_ERR_STATE, "cmg_gmg_damped_jacobi_solve: not a GMG solver");
    if (!iters || !rel_res || max_iters < 0 || g->g.nch < 4) return fail(CMG_ERR_INVALID, "cmg_gmg_damped_jacobi_solve: bad argument");
    if (g->g.nleaf == 0) return fail(CMG_ERR_STATE, "cmg_gmg_damped_jacobi_solve: no LEAF tiles");
    if (int rc = s->s.damped_jacobi_solve(g->g, max_iters, tol, omega, iters, rel_res)) return rc;
    return cmg::check_cuda(cudaGetLastError(), "damped_jacobi_solve");
    GUARD_END
}

int cmg_amg_gauss_seidel(cmg_amg_solver* s, cmg_grid* g, int iters, int order, int level, int x_ch, int rhs_ch) {
    if (!s || !grid_ready(g)) return fail(CMG_ERR_STATE, "solver or grid not ready");
    if (s->s.kind != cmg::kAMG) return fail(CMG_ERR_STATE, "cmg_amg_gauss_seidel: not an AMG solver (use cmg_mg_gauss_seidel)");
    if (level < 0 || level > g->g.max_level() || !chan_ok(g, x_ch) || !chan_ok(g, rhs_ch) || (order != 0 && order != 1))
        return fail(CMG_ERR_INVALID, "cmg_amg_gauss_seidel: bad argument");
    s->s.enqueue_gs(g->g, level, iters, order, g->g.plane(x_ch), g->g.plane(rhs_ch), g->g.stream);
    return cmg::check_cuda(cudaGetLastError(), "gauss_seidel");
}
int cmg_amg_gauss_seidel_masked(cmg_amg_solver* s, cmg_grid* g, int iters, int order, int level, int x_ch, int rhs_ch) {
    if (!s || !grid_ready(g)) return fail(CMG_ERR_STATE, "solver or grid not ready");
    if (s->s.kind != cmg::kAMG) return fail(CMG_ERR_STATE, "cmg_amg_gauss_seidel_masked: not an AMG solver (use cmg_mg_gauss_seidel)");
    if (level < 0 || level > g->g.max_level() || !chan_ok(g, x_ch) || !chan_ok(g, rhs_ch) || (order != 0 && order != 1))
        return fail(CMG_ERR_INVALID, "cmg_amg_gauss_seidel_masked: bad argument");
    if (int rc = s->s.ensure_coeff16(g->g)) return rc;
    if (s->s.storage != cmg::kStorageFP32) cmg::launch_coeff16(g->g.dev(), s->s.coeff_ch, s->s.storage, s->s.coeff16, g->g.stream);
    s->s.enqueue_gs(g->g, level, iters, order, g->g.plane(x_ch), g->g.plane(rhs_ch), g->g.stream, true);
    return cmg::check_cuda(cudaGetLastError(), "gauss_seidel");
}
int cmg_amg_fas_mu_cycle(cmg_amg_solver* s, cmg_grid* g, int x_ch, int rhs_ch, int x0_ch, int level_iters, int coarsest_iters) {
    if (!s || !grid_ready(g)) return fail(CMG_ERR_STATE, "solver or grid not ready");
    if (s->s.kind != cmg::kAMG) return fail(CMG_ERR_STATE, "cmg_amg_fas_mu_cycle: not an AMG solver (use cmg_mg_vcycle)");
    if (!chan_ok(g, x_ch) || !chan_ok(g, rhs_ch) || !chan_ok(g, x0_ch)) return fail(CMG_ERR_INVALID, "cmg_amg_fas_mu_cycle: channel out of range");
    if (int rc = cmg::validate_solver_topology(g->g)) return rc;
    const cmg::MuArgs A = s->s.mu_args(g->g, x_ch, rhs_ch, x0_ch, level_iters, coarsest_iters);
    if (int rc = s->s.ensure_coeff16(g->g)) return rc;
    s->s.enqueue_operand_pack(g->g, g->g.stream);
    s->s.enqueue_mu_cycle(g->g, A, g->g.stream);
    return cmg::check_cuda(cudaGetLastError(), "fas_mu_cycle");
}
static int cycle_args_ok(cmg_amg_solver* s, cmg_grid* g, const char* what) {
    if (!s || !grid_ready(g)) return fail(CMG_ERR_STATE, "solver or grid not ready");
    if (s->s.kind != cmg::kAMG) return fail(CMG_ERR_STATE, (std::string(what) + ": not an AMG solver").c_str());
    return cmg::validate_solver_topology(g->g);
}
int cmg_amg_vcycle(cmg_amg_solver* s, cmg_grid* g, int x_ch, int f_ch, int rhs_ch, int level_iters, int coarsest_iters) {
    GUARD_BEGIN
    if (int rc = cycle_args_ok(s, g, "cmg_amg_vcycle")) return rc;
    if (!chan_ok(g, x_ch) || !chan_ok(g, f_ch) || !chan_ok(g, rhs_ch) || x_ch == f_ch || x_ch == rhs_ch || f_ch == rhs_ch ||
        level_iters < 0 || coarsest_iters < 0)
        return fail(CMG_ERR_INVALID, "cmg_amg_vcycle: bad argument");
    cmg::Grid& G = g->g;
    s->s.enqueue_vcycle_cs(G, G.plane(x_ch), G.plane(f_ch), G.plane(rhs_ch), level_iters, coarsest_iters, G.stream);
    return cmg::check_cuda(cudaGetLastError(), "vcycle");
    GUARD_END
}
int cmg_amg_mu_cycle(cmg_amg_solver* s, cmg_grid* g, int repeat_times, int x_ch, int f_ch, int rhs_ch, int level_iters, int coarsest_iters) {
    GUARD_BEGIN
    if (int rc = cycle_args_ok(s, g, "cmg_amg_mu_cycle")) return rc;
    if (!chan_ok(g, x_ch) || !chan_ok(g, f_ch) || !chan_ok(g, rhs_ch) || x_ch == f_ch || x_ch == rhs_ch || f_ch == rhs_ch ||
        repeat_times < 0 || level_iters < 0 || coarsest_iters < 0)
        return fail(CMG_ERR_INVALID, "cmg_amg_mu_cycle: bad argument");
    cmg::Grid& G = g->g;
    s->s.enqueue_mu_cycle_cs(G, repeat_times, G.plane(x_ch), G.plane(f_ch), G.plane(rhs_ch), level_iters, coarsest_iters, G.stream);
    return cmg::check_cuda(cudaGetLastError(), "mu_cycle");
    GUARD_END
}
int cmg_amg_fas_f_cycle(cmg_amg_solver* s, cmg_grid* g, int x_ch, int rhs_ch, int x0_ch, int level_iters, int coarsest_iters) {
    GUARD_BEGIN
    if (int rc = cycle_args_ok(s, g, "cmg_amg_fas_f_cycle")) return rc;
    if (!chan_ok(g, x_ch) || !chan_ok(g, rhs_ch) || !chan_ok(g, x0_ch) || x_ch == rhs_ch || x_ch == x0_ch || rhs_ch == x0_ch ||
        level_iters < 0 || coarsest_iters < 0)
        return fail(CMG_ERR_INVALID, "cmg_amg_fas_f_cycle: bad argument");
    cmg::Grid& G = g->g;
    const cmg::MuArgs A = s->s.mu_args(G, x_ch, rhs_ch, x0_ch, level_iters, coarsest_iters);
    if (int rc = s->s.ensure_coeff16(G)) return rc;
    s->s.enqueue_operand_pack(G, G.stream);
    s->s.enqueue_fas_f_cycle(G, A, G.stream);
    return cmg::check_cuda(cudaGetLastError(), "fas_f_cycle");
    GUARD_END
}
int cmg_set_dependent_launch(int on) {
    cmg::gs_pipe_set_dependent_launch(on != 0);
    return CMG_OK;
}
int cmg_amg_last_solve_ms(cmg_amg_solver* s, float* ms) {
    if (!s || !ms) return fail(CMG_ERR_INVALID, "null argument");
    *ms = s->s.last_ms;
    return CMG_OK;
}
int cmg_amg_last_solve_launches(cmg_amg_solver* s, long long* launches) {
    if (!s || !launches) return fail(CMG_ERR_INVALID, "null argument");
    *launches = s->s.last_launches;
    return CMG_OK;
}

// ---- 'HAGR' v1 grid blobs (HADeviceGrid::dumpBinaryBlob / loadBinaryBlob, src/HAGrid.h:687-853) ----
// Layout (little endian, the reference's in-memory structs written raw):
//   header, 40 bytes: u32 magic 0x52474148, u32 version 1, u32 num_levels, i32 max_level,
//     u32 tile_size (sizeof(PoissonTile<float,15>) = 44880), u32 coord_size (12), f32 h0,
//     4 bytes of padding, u64 tile_count;
//   num_levels x u32 log2 hash sizes;
//   tile_count records: u32 level, u8 type, 3 x i32 tile coordinate, tile_size bytes of tile:
//     float data[15][736] (cell values in the first 512 of each channel), 6 neighbour
//     descriptors (192 bytes, pointers: meaningless in a file), u8 cell types[512] at byte
//     44352, then flags and status words.
}  // extern "C"

namespace {
constexpr uint32_t kHagrMagic = 0x52474148u;
constexpr size_t kHagrHeader = 40, kHagrTile = 44880, kHagrCoord = 12, kHagrTypes = 44352;
constexpr int kHagrChannels = 15, kHagrChannelStride = 736;
// byte offsets of the header fields: magic, version, num_levels, max_level, tile_size,
// coord_size, h0, tile_count
constexpr size_t kHagrOff[8] = {0, 4, 8, 12, 16, 20, 24, 32};
constexpr size_t kHagrRecord = 4 + 1 + kHagrCoord + kHagrTile;
template <class T>
T rd(const uint8_t* p) {
    T v;
    std::memcpy(&v, p, sizeof(T));
    return v;
}
template <class T>
void wr(uint8_t* p, T v) {
    std::memcpy(p, &v, sizeof(T));
}
}  // namespace

extern "C" {

int cmg_ref_record_layout(long long* out, int n) {
    static_assert(kHagrTile == cmg::kRefTileBytes, "one tile layout for blobs and device views");
    const long long v[] = {(long long)kHagrHeader, (long long)kHagrOff[0], (long long)kHagrOff[1], (long long)kHagrOff[2],
                           (long long)kHagrOff[3], (long long)kHagrOff[4], (long long)kHagrOff[5], (long long)kHagrOff[6],
                           (long long)kHagrOff[7], (long long)kHagrCoord, (long long)kHagrTile, (long long)kHagrTypes,
                           (long long)kHagrChannels, (long long)kHagrChannelStride};
    const int m = (int)(sizeof(v) / sizeof(v[0]));
    if (!out) return m;
    for (int i = 0; i < m && i < n; ++i) out[i] = v[i];
    return m;
}

int cmg_grid_load_hagr(const uint8_t* blob, size_t size, int num_channels, cmg_grid** out) {
    GUARD_BEGIN
    if (!blob || !out || num_channels < 1) return fail(CMG_ERR_INVALID, "cmg_grid_load_hagr: bad argument");
    if (size < kHagrHeader) return fail(CMG_ERR_INVALID, "cmg_grid_load_hagr: buffer too small");
    if (rd<uint32_t>(blob + kHagrOff[0]) != kHagrMagic) return fail(CMG_ERR_INVALID, "cmg_grid_load_hagr: bad magic");
    if (rd<uint32_t>(blob + kHagrOff[1]) != 1) return fail(CMG_ERR_INVALID, "cmg_grid_load_hagr: unsupported version");
    const uint32_t num_levels = rd<uint32_t>(blob + kHagrOff[2]);
    if (rd<uint32_t>(blob + kHagrOff[4]) != kHagrTile) return fail(CMG_ERR_INVALID, "cmg_grid_load_hagr: tile size is not that of PoissonTile<float,15>");
    if (rd<uint32_t>(blob + kHagrOff[5]) != kHagrCoord) return fail(CMG_ERR_INVALID, "cmg_grid_load_hagr: coordinate size mismatch");
    const float h0 = rd<float>(blob + kHagrOff[6]);
    const uint64_t count = rd<uint64_t>(blob + kHagrOff[7]);
    if (num_levels < 1 || num_levels > 16 || !(h0 > 0)) return fail(CMG_ERR_INVALID, "cmg_grid_load_hagr: bad header");
    const size_t body = kHagrHeader + 4 * (size_t)num_levels;
    if (size < body || (size - body) / kHagrRecord < count) return fail(CMG_ERR_INVALID, "cmg_grid_load_hagr: buffer truncated");
    cmg_grid* g = new cmg_grid(h0, (int)num_levels, num_channels);
    auto bail = [&](int code, const char* msg) {
        delete g;
        return fail(code, msg);
    };
    const uint8_t* rec = blob + body;
    for (uint64_t r = 0; r < count; ++r) {
        const uint8_t* p = rec + r * kHagrRecord;
        const int level = (int)rd<uint32_t>(p), type = p[4];
        if (type != CMG_LEAF && type != CMG_NONLEAF && type != CMG_GHOST) return bail(CMG_ERR_INVALID, "cmg_grid_load_hagr: bad tile type");
        if (type == CMG_GHOST) continue;  // GHOST tiles are spawned by the rebuild
        if (g->g.topo.set(level, rd<int32_t>(p + 5), rd<int32_t>(p + 9), rd<int32_t>(p + 13), type) < 0)
            return bail(CMG_ERR_INVALID, "cmg_grid_load_hagr: tile level out of range");
    }
    if (int rc = g->g.rebuild()) return bail(rc, "cmg_grid_load_hagr: rebuild failed");
    const int n = g->g.topo.size();
    const int nc = std::min(num_channels, kHagrChannels);
    std::vector<float> planes((size_t)nc * n * 512, 0.0f);
    std::vector<uint8_t> types((size_t)n * 512, 0);
    for (uint64_t r = 0; r < count; ++r) {
        const uint8_t* p = rec + r * kHagrRecord;
        const int t = g->g.topo.find((int)rd<uint32_t>(p), rd<int32_t>(p + 5), rd<int32_t>(p + 9), rd<int32_t>(p + 13));
        if (t < 0 || g->g.topo.tiles()[t].type != p[4]) return bail(CMG_ERR_TOPOLOGY, "cmg_grid_load_hagr: the blob's tiles are not a graded octree with its ghost layer");
        const uint8_t* tile = p + 17;
        for (int c = 0; c < nc; ++c) std::memcpy(&planes[((size_t)c * n + t) * 512], tile + (size_t)c * kHagrChannelStride * 4, 512 * 4);
        std::memcpy(&types[(size_t)t * 512], tile + kHagrTypes, 512);
    }
    if (!grid_ready(g)) return bail(CMG_ERR_CUDA, "cmg_grid_load_hagr: device allocation failed");
    for (int c = 0; c < num_channels; ++c) {
        cudaError_t e = c < nc ? cudaMemcpyAsync(g->g.plane(c), &planes[(size_t)c * n * 512], sizeof(float) * n * 512, cudaMemcpyHostToDevice, g->g.stream)
                               : cudaMemsetAsync(g->g.plane(c), 0, sizeof(float) * n * 512, g->g.stream);
        if (e != cudaSuccess) return bail(CMG_ERR_CUDA, "cmg_grid_load_hagr: upload failed");
    }
    if (cudaMemcpyAsync(g->g.ctype, types.data(), types.size(), cudaMemcpyHostToDevice, g->g.stream) != cudaSuccess ||
        cudaStreamSynchronize(g->g.stream) != cudaSuccess)
        return bail(CMG_ERR_CUDA, "cmg_grid_load_hagr: upload failed");
    *out = g;
    return CMG_OK;
    GUARD_END
}

int cmg_grid_dump_hagr(cmg_grid* g, uint8_t* buf, size_t capacity, size_t* size) {
    GUARD_BEGIN
    if (!size) return fail(CMG_ERR_INVALID, "cmg_grid_dump_hagr: null size");
    if (!grid_ready(g)) return fail(CMG_ERR_STATE, "cmg_grid_dump_hagr: grid not built");
    const cmg::Grid& G = g->g;
    const int n = G.topo.size(), nl = G.topo.num_levels();
    const size_t total = kHagrHeader + 4 * (size_t)nl + (size_t)n * kHagrRecord;
    *size = total;
    if (!buf) return CMG_OK;
    if (capacity < total) return fail(CMG_ERR_INVALID, "cmg_grid_dump_hagr: buffer too small");
    const int nc = std::min(G.nch, kHagrChannels);
    std::vector<float> planes((size_t)nc * n * 512);
    std::vector<uint8_t> types((size_t)n * 512);
    CKC(cudaMemcpyAsync(planes.data(), G.chan, sizeof(float) * planes.size(), cudaMemcpyDeviceToHost, G.stream));
    CKC(cudaMemcpyAsync(types.data(), G.ctype, types.size(), cudaMemcpyDeviceToHost, G.stream));
    CKC(cudaStreamSynchronize(G.stream));
    std::memset(buf, 0, total);
    wr<uint32_t>(buf + kHagrOff[0], kHagrMagic);
    wr<uint32_t>(buf + kHagrOff[1], 1);
    wr<uint32_t>(buf + kHagrOff[2], (uint32_t)nl);
    wr<int32_t>(buf + kHagrOff[3], G.max_level());
    wr<uint32_t>(buf + kHagrOff[4], (uint32_t)kHagrTile);
    wr<uint32_t>(buf + kHagrOff[5], (uint32_t)kHagrCoord);
    wr<float>(buf + kHagrOff[6], G.topo.h0());
    wr<uint64_t>(buf + kHagrOff[7], (uint64_t)n);
    for (int l = 0; l < nl; ++l) {
        // hash size for the reference's loader: room for twice the level's tiles, at least 2^8
        const int cnt = l <= G.max_level() ? G.level_end(l) - G.level_begin(l) : 0;
        uint32_t lg = 8;
        while ((1u << lg) < 2u * (uint32_t)cnt + 1u && lg < 30) ++lg;
        wr<uint32_t>(buf + kHagrHeader + 4 * l, lg);
    }
    uint8_t* rec = buf + kHagrHeader + 4 * (size_t)nl;
    const auto& T = G.topo.tiles();
    for (int t = 0; t < n; ++t) {
        uint8_t* p = rec + (size_t)t * kHagrRecord;
        wr<uint32_t>(p, (uint32_t)T[t].level);
        p[4] = (uint8_t)T[t].type;
        for (int d = 0; d < 3; ++d) wr<int32_t>(p + 5 + 4 * d, T[t].c[d]);
        uint8_t* tile = p + 17;
        for (int c = 0; c < nc; ++c) std::memcpy(tile + (size_t)c * kHagrChannelStride * 4, &planes[((size_t)c * n + t) * 512], 512 * 4);
        std::memcpy(tile + kHagrTypes, &types[(size_t)t * 512], 512);
    }
    return CMG_OK;
    GUARD_END
}

}  // extern "C"
