// Geometric multigrid preconditioners: GMGSolver (src/GMGSolver.cu) and
// CMGSolver (src/CMGSolver.cu).  Same tile layout and launch shape as the AMG
// kernels: one 128-thread block per 8^3 tile, four cells per thread, the tile and
// its face halo staged in shared memory.
//
// Both operate on raw x (no INTERIOR mask on neighbour values) and compute the
// coefficient of each face from the cell types of its two sides (and, for GMG,
// from the tile types: LEAF-LEAF faces weigh 1/h^2, LEAF-GHOST faces 1/(1.5h h));
// neither reads coefficient channels.  Sums follow the reference's order
// (-x,+x,-y,+y,-z,+z) with fused multiply-adds, as nvcc compiles `sum += c * d`.
#include "kernels.hpp"

namespace cmg {

namespace {

struct GSnap {
    float x[1000];
    uint8_t ct[1000];
    int tt_face[6];  // subtree type across each face (GMG: the tile's own when the neighbour is empty)
};

// HATileInfo::subtreeType (src/HATileInfo.h:79-84): a NONLEAF tile counts as LEAF at its own level
__device__ __forceinline__ int subtree_type(int type, bool sl_is_level) { return (sl_is_level && type == dNonLeaf) ? dLeaf : type; }

// LoadGMGLaplacianTileData (src/GMGSolver.cu:81-134) / LoadCMGLaplacianTileData
// (src/CMGSolver.cu:59-170).  Thread q stages its four own cells and, for r = 0..2,
// halo cell q & 63 of the face of axis r on side q >> 6.
template <int KIND>
__device__ __forceinline__ void load_gsnap(const DevGrid& g, int t, const float* X, bool sl_is_level, int own_tt, GSnap& S, const Quad& Q) {
    const float4 xr = ldcg4(X + Q.base);
    const uchar4 ty = ldt4(g.ctype + Q.base);
    const int side = Q.q >> 6, fa = (Q.q >> 3) & 7, fb = Q.q & 7;
    int desc[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) desc[r] = g.nbx[8 * t + r + 3 * side];
    const int e = side ? 0 : 7;  // the neighbour's cell next to the shared face
    const int nl[3] = {cell_index(e, fa, fb), cell_index(fa, e, fb), cell_index(fa, fb, e)};
    float hv[3];
    uint8_t hc[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        hv[r] = 0.0f;
        hc[r] = dDirichlet;
        if (desc[r] != 0) {
            const size_t o = (size_t)((desc[r] >> 3) - 1) * kCells + nl[r];
            hv[r] = ldcg(X + o);
            hc[r] = g.ctype[o];
        }
    }
    const int s0 = sx(Q.i, Q.j, Q.k0);
    S.x[s0 + 0] = xr.x;
    S.x[s0 + 1] = xr.y;
    S.x[s0 + 2] = xr.z;
    S.x[s0 + 3] = xr.w;
    S.ct[s0 + 0] = ty.x;
    S.ct[s0 + 1] = ty.y;
    S.ct[s0 + 2] = ty.z;
    S.ct[s0 + 3] = ty.w;
    if (Q.q < 6) {
        const int d = g.nbx[8 * t + Q.q];
        S.tt_face[Q.q] = d == 0 ? own_tt : subtree_type(d & 7, sl_is_level);
    }
    __syncthreads();
    const int ie = side ? 7 : 0, hl = side ? 8 : -1;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int fx = r == 0 ? sx(hl, fa, fb) : r == 1 ? sx(fa, hl, fb) : sx(fa, fb, hl);
        float v = hv[r];
        if (KIND == kCMG && desc[r] != 0 && subtree_type(desc[r] & 7, sl_is_level) == dGhost) {
            // x_in + 0.5 * (x_ghost - mean of the 2x2x2 block of own cells at the face)
            int cl[3];
            cl[0] = r == 0 ? ie : fa;
            cl[1] = r == 0 ? fa : r == 1 ? ie : fb;
            cl[2] = r == 2 ? ie : fb;
            float avg = 0.0f;
#pragma unroll
            for (int di = 0; di < 2; ++di)
#pragma unroll
                for (int dj = 0; dj < 2; ++dj)
#pragma unroll
                    for (int dk = 0; dk < 2; ++dk) avg = __fadd_rn(avg, S.x[sx(cl[0] ^ di, cl[1] ^ dj, cl[2] ^ dk)]);
            avg = __fmul_rn(avg, 0.125f);
            v = __fmaf_rn(0.5f, __fsub_rn(hv[r], avg), S.x[sx(cl[0], cl[1], cl[2])]);
        }
        S.x[fx] = v;
        S.ct[fx] = hc[r];
    }
    __syncthreads();
}

// NegativeLaplacianCoeff (src/GMGSolver.cu:3-31, src/CMGSolver.cu:3-7)
template <int KIND>
__device__ __forceinline__ float geo_coeff(float h, float ooh, int tt0, int tt1, int c0, int c1) {
    if ((c0 | c1) & dNeumann) return 0.0f;
    if (KIND == kCMG) return h;
    const bool both = (tt0 & dLeaf) && (tt1 & dLeaf);
    const bool lg = ((tt0 & dLeaf) && (tt1 & dGhost)) || ((tt0 & dGhost) && (tt1 & dLeaf));
    const float oodh = both ? ooh : (lg ? __fdiv_rn(__fmul_rn(2.0f, ooh), 3.0f) : 0.0f);
    return __fmul_rn(oodh, ooh);
}
// negativeLap (src/GMGSolver.cu:46-66, src/CMGSolver.cu:22-45) of cell (i, j, k)
template <int KIND>
__device__ __forceinline__ float geo_neg_lap(const GSnap& S, float h, float ooh, int own_tt, int i, int j, int k, bool diag) {
    const int c = sx(i, j, k);
    const int ct0 = S.ct[c];
    const float x0 = S.x[c];
    const int l[3] = {i, j, k};
    const int step[3] = {100, 10, 1};
    float sum = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const int nc = s ? c + step[a] : c - step[a];
            const bool inside = s ? l[a] < 7 : l[a] > 0;
            const int tt1 = inside ? own_tt : S.tt_face[a + 3 * s];
            const float coeff = geo_coeff<KIND>(h, ooh, own_tt, tt1, ct0, S.ct[nc]);
            sum = diag ? __fadd_rn(sum, coeff) : __fmaf_rn(coeff, __fsub_rn(x0, S.x[nc]), sum);
        }
    if (!(ct0 & dInterior)) return 0.0f;
    return KIND == kCMG ? sum : __fmul_rn(__fmul_rn(__fmul_rn(sum, h), h), h);
}

// NegativeLaplacianSameLevel128Kernel / ConservativeNegativeLaplacianSameLevel128Kernel
// on tiles t0.. whose (subtree) type is in `types`
template <int KIND>
__global__ void __launch_bounds__(128) k_geo_lap(DevGrid g, int t0, const float* X, float* AX, int sl_is_level, int types, int diag) {
    __shared__ GSnap S;
    const int t = t0 + blockIdx.x;
    const int own_tt = subtree_type(tile_type(g, t), sl_is_level);
    if (!(own_tt & types)) return;
    const Quad Q(t, threadIdx.x);
    load_gsnap<KIND>(g, t, X, sl_is_level, own_tt, S, Q);
    const float h = voxel_size(g.h0, tile_level(g, t));
    const float ooh = __fdiv_rn(1.0f, h);
    float4 out;
#pragma unroll
    for (int u = 0; u < 4; ++u) f4set(out, u, geo_neg_lap<KIND>(S, h, ooh, own_tt, Q.i, Q.j, Q.k0 + u, diag != 0));
    st4(AX + Q.base, out);
}

// r = b - r on the cells of LEAF tiles (every cell, or INTERIOR cells only)
__global__ void __launch_bounds__(128) k_leaf_residual(DevGrid g, const int* leaf, const float* B, float* R, int interior_only) {
    const int t = leaf[blockIdx.x];
    const Quad Q(t, threadIdx.x);
    const float4 b = ldcg4(B + Q.base);
    float4 r = ldcg4(R + Q.base);
    const uchar4 ty = ldt4(g.ctype + Q.base);
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if (!interior_only || (t4get(ty, u) & dInterior)) f4set(r, u, __fsub_rn(f4get(b, u), f4get(r, u)));
    st4(R + Q.base, r);
}
// damped Jacobi update (src/GMGSolver.cu:449-465): x += omega r / D on INTERIOR cells, x = 0 where D = 0
__global__ void __launch_bounds__(128) k_jacobi_update(DevGrid g, const int* leaf, float* X, const float* R, const float* D, float omega) {
    const int t = leaf[blockIdx.x];
    const Quad Q(t, threadIdx.x);
    float4 x = ldcg4(X + Q.base);
    const float4 r = ldcg4(R + Q.base), d = ldcg4(D + Q.base);
    const uchar4 ty = ldt4(g.ctype + Q.base);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        if (!(t4get(ty, u) & dInterior)) continue;
        const float dd = f4get(d, u);
        f4set(x, u, dd == 0.0f ? 0.0f : __fadd_rn(f4get(x, u), div_exact(__fmul_rn(omega, f4get(r, u)), dd)));
    }
    st4(X + Q.base, x);
}

// NegativeLaplacianAndGaussSeidelSameLevel128Kernel (src/GMGSolver.cu:173-210, src/CMGSolver.cu:226-262):
// x += (b - Ax) / D on INTERIOR cells of one colour, LEAF and NONLEAF tiles of one level
template <int KIND>
__global__ void __launch_bounds__(128) k_geo_gs(DevGrid g, int t0, float* X, const float* B, int color) {
    __shared__ GSnap S;
    const int t = t0 + blockIdx.x;
    const int own_tt = dLeaf;  // LEAF, or NONLEAF counted as LEAF at its level
    const Quad Q(t, threadIdx.x);
    load_gsnap<KIND>(g, t, X, true, own_tt, S, Q);
    const float h = voxel_size(g.h0, tile_level(g, t));
    const float ooh = __fdiv_rn(1.0f, h);
    const float4 b = ldcg4(B + Q.base);
    float4 out = ldcg4(X + Q.base);
    const int p = (Q.i + Q.j + Q.k0 + color) & 1;
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
        const int u = p + 2 * hh;
        const int k = Q.k0 + u;
        const int c = sx(Q.i, Q.j, k);
        const float ax = geo_neg_lap<KIND>(S, h, ooh, own_tt, Q.i, Q.j, k, false);
        const float dd = geo_neg_lap<KIND>(S, h, ooh, own_tt, Q.i, Q.j, k, true);
        const float delta = (S.ct[c] & dInterior) ? div_exact(__fsub_rn(f4get(b, u), ax), dd) : 0.0f;
        f4set(out, u, __fadd_rn(S.x[c], delta));
    }
    st4(X + Q.base, out);
}

// ResidualAndRestrict128Kernel (src/GMGSolver.cu:225-284), ConservativeResidualAndRestrict128Kernel
// (src/CMGSolver.cu:278-331): coarse rhs = one_over_alpha * sum of 8 residuals; a GMG GHOST tile
// adds its sums to its LEAF parent's rhs instead
template <int KIND>
__global__ void __launch_bounds__(128) k_geo_restrict(DevGrid g, int t0, const float* X, float* RHS, float ooa) {
    __shared__ GSnap S;
    __shared__ float res[kCells];
    const int t = t0 + blockIdx.x;
    const int ty = tile_type(g, t);
    const int own_tt = subtree_type(ty, true);
    const Quad Q(t, threadIdx.x);
    load_gsnap<KIND>(g, t, X, true, own_tt, S, Q);
    const float h = voxel_size(g.h0, tile_level(g, t));
    const float ooh = __fdiv_rn(1.0f, h);
    const float4 rh = ldcg4(RHS + Q.base);
#pragma unroll
    for (int u = 0; u < 4; ++u) res[4 * Q.q + u] = __fsub_rn(f4get(rh, u), geo_neg_lap<KIND>(S, h, ooh, own_tt, Q.i, Q.j, Q.k0 + u, false));
    __syncthreads();
    if (threadIdx.x < 64) {
        const int b = threadIdx.x;
        const int f0 = (b >> 4) * 2, f1 = ((b >> 2) & 3) * 2, f2 = (b & 3) * 2;
        float sum = 0.0f;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) sum = __fadd_rn(sum, res[cell_index(f0 + ii, f1 + jj, f2 + kk)]);
        const int p = g.nb[8 * t + 6];
        if (p >= 0) {
            const int4 m = g.meta[t];
            const size_t o = (size_t)p * kCells + cell_index(parent_local(m.y, f0), parent_local(m.z, f1), parent_local(m.w, f2));
            RHS[o] = (ty & dGhost) ? __fadd_rn(RHS[o], sum) : __fmul_rn(sum, ooa);
        }
    }
}

// ProlongateAndUpdate128Kernel (src/GMGSolver.cu:286-316, src/CMGSolver.cu:339-370)
__global__ void __launch_bounds__(128) k_geo_prolong(DevGrid g, int t0, float* X, float P) {
    const int t = t0 + blockIdx.x;
    const Quad Q(t, threadIdx.x);
    const int4 m = g.meta[t];
    const bool ghost = (m.x >> 8) & dGhost;
    const int p = g.nb[8 * t + 6];
    const float4 xr = ldcg4(X + Q.base);
    const uchar4 ty = ldt4(g.ctype + Q.base);
    const int pi = parent_local(m.y, Q.i), pj = parent_local(m.z, Q.j);
    float4 out;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const float cx = p >= 0 ? ldcg(X + (size_t)p * kCells + cell_index(pi, pj, parent_local(m.w, Q.k0 + u))) : 0.0f;
        const bool in = t4get(ty, u) & dInterior;
        f4set(out, u, ghost ? (in ? cx : 0.0f) : (in ? __fmaf_rn(P, cx, f4get(xr, u)) : 0.0f));
    }
    st4(X + Q.base, out);
}

// V-cycle set-up (src/GMGSolver.cu:327-343): x = 0 everywhere; rhs = f, 0 on GHOST tiles
__global__ void __launch_bounds__(128) k_geo_vinit(DevGrid g, float* X, float* RHS, const float* F) {
    const int t = blockIdx.x;
    const Quad Q(t, threadIdx.x);
    st4(X + Q.base, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    st4(RHS + Q.base, (tile_type(g, t) & dGhost) ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : ldcg4(F + Q.base));
}

// AccumulateToParentsOneStepKernel (src/PoissonGrid.cu:408-449) from the tiles of type `types`:
// parent cell = coeff * sum of its 8 children (added to it when `additive`)
__global__ void __launch_bounds__(64) k_accumulate_cells(DevGrid g, int t0, int types, const float* SRC, float* DST, float coeff, int additive,
                                                         int cell_mask) {
    const int t = t0 + blockIdx.x;
    if (!(tile_type(g, t) & types)) return;
    const int p = g.nb[8 * t + 6];
    if (p < 0) return;
    const int b = threadIdx.x;
    const int f0 = (b >> 4) * 2, f1 = ((b >> 2) & 3) * 2, f2 = (b & 3) * 2;
    float sum = 0.0f;
    for (int ii = 0; ii < 2; ++ii)
        for (int jj = 0; jj < 2; ++jj)
            for (int kk = 0; kk < 2; ++kk) {
                const size_t o = (size_t)t * kCells + cell_index(f0 + ii, f1 + jj, f2 + kk);
                sum = __fadd_rn(sum, (g.ctype[o] & cell_mask) ? ldcg(SRC + o) : 0.0f);
            }
    const int4 m = g.meta[t];
    const size_t po = (size_t)p * kCells + cell_index(parent_local(m.y, f0), parent_local(m.z, f1), parent_local(m.w, f2));
    DST[po] = additive ? __fmaf_rn(sum, coeff, DST[po]) : __fmul_rn(sum, coeff);
}

// CalcCellTypesFromLeafs step 1 (src/PoissonGrid.cu:923-960) on the NONLEAF tiles of one level:
// DIRICHLET if an active child cell is DIRICHLET, else INTERIOR if one is INTERIOR, else NEUMANN
__global__ void __launch_bounds__(128) k_types_from_children(DevGrid g, int t0) {
    const int t = t0 + blockIdx.x;
    if (!(tile_type(g, t) & dNonLeaf)) return;
    for (int v = threadIdx.x; v < kCells; v += blockDim.x) {
        const int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
        const int c = g.child[8 * t + ((i >> 2) << 2) + ((j >> 2) << 1) + (k >> 2)];
        int nd = 0, ni = 0;
        if (c >= 0 && (tile_type(g, c) & (dLeaf | dNonLeaf))) {
            const int b0 = (i & 3) << 1, b1 = (j & 3) << 1, b2 = (k & 3) << 1;
            for (int ii = 0; ii < 2; ++ii)
                for (int jj = 0; jj < 2; ++jj)
                    for (int kk = 0; kk < 2; ++kk) {
                        const int ty = g.ctype[(size_t)c * kCells + cell_index(b0 + ii, b1 + jj, b2 + kk)];
                        if (ty & dDirichlet) ++nd;
                        else if (ty & dInterior) ++ni;
                    }
        }
        g.ctype[(size_t)t * kCells + v] = nd > 0 ? dDirichlet : ni > 0 ? dInterior : dNeumann;
    }
}

}  // namespace

void launch_types_from_children(const DevGrid& g, int t0, int nt, cudaStream_t st) {
    if (nt <= 0) return;
    note_kernel_launch();
    k_types_from_children<<<nt, 128, 0, st>>>(g, t0);
}

void launch_geo_lap(int kind, const DevGrid& g, int t0, int nt, const float* X, float* AX, bool sl_is_level, int types, cudaStream_t st,
                    bool diag) {
    if (nt <= 0) return;
    note_kernel_launch();
    if (kind == kCMG) k_geo_lap<kCMG><<<nt, 128, 0, st>>>(g, t0, X, AX, sl_is_level ? 1 : 0, types, diag ? 1 : 0);
    else k_geo_lap<kGMG><<<nt, 128, 0, st>>>(g, t0, X, AX, sl_is_level ? 1 : 0, types, diag ? 1 : 0);
}
void launch_leaf_residual(const DevGrid& g, const int* leaf, int nleaf, const float* B, float* R, bool interior_only, cudaStream_t st) {
    if (nleaf <= 0) return;
    note_kernel_launch();
    k_leaf_residual<<<nleaf, 128, 0, st>>>(g, leaf, B, R, interior_only ? 1 : 0);
}
void launch_jacobi_update(const DevGrid& g, const int* leaf, int nleaf, float* X, const float* R, const float* D, float omega, cudaStream_t st) {
    if (nleaf <= 0) return;
    note_kernel_launch();
    k_jacobi_update<<<nleaf, 128, 0, st>>>(g, leaf, X, R, D, omega);
}
void launch_geo_gs(int kind, const DevGrid& g, int t0, int nt, float* X, const float* B, int color, cudaStream_t st) {
    if (nt <= 0) return;
    note_kernel_launch();
    if (kind == kCMG) k_geo_gs<kCMG><<<nt, 128, 0, st>>>(g, t0, X, B, color);
    else k_geo_gs<kGMG><<<nt, 128, 0, st>>>(g, t0, X, B, color);
}
void launch_geo_restrict(int kind, const DevGrid& g, int t0, int nt, const float* X, float* RHS, float one_over_alpha, cudaStream_t st) {
    if (nt <= 0) return;
    note_kernel_launch();
    if (kind == kCMG) k_geo_restrict<kCMG><<<nt, 128, 0, st>>>(g, t0, X, RHS, one_over_alpha);
    else k_geo_restrict<kGMG><<<nt, 128, 0, st>>>(g, t0, X, RHS, one_over_alpha);
}
void launch_geo_prolong(const DevGrid& g, int t0, int nt, float* X, float P, cudaStream_t st) {
    if (nt <= 0) return;
    note_kernel_launch();
    k_geo_prolong<<<nt, 128, 0, st>>>(g, t0, X, P);
}
void launch_geo_vinit(const DevGrid& g, float* X, float* RHS, const float* F, cudaStream_t st) {
    if (g.n <= 0) return;
    note_kernel_launch();
    k_geo_vinit<<<g.n, 128, 0, st>>>(g, X, RHS, F);
}
void launch_accumulate_cells(const DevGrid& g, int t0, int nt, int types, const float* SRC, float* DST, float coeff, bool additive,
                             cudaStream_t st, int cell_mask) {
    if (nt <= 0) return;
    note_kernel_launch();
    k_accumulate_cells<<<nt, 64, 0, st>>>(g, t0, types, SRC, DST, coeff, additive ? 1 : 0, cell_mask);
}

}  // namespace cmg
