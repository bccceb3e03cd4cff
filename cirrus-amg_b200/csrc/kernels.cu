// Device kernels of the octree MG-preconditioned CG solve (sm_100a).
//
// Launch shape: one 128-thread block per 8^3 tile; every thread owns four
// consecutive cells along k (one float4 of each channel plane), so each
// channel of a tile moves as one fully coalesced 2 KB transaction set.  Tile
// and halo values are staged in a shared-memory snapshot (device.cuh).
// Reductions are deterministic: one double per block, summed in a fixed order
// by the last block to finish, which then applies the scalar update the
// reference does with one-thread kernels (TernaryOnArray, src/GPUUtils.h:72).
#include "kernels.hpp"
#include "tiles.cuh"

#include <algorithm>
#include <atomic>
#include <cfloat>

namespace cmg {

namespace {

__global__ void __launch_bounds__(128) k_gs(DevGrid g, int t0, float* X, const float* B, int color, SmoothArgs A) {
    __shared__ Snap S;
    tile_gs(g, t0 + blockIdx.x, threadIdx.x, X, B, color, A, S, BlockSync{});
}
__global__ void __launch_bounds__(128) k_restrict(DevGrid g, int t0, float* X, float* RHS, int coeff_ch, float Rr) {
    __shared__ Snap S;
    __shared__ float res[kCells];
    tile_restrict(g, t0 + blockIdx.x, threadIdx.x, X, RHS, coeff_ch, Rr, S, res, BlockSync{});
}
__global__ void __launch_bounds__(128) k_fas_save(DevGrid g, int t0, const float* X, float* RHS, float* X0, int coeff_ch) {
    __shared__ Snap S;
    tile_fas_save(g, t0 + blockIdx.x, threadIdx.x, X, RHS, X0, coeff_ch, S, BlockSync{});
}
__global__ void __launch_bounds__(128) k_prolong(DevGrid g, int t0, float* X, const float* X0, float P) {
    tile_prolong(g, t0 + blockIdx.x, threadIdx.x, X, X0, P);
}

// ---------------------------------------------------------------------------
// Steps of the cycles nothing in the reference's solve calls: AMGSolver::VCycle and
// muCycle (src/AMGSolver.cu:1060-1173), correction schemes with a separate right-hand side
// f, and the prolongation of FASFCycle (src/AMGSolver.cu:1358-1387).
// ---------------------------------------------------------------------------
// the cycle's start: x = 0 on every tile, rhs = f on LEAF and NONLEAF tiles, 0 on GHOST
// tiles (src/AMGSolver.cu:1063-1080)
__global__ void __launch_bounds__(128) k_cycle_init(DevGrid g, float* X, float* RHS, const float* F) {
    const int t = blockIdx.x;
    const size_t base = (size_t)t * kCells + 4 * threadIdx.x;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    st4(X + base, z);
    st4(RHS + base, (tile_type(g, t) & dGhost) ? z : ld4(F + base));
}
// ProlongateAndUpdateAMG128Kernel (src/AMGSolver.cu:1026-1057) on every tile of a level:
// GHOST cells take the parent's x, the others add P times it; 0 on cells that are not INTERIOR
__global__ void __launch_bounds__(128) k_prolong_add(DevGrid g, int t0, float* X, float P) {
    const int t = t0 + blockIdx.x;
    const Quad Q(t, threadIdx.x);
    const int4 m = g.meta[t];
    const bool ghost = (m.x >> 8) & dGhost;
    const int p = g.nb[8 * t + 6];
    const float4 xr = ld4(X + Q.base);
    const uchar4 ty = ldt4(g.ctype + Q.base);
    const int pi = parent_local(m.y, Q.i), pj = parent_local(m.z, Q.j);
    float4 out;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const float cx = p >= 0 ? X[(size_t)p * kCells + cell_index(pi, pj, parent_local(m.w, Q.k0 + u))] : 0.0f;
        const bool in = t4get(ty, u) & dInterior;
        f4set(out, u, ghost ? (in ? cx : 0.0f) : (in ? __fmaf_rn(P, cx, f4get(xr, u)) : 0.0f));
    }
    st4(X + Q.base, out);
}
// DeductFluxOnAbsLeafs128Kernel (src/AMGSolver.cu:966-992) on LEAF tiles: rhs = f minus the
// operator's terms from cells of NONLEAF neighbour tiles (AMGLaplacianTileData::
// negativeLapOuterNonLeaf, src/AMGSolver.cu:384-405: the tile's own cells count 0, each face
// term in the order -x,+x,-y,+y,-z,+z) on INTERIOR cells, 0 elsewhere
__global__ void __launch_bounds__(128) k_deduct_flux(DevGrid g, int t0, const float* X, const float* F, float* RHS, int coeff_ch) {
    __shared__ Snap S;
    const int t = t0 + blockIdx.x;
    const Quad Q(t, threadIdx.x);
    Own o;
    load_snap(g, t, X, coeff_ch, MgHalo{X, g.ctype}, S, Q, o, BlockSync{});
    bool nonleaf[6];  // -x, -y, -z, +x, +y, +z neighbour tile is NONLEAF
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int d = g.nbx[8 * t + f];
        nonleaf[f] = d != 0 && (d & 7) == dNonLeaf;
    }
    const float4 fv = ld4(F + Q.base);
    float4 out;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int i = Q.i, j = Q.j, k = Q.k0 + u;
        const float d = f4get(o.dg, u);
        float s = 0.0f;
        if (d != 0.0f) {
            s = __fmul_rn(0.0f, d);
            // -x, +x
            s = __fmaf_rn(S.c0[i * 64 + j * 8 + k], (i == 0 && nonleaf[0]) ? S.x[sx(i - 1, j, k)] : 0.0f, s);
            s = __fmaf_rn(S.c0[(i + 1) * 64 + j * 8 + k], (i == 7 && nonleaf[3]) ? S.x[sx(i + 1, j, k)] : 0.0f, s);
            // -y, +y
            s = __fmaf_rn(S.c1[i * 72 + j * 8 + k], (j == 0 && nonleaf[1]) ? S.x[sx(i, j - 1, k)] : 0.0f, s);
            s = __fmaf_rn(S.c1[i * 72 + (j + 1) * 8 + k], (j == 7 && nonleaf[4]) ? S.x[sx(i, j + 1, k)] : 0.0f, s);
            // -z, +z
            s = __fmaf_rn(S.c2[i * 72 + j * 9 + k], (k == 0 && nonleaf[2]) ? S.x[sx(i, j, k - 1)] : 0.0f, s);
            s = __fmaf_rn(S.c2[i * 72 + j * 9 + k + 1], (k == 7 && nonleaf[5]) ? S.x[sx(i, j, k + 1)] : 0.0f, s);
        }
        f4set(out, u, (t4get(o.ty, u) & dInterior) ? __fsub_rn(f4get(fv, u), s) : 0.0f);
    }
    st4(RHS + Q.base, out);
}

__global__ void __launch_bounds__(1024) k_coarse(DevGrid g, CoarseArgs A, float* X, float* RHS, float* X0) {
    extern __shared__ __align__(16) unsigned char smraw[];
    coarse_dense(g, A, X, RHS, X0, smraw);
}

// ---------------------------------------------------------------------------
// Persistent kernel for the middle of the hierarchy: FASMuCycleStep of level
// 2 or 3 (all of its mu-recursions) in one cooperative launch.  Each block
// runs four 128-thread slots on four tiles at once; phases (a colour sweep,
// restriction, FAS update, prolongation of one level) are separated by a
// grid barrier, and levels 0-1 run in block 0 with the dense coarse code.
// The barrier spin is bounded: past the limit the kernel records an error
// and every block returns.
// ---------------------------------------------------------------------------
struct PersistArgs {
    int top;
    int lb[4], ab[4], le[4], nlb[4];  // level begin, active end (first GHOST), level end, first NONLEAF
    int mu, level_iters, coarsest_iters;
    SmoothArgs sm;
    CoarseArgs co;
    float Rr, P;
    float *X, *RHS, *X0;
    unsigned int* bar;  // [0] arrivals, [1] generation, [2] error flag
};
constexpr int kSlots = 4;
constexpr size_t kPersistSmem = kCoarseSmem + kSlots * (sizeof(Snap) + sizeof(float) * kCells);

__device__ bool grid_sync(const PersistArgs& A) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = A.bar + 1;
        const unsigned int g0 = *gen;
        __threadfence();
        if (atomicAdd(A.bar, 1u) == gridDim.x - 1) {
            A.bar[0] = 0;
            __threadfence();
            atomicAdd(A.bar + 1, 1u);
        } else {
            unsigned int spins = 0;
            while (*gen == g0) {
                if (++spins > (1u << 24)) {  // ~1 s
                    atomicExch(A.bar + 2, 1u);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *((volatile unsigned int*)A.bar + 2) == 0;
}

struct PersistCtx {
    DevGrid g;
    PersistArgs A;
    Snap* S;
    float* res;
    unsigned char* coarse_smem;
    int slot, tid, gslot, nslot;
    SlotSync sync;
};

__device__ bool p_gs(PersistCtx& C, int l, int iters, int order) {
    for (int it = 0; it < iters; ++it)
        for (int h = 0; h < 2; ++h) {
            const int color = h ? 1 - order : order;
            for (int t = C.A.lb[l] + C.gslot; t < C.A.ab[l]; t += C.nslot) tile_gs(C.g, t, C.tid, C.A.X, C.A.RHS, color, C.A.sm, *C.S, C.sync);
            if (!grid_sync(C.A)) return false;
        }
    return true;
}
__device__ bool p_restrict_and_save(PersistCtx& C, int l) {
    for (int t = C.A.lb[l] + C.gslot; t < C.A.ab[l]; t += C.nslot)
        tile_restrict(C.g, t, C.tid, C.A.X, C.A.RHS, C.A.sm.coeff_ch, C.A.Rr, *C.S, C.res, C.sync);
    if (!grid_sync(C.A)) return false;
    for (int t = C.A.nlb[l - 1] + C.gslot; t < C.A.ab[l - 1]; t += C.nslot)
        tile_fas_save(C.g, t, C.tid, C.A.X, C.A.RHS, C.A.X0, C.A.sm.coeff_ch, *C.S, C.sync);
    return grid_sync(C.A);
}
__device__ bool p_prolong(PersistCtx& C, int l) {
    for (int t = C.A.lb[l] + C.gslot; t < C.A.le[l]; t += C.nslot) tile_prolong(C.g, t, C.tid, C.A.X, C.A.X0, C.A.P);
    return grid_sync(C.A);
}
__device__ bool p_step1(PersistCtx& C) {
    if (blockIdx.x == 0) coarse_dense(C.g, C.A.co, C.A.X, C.A.RHS, C.A.X0, C.coarse_smem);
    return grid_sync(C.A);
}
__device__ bool p_step2(PersistCtx& C) {
    if (!p_gs(C, 2, C.A.level_iters, 0) || !p_restrict_and_save(C, 2)) return false;
    for (int r = 0; r < C.A.mu; ++r)
        if (!p_step1(C)) return false;
    return p_prolong(C, 2) && p_gs(C, 2, C.A.level_iters, 1);
}
__device__ bool p_step3(PersistCtx& C) {
    if (!p_gs(C, 3, C.A.level_iters, 0) || !p_restrict_and_save(C, 3)) return false;
    for (int r = 0; r < C.A.mu; ++r)
        if (!p_step2(C)) return false;
    return p_prolong(C, 3) && p_gs(C, 3, C.A.level_iters, 1);
}

__global__ void __launch_bounds__(512) k_persist(DevGrid g, PersistArgs A) {
    extern __shared__ __align__(16) unsigned char smraw[];
    PersistCtx C;
    C.g = g;
    C.A = A;
    C.slot = threadIdx.x >> 7;
    C.tid = threadIdx.x & 127;
    C.gslot = blockIdx.x * kSlots + C.slot;
    C.nslot = gridDim.x * kSlots;
    C.coarse_smem = smraw;
    C.S = reinterpret_cast<Snap*>(smraw + kCoarseSmem) + C.slot;
    C.res = reinterpret_cast<float*>(smraw + kCoarseSmem + kSlots * sizeof(Snap)) + C.slot * kCells;
    C.sync = SlotSync{1 + C.slot};
    if (A.top == 3) p_step3(C);
    else p_step2(C);
}

// ---------------------------------------------------------------------------
// PCG on LEAF tiles
// ---------------------------------------------------------------------------
// AMGFullNegativeLaplacianOnLeafs (src/AMGSolver.cu:589-632) with the p.Ap dot
// (src/AMGSolver.cu:1455) and alpha = gamma / pAp (src/AMGSolver.cu:1457) fused.
__global__ void __launch_bounds__(128) k_leaf_apply(DevGrid g, const int* leaf, const float* P, float* AP, int coeff_ch, int fuse,
                                                    ReduceScratch rs) {
    __shared__ Snap S;
    __shared__ double red[4];
    const int t = leaf[blockIdx.x];
    const Quad Q(t, threadIdx.x);
    Own o;
    load_snap(g, t, P, coeff_ch, LeafHalo{P, g.ctype}, S, Q, o, BlockSync{});
    float4 ap;
    ap.x = o.ty.x == dInterior ? own_neg_lap<0>(S, Q, o) : 0.0f;
    ap.y = o.ty.y == dInterior ? own_neg_lap<1>(S, Q, o) : 0.0f;
    ap.z = o.ty.z == dInterior ? own_neg_lap<2>(S, Q, o) : 0.0f;
    ap.w = o.ty.w == dInterior ? own_neg_lap<3>(S, Q, o) : 0.0f;
    st4(AP + Q.base, ap);
    if (!fuse) return;
    const double bs = block_sum128(dot4(o.xr, ap), red);
    if (threadIdx.x == 0) rs.partial[blockIdx.x] = bs;
    if (last_block(&rs.s->counter[0])) {
        const double tot = sum_partials(rs.partial, gridDim.x, red);
        if (threadIdx.x == 0) {
            PcgScalars* s = rs.s;
            s->pAp = tot;
            s->alpha = s->gamma / tot;
            s->counter[0] = 0;
        }
    }
}

// x += alpha p, r -= alpha Ap on INTERIOR cells (src/AMGSolver.cu:1462-1485),
// r.r (src/AMGSolver.cu:1488) and the convergence test (src/AMGSolver.cu:1487-1496)
// True-residual replacement (no counterpart in the reference; the mixed-precision solve):
// on iterations that are a multiple of `every`, r = b - A x on the LEAF tiles, the stencil
// summed in double and the difference rounded once to float.  Cells that are not INTERIOR
// keep b, which the recurrence never changes there.  The iteration count is read on the
// device, so every other iteration returns at once.
__global__ void __launch_bounds__(128) k_true_residual(DevGrid g, const int* leaf, const float* X, const float* B, float* R,
                                                       int coeff_ch, PcgScalars* s, int every) {
    const int it = s->iter;
    if (it == 0 || it % every != 0) return;
    __shared__ Snap S;
    const int t = leaf[blockIdx.x];
    const Quad Q(t, threadIdx.x);
    Own o;
    load_snap(g, t, X, coeff_ch, LeafHalo{X, g.ctype}, S, Q, o, BlockSync{});
    const float4 b = ld4(B + Q.base);
    float4 r = b;
    if (o.ty.x == dInterior) r.x = (float)((double)b.x - own_neg_lap64<0>(S, Q, o));
    if (o.ty.y == dInterior) r.y = (float)((double)b.y - own_neg_lap64<1>(S, Q, o));
    if (o.ty.z == dInterior) r.z = (float)((double)b.z - own_neg_lap64<2>(S, Q, o));
    if (o.ty.w == dInterior) r.w = (float)((double)b.w - own_neg_lap64<3>(S, Q, o));
    st4(R + Q.base, r);
    if (blockIdx.x == 0 && threadIdx.x == 0) ++s->replaced;
}

__global__ void __launch_bounds__(128) k_xr_update(DevGrid g, const int* leaf, int nleaf, float* X, float* R, const float* P,
                                                   const float* AP, ReduceScratch rs, cudaGraphConditionalHandle loop_h,
                                                   cudaGraphConditionalHandle body_h, int use_handles) {
    __shared__ double red[4];
    const float alpha = (float)rs.s->alpha;
    // the block walks the leaf list with stride gridDim.x, the next tile's planes in flight
    // while it finishes the current one; tile i's partial is what one block per tile gives
    int i = blockIdx.x;
    Quad Q(leaf[i], threadIdx.x);
    float4 x = ld4(X + Q.base), r = ld4(R + Q.base), p = ld4(P + Q.base), ap = ld4(AP + Q.base);
    uchar4 ty = ldt4(g.ctype + Q.base);
    for (;;) {
        const int in = i + gridDim.x;
        const bool more = in < nleaf;
        const Quad Qn(more ? leaf[in] : 0, threadIdx.x);
        float4 xn = x, rn = r, pn = p, apn = ap;
        uchar4 tyn = ty;
        if (more) {
            xn = ld4(X + Qn.base);
            rn = ld4(R + Qn.base);
            pn = ld4(P + Qn.base);
            apn = ld4(AP + Qn.base);
            tyn = ldt4(g.ctype + Qn.base);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (t4get(ty, u) & dInterior) {
                f4set(x, u, __fmaf_rn(alpha, f4get(p, u), f4get(x, u)));
                f4set(r, u, __fmaf_rn(-alpha, f4get(ap, u), f4get(r, u)));
            }
        }
        st4(X + Q.base, x);
        st4(R + Q.base, r);
        const double bs = block_sum128(dot4(r, r), red);
        if (threadIdx.x == 0) rs.partial[i] = bs;
        if (!more) break;
        i = in;
        Q = Qn;
        x = xn, r = rn, p = pn, ap = apn, ty = tyn;
    }
    if (last_block(&rs.s->counter[1])) {
        const double rr = sum_partials(rs.partial, nleaf, red);
        if (threadIdx.x == 0) {
            PcgScalars* s = rs.s;
            s->rr = rr;
            const int it = ++s->iter;
            const bool bad = !isfinite(rr) || !isfinite(s->alpha);
            const bool conv = s->sync_stride > 0 && (it % s->sync_stride) == 0 && rr < s->thr;
            bool stalled = false;
            if (s->stall_window > 0 && s->sync_stride > 0) {
                const int w = s->stall_window, h = it % w;
                stalled = it > w && !conv && rr > 0.25 * s->rr_hist[h];
                s->rr_hist[h] = rr;
            }
            s->stalled = stalled;
            const bool done = conv || bad || stalled || it >= s->max_iters;
            s->converged = conv;
            s->nonfinite = bad;
            s->done = done;
            s->counter[1] = 0;
            if (use_handles) {
                cudaGraphSetConditional(loop_h, done ? 0u : 1u);
                cudaGraphSetConditional(body_h, done ? 0u : 1u);
            }
        }
    }
}

__global__ void __launch_bounds__(128) k_dot(const int* leaf, int nleaf, const float* A, const float* B, int mode, double* out,
                                             ReduceScratch rs) {
    __shared__ double red[4];
    // grid-stride over the leaf list, the next tile's loads in flight; per-tile partials as
    // with one block per tile
    int i = blockIdx.x;
    size_t base = (size_t)leaf[i] * kCells + 4 * threadIdx.x;
    float4 a = ld4(A + base), b = ld4(B + base);
    for (;;) {
        const int in = i + gridDim.x;
        const bool more = in < nleaf;
        float4 an = a, bn = b;
        if (more) {
            base = (size_t)leaf[in] * kCells + 4 * threadIdx.x;
            an = ld4(A + base);
            bn = ld4(B + base);
        }
        const double bs = block_sum128(dot4(a, b), red);
        if (threadIdx.x == 0) rs.partial[i] = bs;
        if (!more) break;
        i = in;
        a = an, b = bn;
    }
    if (last_block(&rs.s->counter[2])) {
        const double d = sum_partials(rs.partial, nleaf, red);
        if (threadIdx.x == 0) {
            PcgScalars* s = rs.s;
            if (mode == kDotStore) *out = d;
            else if (mode == kDotRR0) s->rr0 = d;
            else if (mode == kDotGammaInit) s->gamma = d;
            else if (mode == kDotAlpha) {  // p.Ap and alpha = gamma / p.Ap (src/GMGSolver.cu:518-521)
                s->pAp = d;
                s->alpha = s->gamma / d;
            } else {  // src/AMGSolver.cu:1513-1520
                s->gamma_old = s->gamma;
                s->gamma = d;
                s->beta = d / s->gamma_old;
            }
            s->counter[2] = 0;
        }
    }
}

// Flexible CG with a non-linear preconditioner (Polak-Ribiere): with r_new = r_old - alpha Ap,
// beta = z.(r_new - r_old) / gamma_old = -alpha (Ap.z) / gamma_old; gamma = r_new.z.
__global__ void __launch_bounds__(128) k_dot_flex(const int* leaf, const float* R, const float* Z, const float* AP, ReduceScratch rs) {
    __shared__ double red[4];
    const int t = leaf[blockIdx.x];
    const size_t base = (size_t)t * kCells + 4 * threadIdx.x;
    const float4 z = ld4(Z + base);
    const double rz = block_sum128(dot4(ld4(R + base), z), red);
    const double az = block_sum128(dot4(ld4(AP + base), z), red);
    if (threadIdx.x == 0) {
        rs.partial[blockIdx.x] = rz;
        rs.partial2[blockIdx.x] = az;
    }
    if (last_block(&rs.s->counter[2])) {
        const double g = sum_partials(rs.partial, gridDim.x, red);
        const double a = sum_partials(rs.partial2, gridDim.x, red);
        if (threadIdx.x == 0) {
            PcgScalars* s = rs.s;
            s->gamma_old = s->gamma;
            s->gamma = g;
            s->beta = -s->alpha * a / s->gamma_old;
            s->counter[2] = 0;
        }
    }
}

// p = z + beta p on INTERIOR cells (src/AMGSolver.cu:1525-1536)
__global__ void __launch_bounds__(128) k_p_update(DevGrid g, const int* leaf, float* P, const float* Z, ReduceScratch rs) {
    const int t = leaf[blockIdx.x];
    const size_t base = (size_t)t * kCells + 4 * threadIdx.x;
    const float beta = (float)rs.s->beta;
    float4 p = ld4(P + base);
    const float4 z = ld4(Z + base);
    const uchar4 ty = ldt4(g.ctype + base);
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if (t4get(ty, u) & dInterior) f4set(p, u, __fmaf_rn(beta, f4get(p, u), f4get(z, u)));
    st4(P + base, p);
}

__global__ void k_leaf_fill(const int* leaf, float* X, float v) {
    const size_t base = (size_t)leaf[blockIdx.x] * kCells + 4 * threadIdx.x;
    st4(X + base, make_float4(v, v, v, v));
}
__global__ void k_leaf_copy(const int* leaf, float* D, const float* Sx) {
    const size_t base = (size_t)leaf[blockIdx.x] * kCells + 4 * threadIdx.x;
    st4(D + base, ld4(Sx + base));
}

// ReCenterLeafCells (src/PoissonGrid.cu:889-921)
__global__ void __launch_bounds__(128) k_mean_partial(DevGrid g, const int* leaf, const float* R, ReduceScratch rs) {
    __shared__ double red[4];
    const size_t base = (size_t)leaf[blockIdx.x] * kCells + 4 * threadIdx.x;
    const float4 r = ld4(R + base);
    const uchar4 ty = ldt4(g.ctype + base);
    float f = 0.0f;
    int c = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const bool in = t4get(ty, u) & dInterior;
        const float v = in ? f4get(r, u) : 0.0f;
        f = (u == 0) ? v : __fadd_rn(f, v);
        c += in;
    }
    const double bs = block_sum128((double)f, red);
    const double bc = block_sum128((double)c, red);
    if (threadIdx.x == 0) {
        rs.partial[blockIdx.x] = bs;
        rs.partial2[blockIdx.x] = bc;
    }
    if (last_block(&rs.s->counter[3])) {
        const double sum = sum_partials(rs.partial, gridDim.x, red);
        const double cnt = sum_partials(rs.partial2, gridDim.x, red);
        if (threadIdx.x == 0) {
            rs.s->mean = sum / cnt;
            rs.s->count = cnt;
            rs.s->counter[3] = 0;
        }
    }
}
__global__ void k_sub_mean(DevGrid g, const int* leaf, float* R, ReduceScratch rs) {
    const size_t base = (size_t)leaf[blockIdx.x] * kCells + 4 * threadIdx.x;
    const double mean = rs.s->mean;
    float4 r = ld4(R + base);
    const uchar4 ty = ldt4(g.ctype + base);
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if (t4get(ty, u) & dInterior) f4set(r, u, (float)((double)f4get(r, u) - mean));
    st4(R + base, r);
}

// threshold (epsilon |b|)^2 and the b == 0 exit (src/AMGSolver.cu:1410-1426), then the loop condition
__global__ void k_loop_gate(ReduceScratch rs, cudaGraphConditionalHandle loop_h, int use_handle) {
    PcgScalars* s = rs.s;
    if (s->sync_stride > 0) {
        const double t = s->tol * s->tol * s->rr0;
        s->thr = t > DBL_MIN ? t : DBL_MIN;
        if (s->rr0 == 0.0) s->done = 1;
    }
    if (s->iter >= s->max_iters) s->done = 1;
    if (use_handle) cudaGraphSetConditional(loop_h, s->done == 0 ? 1u : 0u);
}

// ---------------------------------------------------------------------------
// operator set-up
// ---------------------------------------------------------------------------
// GHOST cell type := parent cell type (src/AMGSolver.cu:265-274)
__global__ void k_ghost_types(DevGrid g, int t0) {
    const int t = t0 + blockIdx.x;
    const int4 m = g.meta[t];
    if (!((m.x >> 8) & dGhost)) return;
    const int p = g.nb[8 * t + 6];
    for (int v = threadIdx.x; v < kCells; v += blockDim.x) {
        uint8_t ty = dDirichlet;
        if (p >= 0)
            ty = g.ctype[(size_t)p * kCells + cell_index(parent_local(m.y, v >> 6), parent_local(m.z, (v >> 3) & 7), parent_local(m.w, v & 7))];
        g.ctype[(size_t)t * kCells + v] = ty;
    }
}

// NegativeLaplacianCoeff (src/AMGSolver.cu:12-24)
__device__ __forceinline__ bool face_valid(int tt0, int tt1, int c0, int c1) {
    const bool both_leafs = (tt0 & dLeaf) && (tt1 & dLeaf);
    const bool leaf_ghost = ((tt0 & dLeaf) && (tt1 & dGhost)) || ((tt0 & dGhost) && (tt1 & dLeaf));
    const bool has_neumann = (c0 & dNeumann) || (c1 & dNeumann);
    const bool has_interior = (c0 & dInterior) || (c1 & dInterior);
    return (both_leafs || leaf_ghost) && !has_neumann && has_interior;
}
// FracInside (cirrus_cutcell/MeshCutCell.cu:262-272)
__device__ __forceinline__ float frac_inside(float a, float b) {
    if (a < 0.0f && b < 0.0f) return 0.0f;
    if (a < 0.0f && b >= 0.0f) return __fdiv_rn(b, __fsub_rn(b, a));
    if (a >= 0.0f && b < 0.0f) return __fdiv_rn(a, __fsub_rn(a, b));
    return 1.0f;
}
// Fluid fraction of a face from its four corner SDFs in cyclic order: the
// marching-squares area rule of FaceFluidRatio (MeshCutCell.cu:305-408).
__device__ float face_fluid_ratio(const float phi[4]) {
    int in[4], nin = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        in[i] = phi[i] < 0.0f;
        nin += in[i];
    }
    float ret;
    if (nin == 4) ret = 0.0f;
    else if (nin == 0) ret = 1.0f;
    else if (nin == 3) {
        int m = 0;
        while (in[m]) ++m;
        ret = (float)(0.5 * (double)frac_inside(phi[m], phi[(m + 3) & 3]) * (double)frac_inside(phi[m], phi[(m + 1) & 3]));
    } else if (nin == 1) {
        int m = 0;
        while (!in[m]) ++m;
        const float e1 = (float)(1.0 - (double)frac_inside(phi[m], phi[(m + 1) & 3]));
        const float e2 = (float)(1.0 - (double)frac_inside(phi[m], phi[(m + 3) & 3]));
        ret = (float)(1.0 - 0.5 * (double)e1 * (double)e2);
    } else if (in[0] == in[2]) {
        const int f0 = in[0] ? 1 : 0, f1 = f0 + 2;
        const double t0 = 0.5 * (double)frac_inside(phi[f0], phi[(f0 + 3) & 3]) * (double)frac_inside(phi[f0], phi[(f0 + 1) & 3]);
        const double t1 = 0.5 * (double)frac_inside(phi[f1], phi[(f1 + 3) & 3]) * (double)frac_inside(phi[f1], phi[(f1 + 1) & 3]);
        ret = (float)(t0 + t1);
    } else {
        // the two crossing edges of a trapezoid, summed in float (the sign of a zero
        // result follows that sum)
        float e[2] = {0.0f, 0.0f};
        int ne = 0;
        for (int i = 0; i < 4; ++i) {
            if (in[i]) continue;
            const int nbc = in[(i + 1) & 3] ? ((i + 1) & 3) : ((i + 3) & 3);
            e[ne++] = frac_inside(phi[i], phi[nbc]);
        }
        ret = (float)(0.5 * (double)__fadd_rn(e[0], e[1]));
    }
    if (ret < 0.1f && ret != 0.0f) ret = 0.1f;
    return ret;
}
// node SDF of a union of spheres at global node (gi, gj, gk) of a level with voxel size h
__device__ __forceinline__ float node_sdf(int gi, int gj, int gk, float h, int ns, const float* sp) {
    const float px = __fmul_rn((float)gi, h), py = __fmul_rn((float)gj, h), pz = __fmul_rn((float)gk, h);
    float best = FLT_MAX;
    for (int s = 0; s < ns; ++s) {
        const float dx = __fsub_rn(px, sp[4 * s]), dy = __fsub_rn(py, sp[4 * s + 1]), dz = __fsub_rn(pz, sp[4 * s + 2]);
        const float d = __fsub_rn(__fsqrt_rn(__fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)))), sp[4 * s + 3]);
        best = fminf(best, d);
    }
    return best;
}

// Face coefficients of LEAF and GHOST cells, 0 on NONLEAF (src/AMGSolver.cu:277-315);
// with spheres, -h times the face fluid fraction (MeshCutCell.cu:452-540).
__global__ void k_face_coeffs(DevGrid g, int t0, int coeff_ch, int ns, const float* sp) {
    const int t = t0 + blockIdx.x;
    const int4 m = g.meta[t];
    const int tt0 = (m.x >> 8) & 0xff, level = m.x & 0xff;
    const float h = voxel_size(g.h0, level);
    for (int v = threadIdx.x; v < kCells; v += blockDim.x) {
        const int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
        const int stride[3] = {64, 8, 1};
        const int c0 = g.ctype[(size_t)t * kCells + v];
        for (int a = 0; a < 3; ++a) {
            float c = 0.0f;  // NONLEAF: 0 (src/AMGSolver.cu:287, MeshCutCell.cu:463)
            if (tt0 != dNonLeaf) {
                c = -0.0f;  // LEAF/GHOST: -coeff with coeff = 0 unless the face is valid (:312)
                int q = t, nv = v - stride[a];
                if (l[a] == 0) {
                    q = g.nb[8 * t + a];
                    nv = v + 7 * stride[a];
                }
                const int tt1 = q < 0 ? tt0 : tile_type(g, q);
                const int c1 = q < 0 ? dDirichlet : g.ctype[(size_t)q * kCells + nv];
                if (face_valid(tt0, tt1, c0, c1)) {
                    if (ns == 0) c = -h;
                    else {
                        // corners of the negative face in cyclic order (FaceCornerSDFs, MeshCutCell.cu:274-303)
                        const int gi = m.y * 8 + l[0], gj = m.z * 8 + l[1], gk = m.w * 8 + l[2];
                        float phi[4];
                        if (a == 0) {
                            phi[0] = node_sdf(gi, gj, gk, h, ns, sp); phi[1] = node_sdf(gi, gj, gk + 1, h, ns, sp);
                            phi[2] = node_sdf(gi, gj + 1, gk + 1, h, ns, sp); phi[3] = node_sdf(gi, gj + 1, gk, h, ns, sp);
                        } else if (a == 1) {
                            phi[0] = node_sdf(gi, gj, gk, h, ns, sp); phi[1] = node_sdf(gi, gj, gk + 1, h, ns, sp);
                            phi[2] = node_sdf(gi + 1, gj, gk + 1, h, ns, sp); phi[3] = node_sdf(gi + 1, gj, gk, h, ns, sp);
                        } else {
                            phi[0] = node_sdf(gi, gj, gk, h, ns, sp); phi[1] = node_sdf(gi, gj + 1, gk, h, ns, sp);
                            phi[2] = node_sdf(gi + 1, gj + 1, gk, h, ns, sp); phi[3] = node_sdf(gi + 1, gj, gk, h, ns, sp);
                        }
                        c = -__fmul_rn(h, face_fluid_ratio(phi));
                    }
                }
            }
            g.plane(coeff_ch + a)[(size_t)t * kCells + v] = c;
        }
    }
}

// LEAF cells with all eight corners inside the solid become NEUMANN (MeshCutCell.cu:421-429)
__global__ void k_cutcell_neumann(DevGrid g, const int* leaf, int ns, const float* sp) {
    const int t = leaf[blockIdx.x];
    const int4 m = g.meta[t];
    const float h = voxel_size(g.h0, m.x & 0xff);
    const float eps = __fmul_rn(h, 1e-3f);
    for (int v = threadIdx.x; v < kCells; v += blockDim.x) {
        const int gi = m.y * 8 + (v >> 6), gj = m.z * 8 + ((v >> 3) & 7), gk = m.w * 8 + (v & 7);
        int cnt = 0;
        for (int d = 0; d < 8; ++d)
            if (__fsub_rn(node_sdf(gi + (d >> 2), gj + ((d >> 1) & 1), gk + (d & 1), h, ns, sp), eps) < 0.0f) ++cnt;
        if (cnt == 8) g.ctype[(size_t)t * kCells + v] = dNeumann;
    }
}

// coarse face += R * (sum of the 4 fine faces) (CoarsenOffDiagCoefficientsOneStepKernel, src/AMGSolver.cu:27-78)
__global__ void k_coarsen_offdiag(DevGrid g, int t0, int coeff_ch, float R) {
    const int t = t0 + blockIdx.x;
    const int b = threadIdx.x;  // 64 threads: one 2x2x2 block each
    const int p = g.nb[8 * t + 6];
    if (p < 0) return;
    const int4 m = g.meta[t];
    const int f[3] = {(b >> 4) * 2, ((b >> 2) & 3) * 2, (b & 3) * 2};
    const size_t pv = (size_t)p * kCells + cell_index(parent_local(m.y, f[0]), parent_local(m.z, f[1]), parent_local(m.w, f[2]));
    for (int a = 0; a < 3; ++a) {
        const float* C = g.plane(coeff_ch + a) + (size_t)t * kCells;
        float s = 0.0f;
        for (int jj = 0; jj < 2; ++jj)
            for (int kk = 0; kk < 2; ++kk) {
                int o[3];
                o[a] = 0;
                o[(a + 1) % 3] = jj;
                o[(a + 2) % 3] = kk;
                s = __fadd_rn(s, C[cell_index(f[0] + o[0], f[1] + o[1], f[2] + o[2])]);
            }
        float* cc = g.plane(coeff_ch + a) + pv;
        *cc = __fmaf_rn(s, R, *cc);
    }
}

// diagonal coefficients and NONLEAF cell types (src/AMGSolver.cu:124-253), one level
__global__ void k_diag(DevGrid g, int t0, int coeff_ch, float R) {
    const int t = t0 + blockIdx.x;
    const int4 m = g.meta[t];
    const int tt = (m.x >> 8) & 0xff;
    const float h = voxel_size(g.h0, m.x & 0xff);
    float* D = g.plane(coeff_ch + 3) + (size_t)t * kCells;
    for (int v = threadIdx.x; v < kCells; v += blockDim.x) {
        const int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
        const int stride[3] = {64, 8, 1};
        if (tt & (dLeaf | dGhost)) {
            float d = 0.0f;
            if (g.ctype[(size_t)t * kCells + v] & dInterior) {
                for (int a = 0; a < 3; ++a) {
                    d = __fsub_rn(d, g.plane(coeff_ch + a)[(size_t)t * kCells + v]);
                    int q = t, nv = v + stride[a];
                    if (l[a] == 7) {
                        q = g.nb[8 * t + 3 + a];
                        nv = v - 7 * stride[a];
                    }
                    const float c1 = q < 0 ? -h : g.plane(coeff_ch + a)[(size_t)q * kCells + nv];
                    d = __fsub_rn(d, c1);
                }
            }
            D[v] = d;
        } else {
            const int q = g.child[8 * t + (l[0] >> 2) * 4 + (l[1] >> 2) * 2 + (l[2] >> 2)];
            int ct[8];
            float off[3][8];
            float dsum = 0.0f;
            int interior_cnt = 0;
            for (int ci = 0; ci < 8; ++ci) {
                if (q >= 0) {
                    const size_t cv = (size_t)q * kCells + cell_index(((l[0] & 3) << 1) + (ci >> 2), ((l[1] & 3) << 1) + ((ci >> 1) & 1),
                                                                       ((l[2] & 3) << 1) + (ci & 1));
                    dsum = __fadd_rn(dsum, g.plane(coeff_ch + 3)[cv]);
                    ct[ci] = g.ctype[cv];
                    interior_cnt += (ct[ci] == dInterior);
                    for (int a = 0; a < 3; ++a) off[a][ci] = g.plane(coeff_ch + a)[cv];
                } else {
                    ct[ci] = dDirichlet;
                    for (int a = 0; a < 3; ++a) off[a][ci] = 0.0f;
                }
            }
            // internal child faces, each counted from both sides of the pair
            for (int ci = 0; ci < 8; ++ci) {
                const int x = ci >> 2, y = (ci >> 1) & 1, z = ci & 1;
                if (ct[0 * 4 + y * 2 + z] == dInterior && ct[1 * 4 + y * 2 + z] == dInterior) dsum = __fadd_rn(dsum, off[0][4 + y * 2 + z]);
                if (ct[x * 4 + 0 * 2 + z] == dInterior && ct[x * 4 + 1 * 2 + z] == dInterior) dsum = __fadd_rn(dsum, off[1][x * 4 + 2 + z]);
                if (ct[x * 4 + y * 2 + 0] == dInterior && ct[x * 4 + y * 2 + 1] == dInterior) dsum = __fadd_rn(dsum, off[2][x * 4 + y * 2 + 1]);
            }
            g.ctype[(size_t)t * kCells + v] = interior_cnt > 0 ? dInterior : dDirichlet;
            D[v] = __fmul_rn(dsum, R);
        }
    }
}

// ---------------------------------------------------------------------------
// right-hand side: face velocity of Fourier modes and its divergence
// ---------------------------------------------------------------------------
__global__ void k_face_velocity(DevGrid g, const int* leaf, int u_ch, int nm, const double* modes) {
    const int t = leaf[blockIdx.x];
    const int4 m = g.meta[t];
    const double h = (double)voxel_size(g.h0, m.x & 0xff);
    const double two_pi = 6.283185307179586;
    const double* kv = modes;
    const double* amp = modes + 3 * nm;
    const double* ph = modes + 6 * nm;
    for (int v = threadIdx.x; v < kCells; v += blockDim.x) {
        const int gc[3] = {m.y * 8 + (v >> 6), m.z * 8 + ((v >> 3) & 7), m.w * 8 + (v & 7)};
        for (int a = 0; a < 3; ++a) {
            double p[3];
            for (int d = 0; d < 3; ++d) p[d] = ((double)gc[d] + (d == a ? 0.0 : 0.5)) * h;
            double u = 0;
            for (int q = 0; q < nm; ++q) {
                const double arg = two_pi * (kv[3 * q] * p[0] + kv[3 * q + 1] * p[1] + kv[3 * q + 2] * p[2]) + ph[q];
                u += amp[3 * q + a] * sin(arg);
            }
            g.plane(u_ch + a)[(size_t)t * kCells + v] = (float)u;
        }
    }
}
// GHOST value := parent value (PropagateToChildren, src/PoissonGrid.cu:377-405)
__global__ void k_propagate_ghost(DevGrid g, int t0, int ch) {
    const int t = t0 + blockIdx.x;
    const int4 m = g.meta[t];
    if (!((m.x >> 8) & dGhost)) return;
    const int p = g.nb[8 * t + 6];
    float* X = g.plane(ch);
    for (int v = threadIdx.x; v < kCells; v += blockDim.x) {
        if (!(g.ctype[(size_t)t * kCells + v] & (dInterior | dDirichlet | dNeumann))) continue;
        float val = 0.0f;
        if (p >= 0) {
            const size_t o = (size_t)p * kCells + cell_index(parent_local(m.y, v >> 6), parent_local(m.z, (v >> 3) & 7), parent_local(m.w, v & 7));
            if (g.ctype[o] & (dInterior | dDirichlet | dNeumann)) val = X[o];
        }
        X[(size_t)t * kCells + v] = val;
    }
}
// coarse face := 1/4 sum of the 4 fine faces of LEAF tiles (AccumulateFacesToParentsOneStepKernel, src/PoissonGrid.cu:523-566)
__global__ void k_accumulate_faces(DevGrid g, const int* leaf, int u_ch) {
    const int t = leaf[blockIdx.x];
    const int b = threadIdx.x;
    const int p = g.nb[8 * t + 6];
    if (p < 0) return;
    const int4 m = g.meta[t];
    const int f[3] = {(b >> 4) * 2, ((b >> 2) & 3) * 2, (b & 3) * 2};
    const size_t pv = (size_t)p * kCells + cell_index(parent_local(m.y, f[0]), parent_local(m.z, f[1]), parent_local(m.w, f[2]));
    for (int a = 0; a < 3; ++a) {
        const float* U = g.plane(u_ch + a) + (size_t)t * kCells;
        float s = 0.0f;
        for (int jj = 0; jj < 2; ++jj)
            for (int kk = 0; kk < 2; ++kk) {
                int o[3];
                o[a] = 0;
                o[(a + 1) % 3] = jj;
                o[(a + 2) % 3] = kk;
                const int v = cell_index(f[0] + o[0], f[1] + o[1], f[2] + o[2]);
                s = __fadd_rn(s, (g.ctype[(size_t)t * kCells + v] & (dInterior | dDirichlet | dNeumann)) ? U[v] : 0.0f);
            }
        g.plane(u_ch + a)[pv] = __fmul_rn(s, 0.25f);
    }
}
// AMGVolumeWeightedDivergenceOnLeafs (src/AMGSolver.cu:797-834)
__global__ void k_divergence(DevGrid g, const int* leaf, int u_ch, int coeff_ch, int out_ch) {
    const int t = leaf[blockIdx.x];
    const int4 m = g.meta[t];
    const float h = voxel_size(g.h0, m.x & 0xff);
    for (int v = threadIdx.x; v < kCells; v += blockDim.x) {
        const int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
        const int stride[3] = {64, 8, 1};
        float sum = 0.0f;
        for (int a = 0; a < 3; ++a) {
            const size_t o = (size_t)t * kCells + v;
            const float u0 = g.plane(u_ch + a)[o];
            // coeff_ch < 0: the coefficient-free variant (src/AMGSolver.cu:750-788), -u0 h h and u1 h h
            sum = coeff_ch < 0 ? __fmaf_rn(__fmul_rn(-u0, h), h, sum) : __fmaf_rn(__fmul_rn(u0, g.plane(coeff_ch + a)[o]), h, sum);
            int q = t, nv = v + stride[a];
            if (l[a] == 7) {
                q = g.nb[8 * t + 3 + a];
                nv = v - 7 * stride[a];
            }
            float u1 = 0.0f, c1 = 0.0f;
            if (q >= 0) {
                u1 = g.plane(u_ch + a)[(size_t)q * kCells + nv];
                if (coeff_ch >= 0) c1 = g.plane(coeff_ch + a)[(size_t)q * kCells + nv];
            }
            sum = coeff_ch < 0 ? __fmaf_rn(__fmul_rn(u1, h), h, sum) : __fmaf_rn(__fmul_rn(-u1, c1), h, sum);
        }
        g.plane(out_ch)[(size_t)t * kCells + v] = (g.ctype[(size_t)t * kCells + v] & dInterior) ? sum : 0.0f;
    }
}

// AMGAddGradientToFace128Kernel (src/AMGSolver.cu:634-678) on LEAF and GHOST
// tiles; GHOST values must already hold their parents' (k_propagate_ghost).
__global__ void __launch_bounds__(128) k_gradient(DevGrid g, const float* X, int coeff_ch, int u_ch) {
    __shared__ Snap S;
    const int t = blockIdx.x;
    if (!(tile_type(g, t) & (dLeaf | dGhost))) return;
    const Quad Q(t, threadIdx.x);
    Own o;
    load_snap(g, t, X, coeff_ch, LeafHalo{X, g.ctype}, S, Q, o, BlockSync{});
    const float h = voxel_size(g.h0, tile_level(g, t));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float* U = g.plane(u_ch + a);
        float4 u = ld4(U + Q.base);
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const int i = Q.i, j = Q.j, k = Q.k0 + w;
            const float pu = S.x[sx(i, j, k)];
            const float pd = S.x[sx(i - (a == 0), j - (a == 1), k - (a == 2))];
            const float c = a == 0 ? S.c0[i * 64 + j * 8 + k] : a == 1 ? S.c1[i * 72 + j * 8 + k] : S.c2[i * 72 + j * 9 + k];
            if (__fdiv_rn(-c, h) > 0.0f) f4set(u, w, __fadd_rn(f4get(u, w), __fdiv_rn(__fsub_rn(pu, pd), h)));
        }
        st4(U + Q.base, u);
    }
}

// cell of source tile for cell (i, j, k) of a new tile at meta m taking data from s levels up:
// the same cell (s = 0), else the ancestor cell that contains it
__device__ __forceinline__ int remap_cell(const int4& m, int s, int v) {
    if (s == 0) return v;
    const int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
    const int ai = ((m.y * 8 + i) >> s) - (m.y >> s) * 8;
    const int aj = ((m.z * 8 + j) >> s) - (m.z >> s) * 8;
    const int ak = ((m.w * 8 + k) >> s) - (m.w >> s) * 8;
    return cell_index(ai, aj, ak);
}
__global__ void k_remap(const float* src, float* dst, const int2* src_of_new, const int4* meta, int n_new, int n_old) {
    const int t = blockIdx.x, c = blockIdx.y;
    const int2 o = src_of_new[t];
    const int4 m = meta[t];
    const size_t dbase = ((size_t)c * n_new + t) * kCells;
    for (int v = threadIdx.x; v < kCells; v += blockDim.x)
        dst[dbase + v] = (o.x >= 0) ? src[((size_t)c * n_old + o.x) * kCells + remap_cell(m, o.y, v)] : 0.0f;
}
__global__ void k_remap_types(const uint8_t* src, uint8_t* dst, const int2* src_of_new, const int4* meta) {
    const int t = blockIdx.x;
    const int2 o = src_of_new[t];
    const int4 m = meta[t];
    for (int v = threadIdx.x; v < kCells; v += blockDim.x)
        dst[(size_t)t * kCells + v] = (o.x >= 0) ? src[(size_t)o.x * kCells + remap_cell(m, o.y, v)] : 0;
}
// Channels of the reference's device tiles (PoissonTile<float,15>: mData[15][736] floats,
// mCellType[512] at byte 44352) to and from the channel planes, one block per (tile, channel).
constexpr int kRefChannelStride = 736;
constexpr size_t kRefTypesOffset = 44352;
__global__ void k_gather_tiles(DevGrid g, const unsigned char* const* ptrs, int first) {
    const int t = blockIdx.x, c = first + (int)blockIdx.y;
    const float4* src = reinterpret_cast<const float4*>(reinterpret_cast<const float*>(ptrs[t]) + (size_t)c * kRefChannelStride);
    reinterpret_cast<float4*>(g.plane(c) + (size_t)t * kCells)[threadIdx.x] = src[threadIdx.x];
}
__global__ void k_gather_types(DevGrid g, const unsigned char* const* ptrs) {
    const int t = blockIdx.x;
    const uint4* src = reinterpret_cast<const uint4*>(ptrs[t] + kRefTypesOffset);
    reinterpret_cast<uint4*>(g.ctype + (size_t)t * kCells)[threadIdx.x] = src[threadIdx.x];
}
__global__ void k_scatter_tiles(DevGrid g, unsigned char* const* ptrs, int first) {
    const int t = blockIdx.x, c = first + (int)blockIdx.y;
    float4* dst = reinterpret_cast<float4*>(reinterpret_cast<float*>(ptrs[t]) + (size_t)c * kRefChannelStride);
    dst[threadIdx.x] = reinterpret_cast<const float4*>(g.plane(c) + (size_t)t * kCells)[threadIdx.x];
}
__global__ void k_fill(float* p, size_t n, float v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void k_count_bad_diag(DevGrid g, int t0, int coeff_ch, int* out) {
    const int t = t0 + blockIdx.x;
    const float* D = g.plane(coeff_ch + 3) + (size_t)t * kCells;
    for (int v = threadIdx.x; v < kCells; v += blockDim.x)
        if ((g.ctype[(size_t)t * kCells + v] & dInterior) && !(D[v] != 0.0f)) atomicAdd(out, 1);
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static std::atomic<long long> g_launches{0};
static inline void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long kernel_launch_count() { return g_launches.load(std::memory_order_relaxed); }

namespace {
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {  // splitmix64 finaliser
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ float make_float(unsigned long long r, int emin, int emax) {
    const unsigned sign = (unsigned)(r >> 63) << 31;
    const int e = emin + (int)((r >> 32) % (unsigned long long)(emax - emin + 1));
    return __uint_as_float(sign | ((unsigned)(e + 127) << 23) | ((unsigned)r & 0x7fffffu));
}
// Compares div_by_recip (with the correctly rounded reciprocal) and div_exact
// (with the Newton-refined one) with the IEEE division on pseudo-random pairs: a quarter
// uniform in sign, exponent and significand; a quarter built to fall within a few
// ulps of a midpoint between two floats (a = RN(d * m) for a midpoint m); a quarter
// shaped like Gauss-Seidel updates; a quarter of zeros, subnormals, huge values,
// infinities and NaNs.
__global__ void k_check_division(long long n, unsigned long long seed, unsigned long long* mism, unsigned int* first) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long r0 = mix64(seed ^ (unsigned long long)i), r1 = mix64(r0), r2 = mix64(r1);
        float a, d;
        switch ((int)(i & 3)) {
            case 0:
                a = make_float(r0, -60, 60);
                d = make_float(r1, -60, 60);
                break;
            case 1: {
                d = make_float(r0, -20, 20);
                const float q = make_float(r1, -20, 20);
                const double m = (double)q + 0.5 * ((double)nextafterf(fabsf(q), INFINITY) - (double)fabsf(q)) * (q < 0 ? -1.0 : 1.0);
                a = __double2float_rn((double)d * m);
                const int off = (int)(r2 % 5ull) - 2;  // a few ulps either side
                for (int s = 0; s < (off < 0 ? -off : off); ++s) a = nextafterf(a, off < 0 ? -INFINITY : INFINITY);
                break;
            }
            case 2:
                a = make_float(r0, -40, 2);
                d = -make_float(r1 & ~(1ull << 63), -14, 0);
                break;
            default: {
                const float pool[10] = {0.0f, -0.0f, 1e-45f, -3e-39f, 1.17549435e-38f, 3.0e38f, INFINITY, -INFINITY, NAN, 1.0f};
                a = (r2 & 1) ? pool[r0 % 10] : make_float(r0, -126, 127);
                d = (r2 & 2) ? pool[r1 % 10] : make_float(r1, -126, 127);
            }
        }
        const float want = __fdiv_rn(a, d);
        const float got = div_by_recip(a, d, 1.0 / (double)d);
        const float got2 = div_exact(a, d);
        const bool same = ((__float_as_uint(want) == __float_as_uint(got)) || (isnan(want) && isnan(got))) &&
                          ((__float_as_uint(want) == __float_as_uint(got2)) || (isnan(want) && isnan(got2)));
        if (!same) {
            if (atomicAdd(mism, 1ull) == 0ull) {
                first[0] = __float_as_uint(a);
                first[1] = __float_as_uint(d);
            }
        }
    }
}
}  // namespace

int check_division(long long n, unsigned long long seed, long long* mismatches, unsigned int* first_pair) {
    unsigned long long* dm = nullptr;
    unsigned int* df = nullptr;
    if (cudaMalloc(&dm, sizeof(unsigned long long)) != cudaSuccess) return 2;
    if (cudaMalloc(&df, 2 * sizeof(unsigned int)) != cudaSuccess) {
        cudaFree(dm);
        return 2;
    }
    cudaMemset(dm, 0, sizeof(unsigned long long));
    cudaMemset(df, 0, 2 * sizeof(unsigned int));
    count_launch(), k_check_division<<<148 * 8, 256>>>(n, seed, dm, df);
    unsigned long long hm = 0;
    unsigned int hf[2] = {0, 0};
    cudaError_t e = cudaMemcpy(&hm, dm, sizeof(hm), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hf, df, sizeof(hf), cudaMemcpyDeviceToHost);
    cudaFree(dm);
    cudaFree(df);
    if (e != cudaSuccess) return 2;
    *mismatches = (long long)hm;
    if (first_pair) {
        first_pair[0] = hf[0];
        first_pair[1] = hf[1];
    }
    return 0;
}
void note_kernel_launch() { count_launch(); }

void launch_gs(const DevGrid& g, int t0, int nt, float* X, const float* B, int coeff_ch, int color, double omega, cudaStream_t st) {
    if (nt <= 0) return;
    SmoothArgs A;
    A.coeff_ch = coeff_ch;
    A.om = (float)omega;
    A.exact = relax_mode(omega);
    A.omega = omega;
    count_launch(), k_gs<<<nt, 128, 0, st>>>(g, t0, X, B, color, A);
}
void launch_restrict(const DevGrid& g, int t0, int nt, float* X, float* RHS, int coeff_ch, float Rr, cudaStream_t st) {
    if (nt > 0) count_launch(), k_restrict<<<nt, 128, 0, st>>>(g, t0, X, RHS, coeff_ch, Rr);
}
void launch_fas_save(const DevGrid& g, int t0, int nt, const float* X, float* RHS, float* X0, int coeff_ch, cudaStream_t st) {
    if (nt > 0) count_launch(), k_fas_save<<<nt, 128, 0, st>>>(g, t0, X, RHS, X0, coeff_ch);
}
void launch_prolong(const DevGrid& g, int t0, int nt, float* X, const float* X0, float P, cudaStream_t st) {
    if (nt > 0) count_launch(), k_prolong<<<nt, 128, 0, st>>>(g, t0, X, X0, P);
}
void launch_cycle_init(const DevGrid& g, float* X, float* RHS, const float* F, cudaStream_t st) {
    if (g.n > 0) count_launch(), k_cycle_init<<<g.n, 128, 0, st>>>(g, X, RHS, F);
}
void launch_prolong_add(const DevGrid& g, int t0, int nt, float* X, float P, cudaStream_t st) {
    if (nt > 0) count_launch(), k_prolong_add<<<nt, 128, 0, st>>>(g, t0, X, P);
}
void launch_deduct_flux(const DevGrid& g, int t0, int nt, const float* X, const float* F, float* RHS, int coeff_ch, cudaStream_t st) {
    if (nt > 0) count_launch(), k_deduct_flux<<<nt, 128, 0, st>>>(g, t0, X, F, RHS, coeff_ch);
}
size_t coarse_step_smem_bytes() { return kCoarseSmem; }
void launch_coarse_step(const DevGrid& g, int top, float* X, float* RHS, float* X0, int coeff_ch, int mu, int level_iters,
                        int coarsest_iters, double omega, float Rr, float P, cudaStream_t st) {
    CoarseArgs A;
    A.top = top;
    A.coeff_ch = coeff_ch;
    A.mu = mu;
    A.level_iters = level_iters;
    A.coarsest_iters = coarsest_iters;
    A.om = (float)omega;
    A.exact = relax_mode(omega);
    A.omega = omega;
    A.Rr = Rr;
    A.P = P;
    count_launch(), k_coarse<<<1, 1024, kCoarseSmem, st>>>(g, A, X, RHS, X0);
}
void launch_leaf_apply(const DevGrid& g, const int* leaf, int nleaf, const float* P, float* AP, int coeff_ch, bool fuse_alpha,
                       ReduceScratch rs, cudaStream_t st) {
    if (nleaf > 0) count_launch(), k_leaf_apply<<<nleaf, 128, 0, st>>>(g, leaf, P, AP, coeff_ch, fuse_alpha ? 1 : 0, rs);
}
void launch_true_residual(const DevGrid& g, const int* leaf, int nleaf, const float* X, const float* B, float* R, int coeff_ch,
                          PcgScalars* s, int every, cudaStream_t st) {
    if (nleaf > 0 && every > 0) count_launch(), k_true_residual<<<nleaf, 128, 0, st>>>(g, leaf, X, B, R, coeff_ch, s, every);
}
// blocks of the grid-stride PCG vector kernels: 8 per SM (a block keeps two tiles' loads in flight)
static int vec_blocks(int nleaf) {
    static int per = 0;
    if (!per) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        per = 8 * (sms > 0 ? sms : 1);
    }
    return nleaf < per ? nleaf : per;
}
void launch_xr_update(const DevGrid& g, const int* leaf, int nleaf, float* X, float* R, const float* P, const float* AP,
                      ReduceScratch rs, cudaGraphConditionalHandle loop_h, cudaGraphConditionalHandle body_h, bool use_handles,
                      cudaStream_t st) {
    if (nleaf > 0)
        count_launch(), k_xr_update<<<vec_blocks(nleaf), 128, 0, st>>>(g, leaf, nleaf, X, R, P, AP, rs, loop_h, body_h, use_handles ? 1 : 0);
}
void launch_dot(const DevGrid& g, const int* leaf, int nleaf, const float* A, const float* B, int mode, double* out, ReduceScratch rs,
                cudaStream_t st) {
    (void)g;
    if (nleaf > 0) count_launch(), k_dot<<<vec_blocks(nleaf), 128, 0, st>>>(leaf, nleaf, A, B, mode, out, rs);
}
void launch_dot_flex(const DevGrid& g, const int* leaf, int nleaf, const float* R, const float* Z, const float* AP, ReduceScratch rs,
                     cudaStream_t st) {
    (void)g;
    if (nleaf > 0) count_launch(), k_dot_flex<<<nleaf, 128, 0, st>>>(leaf, R, Z, AP, rs);
}
void launch_p_update(const DevGrid& g, const int* leaf, int nleaf, float* P, const float* Z, ReduceScratch rs, cudaStream_t st) {
    if (nleaf > 0) count_launch(), k_p_update<<<nleaf, 128, 0, st>>>(g, leaf, P, Z, rs);
}
void launch_leaf_fill(const DevGrid& g, const int* leaf, int nleaf, float* X, float value, cudaStream_t st) {
    (void)g;
    if (nleaf > 0) count_launch(), k_leaf_fill<<<nleaf, 128, 0, st>>>(leaf, X, value);
}
void launch_leaf_copy(const DevGrid& g, const int* leaf, int nleaf, float* dst, const float* src, cudaStream_t st) {
    (void)g;
    if (nleaf > 0) count_launch(), k_leaf_copy<<<nleaf, 128, 0, st>>>(leaf, dst, src);
}
void launch_recenter(const DevGrid& g, const int* leaf, int nleaf, float* R, ReduceScratch rs, cudaStream_t st) {
    if (nleaf <= 0) return;
    count_launch(), k_mean_partial<<<nleaf, 128, 0, st>>>(g, leaf, R, rs);
    count_launch(), k_sub_mean<<<nleaf, 128, 0, st>>>(g, leaf, R, rs);
}
void launch_loop_gate(ReduceScratch rs, cudaGraphConditionalHandle loop_h, bool use_handle, cudaStream_t st) {
    count_launch(), k_loop_gate<<<1, 1, 0, st>>>(rs, loop_h, use_handle ? 1 : 0);
}
void init_kernel_attributes() {
    cudaFuncSetAttribute(k_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmem);
    cudaFuncSetAttribute(k_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPersistSmem);
}
int persist_blocks() {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist, 512, kPersistSmem);
    return per_sm > 0 ? sms * per_sm : 0;
}
cudaError_t launch_persist_step(const DevGrid& g, int top, const int* lb, const int* ab, const int* le, const int* nlb, float* X, float* RHS,
                                float* X0, int coeff_ch, int mu, int level_iters, int coarsest_iters, double omega, float Rr, float P,
                                unsigned int* bar, int nblocks, cudaStream_t st) {
    PersistArgs A;
    A.top = top;
    for (int l = 0; l < 4; ++l) {
        A.lb[l] = lb[l];
        A.ab[l] = ab[l];
        A.le[l] = le[l];
        A.nlb[l] = nlb[l];
    }
    A.mu = mu;
    A.level_iters = level_iters;
    A.coarsest_iters = coarsest_iters;
    A.sm.coeff_ch = coeff_ch;
    A.sm.om = (float)omega;
    A.sm.exact = relax_mode(omega);
    A.sm.omega = omega;
    A.co.top = 1;
    A.co.coeff_ch = coeff_ch;
    A.co.mu = mu;
    A.co.level_iters = level_iters;
    A.co.coarsest_iters = coarsest_iters;
    A.co.om = A.sm.om;
    A.co.exact = A.sm.exact;
    A.co.omega = omega;
    A.co.Rr = Rr;
    A.co.P = P;
    A.Rr = Rr;
    A.P = P;
    A.X = X;
    A.RHS = RHS;
    A.X0 = X0;
    A.bar = bar;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(512);
    cfg.dynamicSmemBytes = kPersistSmem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    count_launch();
    return cudaLaunchKernelEx(&cfg, k_persist, g, A);
}

void launch_ghost_types(const DevGrid& g, int t0, int nt, cudaStream_t st) {
    if (nt > 0) count_launch(), k_ghost_types<<<nt, 128, 0, st>>>(g, t0);
}
void launch_face_coeffs(const DevGrid& g, int t0, int nt, int coeff_ch, int ns, const float* sp, cudaStream_t st) {
    if (nt > 0) count_launch(), k_face_coeffs<<<nt, 128, 0, st>>>(g, t0, coeff_ch, ns, sp);
}
void launch_cutcell_neumann(const DevGrid& g, const int* leaf, int nleaf, int ns, const float* sp, cudaStream_t st) {
    if (nleaf > 0) count_launch(), k_cutcell_neumann<<<nleaf, 128, 0, st>>>(g, leaf, ns, sp);
}
void launch_coarsen_offdiag(const DevGrid& g, int t0, int nt, int coeff_ch, float R, cudaStream_t st) {
    if (nt > 0) count_launch(), k_coarsen_offdiag<<<nt, 64, 0, st>>>(g, t0, coeff_ch, R);
}
void launch_diag(const DevGrid& g, int t0, int nt, int coeff_ch, float R, cudaStream_t st) {
    if (nt > 0) count_launch(), k_diag<<<nt, 128, 0, st>>>(g, t0, coeff_ch, R);
}
void launch_face_velocity(const DevGrid& g, const int* leaf, int nleaf, int u_ch, int nm, const double* modes, cudaStream_t st) {
    if (nleaf > 0) count_launch(), k_face_velocity<<<nleaf, 128, 0, st>>>(g, leaf, u_ch, nm, modes);
}
void launch_propagate_ghost(const DevGrid& g, int t0, int nt, int ch, cudaStream_t st) {
    if (nt > 0) count_launch(), k_propagate_ghost<<<nt, 128, 0, st>>>(g, t0, ch);
}
void launch_accumulate_faces(const DevGrid& g, const int* leaf, int nleaf, int u_ch, cudaStream_t st) {
    if (nleaf > 0) count_launch(), k_accumulate_faces<<<nleaf, 64, 0, st>>>(g, leaf, u_ch);
}
void launch_divergence(const DevGrid& g, const int* leaf, int nleaf, int u_ch, int coeff_ch, int out_ch, cudaStream_t st) {
    if (nleaf > 0) count_launch(), k_divergence<<<nleaf, 128, 0, st>>>(g, leaf, u_ch, coeff_ch, out_ch);
}
void launch_gradient(const DevGrid& g, const float* X, int coeff_ch, int u_ch, cudaStream_t st) {
    if (g.n > 0) count_launch(), k_gradient<<<g.n, 128, 0, st>>>(g, X, coeff_ch, u_ch);
}
void launch_remap(const float* src, float* dst, const int2* src_of_new, const int4* meta, int n_new, int nch, int n_old, cudaStream_t st) {
    if (n_new > 0 && nch > 0) count_launch(), k_remap<<<dim3(n_new, nch), 128, 0, st>>>(src, dst, src_of_new, meta, n_new, n_old);
}
void launch_remap_types(const uint8_t* src, uint8_t* dst, const int2* src_of_new, const int4* meta, int n_new, cudaStream_t st) {
    if (n_new > 0) count_launch(), k_remap_types<<<n_new, 128, 0, st>>>(src, dst, src_of_new, meta);
}
void launch_gather_tiles(const DevGrid& g, const void* const* ptrs, int first, int num, bool types, cudaStream_t st) {
    const auto P = reinterpret_cast<const unsigned char* const*>(ptrs);
    if (g.n > 0 && num > 0) count_launch(), k_gather_tiles<<<dim3(g.n, num), 128, 0, st>>>(g, P, first);
    if (g.n > 0 && types) count_launch(), k_gather_types<<<g.n, 32, 0, st>>>(g, P);
}
void launch_scatter_tiles(const DevGrid& g, void* const* ptrs, int first, int num, cudaStream_t st) {
    if (g.n > 0 && num > 0) count_launch(), k_scatter_tiles<<<dim3(g.n, num), 128, 0, st>>>(g, reinterpret_cast<unsigned char* const*>(ptrs), first);
}
void launch_fill(float* p, size_t n, float v, cudaStream_t st) {
    if (n > 0) count_launch(), k_fill<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, st>>>(p, n, v);
}
void launch_count_bad_diag(const DevGrid& g, int t0, int nt, int coeff_ch, int* out, cudaStream_t st) {
    if (nt > 0) count_launch(), k_count_bad_diag<<<nt, 128, 0, st>>>(g, t0, coeff_ch, out);
}

}  // namespace cmg
