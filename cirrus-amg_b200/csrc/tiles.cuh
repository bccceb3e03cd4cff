// Tile-level device code of the multigrid cycle, shared by the kernels that
// run one tile per block (kernels.cu) and the persistent batched solve
// (batch_persist.cu): the smoothing, restriction, FAS and prolongation steps
// of one 8^3 tile by 128 threads, the dense coarse sub-cycle of levels 0-1,
// and the fixed-order reductions.
#pragma once
#include <cfloat>

#include "kernels.hpp"

namespace cmg {
namespace {
__device__ __forceinline__ bool last_block(unsigned int* counter) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    return is_last;
}
// Thread t sums partials t, t+128, t+256, ... in that order; the loads are issued eight at a
// time before the adds, which keeps the order (and the result) and overlaps the L2 latency.
__device__ __forceinline__ double sum_partials(const double* part, int n, double* red) {
    double s = 0;
    int i = threadIdx.x;
    for (; i + 7 * 128 < n; i += 8 * 128) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = __ldcg(part + i + u * 128);
#pragma unroll
        for (int u = 0; u < 8; ++u) s += v[u];
    }
    for (; i < n; i += 128) s += __ldcg(part + i);
    return block_sum128(s, red);
}
// products of four cells summed in float, the reference's Dot128Kernel (src/PoissonGrid.cu:168-172)
__device__ __forceinline__ double dot4(const float4& a, const float4& b) {
    float f = __fmul_rn(a.x, b.x);
    f = __fmaf_rn(a.y, b.y, f);
    f = __fmaf_rn(a.z, b.z, f);
    f = __fmaf_rn(a.w, b.w, f);
    return (double)f;
}

// ---------------------------------------------------------------------------
// multigrid: one 8^3 tile per 128-thread group.  The tile_* functions are
// shared by the one-tile-per-block kernels and the persistent kernel that
// runs several tiles per block; `sync` is the barrier of the 128 threads.
// Each ends with a barrier so the snapshot can be reused for the next tile.
// ---------------------------------------------------------------------------
struct SmoothArgs {
    int coeff_ch, exact;
    float om;
    double omega;
};

// NegativeLaplacianAndGaussSeidelSameLevelAMG128Kernel (src/AMGSolver.cu:838-877)
template <class Sync>
__device__ __forceinline__ void tile_gs(const DevGrid& g, int t, int tid, float* X, const float* B, int color, const SmoothArgs& A,
                                        Snap& S, const Sync& sync) {
    const Quad Q(t, tid);
    Own o;
    load_snap(g, t, X, A.coeff_ch, MgHalo{X, g.ctype}, S, Q, o, sync);
    const float4 b = ldcg4(B + Q.base);
    float4 out = o.xr;
    // cells of this colour: u = p and u = p + 2
    const int p = (Q.i + Q.j + Q.k0 + color) & 1;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int u = p + 2 * h;
        const float d = f4get(o.dg, u);
        const float ax = own_neg_lap(S, Q, o, u);
        const float delta = (t4get(o.ty, u) & dInterior) ? div_exact(__fsub_rn(f4get(b, u), ax), d) : 0.0f;
        const float xs = f4get(o.xm, u);
        f4set(out, u, relax_rt(A.exact, xs, delta, A.om, A.omega));
    }
    st4(X + Q.base, out);
    sync();
}

// ResidualAndRestrictAMG128Kernel (src/AMGSolver.cu:896-960)
template <class Sync>
__device__ __forceinline__ void tile_restrict(const DevGrid& g, int t, int tid, float* X, float* RHS, int coeff_ch, float Rr, Snap& S,
                                              float* res, const Sync& sync) {
    const Quad Q(t, tid);
    Own o;
    load_snap(g, t, X, coeff_ch, MgHalo{X, g.ctype}, S, Q, o, sync);
    const float4 rh = ldcg4(RHS + Q.base);
    res[4 * Q.q + 0] = __fsub_rn(rh.x, own_neg_lap<0>(S, Q, o));
    res[4 * Q.q + 1] = __fsub_rn(rh.y, own_neg_lap<1>(S, Q, o));
    res[4 * Q.q + 2] = __fsub_rn(rh.z, own_neg_lap<2>(S, Q, o));
    res[4 * Q.q + 3] = __fsub_rn(rh.w, own_neg_lap<3>(S, Q, o));
    sync();
    if (tid < 64) {
        const int b = tid;
        const int f0 = (b >> 4) * 2, f1 = ((b >> 2) & 3) * 2, f2 = (b & 3) * 2;
        float rs = 0.0f, xs = 0.0f;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    rs = __fadd_rn(rs, res[cell_index(f0 + ii, f1 + jj, f2 + kk)]);
                    xs = __fadd_rn(xs, S.x[sx(f0 + ii, f1 + jj, f2 + kk)]);
                }
        const int p = g.nb[8 * t + 6];
        if (p >= 0) {
            const int4 m = g.meta[t];
            const size_t o = (size_t)p * kCells + cell_index(parent_local(m.y, f0), parent_local(m.z, f1), parent_local(m.w, f2));
            RHS[o] = __fmul_rn(rs, Rr);
            // mean of the 8 children (xs / 8), stored as 0 on cells that are not INTERIOR: every read
            // of a multigrid x masks it that way, and keeping the plane masked lets the pipelined
            // smoother read neighbour values without their cell types
            X[o] = (g.ctype[o] & dInterior) ? __fmul_rn(xs, 0.125f) : 0.0f;
        }
    }
    sync();
}

// FASSaveSolutionAndUpdateSource128Kernel (src/AMGSolver.cu:1176-1206)
template <class Sync>
__device__ __forceinline__ void tile_fas_save(const DevGrid& g, int t, int tid, const float* X, float* RHS, float* X0, int coeff_ch,
                                              Snap& S, const Sync& sync) {
    const Quad Q(t, tid);
    Own o;
    load_snap(g, t, X, coeff_ch, MgHalo{X, g.ctype}, S, Q, o, sync);
    float4 rh = ldcg4(RHS + Q.base);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        if (t4get(o.ty, u) & dInterior) {
            f4set(rh, u, __fadd_rn(f4get(rh, u), own_neg_lap(S, Q, o, u)));
            X0[Q.base + u] = f4get(o.xr, u);
        } else {
            f4set(rh, u, 0.0f);
        }
    }
    st4(RHS + Q.base, rh);
    sync();
}

// FASProlongateAndUpdateAMG128Kernel (src/AMGSolver.cu:1216-1248); no snapshot
__device__ __forceinline__ void tile_prolong(const DevGrid& g, int t, int tid, float* X, const float* X0, float P) {
    const Quad Q(t, tid);
    const int4 m = g.meta[t];
    const bool ghost = (m.x >> 8) & dGhost;
    const int p = g.nb[8 * t + 6];
    const float4 xr = ldcg4(X + Q.base);
    const uchar4 ty = ldt4(g.ctype + Q.base);
    const int pi = parent_local(m.y, Q.i), pj = parent_local(m.z, Q.j);
    float4 out;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        float cx = 0.0f, cx0 = 0.0f;
        if (p >= 0) {
            const size_t o = (size_t)p * kCells + cell_index(pi, pj, parent_local(m.w, Q.k0 + u));
            cx = ldcg(X + o);
            cx0 = ldcg(X0 + o);
        }
        const bool in = t4get(ty, u) & dInterior;
        f4set(out, u, ghost ? (in ? cx : 0.0f) : (in ? __fmaf_rn(P, __fsub_rn(cx, cx0), f4get(xr, u)) : 0.0f));
    }
    st4(X + Q.base, out);
}

// ---------------------------------------------------------------------------
// Coarse levels: FASMuCycleStep (src/AMGSolver.cu:1257-1277) of level 0 or 1
// in one 1024-thread block.  A NONLEAF root has all eight children and
// neither level can hold GHOST tiles, so the root and its children are
// complete 8^3 and 16^3 grids.  Both are staged in shared memory as dense
// arrays with a zero halo: the stencil needs no neighbour tables, every
// thread of a colour sweep has a cell, and all mu recursions with their
// 2*coarsest_iters sweeps run between block barriers instead of ~50 kernel
// launches.  A zero halo value is exactly the reference's empty-neighbour rule
// (x = 0, src/AMGSolver.cu:489-493); x is held masked to INTERIOR cells, which
// is how every read of it in the reference sees it.
// ---------------------------------------------------------------------------
struct CoarseArgs {
    int top, coeff_ch, mu, level_iters, coarsest_iters, exact;
    float om, Rr, P;
    double omega;
};

template <int N>  // cells per axis: 16 for level 1, 8 for level 0
struct DenseLevel {
    static constexpr int PD = N + 2;  // padded extent of x
    float* x;                         // PD^3, zero halo
    float* c0;                        // [N+1][N][N]: -x face of cell i (face N: domain boundary, 0)
    float* c1;                        // [N][N+1][N]
    float* c2;                        // [N][N][N+1]
    float* d;                         // [N][N][N]
    float* rhs;
    uint8_t* ty;
    __device__ static int xi(int i, int j, int k) { return ((i + 1) * PD + (j + 1)) * PD + (k + 1); }
    __device__ static int ci(int i, int j, int k) { return (i * N + j) * N + k; }
    __device__ float neg_lap(int i, int j, int k) const {
        const float dd = d[ci(i, j, k)];
        if (dd == 0.0f) return 0.0f;
        const int q = xi(i, j, k);
        float s = x[q] * dd;
        s = __fmaf_rn(c0[(i * N + j) * N + k], x[q - PD * PD], s);
        s = __fmaf_rn(c0[((i + 1) * N + j) * N + k], x[q + PD * PD], s);
        s = __fmaf_rn(c1[(i * (N + 1) + j) * N + k], x[q - PD], s);
        s = __fmaf_rn(c1[(i * (N + 1) + j + 1) * N + k], x[q + PD], s);
        s = __fmaf_rn(c2[(i * N + j) * (N + 1) + k], x[q - 1], s);
        s = __fmaf_rn(c2[(i * N + j) * (N + 1) + k + 1], x[q + 1], s);
        return s;
    }
    // one colour: the N^3/2 cells with (i+j+k)%2 == color, one per thread
    __device__ void gs_pass(int color, const CoarseArgs& A) {
        constexpr int half = N * N * N / 2;
        for (int idx = threadIdx.x; idx < half; idx += blockDim.x) {
            const int i = idx / (N * N / 2), j = (idx / (N / 2)) % N, kh = idx % (N / 2);
            const int k = 2 * kh + ((i + j + color) & 1);
            const int c = ci(i, j, k);
            const float ax = neg_lap(i, j, k);
            const float delta = (ty[c] & dInterior) ? div_exact(__fsub_rn(rhs[c], ax), d[c]) : 0.0f;
            const float xs = x[xi(i, j, k)];
            x[xi(i, j, k)] = relax_rt(A.exact, xs, delta, A.om, A.omega);
        }
        __syncthreads();
    }
    __device__ void gs(int iters, int order, const CoarseArgs& A) {
        for (int it = 0; it < iters; ++it) {
            gs_pass(order, A);
            gs_pass(1 - order, A);
        }
    }
    __device__ void clear_boundary_faces() {
        for (int q = threadIdx.x; q < N * N; q += blockDim.x) {
            const int a = q / N, b = q % N;
            c0[(N * N + a) * N + b] = 0.0f;
            c1[(a * (N + 1) + N) * N + b] = 0.0f;
            c2[(a * N + b) * (N + 1) + N] = 0.0f;
        }
    }
};
constexpr int kCoarseFloats = 18 * 18 * 18 + 3 * 17 * 16 * 16 + 3 * 4096 + 10 * 10 * 10 + 3 * 9 * 8 * 8 + 3 * 512;
constexpr size_t kCoarseSmem = sizeof(float) * kCoarseFloats + sizeof(int) * 8 + 4096 + 512;

// the whole coarse sub-cycle by the calling block (any multiple of 32 threads)
__device__ void coarse_dense(const DevGrid& g, const CoarseArgs& A, float* X, float* RHS, float* X0, unsigned char* smraw) {
    float* f = reinterpret_cast<float*>(smraw);
    DenseLevel<16> L1;
    DenseLevel<8> L0;
    L1.x = f; f += 18 * 18 * 18;
    L1.c0 = f; f += 17 * 256;
    L1.c1 = f; f += 17 * 256;
    L1.c2 = f; f += 17 * 256;
    L1.d = f; f += 4096;
    L1.rhs = f; f += 4096;
    float* res = f; f += 4096;
    L0.x = f; f += 1000;
    L0.c0 = f; f += 576;
    L0.c1 = f; f += 576;
    L0.c2 = f; f += 576;
    L0.d = f; f += 512;
    L0.rhs = f; f += 512;
    float* x00 = f; f += 512;
    int* child = reinterpret_cast<int*>(f);
    L1.ty = reinterpret_cast<uint8_t*>(child + 8);
    L0.ty = L1.ty + 4096;
    const int tid = threadIdx.x;
    const float* C0 = g.plane(A.coeff_ch);
    const float* C1 = g.plane(A.coeff_ch + 1);
    const float* C2 = g.plane(A.coeff_ch + 2);
    const float* C3 = g.plane(A.coeff_ch + 3);

    for (int q = tid; q < 18 * 18 * 18; q += blockDim.x) L1.x[q] = 0.0f;
    for (int q = tid; q < 1000; q += blockDim.x) L0.x[q] = 0.0f;
    if (tid < 8) child[tid] = g.child[tid];
    L1.clear_boundary_faces();
    L0.clear_boundary_faces();
    __syncthreads();
    // root tile (tile 0)
    for (int v = tid; v < kCells; v += blockDim.x) {
        const int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
        const uint8_t t = g.ctype[v];
        L0.ty[v] = t;
        L0.d[v] = C3[v];
        L0.c0[(i * 8 + j) * 8 + k] = C0[v];
        L0.c1[(i * 9 + j) * 8 + k] = C1[v];
        L0.c2[(i * 8 + j) * 9 + k] = C2[v];
        L0.rhs[v] = ldcg(RHS + v);
        x00[v] = ldcg(X0 + v);
        L0.x[DenseLevel<8>::xi(i, j, k)] = t == dInterior ? ldcg(X + v) : 0.0f;
    }
    // the eight level-1 tiles as one 16^3 grid
    if (A.top == 1) {
        for (int idx = tid; idx < 8 * kCells; idx += blockDim.x) {
            const int tci = idx >> 9, v = idx & 511;
            const int tile = child[tci];
            if (tile < 0) continue;
            const size_t o = (size_t)tile * kCells + v;
            const int I = ((tci >> 2) << 3) | (v >> 6), J = (((tci >> 1) & 1) << 3) | ((v >> 3) & 7), K = ((tci & 1) << 3) | (v & 7);
            const int c = DenseLevel<16>::ci(I, J, K);
            const uint8_t t = g.ctype[o];
            L1.ty[c] = t;
            L1.d[c] = C3[o];
            L1.rhs[c] = ldcg(RHS + o);
            L1.c0[(I * 16 + J) * 16 + K] = C0[o];
            L1.c1[(I * 17 + J) * 16 + K] = C1[o];
            L1.c2[(I * 16 + J) * 17 + K] = C2[o];
            L1.x[DenseLevel<16>::xi(I, J, K)] = t == dInterior ? ldcg(X + o) : 0.0f;
        }
    }
    __syncthreads();

    if (A.top == 0) {
        L0.gs(A.coarsest_iters / 2, 0, A);
        L0.gs(A.coarsest_iters / 2, 1, A);
    } else {
        L1.gs(A.level_iters, 0, A);
        // residual on level 1 (ResidualAndRestrictAMG128Kernel) ...
        for (int c = tid; c < 4096; c += blockDim.x) {
            const int I = c >> 8, J = (c >> 4) & 15, K = c & 15;
            res[c] = __fsub_rn(L1.rhs[c], L1.neg_lap(I, J, K));
        }
        __syncthreads();
        // ... restricted to the root: rhs = R * sum of 8 residuals, x = mean of 8 x
        for (int v = tid; v < kCells; v += blockDim.x) {
            const int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
            float rs = 0.0f, xs = 0.0f;
            for (int ii = 0; ii < 2; ++ii)
                for (int jj = 0; jj < 2; ++jj)
                    for (int kk = 0; kk < 2; ++kk) {
                        rs = __fadd_rn(rs, res[DenseLevel<16>::ci(2 * i + ii, 2 * j + jj, 2 * k + kk)]);
                        xs = __fadd_rn(xs, L1.x[DenseLevel<16>::xi(2 * i + ii, 2 * j + jj, 2 * k + kk)]);
                    }
            L0.rhs[v] = __fmul_rn(rs, A.Rr);
            L0.x[DenseLevel<8>::xi(i, j, k)] = L0.ty[v] == dInterior ? __fmul_rn(xs, 0.125f) : 0.0f;
        }
        __syncthreads();
        // FASSaveSolutionAndUpdateSource on the root
        for (int v = tid; v < kCells; v += blockDim.x) {
            const int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
            if (L0.ty[v] & dInterior) {
                L0.rhs[v] = __fadd_rn(L0.rhs[v], L0.neg_lap(i, j, k));
                x00[v] = L0.x[DenseLevel<8>::xi(i, j, k)];
            } else {
                L0.rhs[v] = 0.0f;
            }
        }
        __syncthreads();
        for (int r = 0; r < A.mu; ++r) {
            L0.gs(A.coarsest_iters / 2, 0, A);
            L0.gs(A.coarsest_iters / 2, 1, A);
        }
        // FASProlongateAndUpdate on level 1
        for (int c = tid; c < 4096; c += blockDim.x) {
            const int I = c >> 8, J = (c >> 4) & 15, K = c & 15;
            const int q = DenseLevel<16>::xi(I, J, K);
            const float cx = L0.x[DenseLevel<8>::xi(I >> 1, J >> 1, K >> 1)];
            const float cx0 = x00[DenseLevel<8>::ci(I >> 1, J >> 1, K >> 1)];
            L1.x[q] = (L1.ty[c] & dInterior) ? __fmaf_rn(A.P, __fsub_rn(cx, cx0), L1.x[q]) : 0.0f;
        }
        __syncthreads();
        L1.gs(A.level_iters, 1, A);
    }
    for (int v = tid; v < kCells; v += blockDim.x) {
        X[v] = L0.x[DenseLevel<8>::xi(v >> 6, (v >> 3) & 7, v & 7)];
        RHS[v] = L0.rhs[v];
        X0[v] = x00[v];
    }
    if (A.top == 1) {
        for (int idx = tid; idx < 8 * kCells; idx += blockDim.x) {
            const int tci = idx >> 9, v = idx & 511;
            const int tile = child[tci];
            if (tile < 0) continue;
            const int I = ((tci >> 2) << 3) | (v >> 6), J = (((tci >> 1) & 1) << 3) | ((v >> 3) & 7), K = ((tci & 1) << 3) | (v & 7);
            X[(size_t)tile * kCells + v] = L1.x[DenseLevel<16>::xi(I, J, K)];
        }
    }
    __syncthreads();
}

}  // namespace
}  // namespace cmg
