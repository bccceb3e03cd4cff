// FASMuCycleStep of level 2 (src/AMGSolver.cu:1257-1277) with its whole
// recursion through levels 1 and 0, in one launch of one 8-CTA thread-block
// cluster.
//
// When the root, its eight children and their 64 children all exist (no
// GHOST tile on levels 0-2), levels 2, 1 and 0 are complete 32^3, 16^3 and
// 8^3 grids.  CTA r of the cluster owns octant r of the domain
// (r = 4*oi + 2*oj + ok, the child order of the root): a 16^3 block of level 2,
// the level-1 tile child[r] (8^3) and, on rank 0, the root.  Thread t of a CTA
// owns the 2x2x2 block of level-2 cells that is level-1 cell t, so the
// restriction 2 -> 1 and the prolongation 1 -> 2 need no communication and the
// block's diagonals, right-hand sides, x and face coefficients live in
// registers.  x is mirrored in shared memory with a one-cell halo; after every
// update a CTA stores its octant-boundary cells straight into the halos of the
// neighbouring octants' CTAs (distributed shared memory), and one cluster
// barrier per phase publishes them.  The root (8^3) is restricted into rank 0,
// which runs the coarsest Gauss-Seidel sweeps alone between block barriers.
//
// Every value is computed with the same operations in the same order as the
// per-level tile kernels and the dense coarse kernel (red-black Gauss-Seidel
// does not depend on the order of cells within a colour), so the result equals
// theirs.
#include <cooperative_groups.h>

#include "kernels.hpp"

namespace cmg {

namespace cg = cooperative_groups;

namespace {

constexpr int kClCtas = 8;
constexpr int kClThreads = 512;

struct ClusterArgs {
    int coeff_ch, mu, level_iters, coarsest_iters, exact;
    float om, Rr, P;
    double omega;
};

__device__ __forceinline__ int p18(int i, int j, int k) { return ((i + 1) * 18 + (j + 1)) * 18 + (k + 1); }
__device__ __forceinline__ int p10(int i, int j, int k) { return ((i + 1) * 10 + (j + 1)) * 10 + (k + 1); }

struct ClSmem {
    float x2[18 * 18 * 18];  // level-2 octant, one-cell halo
    float x1[10 * 10 * 10];  // level-1 tile, one-cell halo
    float x0[10 * 10 * 10];  // root x (rank 0), zero halo
    float r1[512];           // level-1 residuals
    float b0[512];           // root right-hand side (rank 0)
    float s0[512];           // root saved x (rank 0)
};

// plane offset of level-2 cell (I, J, K) of the 32^3 grid, -1 outside
__device__ __forceinline__ long long l2_off(const int* child, int I, int J, int K) {
    if ((unsigned)I >= 32u || (unsigned)J >= 32u || (unsigned)K >= 32u) return -1;
    const int t1 = child[((I >> 4) << 2) | ((J >> 4) << 1) | (K >> 4)];
    const int t2 = child[8 * t1 + ((((I >> 3) & 1) << 2) | (((J >> 3) & 1) << 1) | ((K >> 3) & 1))];
    return (long long)t2 * kCells + cell_index(I & 7, J & 7, K & 7);
}
// plane offset of level-1 cell (I, J, K) of the 16^3 grid, -1 outside
__device__ __forceinline__ long long l1_off(const int* child, int I, int J, int K) {
    if ((unsigned)I >= 16u || (unsigned)J >= 16u || (unsigned)K >= 16u) return -1;
    const int t1 = child[((I >> 3) << 2) | ((J >> 3) << 1) | (K >> 3)];
    return (long long)t1 * kCells + cell_index(I & 7, J & 7, K & 7);
}

// AMGLaplacianTileData::negativeLap (src/AMGSolver.cu:346-382), order -x,+x,-y,+y,-z,+z
__device__ __forceinline__ float nlap(float d, float x, float cmx, float xmx, float cpx, float xpx, float cmy, float xmy, float cpy,
                                      float xpy, float cmz, float xmz, float cpz, float xpz) {
    if (d == 0.0f) return 0.0f;
    float s = __fmul_rn(x, d);
    s = __fmaf_rn(cmx, xmx, s);
    s = __fmaf_rn(cpx, xpx, s);
    s = __fmaf_rn(cmy, xmy, s);
    s = __fmaf_rn(cpy, xpy, s);
    s = __fmaf_rn(cmz, xmz, s);
    s = __fmaf_rn(cpz, xpz, s);
    return s;
}
// one Gauss-Seidel update (src/AMGSolver.cu:868-875)
__device__ __forceinline__ float gs_update(float xs, float rhs, float ax, float d, bool interior, const ClusterArgs& A) {
    const float delta = interior ? __fdiv_rn(__fsub_rn(rhs, ax), d) : 0.0f;
    return A.exact ? __fmaf_rn(delta, A.om, xs) : (float)((double)xs + (double)delta * A.omega);
}

// Where this CTA sits: octant bits, and the halo of each neighbouring octant.
struct Geo {
    int r, oi, oj, ok;
    int bi, bj, bk;           // thread's block = level-1 cell
    float* rx2[3];            // neighbour octant's x2 along x, y, z
    float* rx1[3];            // neighbour octant's x1
    float* rb0;               // rank 0's b0, x0, s0
    float* rx0;
    float* rs0;
};

// Level-2 block of one thread.  Cell q = 4*di + 2*dj + dk is (2bi+di, 2bj+dj, 2bk+dk)
// of the octant.  Face planes: cx[4p + 2dj + dk] is the -x face of the cells
// with di = p (p = 2: the +x face of the di = 1 cells); cy[4p + 2di + dk];
// cz[4p + 2di + dj].
struct Blk {
    float x[8], d[8], b[8];
    float cx[12], cy[12], cz[12];
    unsigned in;  // bit q: cell q INTERIOR
};

template <int Q>
__device__ __forceinline__ float blk_nlap(const Blk& o, const ClSmem& sm, const Geo& gm) {
    constexpr int di = Q >> 2, dj = (Q >> 1) & 1, dk = Q & 1;
    const int I = 2 * gm.bi + di, J = 2 * gm.bj + dj, K = 2 * gm.bk + dk;
    const float xmx = di ? o.x[Q - 4] : sm.x2[p18(I - 1, J, K)];
    const float xpx = di ? sm.x2[p18(I + 1, J, K)] : o.x[Q + 4];
    const float xmy = dj ? o.x[Q - 2] : sm.x2[p18(I, J - 1, K)];
    const float xpy = dj ? sm.x2[p18(I, J + 1, K)] : o.x[Q + 2];
    const float xmz = dk ? o.x[Q - 1] : sm.x2[p18(I, J, K - 1)];
    const float xpz = dk ? sm.x2[p18(I, J, K + 1)] : o.x[Q + 1];
    return nlap(o.d[Q], o.x[Q], o.cx[4 * di + 2 * dj + dk], xmx, o.cx[4 * (di + 1) + 2 * dj + dk], xpx, o.cy[4 * dj + 2 * di + dk], xmy,
                o.cy[4 * (dj + 1) + 2 * di + dk], xpy, o.cz[4 * dk + 2 * di + dj], xmz, o.cz[4 * (dk + 1) + 2 * di + dj], xpz);
}

// store cell Q of the block into shared memory and, on an octant face, into the neighbour's halo
template <int Q>
__device__ __forceinline__ void blk_publish(const Blk& o, ClSmem& sm, const Geo& gm) {
    constexpr int di = Q >> 2, dj = (Q >> 1) & 1, dk = Q & 1;
    const int I = 2 * gm.bi + di, J = 2 * gm.bj + dj, K = 2 * gm.bk + dk;
    const float v = o.x[Q];
    sm.x2[p18(I, J, K)] = v;
    if (I == (gm.oi ? 0 : 15)) gm.rx2[0][p18(gm.oi ? 16 : -1, J, K)] = v;
    if (J == (gm.oj ? 0 : 15)) gm.rx2[1][p18(I, gm.oj ? 16 : -1, K)] = v;
    if (K == (gm.ok ? 0 : 15)) gm.rx2[2][p18(I, J, gm.ok ? 16 : -1)] = v;
}

template <int Q>
__device__ __forceinline__ void blk_gs_cell(Blk& o, ClSmem& sm, const Geo& gm, const ClusterArgs& A) {
    const float ax = blk_nlap<Q>(o, sm, gm);
    o.x[Q] = gs_update(o.x[Q], o.b[Q], ax, o.d[Q], (o.in >> Q) & 1u, A);
    blk_publish<Q>(o, sm, gm);
}
// one colour of the level-2 octant; colour of cell q is (di + dj + dk) & 1
__device__ __forceinline__ void blk_gs_pass(Blk& o, ClSmem& sm, const Geo& gm, int color, const ClusterArgs& A) {
    if (color == 0) {
        blk_gs_cell<0>(o, sm, gm, A);
        blk_gs_cell<3>(o, sm, gm, A);
        blk_gs_cell<5>(o, sm, gm, A);
        blk_gs_cell<6>(o, sm, gm, A);
    } else {
        blk_gs_cell<1>(o, sm, gm, A);
        blk_gs_cell<2>(o, sm, gm, A);
        blk_gs_cell<4>(o, sm, gm, A);
        blk_gs_cell<7>(o, sm, gm, A);
    }
}

// Level-1 cell of one thread: cell t of tile child[r]
struct L1Cell {
    float x, d, b, s;  // x, diagonal, rhs, saved x
    float cmx, cpx, cmy, cpy, cmz, cpz;
    bool in;
};
__device__ __forceinline__ float l1_nlap(const L1Cell& c, const ClSmem& sm, const Geo& gm) {
    const int q = p10(gm.bi, gm.bj, gm.bk);
    return nlap(c.d, c.x, c.cmx, sm.x1[q - 100], c.cpx, sm.x1[q + 100], c.cmy, sm.x1[q - 10], c.cpy, sm.x1[q + 10], c.cmz, sm.x1[q - 1],
                c.cpz, sm.x1[q + 1]);
}
__device__ __forceinline__ void l1_publish(const L1Cell& c, ClSmem& sm, const Geo& gm) {
    const int i = gm.bi, j = gm.bj, k = gm.bk;
    sm.x1[p10(i, j, k)] = c.x;
    if (i == (gm.oi ? 0 : 7)) gm.rx1[0][p10(gm.oi ? 8 : -1, j, k)] = c.x;
    if (j == (gm.oj ? 0 : 7)) gm.rx1[1][p10(i, gm.oj ? 8 : -1, k)] = c.x;
    if (k == (gm.ok ? 0 : 7)) gm.rx1[2][p10(i, j, gm.ok ? 8 : -1)] = c.x;
}

// Root cell of one thread of rank 0
struct L0Cell {
    float x, d, b;
    float cmx, cpx, cmy, cpy, cmz, cpz;
    bool in;
};
__device__ __forceinline__ float l0_nlap(const L0Cell& c, const ClSmem& sm, int q) {
    return nlap(c.d, c.x, c.cmx, sm.x0[q - 100], c.cpx, sm.x0[q + 100], c.cmy, sm.x0[q - 10], c.cpy, sm.x0[q + 10], c.cmz, sm.x0[q - 1],
                c.cpz, sm.x0[q + 1]);
}

__global__ void __cluster_dims__(kClCtas, 1, 1) __launch_bounds__(kClThreads, 1)
    k_cluster_step(DevGrid g, ClusterArgs A, float* X, float* RHS, float* X0) {
    __shared__ __align__(16) ClSmem sm;
    cg::cluster_group cluster = cg::this_cluster();
    const int tid = threadIdx.x;
    Geo gm;
    gm.r = (int)cluster.block_rank();
    gm.oi = gm.r >> 2;
    gm.oj = (gm.r >> 1) & 1;
    gm.ok = gm.r & 1;
    gm.bi = tid >> 6;
    gm.bj = (tid >> 3) & 7;
    gm.bk = tid & 7;
    for (int a = 0; a < 3; ++a) {
        gm.rx2[a] = cluster.map_shared_rank(sm.x2, gm.r ^ (4 >> a));
        gm.rx1[a] = cluster.map_shared_rank(sm.x1, gm.r ^ (4 >> a));
    }
    gm.rb0 = cluster.map_shared_rank(sm.b0, 0);
    gm.rx0 = cluster.map_shared_rank(sm.x0, 0);
    gm.rs0 = cluster.map_shared_rank(sm.s0, 0);

    const int* child = g.child;
    const float* C0 = g.plane(A.coeff_ch);
    const float* C1 = g.plane(A.coeff_ch + 1);
    const float* C2 = g.plane(A.coeff_ch + 2);
    const float* C3 = g.plane(A.coeff_ch + 3);
    const uint8_t* ty = g.ctype;

    // ---- zero halos, then load ----
    for (int q = tid; q < 18 * 18 * 18; q += kClThreads) sm.x2[q] = 0.0f;
    for (int q = tid; q < 1000; q += kClThreads) {
        sm.x1[q] = 0.0f;
        sm.x0[q] = 0.0f;
    }
    __syncthreads();

    // level-2 octant coordinates of the block's first cell in the 32^3 grid
    const int G2i = 16 * gm.oi + 2 * gm.bi, G2j = 16 * gm.oj + 2 * gm.bj, G2k = 16 * gm.ok + 2 * gm.bk;
    Blk o;
    o.in = 0u;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int di = q >> 2, dj = (q >> 1) & 1, dk = q & 1;
        const long long off = l2_off(child, G2i + di, G2j + dj, G2k + dk);
        const bool in = ty[off] & dInterior;
        o.in |= (in ? 1u : 0u) << q;
        o.d[q] = C3[off];
        o.b[q] = __ldcg(RHS + off);
        o.x[q] = in ? __ldcg(X + off) : 0.0f;
        o.cx[4 * di + 2 * dj + dk] = C0[off];
        o.cy[4 * dj + 2 * di + dk] = C1[off];
        o.cz[4 * dk + 2 * di + dj] = C2[off];
        sm.x2[p18(2 * gm.bi + di, 2 * gm.bj + dj, 2 * gm.bk + dk)] = o.x[q];
    }
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            // +faces of the block: the -face coefficient of the next block's cells (0 at the domain boundary)
            long long off = l2_off(child, G2i + 2, G2j + u, G2k + v);
            o.cx[8 + 2 * u + v] = off >= 0 ? C0[off] : 0.0f;
            off = l2_off(child, G2i + u, G2j + 2, G2k + v);
            o.cy[8 + 2 * u + v] = off >= 0 ? C1[off] : 0.0f;
            off = l2_off(child, G2i + u, G2j + v, G2k + 2);
            o.cz[8 + 2 * u + v] = off >= 0 ? C2[off] : 0.0f;
        }
    // halo cells that lie in a neighbouring octant (domain-boundary halos stay 0)
    {
        const int hi = gm.oi ? 0 : 7, hj = gm.oj ? 0 : 7, hk = gm.ok ? 0 : 7;
        const int si = gm.oi ? -1 : 2, sj = gm.oj ? -1 : 2, sk = gm.ok ? -1 : 2;  // offset of the halo cell from the block origin
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                if (gm.bi == hi) {
                    const long long off = l2_off(child, G2i + si, G2j + u, G2k + v);
                    sm.x2[p18(2 * gm.bi + si, 2 * gm.bj + u, 2 * gm.bk + v)] = (ty[off] & dInterior) ? __ldcg(X + off) : 0.0f;
                }
                if (gm.bj == hj) {
                    const long long off = l2_off(child, G2i + u, G2j + sj, G2k + v);
                    sm.x2[p18(2 * gm.bi + u, 2 * gm.bj + sj, 2 * gm.bk + v)] = (ty[off] & dInterior) ? __ldcg(X + off) : 0.0f;
                }
                if (gm.bk == hk) {
                    const long long off = l2_off(child, G2i + u, G2j + v, G2k + sk);
                    sm.x2[p18(2 * gm.bi + u, 2 * gm.bj + v, 2 * gm.bk + sk)] = (ty[off] & dInterior) ? __ldcg(X + off) : 0.0f;
                }
            }
    }
    // level-1 cell
    const int G1i = 8 * gm.oi + gm.bi, G1j = 8 * gm.oj + gm.bj, G1k = 8 * gm.ok + gm.bk;
    const long long off1 = l1_off(child, G1i, G1j, G1k);
    L1Cell c1;
    {
        c1.in = ty[off1] & dInterior;
        c1.d = C3[off1];
        c1.cmx = C0[off1];
        c1.cmy = C1[off1];
        c1.cmz = C2[off1];
        long long o2 = l1_off(child, G1i + 1, G1j, G1k);
        c1.cpx = o2 >= 0 ? C0[o2] : 0.0f;
        o2 = l1_off(child, G1i, G1j + 1, G1k);
        c1.cpy = o2 >= 0 ? C1[o2] : 0.0f;
        o2 = l1_off(child, G1i, G1j, G1k + 1);
        c1.cpz = o2 >= 0 ? C2[o2] : 0.0f;
        c1.x = c1.b = c1.s = 0.0f;
    }
    // root cell (rank 0)
    L0Cell c0 = {};
    const int q0 = p10(gm.bi, gm.bj, gm.bk);
    if (gm.r == 0) {
        c0.in = ty[tid] & dInterior;
        c0.d = C3[tid];
        c0.cmx = C0[tid];
        c0.cpx = gm.bi < 7 ? C0[tid + 64] : 0.0f;
        c0.cmy = C1[tid];
        c0.cpy = gm.bj < 7 ? C1[tid + 8] : 0.0f;
        c0.cmz = C2[tid];
        c0.cpz = gm.bk < 7 ? C2[tid + 1] : 0.0f;
        c0.x = c0.b = 0.0f;
        sm.s0[tid] = __ldcg(X0 + tid);
    }
    // every CTA has initialised its halos before any peer writes into them
    cluster.sync();

    // ---- level 2: pre-smoothing ----
    for (int it = 0; it < A.level_iters; ++it) {
        blk_gs_pass(o, sm, gm, 0, A);
        cluster.sync();
        blk_gs_pass(o, sm, gm, 1, A);
        cluster.sync();
    }
    // ---- residual, restriction to level 1 (ResidualAndRestrictAMG128Kernel) ----
    {
        float res[8];
        res[0] = __fsub_rn(o.b[0], blk_nlap<0>(o, sm, gm));
        res[1] = __fsub_rn(o.b[1], blk_nlap<1>(o, sm, gm));
        res[2] = __fsub_rn(o.b[2], blk_nlap<2>(o, sm, gm));
        res[3] = __fsub_rn(o.b[3], blk_nlap<3>(o, sm, gm));
        res[4] = __fsub_rn(o.b[4], blk_nlap<4>(o, sm, gm));
        res[5] = __fsub_rn(o.b[5], blk_nlap<5>(o, sm, gm));
        res[6] = __fsub_rn(o.b[6], blk_nlap<6>(o, sm, gm));
        res[7] = __fsub_rn(o.b[7], blk_nlap<7>(o, sm, gm));
        float rs = 0.0f, xs = 0.0f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            rs = __fadd_rn(rs, res[q]);
            xs = __fadd_rn(xs, o.x[q]);
        }
        c1.b = __fmul_rn(rs, A.Rr);
        c1.x = c1.in ? __fdiv_rn(xs, 8.0f) : 0.0f;
    }
    l1_publish(c1, sm, gm);
    cluster.sync();
    // ---- FASSaveSolutionAndUpdateSource on level 1 ----
    if (c1.in) {
        c1.b = __fadd_rn(c1.b, l1_nlap(c1, sm, gm));
        c1.s = c1.x;
    } else {
        c1.b = 0.0f;
    }
    // the first level-1 sweep overwrites x1 values that the update above reads
    cluster.sync();

    float root_b = 0.0f;
    for (int rep = 0; rep < A.mu; ++rep) {
        // ---- FASMuCycleStep of level 1 ----
        for (int it = 0; it < A.level_iters; ++it)
            for (int h = 0; h < 2; ++h) {
                if (((gm.bi + gm.bj + gm.bk) & 1) == h) {
                    c1.x = gs_update(c1.x, c1.b, l1_nlap(c1, sm, gm), c1.d, c1.in, A);
                    l1_publish(c1, sm, gm);
                }
                cluster.sync();
            }
        sm.r1[tid] = __fsub_rn(c1.b, l1_nlap(c1, sm, gm));
        __syncthreads();
        if (tid < 64) {
            const int a = tid >> 4, b = (tid >> 2) & 3, c = tid & 3;
            float rs = 0.0f, xs = 0.0f;
#pragma unroll
            for (int ii = 0; ii < 2; ++ii)
#pragma unroll
                for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        rs = __fadd_rn(rs, sm.r1[cell_index(2 * a + ii, 2 * b + jj, 2 * c + kk)]);
                        xs = __fadd_rn(xs, sm.x1[p10(2 * a + ii, 2 * b + jj, 2 * c + kk)]);
                    }
            const int ri = 4 * gm.oi + a, rj = 4 * gm.oj + b, rk = 4 * gm.ok + c;
            const int v = cell_index(ri, rj, rk);
            gm.rb0[v] = __fmul_rn(rs, A.Rr);
            gm.rx0[p10(ri, rj, rk)] = (ty[v] & dInterior) ? __fdiv_rn(xs, 8.0f) : 0.0f;
        }
        cluster.sync();
        // ---- root: FAS save, then mu coarsest solves (rank 0 alone) ----
        if (gm.r == 0) {
            c0.x = sm.x0[q0];
            c0.b = sm.b0[tid];
            if (c0.in) {
                c0.b = __fadd_rn(c0.b, l0_nlap(c0, sm, q0));
                sm.s0[tid] = c0.x;
            } else {
                c0.b = 0.0f;
            }
            const int par = (gm.bi + gm.bj + gm.bk) & 1;
            for (int rr = 0; rr < A.mu; ++rr)
                for (int half = 0; half < 2; ++half)
                    for (int it = 0; it < A.coarsest_iters / 2; ++it)
                        for (int h = 0; h < 2; ++h) {
                            __syncthreads();
                            if (par == (h ^ half)) {
                                c0.x = gs_update(c0.x, c0.b, l0_nlap(c0, sm, q0), c0.d, c0.in, A);
                                sm.x0[q0] = c0.x;
                            }
                        }
            root_b = c0.b;
        }
        cluster.sync();
        // ---- FASProlongateAndUpdate on level 1 from the root ----
        {
            const int pi = G1i >> 1, pj = G1j >> 1, pk = G1k >> 1;
            const float cx = gm.rx0[p10(pi, pj, pk)];
            const float cx0 = gm.rs0[cell_index(pi, pj, pk)];
            c1.x = c1.in ? __fmaf_rn(A.P, __fsub_rn(cx, cx0), c1.x) : 0.0f;
            l1_publish(c1, sm, gm);
        }
        cluster.sync();
        for (int it = 0; it < A.level_iters; ++it)
            for (int h = 0; h < 2; ++h) {
                if (((gm.bi + gm.bj + gm.bk) & 1) == (h ^ 1)) {
                    c1.x = gs_update(c1.x, c1.b, l1_nlap(c1, sm, gm), c1.d, c1.in, A);
                    l1_publish(c1, sm, gm);
                }
                cluster.sync();
            }
    }
    // ---- FASProlongateAndUpdate on level 2 ----
    {
        const float dlt = __fsub_rn(c1.x, c1.s);
#pragma unroll
        for (int q = 0; q < 8; ++q) o.x[q] = ((o.in >> q) & 1u) ? __fmaf_rn(A.P, dlt, o.x[q]) : 0.0f;
        blk_publish<0>(o, sm, gm);
        blk_publish<1>(o, sm, gm);
        blk_publish<2>(o, sm, gm);
        blk_publish<3>(o, sm, gm);
        blk_publish<4>(o, sm, gm);
        blk_publish<5>(o, sm, gm);
        blk_publish<6>(o, sm, gm);
        blk_publish<7>(o, sm, gm);
    }
    cluster.sync();
    // ---- level 2: post-smoothing ----
    for (int it = 0; it < A.level_iters; ++it) {
        blk_gs_pass(o, sm, gm, 1, A);
        cluster.sync();
        blk_gs_pass(o, sm, gm, 0, A);
        cluster.sync();
    }

    // ---- write back: level-2 x; level-1 x, rhs, saved x; root x, rhs, saved x ----
#pragma unroll
    for (int q = 0; q < 8; ++q) X[l2_off(child, G2i + (q >> 2), G2j + ((q >> 1) & 1), G2k + (q & 1))] = o.x[q];
    X[off1] = c1.x;
    RHS[off1] = c1.b;
    if (c1.in) X0[off1] = c1.s;
    if (gm.r == 0 && A.mu > 0) {
        X[tid] = sm.x0[q0];
        RHS[tid] = root_b;
        X0[tid] = sm.s0[tid];
    }
}

}  // namespace

void launch_cluster_step(const DevGrid& g, float* X, float* RHS, float* X0, int coeff_ch, int mu, int level_iters, int coarsest_iters,
                         double omega, float Rr, float P, cudaStream_t st) {
    ClusterArgs A;
    A.coeff_ch = coeff_ch;
    A.mu = mu;
    A.level_iters = level_iters;
    A.coarsest_iters = coarsest_iters;
    A.om = (float)omega;
    A.exact = ((double)A.om == omega);
    A.omega = omega;
    A.Rr = Rr;
    A.P = P;
    note_kernel_launch();
    k_cluster_step<<<kClCtas, kClThreads, 0, st>>>(g, A, X, RHS, X0);
}

bool cluster_step_supported() {
    int dev = 0, cc = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&cc, cudaDevAttrClusterLaunch, dev) != cudaSuccess || !cc) return false;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClCtas);
    cfg.blockDim = dim3(kClThreads);
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = kClCtas;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_cluster_step, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return nclusters > 0;
}

}  // namespace cmg
