// FASMuCycleStep of level 2 (src/AMGSolver.cu:1257-1277) with its whole
// recursion through levels 1 and 0, in one launch of one 9-CTA thread-block
// cluster.
//
// When the root, its eight children and their 64 children all exist (no GHOST
// tile on levels 0-2), levels 2, 1 and 0 are complete 32^3, 16^3 and 8^3
// grids.  CTAs 0-7 of the cluster own the octants of level 2
// (r = 4*oi + 2*oj + ok, the child order of the root): a 16^3 block each.  CTA
// 8, the coarse CTA, owns all of level 1 and the root and runs the level-1
// cycles and the coarsest sweeps between block barriers.
//
// In an octant CTA, thread t owns the 2x2x2 block of level-2 cells that is
// level-1 cell t of tile child[r]; in the coarse CTA, thread t owns root cell t
// and the 2x2x2 block of level-1 cells under it.  Restriction and prolongation
// therefore stay inside a thread, and a block's diagonals, right-hand sides, x
// and face coefficients live in registers.  x is mirrored in shared memory with
// a one-cell halo.  After every level-2 update an octant CTA stores its octant-
// boundary cells straight into the halos of the neighbouring octants' CTAs
// (distributed shared memory); one cluster barrier per phase publishes them.
// The level-1 x and rhs made by the restriction go straight into the coarse
// CTA's shared memory, and the corrected level-1 x comes back the same way.
//
// The static operands (diagonals, face coefficients, 1/diagonal in double,
// INTERIOR masks) are packed once per solve by k_cluster_pack into
// thread-major arrays, so each CTA loads them with coalesced loads and no
// divisions.  Every value is computed with the same operations in the same
// order as the per-level tile kernels and the dense coarse kernel (red-black
// Gauss-Seidel does not depend on the order of cells within a colour, and
// div_by_recip equals IEEE division), so the result equals theirs bit for bit.
#include <cooperative_groups.h>

#include "kernels.hpp"

namespace cmg {

namespace cg = cooperative_groups;

namespace {

constexpr int kOct = 8;        // octant CTAs
constexpr int kCoarse = 8;     // rank of the coarse CTA
constexpr int kClCtas = 9;
constexpr int kClThreads = 512;

// Shared-memory layout of a 16^3 grid with a one-cell halo (cells -1..16 per
// axis): split by cell parity, q = 4*(I&1) + 2*(J&1) + (K&1), each parity class
// indexed by the 2x2x2 block (I>>1)+1 etc. in 0..9 with strides 240, 24, 1.  The
// thread-to-block map below puts a warp on blocks (bi0+0..1, bj0+0..1, 0..7),
// whose offsets 240*bi + 24*bj + bk fall on 32 distinct banks, so every
// neighbour access of a sweep is free of bank conflicts.
constexpr int kPar = 2400;  // floats per parity class
__device__ __forceinline__ int xo(int I, int J, int K) {
    return (((I & 1) << 2) | ((J & 1) << 1) | (K & 1)) * kPar + ((I >> 1) + 1) * 240 + ((J >> 1) + 1) * 24 + ((K >> 1) + 1);
}
// root grid (8^3, zero halo): strides 240, 24, 1 as well
__device__ __forceinline__ int ro(int i, int j, int k) { return (i + 1) * 240 + (j + 1) * 24 + (k + 1); }
// thread t <-> block (bi, bj, bk) of an 8^3 block grid: lane = 16*(bi&1) + 8*(bj&1) + bk,
// warp = 4*(bi>>1) + (bj>>1)
__device__ __forceinline__ void blk_of_thread(int t, int& bi, int& bj, int& bk) {
    const int w = t >> 5, lane = t & 31;
    bk = lane & 7;
    bj = ((w & 3) << 1) | ((lane >> 3) & 1);
    bi = ((w >> 2) << 1) | (lane >> 4);
}
__device__ __forceinline__ int thread_of_blk(int bi, int bj, int bk) {
    return ((((bi >> 1) << 2) | (bj >> 1)) << 5) | ((bi & 1) << 4) | ((bj & 1) << 3) | bk;
}

// Packed static operands of one CTA, [field][thread].
//   f[0..7]   diagonal of block cell q = 4*di + 2*dj + dk
//   f[8..19]  x-face coefficients cx[4p + 2dj + dk]: -x face of the cells with di = p,
//             p = 2: the +x face of the di = 1 cells (0 at the domain boundary)
//   f[20..31] cy[4p + 2di + dk]   f[32..43] cz[4p + 2di + dj]
//   f[44..50] coarse CTA: root cell diagonal, then its -x,+x,-y,+y,-z,+z coefficients
//   y[0..7]   1/diagonal (double) of the block cells; y[8]: of the root cell
//   m         bits 0-7: block cell q INTERIOR; bit 8: the level-1 cell (octant CTAs)
//             or the root cell (coarse CTA) INTERIOR; bits 9-20 (octant CTAs): halo
//             cell (axis a, u, v) INTERIOR at bit 9 + 4a + 2u + v
struct ClPack {
    float f[52][kClThreads];
    double y[9][kClThreads];
    unsigned m[kClThreads];
};

struct ClusterArgs {
    int coeff_ch, mu, level_iters, coarsest_iters, exact, fas2;
    float om, Rr, P;
    double omega;
    // direct coarsest solve (mixed-precision mode): the inverse of the root operator in
    // double, [j][t] = (A0^-1)[cell of thread j][cell of thread t]; null: Gauss-Seidel
    const double* root_inv;
    int tile1[8];   // level-1 tiles by octant (root child order)
    int tile2[64];  // level-2 tiles by (I>>3)*16 + (J>>3)*4 + (K>>3) over the 32^3 grid
};

// plane offset of level-2 cell (I, J, K) of the 32^3 grid, -1 outside
__device__ __forceinline__ long long l2_off(const ClusterArgs& A, int I, int J, int K) {
    if ((unsigned)I >= 32u || (unsigned)J >= 32u || (unsigned)K >= 32u) return -1;
    return (long long)A.tile2[((I >> 3) << 4) | ((J >> 3) << 2) | (K >> 3)] * kCells + cell_index(I & 7, J & 7, K & 7);
}
// plane offset of level-1 cell (I, J, K) of the 16^3 grid, -1 outside
__device__ __forceinline__ long long l1_off(const ClusterArgs& A, int I, int J, int K) {
    if ((unsigned)I >= 16u || (unsigned)J >= 16u || (unsigned)K >= 16u) return -1;
    return (long long)A.tile1[((I >> 3) << 2) | ((J >> 3) << 1) | (K >> 3)] * kCells + cell_index(I & 7, J & 7, K & 7);
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
// one Gauss-Seidel update (src/AMGSolver.cu:868-875); kRelax: how omega is applied (relax<>)
template <int kRelax>
__device__ __forceinline__ float gs_update(float xs, float rhs, float ax, float d, double yd, bool interior, const ClusterArgs& A) {
    const float delta = interior ? div_by_recip(__fsub_rn(rhs, ax), d, yd) : 0.0f;
    return relax<kRelax>(xs, delta, A.om, A.omega);
}

// Shared memory.  Octant CTA: x (the level-2 octant, halo from the neighbouring
// octants) and yd.  Coarse CTA: x (level 1, zero halo), yd, b1 and s1 ([q][t]), x0.
struct ClSmem {
    double yd[9][kClThreads];  // 1/diagonal of the block cells ([q][t]) and of the root cell
    float x[8 * kPar];         // 16^3 grid with halo, layout xo()
    float b1[8][kClThreads];   // coarse: restricted level-1 rhs, written by the octant CTAs
    float s1[8][kClThreads];   // coarse: saved level-1 x, read back by the octant CTAs
    float x0[kPar];            // coarse: root x, zero halo, layout ro()
    float b0[kClThreads];      // coarse: root rhs by owning thread (direct coarsest solve)
};
constexpr size_t kClSmem = sizeof(ClSmem);

// A 2x2x2 block of one thread on a 16^3 grid held in shared memory (layout xo()).
struct Blk {
    float x[8], d[8], b[8];
    float cx[12], cy[12], cz[12];
    unsigned in;  // bit q: cell q INTERIOR
    int bi, bj, bk;
};

// the three neighbours of block cell Q outside the block: x side, y side, z side
template <int Q>
__device__ __forceinline__ void blk_outer(const Blk& o, const float* xs, float v[3]) {
    constexpr int di = Q >> 2, dj = (Q >> 1) & 1, dk = Q & 1;
    // the cell of opposite parity along the axis, one block over
    const int b = (o.bi + 1) * 240 + (o.bj + 1) * 24 + (o.bk + 1);
    v[0] = di ? xs[(Q & 3) * kPar + b + 240] : xs[(Q | 4) * kPar + b - 240];
    v[1] = dj ? xs[(Q & 5) * kPar + b + 24] : xs[(Q | 2) * kPar + b - 24];
    v[2] = dk ? xs[(Q & 6) * kPar + b + 1] : xs[(Q | 1) * kPar + b - 1];
}
template <int Q>
__device__ __forceinline__ float blk_nlap_v(const Blk& o, const float v[3]) {
    constexpr int di = Q >> 2, dj = (Q >> 1) & 1, dk = Q & 1;
    const float xmx = di ? o.x[Q - 4] : v[0];
    const float xpx = di ? v[0] : o.x[Q + 4];
    const float xmy = dj ? o.x[Q - 2] : v[1];
    const float xpy = dj ? v[1] : o.x[Q + 2];
    const float xmz = dk ? o.x[Q - 1] : v[2];
    const float xpz = dk ? v[2] : o.x[Q + 1];
    return nlap(o.d[Q], o.x[Q], o.cx[4 * di + 2 * dj + dk], xmx, o.cx[4 * (di + 1) + 2 * dj + dk], xpx, o.cy[4 * dj + 2 * di + dk], xmy,
                o.cy[4 * (dj + 1) + 2 * di + dk], xpy, o.cz[4 * dk + 2 * di + dj], xmz, o.cz[4 * (dk + 1) + 2 * di + dj], xpz);
}
template <int Q>
__device__ __forceinline__ float blk_nlap(const Blk& o, const float* xs) {
    float v[3];
    blk_outer<Q>(o, xs, v);
    return blk_nlap_v<Q>(o, v);
}

// 32-bit shared::cluster address of `p` (this CTA's shared memory) in CTA `rank`
__device__ __forceinline__ unsigned peer_addr(const void* p, int rank) {
    unsigned a;
    asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"((unsigned)__cvta_generic_to_shared(p)), "r"(rank));
    return a;
}
__device__ __forceinline__ void st_peer(unsigned a, float v) { asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory"); }

// Neighbouring octants' halos (octant CTAs only).
struct Peers {
    int oi, oj, ok;
    unsigned rx[3];  // x of the neighbouring octant along x, y, z (shared::cluster addresses)
};

// store cell Q of the block into shared memory and, for an octant CTA on an octant face, into the neighbour's halo
template <int Q, bool kRemote>
__device__ __forceinline__ void blk_publish(const Blk& o, float* xs, const Peers& pr) {
    constexpr int di = Q >> 2, dj = (Q >> 1) & 1, dk = Q & 1;
    const int I = 2 * o.bi + di, J = 2 * o.bj + dj, K = 2 * o.bk + dk;
    const float v = o.x[Q];
    xs[Q * kPar + (o.bi + 1) * 240 + (o.bj + 1) * 24 + (o.bk + 1)] = v;
    if (kRemote) {
        if (I == (pr.oi ? 0 : 15)) st_peer(pr.rx[0] + 4 * xo(pr.oi ? 16 : -1, J, K), v);
        if (J == (pr.oj ? 0 : 15)) st_peer(pr.rx[1] + 4 * xo(I, pr.oj ? 16 : -1, K), v);
        if (K == (pr.ok ? 0 : 15)) st_peer(pr.rx[2] + 4 * xo(I, J, pr.ok ? 16 : -1), v);
    }
}
template <bool kRemote>
__device__ __forceinline__ void blk_publish_all(const Blk& o, float* xs, const Peers& pr) {
    blk_publish<0, kRemote>(o, xs, pr);
    blk_publish<1, kRemote>(o, xs, pr);
    blk_publish<2, kRemote>(o, xs, pr);
    blk_publish<3, kRemote>(o, xs, pr);
    blk_publish<4, kRemote>(o, xs, pr);
    blk_publish<5, kRemote>(o, xs, pr);
    blk_publish<6, kRemote>(o, xs, pr);
    blk_publish<7, kRemote>(o, xs, pr);
}

// one colour of the block, cells Q0..Q3 (the colour of cell q is (di + dj + dk) & 1).  The
// four cells are not neighbours of one another, so every neighbour load comes first, then
// the four updates, then the stores: the updates overlap instead of each waiting on the
// previous cell's shared-memory store.
template <int Q0, int Q1, int Q2, int Q3, bool kRemote, int kExact>
__device__ __forceinline__ void blk_gs_colour(Blk& o, float* xs, const double* yd, const Peers& pr, const ClusterArgs& A) {
    float v0[3], v1[3], v2[3], v3[3];
    blk_outer<Q0>(o, xs, v0);
    blk_outer<Q1>(o, xs, v1);
    blk_outer<Q2>(o, xs, v2);
    blk_outer<Q3>(o, xs, v3);
    const double y0 = yd[Q0 * kClThreads + threadIdx.x], y1 = yd[Q1 * kClThreads + threadIdx.x];
    const double y2 = yd[Q2 * kClThreads + threadIdx.x], y3 = yd[Q3 * kClThreads + threadIdx.x];
    const float a0 = blk_nlap_v<Q0>(o, v0), a1 = blk_nlap_v<Q1>(o, v1), a2 = blk_nlap_v<Q2>(o, v2), a3 = blk_nlap_v<Q3>(o, v3);
    o.x[Q0] = gs_update<kExact>(o.x[Q0], o.b[Q0], a0, o.d[Q0], y0, (o.in >> Q0) & 1u, A);
    o.x[Q1] = gs_update<kExact>(o.x[Q1], o.b[Q1], a1, o.d[Q1], y1, (o.in >> Q1) & 1u, A);
    o.x[Q2] = gs_update<kExact>(o.x[Q2], o.b[Q2], a2, o.d[Q2], y2, (o.in >> Q2) & 1u, A);
    o.x[Q3] = gs_update<kExact>(o.x[Q3], o.b[Q3], a3, o.d[Q3], y3, (o.in >> Q3) & 1u, A);
    blk_publish<Q0, kRemote>(o, xs, pr);
    blk_publish<Q1, kRemote>(o, xs, pr);
    blk_publish<Q2, kRemote>(o, xs, pr);
    blk_publish<Q3, kRemote>(o, xs, pr);
}
template <bool kRemote, int kExact>
__device__ __forceinline__ void blk_gs_pass(Blk& o, float* xs, const double* yd, const Peers& pr, int color, const ClusterArgs& A) {
    if (color == 0)
        blk_gs_colour<0, 3, 5, 6, kRemote, kExact>(o, xs, yd, pr, A);
    else
        blk_gs_colour<1, 2, 4, 7, kRemote, kExact>(o, xs, yd, pr, A);
}
// ResidualAndRestrictAMG128Kernel (src/AMGSolver.cu:896-960) of the block into its parent cell:
// rhs = R * sum of the 8 residuals, x = mean of the 8 x (0 unless the parent is INTERIOR)
__device__ __forceinline__ void blk_restrict(const Blk& o, const float* xs, bool parent_in, float Rr, float& rhs, float& x) {
    float res[8];
    res[0] = __fsub_rn(o.b[0], blk_nlap<0>(o, xs));
    res[1] = __fsub_rn(o.b[1], blk_nlap<1>(o, xs));
    res[2] = __fsub_rn(o.b[2], blk_nlap<2>(o, xs));
    res[3] = __fsub_rn(o.b[3], blk_nlap<3>(o, xs));
    res[4] = __fsub_rn(o.b[4], blk_nlap<4>(o, xs));
    res[5] = __fsub_rn(o.b[5], blk_nlap<5>(o, xs));
    res[6] = __fsub_rn(o.b[6], blk_nlap<6>(o, xs));
    res[7] = __fsub_rn(o.b[7], blk_nlap<7>(o, xs));
    float rs = 0.0f, xsum = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        rs = __fadd_rn(rs, res[q]);
        xsum = __fadd_rn(xsum, o.x[q]);
    }
    rhs = __fmul_rn(rs, Rr);
    x = parent_in ? __fmul_rn(xsum, 0.125f) : 0.0f;  // equals xsum / 8
}
// FASProlongateAndUpdateAMG128Kernel (src/AMGSolver.cu:1216-1248) from the parent cell
__device__ __forceinline__ void blk_prolong(Blk& o, float P, float cx, float cx0) {
    const float dlt = __fsub_rn(cx, cx0);
#pragma unroll
    for (int q = 0; q < 8; ++q) o.x[q] = ((o.in >> q) & 1u) ? __fmaf_rn(P, dlt, o.x[q]) : 0.0f;
}

__device__ __forceinline__ void blk_load_static(Blk& o, const ClPack& pk, int t) {
#pragma unroll
    for (int q = 0; q < 8; ++q) o.d[q] = pk.f[q][t];
#pragma unroll
    for (int c = 0; c < 12; ++c) {
        o.cx[c] = pk.f[8 + c][t];
        o.cy[c] = pk.f[20 + c][t];
        o.cz[c] = pk.f[32 + c][t];
    }
}

// ---------------------------------------------------------------------------
// Packing of the static operands (once per solve)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kClThreads) k_cluster_pack(DevGrid g, const __grid_constant__ ClusterArgs A, ClPack* packs) {
    const int r = blockIdx.x, t = threadIdx.x;
    ClPack& pk = packs[r];
    const float* C0 = g.plane(A.coeff_ch);
    const float* C1 = g.plane(A.coeff_ch + 1);
    const float* C2 = g.plane(A.coeff_ch + 2);
    const float* C3 = g.plane(A.coeff_ch + 3);
    const uint8_t* ty = g.ctype;
    int bi, bj, bk;
    blk_of_thread(t, bi, bj, bk);
    unsigned m = 0;
    if (r < kOct) {
        const int oi = r >> 2, oj = (r >> 1) & 1, ok = r & 1;
        const int Gi = 16 * oi + 2 * bi, Gj = 16 * oj + 2 * bj, Gk = 16 * ok + 2 * bk;
        for (int q = 0; q < 8; ++q) {
            const int di = q >> 2, dj = (q >> 1) & 1, dk = q & 1;
            const long long o = l2_off(A, Gi + di, Gj + dj, Gk + dk);
            pk.f[q][t] = C3[o];
            pk.y[q][t] = 1.0 / (double)C3[o];
            pk.f[8 + 4 * di + 2 * dj + dk][t] = C0[o];
            pk.f[20 + 4 * dj + 2 * di + dk][t] = C1[o];
            pk.f[32 + 4 * dk + 2 * di + dj][t] = C2[o];
            if (ty[o] & dInterior) m |= 1u << q;
        }
        for (int u = 0; u < 2; ++u)
            for (int v = 0; v < 2; ++v) {
                long long o = l2_off(A, Gi + 2, Gj + u, Gk + v);
                pk.f[8 + 8 + 2 * u + v][t] = o >= 0 ? C0[o] : 0.0f;
                o = l2_off(A, Gi + u, Gj + 2, Gk + v);
                pk.f[20 + 8 + 2 * u + v][t] = o >= 0 ? C1[o] : 0.0f;
                o = l2_off(A, Gi + u, Gj + v, Gk + 2);
                pk.f[32 + 8 + 2 * u + v][t] = o >= 0 ? C2[o] : 0.0f;
            }
        if (ty[l1_off(A, 8 * oi + bi, 8 * oj + bj, 8 * ok + bk)] & dInterior) m |= 1u << 8;
        for (int f = 44; f < 52; ++f) pk.f[f][t] = 0.0f;
        pk.y[8][t] = 0.0;
        // halo cells in the neighbouring octants
        const int si = oi ? -1 : 2, sj = oj ? -1 : 2, sk = ok ? -1 : 2;
        for (int u = 0; u < 2; ++u)
            for (int v = 0; v < 2; ++v) {
                if (bi == (oi ? 0 : 7) && (ty[l2_off(A, Gi + si, Gj + u, Gk + v)] & dInterior)) m |= 1u << (9 + 2 * u + v);
                if (bj == (oj ? 0 : 7) && (ty[l2_off(A, Gi + u, Gj + sj, Gk + v)] & dInterior)) m |= 1u << (13 + 2 * u + v);
                if (bk == (ok ? 0 : 7) && (ty[l2_off(A, Gi + u, Gj + v, Gk + sk)] & dInterior)) m |= 1u << (17 + 2 * u + v);
            }
    } else {
        const int Gi = 2 * bi, Gj = 2 * bj, Gk = 2 * bk;
        for (int q = 0; q < 8; ++q) {
            const int di = q >> 2, dj = (q >> 1) & 1, dk = q & 1;
            const long long o = l1_off(A, Gi + di, Gj + dj, Gk + dk);
            pk.f[q][t] = C3[o];
            pk.y[q][t] = 1.0 / (double)C3[o];
            pk.f[8 + 4 * di + 2 * dj + dk][t] = C0[o];
            pk.f[20 + 4 * dj + 2 * di + dk][t] = C1[o];
            pk.f[32 + 4 * dk + 2 * di + dj][t] = C2[o];
            if (ty[o] & dInterior) m |= 1u << q;
        }
        for (int u = 0; u < 2; ++u)
            for (int v = 0; v < 2; ++v) {
                long long o = l1_off(A, Gi + 2, Gj + u, Gk + v);
                pk.f[8 + 8 + 2 * u + v][t] = o >= 0 ? C0[o] : 0.0f;
                o = l1_off(A, Gi + u, Gj + 2, Gk + v);
                pk.f[20 + 8 + 2 * u + v][t] = o >= 0 ? C1[o] : 0.0f;
                o = l1_off(A, Gi + u, Gj + v, Gk + 2);
                pk.f[32 + 8 + 2 * u + v][t] = o >= 0 ? C2[o] : 0.0f;
            }
        // root cell (bi, bj, bk) (the root is tile 0)
        const int v = cell_index(bi, bj, bk);
        pk.f[44][t] = C3[v];
        pk.y[8][t] = 1.0 / (double)C3[v];
        pk.f[45][t] = C0[v];
        pk.f[46][t] = bi < 7 ? C0[v + 64] : 0.0f;
        pk.f[47][t] = C1[v];
        pk.f[48][t] = bj < 7 ? C1[v + 8] : 0.0f;
        pk.f[49][t] = C2[v];
        pk.f[50][t] = bk < 7 ? C2[v + 1] : 0.0f;
        pk.f[51][t] = 0.0f;
        if (ty[v] & dInterior) m |= 1u << 8;
    }
    pk.m[t] = m;
}

// ---------------------------------------------------------------------------
// The cluster step
// ---------------------------------------------------------------------------
template <int kExact>
__global__ void __launch_bounds__(kClThreads, 1)
    k_cluster_step(DevGrid g, const __grid_constant__ ClusterArgs A, const ClPack* packs, float* X, float* RHS, float* X0) {
    extern __shared__ __align__(16) unsigned char cl_smem[];
    ClSmem& sm = *reinterpret_cast<ClSmem*>(cl_smem);
    cg::cluster_group cluster = cg::this_cluster();
    const int t = threadIdx.x;
    const int r = (int)cluster.block_rank();
    const ClPack& pk = packs[r];
    Blk o;
    blk_of_thread(t, o.bi, o.bj, o.bk);
    Peers pr;
    pr.oi = r >> 2;
    pr.oj = (r >> 1) & 1;
    pr.ok = r & 1;
    float* xs = sm.x;
    const double* yd = &sm.yd[0][0];
    ClSmem& cs = *cluster.map_shared_rank(&sm, kCoarse);  // the coarse CTA's shared memory

    for (int q = t; q < 8 * kPar; q += kClThreads) xs[q] = 0.0f;
    if (r == kCoarse)
        for (int q = t; q < kPar; q += kClThreads) sm.x0[q] = 0.0f;
    blk_load_static(o, pk, t);
    const unsigned m = pk.m[t];
    o.in = m & 0xffu;
#pragma unroll
    for (int q = 0; q < 9; ++q) sm.yd[q][t] = pk.y[q][t];

    if (r < kOct) {
        // ============================ octant CTA ============================
        for (int a = 0; a < 3; ++a) pr.rx[a] = peer_addr(sm.x, r ^ (4 >> a));
        const int Gi = 16 * pr.oi + 2 * o.bi, Gj = 16 * pr.oj + 2 * o.bj, Gk = 16 * pr.ok + 2 * o.bk;
        float xin[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const long long off = l2_off(A, Gi + (q >> 2), Gj + ((q >> 1) & 1), Gk + (q & 1));
            o.b[q] = __ldcg(RHS + off);
            xin[q] = __ldcg(X + off);
        }
        // halo cells in the neighbouring octants (domain-boundary halos stay 0)
        float hv[12];
        const int si = pr.oi ? -1 : 2, sj = pr.oj ? -1 : 2, sk = pr.ok ? -1 : 2;
        const bool fi = o.bi == (pr.oi ? 0 : 7), fj = o.bj == (pr.oj ? 0 : 7), fk = o.bk == (pr.ok ? 0 : 7);
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                // the offsets are in range exactly when the face flag is set; 0 stands in otherwise
                const long long oi_ = fi ? l2_off(A, Gi + si, Gj + u, Gk + v) : 0;
                const long long oj_ = fj ? l2_off(A, Gi + u, Gj + sj, Gk + v) : 0;
                const long long ok_ = fk ? l2_off(A, Gi + u, Gj + v, Gk + sk) : 0;
                hv[2 * u + v] = fi ? __ldcg(X + oi_) : 0.0f;
                hv[4 + 2 * u + v] = fj ? __ldcg(X + oj_) : 0.0f;
                hv[8 + 2 * u + v] = fk ? __ldcg(X + ok_) : 0.0f;
            }
#pragma unroll
        for (int q = 0; q < 8; ++q) o.x[q] = ((m >> q) & 1u) ? xin[q] : 0.0f;
        blk_publish_all<false>(o, xs, pr);
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                if (fi) xs[xo(2 * o.bi + si, 2 * o.bj + u, 2 * o.bk + v)] = ((m >> (9 + 2 * u + v)) & 1u) ? hv[2 * u + v] : 0.0f;
                if (fj) xs[xo(2 * o.bi + u, 2 * o.bj + sj, 2 * o.bk + v)] = ((m >> (13 + 2 * u + v)) & 1u) ? hv[4 + 2 * u + v] : 0.0f;
                if (fk) xs[xo(2 * o.bi + u, 2 * o.bj + v, 2 * o.bk + sk)] = ((m >> (17 + 2 * u + v)) & 1u) ? hv[8 + 2 * u + v] : 0.0f;
            }
        if (A.fas2) {
            // ---- FASSaveSolutionAndUpdateSource on level 2: rhs += A x, saved x = x on INTERIOR cells ----
            __syncthreads();
            float ax[8];
            ax[0] = blk_nlap<0>(o, xs);
            ax[1] = blk_nlap<1>(o, xs);
            ax[2] = blk_nlap<2>(o, xs);
            ax[3] = blk_nlap<3>(o, xs);
            ax[4] = blk_nlap<4>(o, xs);
            ax[5] = blk_nlap<5>(o, xs);
            ax[6] = blk_nlap<6>(o, xs);
            ax[7] = blk_nlap<7>(o, xs);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const long long off = l2_off(A, Gi + (q >> 2), Gj + ((q >> 1) & 1), Gk + (q & 1));
                if ((o.in >> q) & 1u) {
                    o.b[q] = __fadd_rn(o.b[q], ax[q]);
                    X0[off] = o.x[q];
                } else {
                    o.b[q] = 0.0f;
                }
                RHS[off] = o.b[q];
            }
        }
        // every CTA has initialised its halos before any peer writes into them
        cluster.sync();

        // ---- level 2: pre-smoothing ----
        for (int it = 0; it < A.level_iters; ++it) {
            blk_gs_pass<true, kExact>(o, xs, yd, pr, 0, A);
            cluster.sync();
            blk_gs_pass<true, kExact>(o, xs, yd, pr, 1, A);
            cluster.sync();
        }
        // ---- residual, restriction into the coarse CTA's level-1 grid ----
        const int G1i = 8 * pr.oi + o.bi, G1j = 8 * pr.oj + o.bj, G1k = 8 * pr.ok + o.bk;
        const int ct = thread_of_blk(G1i >> 1, G1j >> 1, G1k >> 1);        // coarse thread of the parent root cell
        const int cq = ((G1i & 1) << 2) | ((G1j & 1) << 1) | (G1k & 1);     // cell within it
        {
            float b1, x1;
            blk_restrict(o, xs, (m >> 8) & 1u, A.Rr, b1, x1);
            cs.x[xo(G1i, G1j, G1k)] = x1;
            cs.b1[cq][ct] = b1;
        }
        cluster.sync();  // level-1 data delivered
        cluster.sync();  // coarse CTA done with levels 1 and 0
        // ---- FASProlongateAndUpdate on level 2 ----
        blk_prolong(o, A.P, cs.x[xo(G1i, G1j, G1k)], cs.s1[cq][ct]);
        blk_publish_all<true>(o, xs, pr);
        cluster.sync();
        // ---- level 2: post-smoothing ----
        for (int it = 0; it < A.level_iters; ++it) {
            blk_gs_pass<true, kExact>(o, xs, yd, pr, 1, A);
            cluster.sync();
            blk_gs_pass<true, kExact>(o, xs, yd, pr, 0, A);
            cluster.sync();
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) X[l2_off(A, Gi + (q >> 2), Gj + ((q >> 1) & 1), Gk + (q & 1))] = o.x[q];
    } else {
        // ============================ coarse CTA ============================
        pr.rx[0] = pr.rx[1] = pr.rx[2] = 0u;
        const bool in0 = (m >> 8) & 1u;
        const float d0 = pk.f[44][t], c0mx = pk.f[45][t], c0px = pk.f[46][t], c0my = pk.f[47][t], c0py = pk.f[48][t], c0mz = pk.f[49][t],
                    c0pz = pk.f[50][t];
        const int v0 = cell_index(o.bi, o.bj, o.bk);  // root cell of this thread
        float s0 = __ldcg(X0 + v0);                     // root saved x: INTERIOR cells are overwritten below
        const int q0 = ro(o.bi, o.bj, o.bk);
        float x0 = 0.0f, b0 = 0.0f;
        float s1[8];
        cluster.sync();  // halos initialised
        for (int it = 0; it < A.level_iters; ++it) {
            cluster.sync();
            cluster.sync();
        }
        cluster.sync();  // level-1 data delivered
        // ---- FASSaveSolutionAndUpdateSource on level 1 ----
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            o.x[q] = xs[q * kPar + (o.bi + 1) * 240 + (o.bj + 1) * 24 + (o.bk + 1)];
            o.b[q] = sm.b1[q][t];
        }
        {
            float ax[8];
            ax[0] = blk_nlap<0>(o, xs);
            ax[1] = blk_nlap<1>(o, xs);
            ax[2] = blk_nlap<2>(o, xs);
            ax[3] = blk_nlap<3>(o, xs);
            ax[4] = blk_nlap<4>(o, xs);
            ax[5] = blk_nlap<5>(o, xs);
            ax[6] = blk_nlap<6>(o, xs);
            ax[7] = blk_nlap<7>(o, xs);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const bool in = (o.in >> q) & 1u;
                o.b[q] = in ? __fadd_rn(o.b[q], ax[q]) : 0.0f;
                s1[q] = o.x[q];
            }
        }
        __syncthreads();  // the first sweep overwrites x that the update above reads
        for (int rep = 0; rep < A.mu; ++rep) {
            // ---- FASMuCycleStep of level 1 ----
            for (int it = 0; it < A.level_iters; ++it) {
                blk_gs_pass<false, kExact>(o, xs, yd, pr, 0, A);
                __syncthreads();
                blk_gs_pass<false, kExact>(o, xs, yd, pr, 1, A);
                __syncthreads();
            }
            {
                float rb, rx;
                blk_restrict(o, xs, in0, A.Rr, rb, rx);
                b0 = rb;
                x0 = rx;
                sm.x0[q0] = x0;
            }
            __syncthreads();
            // FASSaveSolutionAndUpdateSource on the root
            if (in0) {
                b0 = __fadd_rn(b0, nlap(d0, x0, c0mx, sm.x0[q0 - 240], c0px, sm.x0[q0 + 240], c0my, sm.x0[q0 - 24], c0py, sm.x0[q0 + 24],
                                        c0mz, sm.x0[q0 - 1], c0pz, sm.x0[q0 + 1]));
                s0 = x0;
            } else {
                b0 = 0.0f;
            }
            // mu coarsest solves: coarsest_iters/2 sweeps in order 0, then in order 1; or, in
            // the mixed-precision mode, one exact solve x0 = A0^-1 b0 in double (the later mu
            // visits of the same right-hand side would leave it unchanged)
            const int par = (o.bi + o.bj + o.bk) & 1;
            const double y0 = sm.yd[8][t];
            if (A.root_inv) {
                sm.b0[t] = b0;
                __syncthreads();
                if (in0) {
                    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
                    const double* M = A.root_inv + t;
                    for (int j = 0; j < kClThreads; j += 4) {
                        a0 = fma(__ldg(M + (size_t)j * kClThreads), (double)sm.b0[j], a0);
                        a1 = fma(__ldg(M + (size_t)(j + 1) * kClThreads), (double)sm.b0[j + 1], a1);
                        a2 = fma(__ldg(M + (size_t)(j + 2) * kClThreads), (double)sm.b0[j + 2], a2);
                        a3 = fma(__ldg(M + (size_t)(j + 3) * kClThreads), (double)sm.b0[j + 3], a3);
                    }
                    x0 = __double2float_rn((a0 + a1) + (a2 + a3));
                }
                sm.x0[q0] = x0;
            } else
            for (int rr = 0; rr < A.mu; ++rr)
                for (int half = 0; half < 2; ++half)
                    for (int it = 0; it < A.coarsest_iters / 2; ++it)
                        for (int h = 0; h < 2; ++h) {
                            __syncthreads();
                            if (par == (h ^ half)) {
                                const float ax = nlap(d0, x0, c0mx, sm.x0[q0 - 240], c0px, sm.x0[q0 + 240], c0my, sm.x0[q0 - 24], c0py,
                                                      sm.x0[q0 + 24], c0mz, sm.x0[q0 - 1], c0pz, sm.x0[q0 + 1]);
                                x0 = gs_update<kExact>(x0, b0, ax, d0, y0, in0, A);
                                sm.x0[q0] = x0;
                            }
                        }
            // FASProlongateAndUpdate on level 1 from the root
            blk_prolong(o, A.P, x0, s0);
            blk_publish_all<false>(o, xs, pr);
            __syncthreads();
            for (int it = 0; it < A.level_iters; ++it) {
                blk_gs_pass<false, kExact>(o, xs, yd, pr, 1, A);
                __syncthreads();
                blk_gs_pass<false, kExact>(o, xs, yd, pr, 0, A);
                __syncthreads();
            }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) sm.s1[q][t] = s1[q];
        cluster.sync();  // coarse CTA done: octant CTAs read x1 and s1
        cluster.sync();  // prolongation published
        for (int it = 0; it < A.level_iters; ++it) {
            cluster.sync();
            cluster.sync();
        }
        // ---- write back: level-1 x, rhs, saved x; root x, rhs, saved x ----
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const long long o1 = l1_off(A, 2 * o.bi + (q >> 2), 2 * o.bj + ((q >> 1) & 1), 2 * o.bk + (q & 1));
            X[o1] = o.x[q];
            RHS[o1] = o.b[q];
            if ((o.in >> q) & 1u) X0[o1] = s1[q];
        }
        if (A.mu > 0) {
            X[v0] = x0;
            RHS[v0] = b0;
            X0[v0] = s0;
        }
    }
}

}  // namespace

size_t cluster_pack_bytes() { return sizeof(ClPack) * kClCtas; }

static void fill_args(ClusterArgs& A, const int* tile1, const int* tile2, int coeff_ch, int mu, int level_iters, int coarsest_iters,
                      double omega, float Rr, float P, bool fas2, const double* root_inv = nullptr) {
    A.root_inv = root_inv;
    for (int i = 0; i < 8; ++i) A.tile1[i] = tile1[i];
    for (int i = 0; i < 64; ++i) A.tile2[i] = tile2[i];
    A.coeff_ch = coeff_ch;
    A.mu = mu;
    A.level_iters = level_iters;
    A.coarsest_iters = coarsest_iters;
    A.om = (float)omega;
    A.exact = relax_mode(omega);
    A.omega = omega;
    A.Rr = Rr;
    A.P = P;
    A.fas2 = fas2 ? 1 : 0;
}

void launch_cluster_pack(const DevGrid& g, const int* tile1, const int* tile2, int coeff_ch, void* pack, cudaStream_t st) {
    ClusterArgs A;
    fill_args(A, tile1, tile2, coeff_ch, 0, 0, 0, 1.0, 1.0f, 1.0f, false);
    note_kernel_launch();
    k_cluster_pack<<<kClCtas, kClThreads, 0, st>>>(g, A, reinterpret_cast<ClPack*>(pack));
}

int cluster_thread_cell(int t) {
    const int w = t >> 5, lane = t & 31;
    const int bk = lane & 7, bj = ((w & 3) << 1) | ((lane >> 3) & 1), bi = ((w >> 2) << 1) | (lane >> 4);
    return (bi << 6) | (bj << 3) | bk;
}

cudaError_t launch_cluster_step(const DevGrid& g, const int* tile1, const int* tile2, const void* pack, float* X, float* RHS, float* X0,
                                int coeff_ch, int mu, int level_iters, int coarsest_iters, double omega, float Rr, float P, bool fas2,
                                cudaStream_t st, const double* root_inv) {
    ClusterArgs A;
    fill_args(A, tile1, tile2, coeff_ch, mu, level_iters, coarsest_iters, omega, Rr, P, fas2, root_inv);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClCtas);
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = kClSmem;
    cfg.stream = st;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = kClCtas;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    note_kernel_launch();
    const ClPack* pk = reinterpret_cast<const ClPack*>(pack);
    if (A.exact == kRelaxRef) return cudaLaunchKernelEx(&cfg, k_cluster_step<kRelaxRef>, g, A, pk, X, RHS, X0);
    return cudaLaunchKernelEx(&cfg, k_cluster_step<kRelaxDouble>, g, A, pk, X, RHS, X0);
}

bool cluster_step_supported() {
    int dev = 0, cc = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&cc, cudaDevAttrClusterLaunch, dev) != cudaSuccess || !cc) return false;
    if (cudaFuncSetAttribute(k_cluster_step<kRelaxRef>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClSmem) != cudaSuccess ||
        cudaFuncSetAttribute(k_cluster_step<kRelaxRef>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
        cudaFuncSetAttribute(k_cluster_step<kRelaxDouble>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClSmem) != cudaSuccess ||
        cudaFuncSetAttribute(k_cluster_step<kRelaxDouble>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClCtas);
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = kClSmem;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = kClCtas;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_cluster_step<kRelaxRef>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return nclusters > 0;
}

}  // namespace cmg
