// Device-side layout of the octree and the tile snapshot used by every
// stencil kernel.
//
// HBM layout: a channel is a plane of num_tiles * 512 floats; tile t's cells
// are the 2 KB block [t*512, t*512+512), cell index i*64 + j*8 + k
// (src/HAAccessor.h:32).  Cell types are one uint8 plane.  Per tile the device
// also holds meta = {level | type << 8, cx, cy, cz}, nb[8] = same-level
// neighbours (-x,-y,-z,+x,+y,+z), parent tile and -1, child[8] (dx*4+dy*2+dz).
// These tables replace the reference's per-voxel hash probes
// (HATileAccessor::findVoxel, src/HAAccessor.h:278).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cmg {

constexpr int kCells = 512;
enum : int { dLeaf = 1, dNonLeaf = 2, dGhost = 4 };
enum : int { dDirichlet = 1, dInterior = 2, dNeumann = 4 };

struct DevGrid {
    int n;
    int nch;
    float h0;
    float* chan;
    uint8_t* ctype;
    const int4* meta;
    const int* nb;
    const int* child;
    const int* nbx;  // [n][8]: face neighbours packed as (tile + 1) << 3 | tile type, 0 = none
    __host__ __device__ float* plane(int c) const { return chan + (size_t)c * (size_t)n * kCells; }
};

__device__ __forceinline__ int tile_level(const DevGrid& g, int t) { return g.meta[t].x & 0xff; }
__device__ __forceinline__ int tile_type(const DevGrid& g, int t) { return (g.meta[t].x >> 8) & 0xff; }
// HACoordAccessor::voxelSize (src/HAAccessor.h:75): h0 / 2^level in float
__device__ __forceinline__ float voxel_size(float h0, int level) { return h0 / (float)(1 << level); }

// local cell of the parent tile holding the parent of local cell l (per axis)
__device__ __forceinline__ int parent_local(int tile_coord, int l) { return ((tile_coord & 1) << 2) | (l >> 1); }
__device__ __forceinline__ int cell_index(int i, int j, int k) { return (i << 6) | (j << 3) | k; }

// Tile snapshot with a one-cell halo (the role of AMGLaplacianTileData,
// src/AMGSolver.cu:320-406).  x: 10^3 values, index (i+1)*100+(j+1)*10+(k+1).
// c0/c1/c2: negative-face coefficient of each cell; slot 8 along the axis
// holds the positive face of cell 7 taken from the neighbour tile.
struct __align__(16) Snap {  // 16-byte aligned: c0/c1 rows are written as float4
    float x[1000];
    float c0[576];  // [i 0..8][j][k] -> i*64 + j*8 + k
    float c1[576];  // [i][j 0..8][k] -> i*72 + j*8 + k
    float c2[576];  // [i][j][k 0..8] -> i*72 + j*9 + k
};
__device__ __forceinline__ int sx(int i, int j, int k) { return (i + 1) * 100 + (j + 1) * 10 + (k + 1); }

// AMGLaplacianTileData::negativeLap (src/AMGSolver.cu:346-382): diag*x plus
// the six off-diagonal terms in the order -x,+x,-y,+y,-z,+z, fused multiply-adds.
__device__ __forceinline__ float snap_neg_lap(const Snap& S, int i, int j, int k, float d) {
    if (d == 0.0f) return 0.0f;
    const int c = sx(i, j, k);
    float s = S.x[c] * d;
    s = __fmaf_rn(S.c0[i * 64 + j * 8 + k], S.x[c - 100], s);
    s = __fmaf_rn(S.c0[(i + 1) * 64 + j * 8 + k], S.x[c + 100], s);
    s = __fmaf_rn(S.c1[i * 72 + j * 8 + k], S.x[c - 10], s);
    s = __fmaf_rn(S.c1[i * 72 + (j + 1) * 8 + k], S.x[c + 10], s);
    s = __fmaf_rn(S.c2[i * 72 + j * 9 + k], S.x[c - 1], s);
    s = __fmaf_rn(S.c2[i * 72 + j * 9 + k + 1], S.x[c + 1], s);
    return s;
}

// Per-thread view of the four consecutive cells (along k) a thread of a
// 128-thread tile block owns: cells 4q .. 4q+3.
struct Quad {
    int q, i, j, k0;
    size_t base;  // t*512 + 4q
    __device__ __forceinline__ Quad(int t, int tid) {
        q = tid;
        i = q >> 4;
        j = (q >> 1) & 7;
        k0 = (q & 1) << 2;
        base = (size_t)t * kCells + 4 * q;
    }
};

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
// loads of fields other blocks of the same kernel may have written (the
// persistent multi-level kernel): straight from L2, never a stale L1 line
__device__ __forceinline__ float4 ldcg4(const float* p) { return __ldcg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ uchar4 ldt4(const uint8_t* p) { return *reinterpret_cast<const uchar4*>(p); }
__device__ __forceinline__ float f4get(const float4& v, int u) { return u == 0 ? v.x : u == 1 ? v.y : u == 2 ? v.z : v.w; }
__device__ __forceinline__ void f4set(float4& v, int u, float x) {
    if (u == 0) v.x = x; else if (u == 1) v.y = x; else if (u == 2) v.z = x; else v.w = x;
}
__device__ __forceinline__ int t4get(const uchar4& v, int u) { return u == 0 ? v.x : u == 1 ? v.y : u == 2 ? v.z : v.w; }

// Halo value rules.
// MgHalo: the multigrid kernels read the neighbour's channel directly; a
// LEAF/NONLEAF neighbour contributes only INTERIOR cells, a GHOST neighbour
// its raw value (LoadAMGLaplacianTileData, src/AMGSolver.cu:489-541).
struct MgHalo {
    const float* X;
    const uint8_t* ct;
    __device__ __forceinline__ float active(const DevGrid&, int qn, int nl, int) const {
        const size_t o = (size_t)qn * kCells + nl;
        const float v = ldcg(X + o);
        return ct[o] == dInterior ? v : 0.0f;
    }
    __device__ __forceinline__ float ghost(const DevGrid&, int qn, int nl) const { return ldcg(X + (size_t)qn * kCells + nl); }
};
// LeafHalo: A*p on LEAF tiles.  The reference first writes GHOST cells from
// their LEAF parents (PropagateToChildren, src/PoissonGrid.cu:377) and NONLEAF
// cells as 1/8 of their LEAF children (AccumulateToParentsOneStep,
// src/PoissonGrid.cu:408); here the halo computes those values on the fly.
struct LeafHalo {
    const float* X;
    const uint8_t* ct;
    __device__ __forceinline__ float active(const DevGrid& g, int qn, int nl, int ntype) const {
        const size_t o = (size_t)qn * kCells + nl;
        if (ntype & dLeaf) return ct[o] == dInterior ? ldcg(X + o) : 0.0f;
        if (ct[o] != dInterior) return 0.0f;
        const int l0 = nl >> 6, l1 = (nl >> 3) & 7, l2 = nl & 7;
        const int c = g.child[8 * qn + (l0 >> 2) * 4 + (l1 >> 2) * 2 + (l2 >> 2)];
        if (c < 0) return 0.0f;
        const float* Xc = X + (size_t)c * kCells;
        const int b0 = (l0 & 3) << 1, b1 = (l1 & 3) << 1, b2 = (l2 & 3) << 1;
        float s = 0.0f;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) s = __fadd_rn(s, ldcg(Xc + cell_index(b0 + ii, b1 + jj, b2 + kk)));
        return __fmul_rn(s, 0.125f);
    }
    __device__ __forceinline__ float ghost(const DevGrid& g, int qn, int nl) const {
        const int p = g.nb[8 * qn + 6];
        if (p < 0) return 0.0f;
        const int4 m = g.meta[qn];
        const int pv = cell_index(parent_local(m.y, nl >> 6), parent_local(m.z, (nl >> 3) & 7), parent_local(m.w, nl & 7));
        return ldcg(X + (size_t)p * kCells + pv);
    }
};

// Barrier scopes of the tile code: the whole block (one tile per block) or
// one 128-thread slot of a block that works on several tiles at once.
struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct SlotSync {
    int id;  // named barrier 1..15
    __device__ __forceinline__ void operator()() const { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
};

// What a thread of a 128-thread tile block holds for its four cells after the
// snapshot load: raw x, x masked to INTERIOR cells (as the snapshot holds it),
// cell types, diagonal, and the negative-face coefficients c0, c1, c2.
struct Own {
    float4 xr, xm, dg, a0, a1, a2;
    uchar4 ty;
};

// Load the snapshot of tile t (128 threads).  LoadAMGLaplacianTileData,
// src/AMGSolver.cu:419-543.  Latency: the neighbour descriptors are the only
// loads the halo values depend on, so the tile's own loads and the halo loads
// are all in flight before the first barrier; only the GHOST extrapolation,
// which needs the tile's own values, waits for it.
// Halo cells: thread q handles, for r = 0, 1, 2, cell q & 63 of the face of
// axis r on side q >> 6 (the 384 halo cells of the six faces).
template <class Halo, class Sync>
__device__ __forceinline__ void load_snap(const DevGrid& g, int t, const float* X, int coeff_ch, const Halo& halo, Snap& S,
                                          const Quad& Q, Own& o, const Sync& sync) {
    const float* C0 = g.plane(coeff_ch);
    const float* C1 = g.plane(coeff_ch + 1);
    const float* C2 = g.plane(coeff_ch + 2);
    const float* C3 = g.plane(coeff_ch + 3);
    const int side = Q.q >> 6, fa = (Q.q >> 3) & 7, fb = Q.q & 7;
    int desc[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) desc[r] = g.nbx[8 * t + r + 3 * side];
    o.xr = ldcg4(X + Q.base);
    o.ty = ldt4(g.ctype + Q.base);
    o.a0 = ld4(C0 + Q.base);
    o.a1 = ld4(C1 + Q.base);
    o.a2 = ld4(C2 + Q.base);
    o.dg = ld4(C3 + Q.base);
    const float h = voxel_size(g.h0, tile_level(g, t));
    // the neighbour's cell across face (r, side) at face position (fa, fb)
    const int nl0 = cell_index(side ? 0 : 7, fa, fb), nl1 = cell_index(fa, side ? 0 : 7, fb), nl2 = cell_index(fa, fb, side ? 0 : 7);
    float hv[3], hc[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int nl = r == 0 ? nl0 : r == 1 ? nl1 : nl2;
        hv[r] = 0.0f;
        hc[r] = h;
        if (desc[r] != 0) {
            const int qn = (desc[r] >> 3) - 1, ntype = desc[r] & 7;
            hv[r] = (ntype & dGhost) ? halo.ghost(g, qn, nl) : halo.active(g, qn, nl, ntype);
            if (side) hc[r] = g.plane(coeff_ch + r)[(size_t)qn * kCells + nl];
        }
    }
    o.xm.x = o.ty.x == dInterior ? o.xr.x : 0.0f;
    o.xm.y = o.ty.y == dInterior ? o.xr.y : 0.0f;
    o.xm.z = o.ty.z == dInterior ? o.xr.z : 0.0f;
    o.xm.w = o.ty.w == dInterior ? o.xr.w : 0.0f;
    const int s0 = sx(Q.i, Q.j, Q.k0);
    S.x[s0 + 0] = o.xm.x;
    S.x[s0 + 1] = o.xm.y;
    S.x[s0 + 2] = o.xm.z;
    S.x[s0 + 3] = o.xm.w;
    *reinterpret_cast<float4*>(&S.c0[Q.i * 64 + Q.j * 8 + Q.k0]) = o.a0;
    *reinterpret_cast<float4*>(&S.c1[Q.i * 72 + Q.j * 8 + Q.k0]) = o.a1;
    const int c2o = Q.i * 72 + Q.j * 9 + Q.k0;
    S.c2[c2o + 0] = o.a2.x;
    S.c2[c2o + 1] = o.a2.y;
    S.c2[c2o + 2] = o.a2.z;
    S.c2[c2o + 3] = o.a2.w;
    sync();

    const int e = side ? 7 : 0;     // own boundary layer next to the face
    const int hx = side ? 8 : -1;   // halo layer
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        int cl[3];
        cl[0] = r == 0 ? e : fa;
        cl[1] = r == 0 ? fa : r == 1 ? e : fb;
        cl[2] = r == 2 ? e : fb;
        const int fx = r == 0 ? sx(hx, fa, fb) : r == 1 ? sx(fa, hx, fb) : sx(fa, fb, hx);
        float v = hv[r];
        if (desc[r] != 0 && (desc[r] & dGhost)) {
            // T-junction: x_in + 0.5 * (x_ghost - mean of the 2x2x2 block of own cells at the face)
            float avg = 0.0f;
#pragma unroll
            for (int di = 0; di < 2; ++di)
#pragma unroll
                for (int dj = 0; dj < 2; ++dj)
#pragma unroll
                    for (int dk = 0; dk < 2; ++dk) avg = __fadd_rn(avg, S.x[sx(cl[0] ^ di, cl[1] ^ dj, cl[2] ^ dk)]);
            avg = __fmul_rn(avg, 0.125f);  // equals avg / 8 (scaling by a power of two)
            v = __fmaf_rn(0.5f, __fsub_rn(hv[r], avg), S.x[sx(cl[0], cl[1], cl[2])]);
        }
        S.x[fx] = v;
        if (side) {
            float* cslot = r == 0 ? &S.c0[8 * 64 + fa * 8 + fb] : r == 1 ? &S.c1[fa * 72 + 64 + fb] : &S.c2[fa * 72 + fb * 9 + 8];
            *cslot = hc[r];
        }
    }
    sync();
}

// negativeLap of own cell u (0..3) of the thread: the snapshot's stencil with the
// thread's own x and negative-face coefficients taken from registers; same
// operands in the same order as snap_neg_lap.
template <int U>
__device__ __forceinline__ float own_neg_lap(const Snap& S, const Quad& Q, const Own& o) {
    const float d = f4get(o.dg, U);
    if (d == 0.0f) return 0.0f;
    const int k = Q.k0 + U;
    const int c = sx(Q.i, Q.j, k);
    float s = __fmul_rn(f4get(o.xm, U), d);
    s = __fmaf_rn(f4get(o.a0, U), S.x[c - 100], s);
    s = __fmaf_rn(S.c0[(Q.i + 1) * 64 + Q.j * 8 + k], S.x[c + 100], s);
    s = __fmaf_rn(f4get(o.a1, U), S.x[c - 10], s);
    s = __fmaf_rn(S.c1[Q.i * 72 + (Q.j + 1) * 8 + k], S.x[c + 10], s);
    s = __fmaf_rn(f4get(o.a2, U), U > 0 ? f4get(o.xm, U - 1) : S.x[c - 1], s);
    s = __fmaf_rn(U < 3 ? f4get(o.a2, U + 1) : S.c2[Q.i * 72 + Q.j * 9 + k + 1], U < 3 ? f4get(o.xm, U + 1) : S.x[c + 1], s);
    return s;
}
// the same stencil accumulated in double (the FP64 true residual of residual replacement)
template <int U>
__device__ __forceinline__ double own_neg_lap64(const Snap& S, const Quad& Q, const Own& o) {
    const float d = f4get(o.dg, U);
    if (d == 0.0f) return 0.0;
    const int k = Q.k0 + U;
    const int c = sx(Q.i, Q.j, k);
    double s = (double)f4get(o.xm, U) * (double)d;
    s = fma((double)f4get(o.a0, U), (double)S.x[c - 100], s);
    s = fma((double)S.c0[(Q.i + 1) * 64 + Q.j * 8 + k], (double)S.x[c + 100], s);
    s = fma((double)f4get(o.a1, U), (double)S.x[c - 10], s);
    s = fma((double)S.c1[Q.i * 72 + (Q.j + 1) * 8 + k], (double)S.x[c + 10], s);
    s = fma((double)f4get(o.a2, U), (double)(U > 0 ? f4get(o.xm, U - 1) : S.x[c - 1]), s);
    s = fma((double)(U < 3 ? f4get(o.a2, U + 1) : S.c2[Q.i * 72 + Q.j * 9 + k + 1]), (double)(U < 3 ? f4get(o.xm, U + 1) : S.x[c + 1]), s);
    return s;
}
__device__ __forceinline__ float own_neg_lap(const Snap& S, const Quad& Q, const Own& o, int u) {
    return u == 0 ? own_neg_lap<0>(S, Q, o) : u == 1 ? own_neg_lap<1>(S, Q, o) : u == 2 ? own_neg_lap<2>(S, Q, o) : own_neg_lap<3>(S, Q, o);
}

// Block-wide deterministic double reduction for 128 threads; result valid in thread 0.
__device__ __forceinline__ double block_sum128(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[w] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x == 0) r = (red[0] + red[1]) + (red[2] + red[3]);
    __syncthreads();
    return r;
}

// a / d rounded to the nearest float -- bit-identical to IEEE division -- given
// yd = 1/d rounded to the nearest double (1.0 / (double)d), for a divisor that is
// reused many times.  q = RN_double(a * yd) differs from a/d by less than 2^-51.9
// relative (two double roundings).  A quotient of two 24-bit floats is never a
// midpoint of adjacent normal floats and stays more than 2^-49 (relative) away
// from every midpoint: writing the midpoint as M*2^m (M odd, 25 bits), d = D*2^e,
// a - d*M*2^m is a nonzero multiple of 2^(e+m), so |a/d - M*2^m| >= 2^m / D.
// Hence q and a/d round to the same float.  This is the argument behind the
// double-rounding bound for division (S. A. Figueroa, "When is double rounding
// innocuous?", ACM SIGNUM Newsletter 30(3), 1995), applied to the product with a
// correctly rounded reciprocal.  Zero, subnormal, huge and non-finite cases take
// the IEEE division itself.
// The argument holds for any yd within 2^-52 (relative) of 1/d, not only for the
// correctly rounded one.
__device__ __forceinline__ float div_by_recip(float a, float d, double yd) {
    const float q = __double2float_rn(__dmul_rn((double)a, yd));
    const float m = fabsf(q);
    if (m >= 0x1p-125f && m <= 0x1p127f) return q;
    // 0 / d for nonzero, non-NaN d: zero with the sign of a * d
    if (a == 0.0f && d != 0.0f && !isnan(d)) return __int_as_float((__float_as_int(a) ^ __float_as_int(d)) & 0x80000000);
    return __fdiv_rn(a, d);
}
// 1/d in double within 2^-52 (relative) for normal d: the single-precision
// hardware reciprocal (relative error below 2^-22) refined by two Newton-Raphson
// steps y <- y + y*(1 - d*y) in double (the error squares at each step, then one
// double rounding remains).  Zero, subnormal, infinite and huge d give inf, NaN or
// 0 here, which div_by_recip sends to the IEEE division.
__device__ __forceinline__ double recip_f64(float d) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
    const double dd = (double)d;
    double y = (double)r;
    y = __fma_rn(y, __fma_rn(-dd, y, 1.0), y);
    y = __fma_rn(y, __fma_rn(-dd, y, 1.0), y);
    return y;
}
// a / d, bit-identical to the IEEE division, without the long latency of the
// division routine on the dependent chain of a Gauss-Seidel update
__device__ __forceinline__ float div_exact(float a, float d) { return div_by_recip(a, d, recip_f64(d)); }

// The Gauss-Seidel relaxation x + delta * omega as the reference evaluates it
// (src/AMGSolver.cu:874): delta and x are floats, omega a float held in a double, so the
// product is exact in double, the sum is rounded once to double and then once to float.
// A single-precision fused multiply-add rounds once to float and can differ from that in
// the last bit (a sum within half a double ulp of a float midpoint), so it is not used.
__device__ __forceinline__ float relax_ref(float xs, float delta, float om) {
    return __double2float_rn(__fma_rn((double)delta, (double)om, (double)xs));
}

// how a smoother applies omega: a float (relax_ref, as the reference's AMGSolver::omega
// always is), or not a float (x + delta * omega in double, the product rounded too)
enum : int { kRelaxDouble = 0, kRelaxRef = 1 };
inline int relax_mode(double omega) { return (double)(float)omega == omega ? kRelaxRef : kRelaxDouble; }
template <int M>
__device__ __forceinline__ float relax(float xs, float delta, float om, double omega) {
    if constexpr (M == kRelaxRef) return relax_ref(xs, delta, om);
    else return (float)((double)xs + (double)delta * omega);
}
__device__ __forceinline__ float relax_rt(int mode, float xs, float delta, float om, double omega) {
    return mode == kRelaxRef ? relax_ref(xs, delta, om) : (float)((double)xs + (double)delta * omega);
}

}  // namespace cmg
