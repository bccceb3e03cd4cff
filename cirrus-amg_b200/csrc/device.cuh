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

// Load the snapshot of tile t (128 threads).  Returns the thread's raw x,
// cell types and diagonal for its four cells.  LoadAMGLaplacianTileData,
// src/AMGSolver.cu:419-543.  Latency: the neighbour descriptors are the only
// loads the halo values depend on, so the tile's own loads and the halo loads
// are all in flight before the first barrier; only the GHOST extrapolation,
// which needs the tile's own values, waits for it.
template <class Halo, class Sync>
__device__ __forceinline__ void load_snap(const DevGrid& g, int t, const float* X, int coeff_ch, const Halo& halo, Snap& S,
                                          const Quad& Q, float4& xr, uchar4& ty, float4& dg, const Sync& sync) {
    const float* C0 = g.plane(coeff_ch);
    const float* C1 = g.plane(coeff_ch + 1);
    const float* C2 = g.plane(coeff_ch + 2);
    const float* C3 = g.plane(coeff_ch + 3);
    // halo cell r of this thread: face f = hh / 64 (axis f/2, side f%2), cell (a, b) on the face
    int desc[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int f = (Q.q + 128 * r) >> 6;
        desc[r] = g.nbx[8 * t + (f >> 1) + 3 * (f & 1)];
    }
    xr = ldcg4(X + Q.base);
    ty = ldt4(g.ctype + Q.base);
    const float4 a0 = ld4(C0 + Q.base), a1 = ld4(C1 + Q.base), a2 = ld4(C2 + Q.base);
    dg = ld4(C3 + Q.base);
    const float h = voxel_size(g.h0, tile_level(g, t));
    float hv[3], hc[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int hh = Q.q + 128 * r;
        const int f = hh >> 6, fi = hh & 63;
        const int axis = f >> 1, s = f & 1;
        const int a = fi >> 3, b = fi & 7;
        int nlc[3];
        nlc[axis] = s ? 0 : 7;
        if (axis == 0) { nlc[1] = a; nlc[2] = b; }
        else if (axis == 1) { nlc[0] = a; nlc[2] = b; }
        else { nlc[0] = a; nlc[1] = b; }
        const int nl = cell_index(nlc[0], nlc[1], nlc[2]);
        hv[r] = 0.0f;
        hc[r] = h;
        if (desc[r] != 0) {
            const int qn = (desc[r] >> 3) - 1, ntype = desc[r] & 7;
            hv[r] = (ntype & dGhost) ? halo.ghost(g, qn, nl) : halo.active(g, qn, nl, ntype);
            if (s) hc[r] = g.plane(coeff_ch + axis)[(size_t)qn * kCells + nl];
        }
    }
    const int s0 = sx(Q.i, Q.j, Q.k0);
    S.x[s0 + 0] = ty.x == dInterior ? xr.x : 0.0f;
    S.x[s0 + 1] = ty.y == dInterior ? xr.y : 0.0f;
    S.x[s0 + 2] = ty.z == dInterior ? xr.z : 0.0f;
    S.x[s0 + 3] = ty.w == dInterior ? xr.w : 0.0f;
    *reinterpret_cast<float4*>(&S.c0[Q.i * 64 + Q.j * 8 + Q.k0]) = a0;
    *reinterpret_cast<float4*>(&S.c1[Q.i * 72 + Q.j * 8 + Q.k0]) = a1;
    const int c2o = Q.i * 72 + Q.j * 9 + Q.k0;
    S.c2[c2o + 0] = a2.x;
    S.c2[c2o + 1] = a2.y;
    S.c2[c2o + 2] = a2.z;
    S.c2[c2o + 3] = a2.w;
    sync();

#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int hh = Q.q + 128 * r;
        const int f = hh >> 6, fi = hh & 63;
        const int axis = f >> 1, s = f & 1;
        const int a = fi >> 3, b = fi & 7;
        const int axk = s ? 8 : -1;
        int fl[3], cl[3];
        if (axis == 0) { fl[0] = axk; fl[1] = a; fl[2] = b; }
        else if (axis == 1) { fl[0] = a; fl[1] = axk; fl[2] = b; }
        else { fl[0] = a; fl[1] = b; fl[2] = axk; }
        cl[0] = fl[0]; cl[1] = fl[1]; cl[2] = fl[2];
        cl[axis] = s ? 7 : 0;
        const int fx = sx(fl[0], fl[1], fl[2]);
        float v = hv[r];
        if (desc[r] != 0 && (desc[r] & dGhost)) {
            float avg = 0.0f;
#pragma unroll
            for (int di = 0; di < 2; ++di)
#pragma unroll
                for (int dj = 0; dj < 2; ++dj)
#pragma unroll
                    for (int dk = 0; dk < 2; ++dk) avg = __fadd_rn(avg, S.x[sx(cl[0] ^ di, cl[1] ^ dj, cl[2] ^ dk)]);
            avg = __fdiv_rn(avg, 8.0f);
            v = __fmaf_rn(0.5f, __fsub_rn(hv[r], avg), S.x[sx(cl[0], cl[1], cl[2])]);
        }
        S.x[fx] = v;
        if (s) {
            float* cslot = axis == 0 ? &S.c0[8 * 64 + a * 8 + b] : axis == 1 ? &S.c1[a * 72 + 64 + b] : &S.c2[a * 72 + b * 9 + 8];
            *cslot = hc[r];
        }
    }
    sync();
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
__device__ __forceinline__ float div_by_recip(float a, float d, double yd) {
    const float q = __double2float_rn(__dmul_rn((double)a, yd));
    const float m = fabsf(q);
    if (m >= 0x1p-125f && m <= 0x1p127f) return q;
    if (a == 0.0f && d != 0.0f) return q;
    return __fdiv_rn(a, d);
}

}  // namespace cmg
