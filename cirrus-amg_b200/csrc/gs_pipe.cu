// Red-black Gauss-Seidel colour pass on the LEAF and NONLEAF tiles of one level
// (NegativeLaplacianAndGaussSeidelSameLevelAMG128Kernel, src/AMGSolver.cu:838-877),
// as a persistent, software-pipelined kernel for the multigrid cycle.
//
// k_gs spends most of a tile's life waiting: the neighbour descriptors arrive, then
// the halo loads go out, then the block computes.  Here each 128-thread block walks a
// strided list of tiles and keeps the next tile's planes and halo in flight (into a
// second shared-memory stage) while it computes the current one.  A tile's own data are
// seven contiguous blocks (x, rhs, the four operator planes, the cell types: 2 KB, or
// 1 KB for a 16-bit plane, and 512 B): one thread moves them with 1-D bulk copies
// (cp.async.bulk, the TMA engine) that complete on the stage's mbarrier; the halo words
// are scattered and keep per-thread cp.async.  No register holds data in flight.  The
// mbarrier waits are bounded: a wait that gives up sets an error flag that the solve
// reports, and the block stops.
//
// Halo values are read without the neighbour's cell types.  That relies on the
// multigrid x plane holding 0 on every cell that is not INTERIOR, which the cycle keeps
// true (x starts at 0; restriction, prolongation and the sweeps write masked values),
// and on GHOST neighbours being read raw, as the reference does.  The public
// cmg_amg_gauss_seidel, which takes arbitrary x, keeps using k_gs.
//
// The operator planes (diagonal and the three face coefficients) are read either as
// float (the reference's arithmetic) or, in the mixed-precision mode, from BF16 or FP16
// copies made once per solve: 8 of the 27 bytes a cell costs per pass.  Every value is
// widened to float on load and all arithmetic stays FP32, so a 16-bit run equals a
// float run on coefficients rounded to 16 bits beforehand, bit for bit.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstddef>
#include <type_traits>
#include <utility>

#include "kernels.hpp"

namespace cmg {

namespace {

template <typename CT, typename XT = float>
struct alignas(16) PipeStage {
    XT x[512], b[512];
    CT d[512];        // diagonal
    CT c0[512];       // -x faces
    CT c1[512];       // -y faces
    CT c2[512];       // -z faces
    // faces taken from the neighbours: +x faces of row i = 7 [j][k], +y faces of row j = 7
    // [i][k], +z faces of row k = 7 [i][j]; a word holds the float, or for 16-bit storage
    // the 4-byte-aligned pair of plane elements that contains the face
    unsigned c0h[64], c1h[64], c2h[64];
    unsigned hx[384];  // halo x of the six faces, [axis][side][a][b]: the float, or the BF16 pair
    unsigned ty[128];
};
// bulk-copy destinations: 16-byte aligned offsets
template <typename CT, typename XT>
constexpr bool stage_aligned() {
    using S = PipeStage<CT, XT>;
    return offsetof(S, b) % 16 == 0 && offsetof(S, d) % 16 == 0 && offsetof(S, c0) % 16 == 0 && offsetof(S, c1) % 16 == 0 &&
           offsetof(S, c2) % 16 == 0 && offsetof(S, ty) % 16 == 0 && sizeof(S) % 16 == 0;
}
static_assert(stage_aligned<float, float>() && stage_aligned<__nv_bfloat16, float>() && stage_aligned<__half, float>() &&
                  stage_aligned<float, __nv_bfloat16>() && stage_aligned<__nv_bfloat16, __nv_bfloat16>() &&
                  stage_aligned<__half, __nv_bfloat16>(),
              "stage layout");
// The snapshot: masked x of the tile with its one-cell halo, split into four planes by
// k mod 4 (k = 4h + u: u the plane, h = -1..2 the slot), rows j of 4 slots, layers i of
// 42 floats, planes of 448 floats.  A warp's threads own (i0..i0+1, j 0..7, h 0..1) and
// touch one plane per lane at a time: the offsets 4j + h and 42 + 4j + h fill the 32
// banks once each, and the plane stride is a multiple of 32, so the stores of its own
// cells and the i/j neighbour loads of a colour pass are free of bank conflicts.
constexpr int kSxI = 42, kSxJ = 4, kSxP = 448;
__device__ __forceinline__ int sxp(int i, int j, int k) { return ((k + 4) & 3) * kSxP + (i + 1) * kSxI + (j + 1) * kSxJ + ((k + 4) >> 2); }

template <typename CT, typename XT>
struct PipeSmem {
    PipeStage<CT, XT> st[2];
    float x[4 * kSxP];
};
// the restriction pass also keeps the tile's residuals (operator in float)
template <typename XT>
struct PipeSmemR {
    PipeStage<float, XT> st[2];
    float x[4 * kSxP];
    float res[512];
};

__device__ __forceinline__ void cp4(void* dst, const void* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// 1-D bulk copies onto an mbarrier (both addresses 16-byte aligned, sizes multiples of 16)
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned mb) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned mb, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned mb) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(mb) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned mb, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(ok) : "r"(mb), "r"(parity) : "memory");
    return ok != 0;
}
// bounded wait for phase `parity` of an mbarrier (each try_wait suspends for a while)
constexpr int kMbarTries = 1 << 20;
__device__ __forceinline__ bool mbar_wait(unsigned mb, unsigned parity) {
    for (int i = 0; i < kMbarTries; ++i)
        if (mbar_try(mb, parity)) return true;
    return false;
}
__device__ int g_pipe_error;  // set when a stage's bulk copies did not arrive in time
__device__ __forceinline__ void cp_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Storage of the operator planes: copies into a stage and widening to float.
template <typename CT>
struct Coef;
template <>
struct Coef<float> {
    __device__ static void cp_face(unsigned* dst, const float* plane, size_t o) { cp4(dst, plane + o); }
    __device__ static unsigned word(float v) { return __float_as_uint(v); }
    __device__ static float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
    __device__ static float at(const float* p) { return *p; }
    __device__ static float face(unsigned w, int) { return __uint_as_float(w); }
};
// 16-bit storage: 4 elements move as 8 bytes; a face element moves inside its aligned pair
template <typename CT>
struct Coef16 {
    __device__ static void cp_face(unsigned* dst, const CT* plane, size_t o) { cp4(dst, plane + (o & ~(size_t)1)); }
    __device__ static float4 ld4(const CT* p) {
        const uint2 w = *reinterpret_cast<const uint2*>(p);
        return make_float4(Coef<CT>::wide(w.x & 0xffffu), Coef<CT>::wide(w.x >> 16), Coef<CT>::wide(w.y & 0xffffu), Coef<CT>::wide(w.y >> 16));
    }
    __device__ static float at(const CT* p) { return Coef<CT>::wide(*reinterpret_cast<const unsigned short*>(p)); }
    __device__ static float face(unsigned w, int odd) { return Coef<CT>::wide(odd ? w >> 16 : w & 0xffffu); }
};
template <>
struct Coef<__nv_bfloat16> : Coef16<__nv_bfloat16> {
    __device__ static float wide(unsigned bits) { return __uint_as_float(bits << 16); }
    __device__ static unsigned word(float v) {
        const unsigned b = __bfloat16_as_ushort(__float2bfloat16_rn(v));
        return b | (b << 16);
    }
};
template <>
struct Coef<__half> : Coef16<__half> {
    __device__ static float wide(unsigned bits) { return __half2float(__ushort_as_half((unsigned short)bits)); }
    __device__ static unsigned word(float v) {
        const unsigned b = __half_as_ushort(__float2half_rn(v));
        return b | (b << 16);
    }
};

// Storage of x and rhs (the mixed-precision cycle keeps them in BF16 on levels >= 3).
template <typename XT>
struct XStore;
template <>
struct XStore<float> {
    __device__ static void cp_halo(unsigned* dst, const float* X, size_t o) { cp4(dst, X + o); }
    __device__ static float halo(unsigned w, int) { return __uint_as_float(w); }
    __device__ static float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
    __device__ static void st4g(float* p, float4 v) { st4(p, v); }
    __device__ static void st1(float* p, float v) { *p = v; }
};
template <>
struct XStore<__nv_bfloat16> {
    // a halo element moves inside its 4-byte-aligned pair
    __device__ static void cp_halo(unsigned* dst, const __nv_bfloat16* X, size_t o) { cp4(dst, X + (o & ~(size_t)1)); }
    __device__ static float wide(unsigned bits) { return __uint_as_float(bits << 16); }
    __device__ static float halo(unsigned w, int odd) { return wide(odd ? w >> 16 : w & 0xffffu); }
    __device__ static float4 ld4(const __nv_bfloat16* p) {
        const uint2 w = *reinterpret_cast<const uint2*>(p);
        return make_float4(wide(w.x & 0xffffu), wide(w.x >> 16), wide(w.y & 0xffffu), wide(w.y >> 16));
    }
    __device__ static unsigned bits(float v) { return (unsigned)__bfloat16_as_ushort(__float2bfloat16_rn(v)); }
    __device__ static void st4g(__nv_bfloat16* p, float4 v) {
        *reinterpret_cast<uint2*>(p) = make_uint2(bits(v.x) | (bits(v.y) << 16), bits(v.z) | (bits(v.w) << 16));
    }
    __device__ static void st1(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
};

struct PipeArgs {
    int t0, nt, color, exact;  // exact: the relaxation mode (kRelax*)
    float om;
    double omega;
    const void* coef;  // first of the four operator planes (-x, -y, -z faces, diagonal)
    size_t cstride;    // elements from one operator plane to the next
    void* xp;          // restriction pass: the x plane of the parent tiles
    void* rhsp;        // restriction pass: the rhs plane of the parent tiles; FAS pass: the tiles' own rhs
    void* x0p;         // FAS pass: the saved-x plane
    float Rr;          // restriction pass: R_restrict
};

// neighbour descriptors of the thread's three halo cells: face r on side q >> 6
__device__ __forceinline__ void load_desc(const DevGrid& g, int t, int side, int d[3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r) d[r] = __ldg(g.nbx + 8 * t + r + 3 * side);
}

// start the copies of tile t into stage S (mbarrier mb takes the bulk part), in two halves:
// issue_static moves what no kernel of a solve writes (the operator planes, the cell types,
// the neighbours' face coefficients), issue_dynamic x, rhs and the halo x
template <typename CT, typename XT>
__device__ __forceinline__ void issue_static(PipeStage<CT, XT>& S, unsigned mb, const DevGrid& g, int t, const CT* C0, const CT* C1,
                                             const CT* C2, const CT* C3, const int d[3], int q, float h) {
    const size_t tb = (size_t)t * kCells;
    if (q == 0) {
        constexpr unsigned kX = kCells * sizeof(XT), kC = kCells * sizeof(CT), kT = kCells;
        // the stage was last read through ordinary loads; order them before the async writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect(mb, 2 * kX + 4 * kC + kT);
        bulk_g2s(S.d, C3 + tb, kC, mb);
        bulk_g2s(S.c0, C0 + tb, kC, mb);
        bulk_g2s(S.c1, C1 + tb, kC, mb);
        bulk_g2s(S.c2, C2 + tb, kC, mb);
        bulk_g2s(S.ty, g.ctype + tb, kT, mb);
    }
    const int side = q >> 6, fa = (q >> 3) & 7, fb = q & 7;
    if (!side) return;
    const int nl[3] = {cell_index(0, fa, fb), cell_index(fa, 0, fb), cell_index(fa, fb, 0)};
    unsigned* hc[3] = {&S.c0h[fa * 8 + fb], &S.c1h[fa * 8 + fb], &S.c2h[fa * 8 + fb]};
    const CT* Cr[3] = {C0, C1, C2};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        if (d[r] != 0) Coef<CT>::cp_face(hc[r], Cr[r], (size_t)((d[r] >> 3) - 1) * kCells + nl[r]);
        else *hc[r] = Coef<CT>::word(h);
    }
}
template <typename CT, typename XT>
__device__ __forceinline__ void issue_dynamic(PipeStage<CT, XT>& S, unsigned mb, int t, const XT* X, const XT* B, const int d[3], int q) {
    const size_t tb = (size_t)t * kCells;
    if (q == 0) {
        constexpr unsigned kX = kCells * sizeof(XT);
        bulk_g2s(S.x, X + tb, kX, mb);
        bulk_g2s(S.b, B + tb, kX, mb);
    }
    const int side = q >> 6, fa = (q >> 3) & 7, fb = q & 7;
    const int e = side ? 0 : 7;  // the neighbour's cell next to the shared face
    const int nl[3] = {cell_index(e, fa, fb), cell_index(fa, e, fb), cell_index(fa, fb, e)};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        unsigned* hxd = &S.hx[r * 128 + q];
        if (d[r] != 0) XStore<XT>::cp_halo(hxd, X, (size_t)((d[r] >> 3) - 1) * kCells + nl[r]);
        else *hxd = 0u;
    }
    cp_commit();
}
template <typename CT, typename XT>
__device__ __forceinline__ void issue(PipeStage<CT, XT>& S, unsigned mb, const DevGrid& g, int t, const XT* X, const XT* B,
                                      const CT* C0, const CT* C1, const CT* C2, const CT* C3, const int d[3], int q, float h) {
    issue_static(S, mb, g, t, C0, C1, C2, C3, d, q, h);
    issue_dynamic(S, mb, t, X, B, d, q);
}

// The masked snapshot of the staged tile in SX: own cells (x is 0 on cells that are not
// INTERIOR) and the one-cell halo, GHOST faces by the T-junction rule.  Returns the
// thread's masked quad and the plane-0 offset s0 of its first cell.
template <typename CT, typename XT>
__device__ __forceinline__ void build_snapshot(const PipeStage<CT, XT>& S, float* SX, const int d[3], int q, const Quad& Q, float4& xm,
                                               int& s0) {
    const float4 xr = XStore<XT>::ld4(&S.x[4 * q]);
    const unsigned tyw = S.ty[q];
    xm.x = (tyw & 0xffu) == dInterior ? xr.x : 0.0f;
    xm.y = ((tyw >> 8) & 0xffu) == dInterior ? xr.y : 0.0f;
    xm.z = ((tyw >> 16) & 0xffu) == dInterior ? xr.z : 0.0f;
    xm.w = ((tyw >> 24) & 0xffu) == dInterior ? xr.w : 0.0f;
    // own cells (i, j, k0 + u): plane u, slot h + 1
    s0 = (Q.i + 1) * kSxI + (Q.j + 1) * kSxJ + (Q.k0 >> 2) + 1;
    SX[s0] = xm.x;
    SX[s0 + kSxP] = xm.y;
    SX[s0 + 2 * kSxP] = xm.z;
    SX[s0 + 3 * kSxP] = xm.w;
    const int side = q >> 6, fa = (q >> 3) & 7, fb = q & 7;
    const int e = side ? 7 : 0, hxl = side ? 8 : -1;
    const int fx[3] = {sxp(hxl, fa, fb), sxp(fa, hxl, fb), sxp(fa, fb, hxl)};
    // the halo cell's position in its 4-byte pair (16-bit storage): the parity of its last index
    const int odd[3] = {fb & 1, fb & 1, side ? 0 : 1};
    float hxv[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) hxv[r] = XStore<XT>::halo(S.hx[r * 128 + q], odd[r]);
#pragma unroll
    for (int r = 0; r < 3; ++r)
        if (!(d[r] & dGhost)) SX[fx[r]] = hxv[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        if (d[r] & dGhost) {
            // T-junction: x_in + 0.5 * (x_ghost - mean of the 2x2x2 block of own cells at the face)
            int cl[3];
            cl[0] = r == 0 ? e : fa;
            cl[1] = r == 0 ? fa : r == 1 ? e : fb;
            cl[2] = r == 2 ? e : fb;
            float avg = 0.0f;
#pragma unroll
            for (int di = 0; di < 2; ++di)
#pragma unroll
                for (int dj = 0; dj < 2; ++dj)
#pragma unroll
                    for (int dk = 0; dk < 2; ++dk) avg = __fadd_rn(avg, SX[sxp(cl[0] ^ di, cl[1] ^ dj, cl[2] ^ dk)]);
            avg = __fmul_rn(avg, 0.125f);
            SX[fx[r]] = __fmaf_rn(0.5f, __fsub_rn(hxv[r], avg), SX[sxp(cl[0], cl[1], cl[2])]);
        }
    }
    __syncthreads();
}

// The operator of the thread's quad: diagonal, -x/-y/-z faces, and the +x/+y faces and the
// +z face of the quad's last cell.
struct QuadOps {
    float4 dg, a0, a1, a2, px, py;
    float pz3;
};
template <typename CT, typename XT>
__device__ __forceinline__ void load_ops(const PipeStage<CT, XT>& S, int q, const Quad& Q, QuadOps& o) {
    o.dg = Coef<CT>::ld4(&S.d[4 * q]);
    o.a0 = Coef<CT>::ld4(&S.c0[4 * q]);
    o.a1 = Coef<CT>::ld4(&S.c1[4 * q]);
    o.a2 = Coef<CT>::ld4(&S.c2[4 * q]);
    // +x faces: the -x faces of the cells at i + 1 (thread q + 16), or from the +x neighbour on row i = 7
    o.px = Q.i < 7 ? Coef<CT>::ld4(&S.c0[4 * (q + 16)])
                   : make_float4(Coef<CT>::face(S.c0h[Q.j * 8 + Q.k0], 0), Coef<CT>::face(S.c0h[Q.j * 8 + Q.k0 + 1], 1),
                                 Coef<CT>::face(S.c0h[Q.j * 8 + Q.k0 + 2], 0), Coef<CT>::face(S.c0h[Q.j * 8 + Q.k0 + 3], 1));
    // +y faces: the -y faces at j + 1 (thread q + 2), or from the +y neighbour on row j = 7
    o.py = Q.j < 7 ? Coef<CT>::ld4(&S.c1[4 * (q + 2)])
                   : make_float4(Coef<CT>::face(S.c1h[Q.i * 8 + Q.k0], 0), Coef<CT>::face(S.c1h[Q.i * 8 + Q.k0 + 1], 1),
                                 Coef<CT>::face(S.c1h[Q.i * 8 + Q.k0 + 2], 0), Coef<CT>::face(S.c1h[Q.i * 8 + Q.k0 + 3], 1));
    // +z face of the last cell of the quad: the next quad's first -z face, or the +z neighbour's
    o.pz3 = Q.k0 == 0 ? Coef<CT>::at(&S.c2[4 * (q + 1)]) : Coef<CT>::face(S.c2h[Q.i * 8 + Q.j], 0);
}

// negativeLap (src/AMGSolver.cu:346-382) of own cell u: diag*x, then -x,+x,-y,+y,-z,+z; the
// k neighbours inside the quad are the thread's own cells
__device__ __forceinline__ float quad_neg_lap(const float* SX, const QuadOps& o, const float4& xm, int s0, int u) {
    const float dd = f4get(o.dg, u);
    if (dd == 0.0f) return 0.0f;
    const int c = s0 + u * kSxP;
    const float xmz = u > 0 ? f4get(xm, u - 1) : SX[s0 - 1 + 3 * kSxP];
    const float xpz = u < 3 ? f4get(xm, u + 1) : SX[s0 + 1];
    const float cpz = u < 3 ? f4get(o.a2, u + 1) : o.pz3;
    float ax = __fmul_rn(f4get(xm, u), dd);
    ax = __fmaf_rn(f4get(o.a0, u), SX[c - kSxI], ax);
    ax = __fmaf_rn(f4get(o.px, u), SX[c + kSxI], ax);
    ax = __fmaf_rn(f4get(o.a1, u), SX[c - kSxJ], ax);
    ax = __fmaf_rn(f4get(o.py, u), SX[c + kSxJ], ax);
    ax = __fmaf_rn(f4get(o.a2, u), xmz, ax);
    ax = __fmaf_rn(cpz, xpz, ax);
    return ax;
}

// one colour pass over the staged tile; kRelax: how omega is applied (relax<>)
template <typename CT, typename XT, int kRelax>
__device__ __forceinline__ void process(const PipeStage<CT, XT>& S, float* SX, const DevGrid& g, int t, XT* X, const int d[3], int q,
                                        const PipeArgs& A) {
    const Quad Q(t, q);
    float4 xm;
    int s0;
    build_snapshot(S, SX, d, q, Q, xm, s0);
    const float4 xr = XStore<XT>::ld4(&S.x[4 * q]);
    const unsigned tyw = S.ty[q];
    const float4 b = XStore<XT>::ld4(&S.b[4 * q]);
    QuadOps o;
    load_ops(S, q, Q, o);
    float4 out = xr;
    const int p = (Q.i + Q.j + Q.k0 + A.color) & 1;  // own cells of this colour: u = p, p + 2
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
        const int u = p + 2 * hh;
        const float ax = quad_neg_lap(SX, o, xm, s0, u);
        const bool in = ((tyw >> (8 * u)) & 0xffu) & dInterior;
        const float delta = in ? div_exact(__fsub_rn(f4get(b, u), ax), f4get(o.dg, u)) : 0.0f;
        const float xs = f4get(xm, u);
        f4set(out, u, relax<kRelax>(xs, delta, A.om, A.omega));
    }
    XStore<XT>::st4g(X + Q.base, out);
}

// ResidualAndRestrictAMG128Kernel (src/AMGSolver.cu:896-960) of the staged tile into its
// parent: rhs = R * sum of the 8 children's residuals, x = their mean (0 unless the parent
// cell is INTERIOR), summed in the order of the per-tile kernel (tile_restrict)
template <typename XT, typename PT>
__device__ __forceinline__ void process_restrict(const PipeStage<float, XT>& S, float* SX, float* res, const DevGrid& g, int t, PT* X,
                                                 PT* RHS, const int d[3], int q, float Rr) {
    const Quad Q(t, q);
    float4 xm;
    int s0;
    build_snapshot(S, SX, d, q, Q, xm, s0);
    const float4 b = XStore<XT>::ld4(&S.b[4 * q]);
    QuadOps o;
    load_ops(S, q, Q, o);
    float4 r;
    r.x = __fsub_rn(b.x, quad_neg_lap(SX, o, xm, s0, 0));
    r.y = __fsub_rn(b.y, quad_neg_lap(SX, o, xm, s0, 1));
    r.z = __fsub_rn(b.z, quad_neg_lap(SX, o, xm, s0, 2));
    r.w = __fsub_rn(b.w, quad_neg_lap(SX, o, xm, s0, 3));
    *reinterpret_cast<float4*>(&res[4 * q]) = r;
    __syncthreads();
    if (q < 64) {
        const int f0 = (q >> 4) * 2, f1 = ((q >> 2) & 3) * 2, f2 = (q & 3) * 2;
        float rs = 0.0f, xs = 0.0f;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    rs = __fadd_rn(rs, res[cell_index(f0 + ii, f1 + jj, f2 + kk)]);
                    xs = __fadd_rn(xs, SX[sxp(f0 + ii, f1 + jj, f2 + kk)]);
                }
        const int p = __ldg(g.nb + 8 * t + 6);
        if (p >= 0) {
            const int4 m = __ldg(g.meta + t);
            const size_t po = (size_t)p * kCells + cell_index(parent_local(m.y, f0), parent_local(m.z, f1), parent_local(m.w, f2));
            XStore<PT>::st1(RHS + po, __fmul_rn(rs, Rr));
            XStore<PT>::st1(X + po, (g.ctype[po] & dInterior) ? __fmul_rn(xs, 0.125f) : 0.0f);
        }
    }
}

// FASSaveSolutionAndUpdateSource128Kernel (src/AMGSolver.cu:1176-1206) of the staged NONLEAF
// tile: rhs += A x and x0 = x on INTERIOR cells, rhs = 0 elsewhere (the cycle's 16-bit levels)
template <typename XT>
__device__ __forceinline__ void process_fas(const PipeStage<float, XT>& S, float* SX, const DevGrid& g, int t, XT* RHS, XT* X0,
                                            const int d[3], int q) {
    const Quad Q(t, q);
    float4 xm;
    int s0;
    build_snapshot(S, SX, d, q, Q, xm, s0);
    const float4 b = XStore<XT>::ld4(&S.b[4 * q]);
    const float4 xr = XStore<XT>::ld4(&S.x[4 * q]);
    const unsigned tyw = S.ty[q];
    QuadOps o;
    load_ops(S, q, Q, o);
    float4 rh;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const bool in = ((tyw >> (8 * u)) & 0xffu) & dInterior;
        f4set(rh, u, in ? __fadd_rn(f4get(b, u), quad_neg_lap(SX, o, xm, s0, u)) : 0.0f);
        if (in) XStore<XT>::st1(X0 + Q.base + u, f4get(xr, u));
    }
    XStore<XT>::st4g(RHS + Q.base, rh);
}

// MODE 0: one red-black colour pass; MODE 1: residual and restriction into the parents (PT:
// the parents' x/rhs storage); MODE 2: the FAS update of NONLEAF tiles.  XT: x/rhs storage.
template <typename CT, int MODE, int kRelax = kRelaxRef, typename XT = float, typename PT = float>
__global__ void __launch_bounds__(128, 6) k_gs_pipe(DevGrid g, XT* X, const XT* B, PipeArgs A) {
    extern __shared__ __align__(128) unsigned char pipe_smem[];
    __shared__ __align__(8) unsigned long long mbar[2];
    using Smem = typename std::conditional<MODE == 0, PipeSmem<CT, XT>, PipeSmemR<XT>>::type;
    static_assert(MODE == 0 || std::is_same<CT, float>::value, "restriction and FAS read the float operator");
    Smem& sm = *reinterpret_cast<Smem*>(pipe_smem);
    const int q = threadIdx.x, side = q >> 6;
    const int stride = gridDim.x, tend = A.t0 + A.nt;
    int tcur = A.t0 + blockIdx.x;
    if (tcur >= tend) return;
    const unsigned mb0 = smem_addr(&mbar[0]);  // stage s: mb0 + 8 s
    if (q == 0) {
        mbar_init(mb0);
        mbar_init(mb0 + 8);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const CT* C0 = static_cast<const CT*>(A.coef);
    const CT* C1 = C0 + A.cstride;
    const CT* C2 = C1 + A.cstride;
    const CT* C3 = C2 + A.cstride;
    const float h = voxel_size(g.h0, tile_level(g, tcur));  // all tiles of the launch share the level
    int dcur[3], dnext[3] = {0, 0, 0};
    load_desc(g, tcur, side, dcur);
    int tnext = tcur + stride;
    if (tnext < tend) load_desc(g, tnext, side, dnext);
    // Launched as a programmatic dependent of the previous kernel, the block may start while
    // that kernel still runs: the first tile's static planes go out now, x and rhs only once
    // the previous kernel has finished (a no-op for an ordinary launch).
    issue_static(sm.st[0], mb0, g, tcur, C0, C1, C2, C3, dcur, q, h);
    asm volatile("griddepcontrol.wait;" ::: "memory");
    issue_dynamic(sm.st[0], mb0, tcur, X, B, dcur, q);
    bool pending_other = false;  // bulk copies in flight into the other stage
    for (int k = 0;; ++k) {
        const int s = k & 1;
        pending_other = tnext < tend;
        if (pending_other) issue(sm.st[s ^ 1], mb0 + 8 * (s ^ 1), g, tnext, X, B, C0, C1, C2, C3, dnext, q, h);
        else cp_commit();
        const int tn2 = tnext + stride;
        int dn2[3] = {0, 0, 0};
        if (tn2 < tend) load_desc(g, tn2, side, dn2);
        // on its last tile the block lets the next pass be scheduled (it reads nothing of this
        // one before its own wait); a block that exits counts as triggered
        if (tnext >= tend) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
        cp_wait_prev();
        // stage s is the (k >> 1)-th use of its mbarrier
        const bool ok = mbar_wait(mb0 + 8 * s, (unsigned)(k >> 1) & 1u);
        if (__syncthreads_or(!ok)) {
            if (q == 0) atomicExch(&g_pipe_error, 1);
            if (pending_other) mbar_wait(mb0 + 8 * (s ^ 1), (unsigned)((k + 1) >> 1) & 1u);
            break;
        }
        if constexpr (MODE == 0)
            process<CT, XT, kRelax>(sm.st[s], sm.x, g, tcur, X, dcur, q, A);
        else if constexpr (MODE == 1)
            process_restrict<XT, PT>(sm.st[s], sm.x, sm.res, g, tcur, static_cast<PT*>(A.xp), static_cast<PT*>(A.rhsp), dcur, q, A.Rr);
        else
            process_fas<XT>(sm.st[s], sm.x, g, tcur, static_cast<XT*>(A.rhsp), static_cast<XT*>(A.x0p), dcur, q);
        __syncthreads();
        if (tnext >= tend) break;
        tcur = tnext;
        tnext = tn2;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            dcur[r] = dnext[r];
            dnext[r] = dn2[r];
        }
    }
    cp_wait_all();
}

__device__ __forceinline__ void store16(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
__device__ __forceinline__ void store16(__half* p, float v) { *p = __float2half_rn(v); }
// the operator planes rounded to 16 bits (round to nearest even), plane after plane
template <typename CT>
__global__ void k_coeff16(const float* __restrict__ C, CT* __restrict__ out, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) store16(out + i, C[i]);
}

int g_pipe_blocks = 0;  // resident blocks of k_gs_pipe on the device
int g_pipe_dependent = 1;  // launch the passes as programmatic dependents of the previous kernel

// A pass launched as a programmatic dependent starts its blocks as soon as the previous
// kernel's blocks have all started (or exited) and resources free up, instead of after that
// kernel has drained: the launch latency and the first tile's static copies overlap its tail.
template <typename... P, typename... A>
void launch_pass_kernel(void (*kernel)(P...), int blocks, size_t smem, cudaStream_t st, A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = g_pipe_dependent ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

using bf16 = __nv_bfloat16;

template <typename K>
bool set_smem(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess;
}
template <typename CT, typename XT>
bool set_pipe_smem() {
    const size_t b = sizeof(PipeSmem<CT, XT>);
    return set_smem(k_gs_pipe<CT, 0, kRelaxRef, XT>, b) && set_smem(k_gs_pipe<CT, 0, kRelaxDouble, XT>, b);
}
template <typename CT, typename XT>
void launch_pass(int blocks, cudaStream_t st, const DevGrid& g, XT* X, const XT* B, const PipeArgs& A) {
    const size_t sm = sizeof(PipeSmem<CT, XT>);
    if (A.exact == kRelaxRef)
        launch_pass_kernel(k_gs_pipe<CT, 0, kRelaxRef, XT>, blocks, sm, st, g, X, B, A);
    else
        launch_pass_kernel(k_gs_pipe<CT, 0, kRelaxDouble, XT>, blocks, sm, st, g, X, B, A);
}
int g_restrict_blocks = 0;  // resident blocks of the restriction pass

}  // namespace

void gs_pipe_set_dependent_launch(bool on) { g_pipe_dependent = on ? 1 : 0; }
bool gs_pipe_dependent_launch() { return g_pipe_dependent != 0; }

int gs_pipe_take_error() {
    int v = 0, z = 0;
    if (cudaMemcpyFromSymbol(&v, g_pipe_error, sizeof(int)) != cudaSuccess) return -1;
    if (v) cudaMemcpyToSymbol(g_pipe_error, &z, sizeof(int));
    return v;
}

int gs_pipe_init() {
    if (!set_pipe_smem<float, float>() || !set_pipe_smem<bf16, float>() || !set_pipe_smem<__half, float>() ||
        !set_pipe_smem<float, bf16>() || !set_pipe_smem<bf16, bf16>() || !set_pipe_smem<__half, bf16>())
        return 0;
    if (!set_smem(k_gs_pipe<float, 1>, sizeof(PipeSmemR<float>)) || !set_smem(k_gs_pipe<float, 1, kRelaxRef, bf16, bf16>, sizeof(PipeSmemR<bf16>)) ||
        !set_smem(k_gs_pipe<float, 1, kRelaxRef, bf16, float>, sizeof(PipeSmemR<bf16>)) ||
        !set_smem(k_gs_pipe<float, 2, kRelaxRef, bf16>, sizeof(PipeSmemR<bf16>)))
        return 0;
    int dev = 0, sms = 0, per_sm = 0, per_sm_r = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs_pipe<float, 0, kRelaxRef>, 128, sizeof(PipeSmem<float, float>)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_r, k_gs_pipe<float, 1>, 128, sizeof(PipeSmemR<float>)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    g_pipe_blocks = sms * per_sm;
    g_restrict_blocks = sms * per_sm_r;
    return per_sm_r > 0 ? g_pipe_blocks : 0;
}

size_t coeff16_bytes(const DevGrid& g) { return (size_t)4 * g.n * kCells * 2; }

void launch_coeff16(const DevGrid& g, int coeff_ch, int storage, void* out, cudaStream_t st) {
    const size_t n = (size_t)4 * g.n * kCells;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    note_kernel_launch();
    if (storage == kStorageBF16)
        k_coeff16<__nv_bfloat16><<<blocks, 256, 0, st>>>(g.plane(coeff_ch), static_cast<__nv_bfloat16*>(out), n);
    else
        k_coeff16<__half><<<blocks, 256, 0, st>>>(g.plane(coeff_ch), static_cast<__half*>(out), n);
}

void launch_gs_pipe(const DevGrid& g, int t0, int nt, void* X, const void* B, bool x16, int coeff_ch, int color, double omega,
                    cudaStream_t st, int storage, const void* coeff16) {
    if (nt <= 0) return;
    PipeArgs A = {};
    A.t0 = t0;
    A.nt = nt;
    A.color = color;
    A.om = (float)omega;
    A.exact = relax_mode(omega);
    A.omega = omega;
    A.cstride = (size_t)g.n * kCells;
    A.Rr = 1.0f;
    A.coef = storage == kStorageFP32 ? (const void*)g.plane(coeff_ch) : coeff16;
    const int blocks = nt < g_pipe_blocks ? nt : g_pipe_blocks;
    note_kernel_launch();
    if (!x16) {
        float* Xf = static_cast<float*>(X);
        const float* Bf = static_cast<const float*>(B);
        if (storage == kStorageFP32) launch_pass<float>(blocks, st, g, Xf, Bf, A);
        else if (storage == kStorageBF16) launch_pass<bf16>(blocks, st, g, Xf, Bf, A);
        else launch_pass<__half>(blocks, st, g, Xf, Bf, A);
    } else {
        bf16* Xh = static_cast<bf16*>(X);
        const bf16* Bh = static_cast<const bf16*>(B);
        if (storage == kStorageFP32) launch_pass<float>(blocks, st, g, Xh, Bh, A);
        else if (storage == kStorageBF16) launch_pass<bf16>(blocks, st, g, Xh, Bh, A);
        else launch_pass<__half>(blocks, st, g, Xh, Bh, A);
    }
}

void launch_restrict_pipe(const DevGrid& g, int t0, int nt, const void* X, const void* B, bool x16, void* Xp, void* RHSp, bool p16,
                          int coeff_ch, float Rr, cudaStream_t st) {
    if (nt <= 0) return;
    PipeArgs A = {};
    A.t0 = t0;
    A.nt = nt;
    A.exact = kRelaxRef;
    A.om = 1.0f;
    A.omega = 1.0;
    A.coef = g.plane(coeff_ch);
    A.cstride = (size_t)g.n * kCells;
    A.xp = Xp;
    A.rhsp = RHSp;
    A.Rr = Rr;
    const int blocks = nt < g_restrict_blocks ? nt : g_restrict_blocks;
    note_kernel_launch();
    if (!x16) {
        launch_pass_kernel(k_gs_pipe<float, 1>, blocks, sizeof(PipeSmemR<float>), st, g, (float*)X, (const float*)B, A);
    } else if (p16) {
        launch_pass_kernel(k_gs_pipe<float, 1, kRelaxRef, bf16, bf16>, blocks, sizeof(PipeSmemR<bf16>), st, g, (bf16*)X, (const bf16*)B, A);
    } else {
        launch_pass_kernel(k_gs_pipe<float, 1, kRelaxRef, bf16, float>, blocks, sizeof(PipeSmemR<bf16>), st, g, (bf16*)X, (const bf16*)B,
                           A);
    }
}

namespace {
__device__ __forceinline__ float ldx(const float* p) { return *p; }
__device__ __forceinline__ float ldx(const bf16* p) { return __bfloat162float(*p); }
// FASProlongateAndUpdateAMG128Kernel (src/AMGSolver.cu:1216-1248) on a level whose x is BF16;
// the parent level's x and saved x are BF16 or float (PT)
template <typename PT>
__global__ void __launch_bounds__(128) k_prolong_x16(DevGrid g, int t0, bf16* X, const PT* Xc, const PT* X0c, float P) {
    const int t = t0 + blockIdx.x;
    const Quad Q(t, threadIdx.x);
    const int4 m = g.meta[t];
    const bool ghost = (m.x >> 8) & dGhost;
    const int p = g.nb[8 * t + 6];
    const float4 xr = XStore<bf16>::ld4(X + Q.base);
    const uchar4 ty = ldt4(g.ctype + Q.base);
    const int pi = parent_local(m.y, Q.i), pj = parent_local(m.z, Q.j);
    float4 out;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        float cx = 0.0f, cx0 = 0.0f;
        if (p >= 0) {
            const size_t o = (size_t)p * kCells + cell_index(pi, pj, parent_local(m.w, Q.k0 + u));
            cx = ldx(Xc + o);
            cx0 = ldx(X0c + o);
        }
        const bool in = t4get(ty, u) & dInterior;
        f4set(out, u, ghost ? (in ? cx : 0.0f) : (in ? __fmaf_rn(P, __fsub_rn(cx, cx0), f4get(xr, u)) : 0.0f));
    }
    XStore<bf16>::st4g(X + Q.base, out);
}
// the cycle's right-hand side in BF16 on the given LEAF tiles, and the cycle's result back
__global__ void __launch_bounds__(128) k_leaf_to_bf16(const int* leaf, const float* R, bf16* R16) {
    const size_t base = (size_t)leaf[blockIdx.x] * kCells + 4 * threadIdx.x;
    XStore<bf16>::st4g(R16 + base, *reinterpret_cast<const float4*>(R + base));
}
__global__ void __launch_bounds__(128) k_leaf_from_bf16(const int* leaf, const bf16* X16, float* Z) {
    const size_t base = (size_t)leaf[blockIdx.x] * kCells + 4 * threadIdx.x;
    st4(Z + base, XStore<bf16>::ld4(X16 + base));
}
}  // namespace

void launch_prolong_x16(const DevGrid& g, int t0, int nt, void* X, const void* Xc, const void* X0c, bool p16, float P, cudaStream_t st) {
    if (nt <= 0) return;
    note_kernel_launch();
    if (p16) k_prolong_x16<bf16><<<nt, 128, 0, st>>>(g, t0, (bf16*)X, (const bf16*)Xc, (const bf16*)X0c, P);
    else k_prolong_x16<float><<<nt, 128, 0, st>>>(g, t0, (bf16*)X, (const float*)Xc, (const float*)X0c, P);
}
void launch_leaf_to_bf16(const int* leaf, int nleaf, const float* R, void* R16, cudaStream_t st) {
    if (nleaf <= 0) return;
    note_kernel_launch();
    k_leaf_to_bf16<<<nleaf, 128, 0, st>>>(leaf, R, (bf16*)R16);
}
void launch_leaf_from_bf16(const int* leaf, int nleaf, const void* X16, float* Z, cudaStream_t st) {
    if (nleaf <= 0) return;
    note_kernel_launch();
    k_leaf_from_bf16<<<nleaf, 128, 0, st>>>(leaf, (const bf16*)X16, Z);
}

void launch_fas_pipe_x16(const DevGrid& g, int t0, int nt, const void* X, void* RHS, void* X0, int coeff_ch, cudaStream_t st) {
    if (nt <= 0) return;
    PipeArgs A = {};
    A.t0 = t0;
    A.nt = nt;
    A.exact = kRelaxRef;
    A.om = 1.0f;
    A.omega = 1.0;
    A.coef = g.plane(coeff_ch);
    A.cstride = (size_t)g.n * kCells;
    A.rhsp = RHS;
    A.x0p = X0;
    const int blocks = nt < g_restrict_blocks ? nt : g_restrict_blocks;
    note_kernel_launch();
    launch_pass_kernel(k_gs_pipe<float, 2, kRelaxRef, bf16>, blocks, sizeof(PipeSmemR<bf16>), st, g, (bf16*)X, (const bf16*)RHS, A);
}

}  // namespace cmg
