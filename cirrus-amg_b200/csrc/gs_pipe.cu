// Red-black Gauss-Seidel colour pass on the LEAF and NONLEAF tiles of one level
// (NegativeLaplacianAndGaussSeidelSameLevelAMG128Kernel, src/AMGSolver.cu:838-877),
// as a persistent, software-pipelined kernel for the multigrid cycle.
//
// k_gs spends most of a tile's life waiting: the neighbour descriptors arrive, then
// the halo loads go out, then the block computes.  Here each 128-thread block walks a
// strided list of tiles and keeps the next tile's planes and halo in flight (cp.async
// into a second shared-memory stage) while it computes the current one.  No register
// holds data in flight and nothing spins: cp.async.wait_group is the only wait.
//
// Halo values are read without the neighbour's cell types.  That relies on the
// multigrid x plane holding 0 on every cell that is not INTERIOR, which the cycle keeps
// true (x starts at 0; restriction, prolongation and the sweeps write masked values),
// and on GHOST neighbours being read raw, as the reference does.  The public
// cmg_amg_gauss_seidel, which takes arbitrary x, keeps using k_gs.
#include "kernels.hpp"

namespace cmg {

namespace {

struct PipeStage {
    float x[512], b[512], d[512];
    float c0[576];   // -x faces of the tile, then the +x faces of row i = 7 (from the +x neighbour)
    float c1[512];   // -y faces
    float c2[512];   // -z faces
    float c1h[64];   // +y faces of row j = 7, [i][k]
    float c2h[64];   // +z faces of row k = 7, [i][j]
    float hx[384];   // halo x of the six faces, [axis][side][a][b]
    unsigned ty[128];
};
// The snapshot: masked x of the tile with its one-cell halo, split into four planes by
// k mod 4 (k = 4h + u: u the plane, h = -1..2 the slot), rows j of 4 slots, layers i of
// 42 floats, planes of 448 floats.  A warp's threads own (i0..i0+1, j 0..7, h 0..1) and
// touch one plane per lane at a time: the offsets 4j + h and 42 + 4j + h fill the 32
// banks once each, and the plane stride is a multiple of 32, so the stores of its own
// cells and the i/j neighbour loads of a colour pass are free of bank conflicts.
constexpr int kSxI = 42, kSxJ = 4, kSxP = 448;
__device__ __forceinline__ int sxp(int i, int j, int k) { return ((k + 4) & 3) * kSxP + (i + 1) * kSxI + (j + 1) * kSxJ + ((k + 4) >> 2); }

struct PipeSmem {
    PipeStage st[2];
    float x[4 * kSxP];
};
constexpr size_t kPipeSmem = sizeof(PipeSmem);

__device__ __forceinline__ void cp16(void* dst, const void* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp4(void* dst, const void* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

struct PipeArgs {
    int t0, nt, coeff_ch, color, exact;
    float om;
    double omega;
};

// neighbour descriptors of the thread's three halo cells: face r on side q >> 6
__device__ __forceinline__ void load_desc(const DevGrid& g, int t, int side, int d[3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r) d[r] = __ldg(g.nbx + 8 * t + r + 3 * side);
}

// start the copies of tile t into stage S
__device__ __forceinline__ void issue(PipeStage& S, const DevGrid& g, int t, const float* X, const float* B, const float* C0,
                                      const float* C1, const float* C2, const float* C3, const int d[3], int q, float h) {
    const size_t base = (size_t)t * kCells + 4 * q;
    cp16(&S.x[4 * q], X + base);
    cp16(&S.b[4 * q], B + base);
    cp16(&S.d[4 * q], C3 + base);
    cp16(&S.c0[4 * q], C0 + base);
    cp16(&S.c1[4 * q], C1 + base);
    cp16(&S.c2[4 * q], C2 + base);
    cp4(&S.ty[q], g.ctype + base);
    const int side = q >> 6, fa = (q >> 3) & 7, fb = q & 7;
    const int e = side ? 0 : 7;  // the neighbour's cell next to the shared face
    const int nl[3] = {cell_index(e, fa, fb), cell_index(fa, e, fb), cell_index(fa, fb, e)};
    float* hc[3] = {&S.c0[512 + fa * 8 + fb], &S.c1h[fa * 8 + fb], &S.c2h[fa * 8 + fb]};
    const float* Cr[3] = {C0, C1, C2};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        float* hxd = &S.hx[r * 128 + q];
        if (d[r] != 0) {
            const size_t o = (size_t)((d[r] >> 3) - 1) * kCells + nl[r];
            cp4(hxd, X + o);
            if (side) cp4(hc[r], Cr[r] + o);
        } else {
            *hxd = 0.0f;
            if (side) *hc[r] = h;
        }
    }
    cp_commit();
}

// the snapshot of the staged tile and one colour pass over it
__device__ __forceinline__ void process(const PipeStage& S, float* SX, const DevGrid& g, int t, float* X, const int d[3], int q,
                                        const PipeArgs& A) {
    const Quad Q(t, q);
    const float4 xr = *reinterpret_cast<const float4*>(&S.x[4 * q]);
    const unsigned tyw = S.ty[q];
    float4 xm;
    xm.x = (tyw & 0xffu) == dInterior ? xr.x : 0.0f;
    xm.y = ((tyw >> 8) & 0xffu) == dInterior ? xr.y : 0.0f;
    xm.z = ((tyw >> 16) & 0xffu) == dInterior ? xr.z : 0.0f;
    xm.w = ((tyw >> 24) & 0xffu) == dInterior ? xr.w : 0.0f;
    // own cells (i, j, k0 + u): plane u, slot h + 1
    const int s0 = (Q.i + 1) * kSxI + (Q.j + 1) * kSxJ + (Q.k0 >> 2) + 1;
    SX[s0] = xm.x;
    SX[s0 + kSxP] = xm.y;
    SX[s0 + 2 * kSxP] = xm.z;
    SX[s0 + 3 * kSxP] = xm.w;
    const int side = q >> 6, fa = (q >> 3) & 7, fb = q & 7;
    const int e = side ? 7 : 0, hxl = side ? 8 : -1;
    const int fx[3] = {sxp(hxl, fa, fb), sxp(fa, hxl, fb), sxp(fa, fb, hxl)};
#pragma unroll
    for (int r = 0; r < 3; ++r)
        if (!(d[r] & dGhost)) SX[fx[r]] = S.hx[r * 128 + q];
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
            SX[fx[r]] = __fmaf_rn(0.5f, __fsub_rn(S.hx[r * 128 + q], avg), SX[sxp(cl[0], cl[1], cl[2])]);
        }
    }
    __syncthreads();
    const float4 b = *reinterpret_cast<const float4*>(&S.b[4 * q]);
    const float4 dg = *reinterpret_cast<const float4*>(&S.d[4 * q]);
    const float4 a0 = *reinterpret_cast<const float4*>(&S.c0[4 * q]);
    const float4 a1 = *reinterpret_cast<const float4*>(&S.c1[4 * q]);
    const float4 a2 = *reinterpret_cast<const float4*>(&S.c2[4 * q]);
    // +x faces: the -x faces of the cells at i + 1 (thread q + 16; row i = 7: from the +x
    // neighbour, stored after the tile's faces in the same order)
    const float4 px = *reinterpret_cast<const float4*>(&S.c0[4 * (q + 16)]);
    // +y faces: the -y faces at j + 1 (thread q + 2), or from the +y neighbour on row j = 7
    const float4 py = Q.j < 7 ? *reinterpret_cast<const float4*>(&S.c1[4 * (q + 2)])
                              : *reinterpret_cast<const float4*>(&S.c1h[Q.i * 8 + Q.k0]);
    // +z face of the last cell of the quad: the next quad's first -z face, or the +z neighbour's
    const float pz3 = Q.k0 == 0 ? S.c2[4 * (q + 1)] : S.c2h[Q.i * 8 + Q.j];
    float4 out = xr;
    const int p = (Q.i + Q.j + Q.k0 + A.color) & 1;  // own cells of this colour: u = p, p + 2
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
        const int u = p + 2 * hh;
        const float dd = f4get(dg, u);
        float ax = 0.0f;
        if (dd != 0.0f) {
            // negativeLap (src/AMGSolver.cu:346-382): diag*x, then -x,+x,-y,+y,-z,+z; the k
            // neighbours inside the quad are the thread's own cells of the other colour
            const int c = s0 + u * kSxP;
            const float xmz = u > 0 ? f4get(xm, u - 1) : SX[s0 - 1 + 3 * kSxP];
            const float xpz = u < 3 ? f4get(xm, u + 1) : SX[s0 + 1];
            const float cpz = u < 3 ? f4get(a2, u + 1) : pz3;
            ax = __fmul_rn(f4get(xm, u), dd);
            ax = __fmaf_rn(f4get(a0, u), SX[c - kSxI], ax);
            ax = __fmaf_rn(f4get(px, u), SX[c + kSxI], ax);
            ax = __fmaf_rn(f4get(a1, u), SX[c - kSxJ], ax);
            ax = __fmaf_rn(f4get(py, u), SX[c + kSxJ], ax);
            ax = __fmaf_rn(f4get(a2, u), xmz, ax);
            ax = __fmaf_rn(cpz, xpz, ax);
        }
        const bool in = ((tyw >> (8 * u)) & 0xffu) & dInterior;
        const float delta = in ? div_exact(__fsub_rn(f4get(b, u), ax), dd) : 0.0f;
        const float xs = f4get(xm, u);
        f4set(out, u, A.exact ? __fmaf_rn(delta, A.om, xs) : (float)((double)xs + (double)delta * A.omega));
    }
    st4(X + Q.base, out);
}
__global__ void __launch_bounds__(128, 6) k_gs_pipe(DevGrid g, float* X, const float* B, PipeArgs A) {
    extern __shared__ __align__(16) unsigned char pipe_smem[];
    PipeSmem& sm = *reinterpret_cast<PipeSmem*>(pipe_smem);
    const int q = threadIdx.x, side = q >> 6;
    const int stride = gridDim.x, tend = A.t0 + A.nt;
    int tcur = A.t0 + blockIdx.x;
    if (tcur >= tend) return;
    const float* C0 = g.plane(A.coeff_ch);
    const float* C1 = g.plane(A.coeff_ch + 1);
    const float* C2 = g.plane(A.coeff_ch + 2);
    const float* C3 = g.plane(A.coeff_ch + 3);
    const float h = voxel_size(g.h0, tile_level(g, tcur));  // all tiles of the launch share the level
    int dcur[3], dnext[3] = {0, 0, 0};
    load_desc(g, tcur, side, dcur);
    int tnext = tcur + stride;
    if (tnext < tend) load_desc(g, tnext, side, dnext);
    issue(sm.st[0], g, tcur, X, B, C0, C1, C2, C3, dcur, q, h);
    for (int k = 0;; ++k) {
        const int s = k & 1;
        if (tnext < tend) issue(sm.st[s ^ 1], g, tnext, X, B, C0, C1, C2, C3, dnext, q, h);
        else cp_commit();
        const int tn2 = tnext + stride;
        int dn2[3] = {0, 0, 0};
        if (tn2 < tend) load_desc(g, tn2, side, dn2);
        cp_wait_prev();
        __syncthreads();
        process(sm.st[s], sm.x, g, tcur, X, dcur, q, A);
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

int g_pipe_blocks = 0;  // resident blocks of k_gs_pipe on the device

}  // namespace

int gs_pipe_init() {
    if (cudaFuncSetAttribute(k_gs_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPipeSmem) != cudaSuccess) return 0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs_pipe, 128, kPipeSmem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    g_pipe_blocks = sms * per_sm;
    return g_pipe_blocks;
}

void launch_gs_pipe(const DevGrid& g, int t0, int nt, float* X, const float* B, int coeff_ch, int color, double omega, cudaStream_t st) {
    if (nt <= 0) return;
    PipeArgs A;
    A.t0 = t0;
    A.nt = nt;
    A.coeff_ch = coeff_ch;
    A.color = color;
    A.om = (float)omega;
    A.exact = ((double)A.om == omega);
    A.omega = omega;
    const int blocks = nt < g_pipe_blocks ? nt : g_pipe_blocks;
    note_kernel_launch();
    k_gs_pipe<<<blocks, 128, kPipeSmem, st>>>(g, X, B, A);
}

}  // namespace cmg
