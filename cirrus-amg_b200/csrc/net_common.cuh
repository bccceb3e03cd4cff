// Device code shared by the learned smoother's kernels (learned.cu: the small nets on
// mma.sync and tcgen05; learned_deep.cu: the 32-channel residual net on tcgen05): the
// padded 10^3 voxel grid of a tile, the feature staging from the grid or the samples, and
// the tcgen05 / mbarrier primitives.
#pragma once
#include <cuda_bf16.h>

#include "kernels.hpp"

namespace cmg {
namespace {

constexpr int kNetThreads = 128;
constexpr int kPadVox = 1000;  // 10^3 padded voxels per tile

// tap = dx*9 + dy*3 + dz (each 0..2), offset in the padded voxel grid
__device__ __forceinline__ int tap_off(int tap) { return (tap / 9 - 1) * 100 + ((tap / 3) % 3 - 1) * 10 + (tap % 3 - 1); }
__device__ __forceinline__ int pad_vox(int i, int j, int k) { return (i + 1) * 100 + (j + 1) * 10 + (k + 1); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// fixed-order block reductions over 128 threads
__device__ __forceinline__ float block_sum_f(float v, float* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const float r = (red[0] + red[1]) + (red[2] + red[3]);
    __syncthreads();
    return r;
}
__device__ __forceinline__ float block_max_f(float v, float* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const float r = fmaxf(fmaxf(red[0], red[1]), fmaxf(red[2], red[3]));
    __syncthreads();
    return r;
}

// Where one tile's inputs come from: sample s is tile (idx ? idx[s] : t0 + s) of planes of
// 512 floats; rho = r - az (az may be null: r already holds rho).  ex: the face coefficients
// and the residual's 1-cell halo (NetExtra), each optional.
struct NetIn {
    const float* r;
    const float* az;
    const float* diag;
    const uint8_t* types;
    const float* target;
    const int* idx;
    int t0;
    NetExtra ex;
};

struct Staged {
    float rho[4];
    float tgt[4];
    bool in[4];
    float S, D;  // S = 0: nothing to do on this tile
};

// Stage one tile's features into x0 (8-channel layout); thread q owns cells 4q..4q+3.
__device__ __forceinline__ Staged stage_features(const NetIn& I, int s, __nv_bfloat16* x0, float* red) {
    Staged o;
    const int t = I.idx ? I.idx[s] : I.t0 + s;
    const size_t base = (size_t)t * kCells + 4 * threadIdx.x;
    float4 r4 = ldcg4(I.r + base);
    if (I.az) {
        const float4 a4 = ldcg4(I.az + base);
        r4 = make_float4(__fsub_rn(r4.x, a4.x), __fsub_rn(r4.y, a4.y), __fsub_rn(r4.z, a4.z), __fsub_rn(r4.w, a4.w));
    }
    const float4 dg = ldcg4(I.diag + base);
    const uchar4 ty = ldt4(I.types + base);
    const float rr[4] = {r4.x, r4.y, r4.z, r4.w}, dd[4] = {dg.x, dg.y, dg.z, dg.w};
    const uint8_t tt[4] = {ty.x, ty.y, ty.z, ty.w};
    float ss = 0.0f, dm = 0.0f, cnt = 0.0f;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        o.in[u] = (tt[u] & dInterior) != 0;
        o.rho[u] = o.in[u] ? rr[u] : 0.0f;
        ss = __fmaf_rn(o.rho[u], o.rho[u], ss);
        if (o.in[u]) {
            dm = fmaxf(dm, fabsf(dd[u]));
            cnt += 1.0f;
        }
    }
    if (I.target) {
        const float4 tg = ldcg4(I.target + base);
        o.tgt[0] = tg.x, o.tgt[1] = tg.y, o.tgt[2] = tg.z, o.tgt[3] = tg.w;
    }
    const float sum = block_sum_f(ss, red), n = block_sum_f(cnt, red);
    o.D = block_max_f(dm, red);
    o.S = (n > 0.0f && sum > 0.0f && o.D > 0.0f) ? sqrtf(sum / n) : 0.0f;
    if (o.S == 0.0f) return o;
    // the -x, -y, -z face coefficients (cut cells: scaled by their face fractions)
    float fc[3][4] = {};
    if (I.ex.faces) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float4 f4 = ldcg4(I.ex.faces + (size_t)a * I.ex.fstride + (size_t)t * I.ex.ftile + 4 * threadIdx.x);
            fc[a][0] = f4.x, fc[a][1] = f4.y, fc[a][2] = f4.z, fc[a][3] = f4.w;
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int cell = 4 * threadIdx.x + u;
        const int v = pad_vox(cell >> 6, (cell >> 3) & 7, cell & 7);
        __nv_bfloat162 f[4];
        f[0] = __floats2bfloat162_rn(o.rho[u] / o.S, o.in[u] ? 1.0f : 0.0f);
        f[1] = __floats2bfloat162_rn((tt[u] & dDirichlet) ? 1.0f : 0.0f, o.in[u] ? dd[u] / o.D : 0.0f);
        f[2] = __floats2bfloat162_rn(o.in[u] ? fc[0][u] / o.D : 0.0f, o.in[u] ? fc[1][u] / o.D : 0.0f);
        f[3] = __floats2bfloat162_rn(o.in[u] ? fc[2][u] / o.D : 0.0f, 0.0f);
        *reinterpret_cast<uint4*>(x0 + v * 8) = *reinterpret_cast<const uint4*>(f);
    }
    // the residual's 1-cell halo: thread q owns cell (fa, fb) of the face of axis r on side
    // q >> 6 for r = 0, 1, 2 (channel 0: rho / S of the neighbour cell, channel 1: 1 when it
    // is an INTERIOR cell of a LEAF neighbour tile, else both 0)
    if (I.ex.halo || I.ex.nbx) {
        const int q = threadIdx.x, side = q >> 6, fa = (q >> 3) & 7, fb = q & 7;
        const int e = side ? 0 : 7, hx = side ? 8 : -1;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            float hv = 0.0f, ok = 0.0f;
            if (I.ex.halo) {
                const float* hs = I.ex.halo + (size_t)t * 768;
                hv = __ldcg(hs + r * 128 + q);
                ok = __ldcg(hs + 384 + r * 128 + q);
            } else {
                const int d = I.ex.nbx[8 * t + r + 3 * side];
                if (d != 0 && (d & 7) == dLeaf) {
                    const size_t on = (size_t)((d >> 3) - 1) * kCells +
                                      (r == 0 ? cell_index(e, fa, fb) : r == 1 ? cell_index(fa, e, fb) : cell_index(fa, fb, e));
                    if (I.types[on] & dInterior) {
                        hv = __ldcg(I.r + on);
                        if (I.az) hv = __fsub_rn(hv, __ldcg(I.az + on));
                        ok = 1.0f;
                    }
                }
            }
            const int v = r == 0 ? pad_vox(hx, fa, fb) : r == 1 ? pad_vox(fa, hx, fb) : pad_vox(fa, fb, hx);
            __nv_bfloat162 f[4];
            f[0] = __floats2bfloat162_rn(ok != 0.0f ? hv / o.S : 0.0f, ok);
            f[1] = f[2] = f[3] = __floats2bfloat162_rn(0.0f, 0.0f);
            *reinterpret_cast<uint4*>(x0 + v * 8) = *reinterpret_cast<const uint4*>(f);
        }
    }
    return o;
}
// Loss of one tile and its gradient dL/df / 2 on this thread's cells 4q..4q+3, from the net's
// output f in ys: e = f - target D/S on INTERIOR cells (0 elsewhere).  Kind 0: sum e^2, g = e.
// Kind 1 (energy): e^T L e with L the 7-point Laplacian of the tile (6 on the diagonal, -1
// per neighbour inside the tile, zero outside), g = L e on INTERIOR cells.  Returns this
// thread's share of the loss; ys holds e afterwards with kind 1.
__device__ __forceinline__ float tile_loss_grad(const Staged& st, float* ys, int loss_kind, float (&g)[4]) {
    const float sc = st.D / st.S;
    float e[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) e[u] = st.in[u] ? __fsub_rn(ys[4 * threadIdx.x + u], __fmul_rn(st.tgt[u], sc)) : 0.0f;
    if (loss_kind == 1) {
        __syncthreads();  // every thread has read its f
#pragma unroll
        for (int u = 0; u < 4; ++u) ys[4 * threadIdx.x + u] = e[u];
        __syncthreads();
    }
    float l = 0.0f;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int cell = 4 * threadIdx.x + u, ci = cell >> 6, cj = (cell >> 3) & 7, ck = cell & 7;
        g[u] = e[u];
        if (loss_kind == 1) {
            float nbs = 0.0f;
            if (ci > 0) nbs += ys[cell - 64];
            if (ci < 7) nbs += ys[cell + 64];
            if (cj > 0) nbs += ys[cell - 8];
            if (cj < 7) nbs += ys[cell + 8];
            if (ck > 0) nbs += ys[cell - 1];
            if (ck < 7) nbs += ys[cell + 1];
            g[u] = st.in[u] ? __fsub_rn(6.0f * e[u], nbs) : 0.0f;
        }
        l = __fmaf_rn(e[u], g[u], l);
    }
    return l;
}

// zero the face halo voxels of an 8-channel buffer (whose other use needs zero padding)
__device__ __forceinline__ void clear_face_halo(__nv_bfloat16* x0) {
    const int q = threadIdx.x, side = q >> 6, fa = (q >> 3) & 7, fb = q & 7, hx = side ? 8 : -1;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int v = r == 0 ? pad_vox(hx, fa, fb) : r == 1 ? pad_vox(fa, hx, fb) : pad_vox(fa, fb, hx);
        *reinterpret_cast<uint4*>(x0 + v * 8) = make_uint4(0, 0, 0, 0);
    }
}

__device__ __forceinline__ void zero_smem(void* p, int bytes) {
    for (int i = threadIdx.x; i < bytes / 16; i += kNetThreads) reinterpret_cast<uint4*>(p)[i] = make_uint4(0, 0, 0, 0);
}

constexpr int kTcVox = 1008;  // padded voxels per group plane (16 beyond the grid: K padding reads there)

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) |
           (1ull << 46);  // no swizzle, version 1
}
// kind::f16 instruction descriptor: F32 accumulator, BF16 A and B, both K-major, M = 64
__host__ __device__ constexpr uint32_t umma_idesc(int N) { return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | (4u << 24); }

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(done)
                 : "r"(mbar), "r"(parity)
                 : "memory");
    return done != 0;
}
// bounded wait for an MMA completion phase
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (int i = 0; i < (1 << 20); ++i)
        if (mbar_try(mbar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }


}  // namespace
}  // namespace cmg
