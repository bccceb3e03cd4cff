// Learned finest-level smoother: a per-tile 3-D convolutional network on BF16 tensor
// cores (the reference has no counterpart; it is the learned preconditioner of the
// learned-versus-plain comparison).
//
// After the FAS mu-cycle has produced z = M r, the residual it leaves on the LEAF tiles of
// the finest level, rho = r - A z, is fed tile by tile to a small network whose output is
// added to z on INTERIOR cells:
//     z_t += (S_t / D_t) * f(features_t)
// features (8 input channels on the 10^3 grid of the tile and its 1-cell border):
//     0: rho / S_t   (S_t = root mean square of rho over the tile's INTERIOR cells)
//     1: INTERIOR flag   2: DIRICHLET flag   3: diagonal of A / D_t (D_t = its maximum)
//     4-6: the -x/-y/-z face coefficients of A / D_t (on cut cells they carry the face
//          fractions of the cut-cell operator)   7: 0
//     border: channel 0 the residual rho / S_t of the neighbour cell across each face and
//     channel 1 a flag for it (INTERIOR cells of same-level LEAF neighbours), 0 elsewhere;
//     the hidden layers are zero-padded
// network: conv3x3x3 8->H, bias, ReLU; conv3x3x3 H->H, bias, ReLU; conv3x3x3 H->1
// (H = 8 or 16).  The target of f is the error the cycle leaves, d = A^-1 rho, scaled
// by D_t / S_t; the network is trained on (rho, d) pairs made by the plain solver.
// The preconditioner is no longer linear, so the solve runs flexible CG (Polak-Ribiere
// beta) and judges its result by the true residual, with the plain solve as fallback.
//
// Every convolution is an implicit GEMM on mma.sync m16n8k16 (BF16 operands, FP32
// accumulation): M = the tile's 512 voxels in 16-voxel fragments (two rows of 8 along
// the innermost axis), N = output channels, K = (tap, input channel).  Activations live
// in shared memory as a zero-padded 10^3 voxel grid, channels innermost (16 bytes per
// 8-channel group); ldmatrix gathers the shifted rows of each tap directly, so no
// im2col buffer exists.  With 16 channels the two 16-byte groups of a voxel swap places
// on voxels whose bit 2 is set, which makes every 8-row ldmatrix phase conflict-free.
// Training uses the same routine for the input gradients (a convolution with the
// flipped, transposed kernel) and a transposed-operand GEMM (ldmatrix .trans) for the
// weight gradients, reduced over the batch in a fixed order and applied by Adam.
#include <cuda_bf16.h>

#include <cmath>
#include <type_traits>

#include "net_common.cuh"

namespace cmg {

namespace {

// element offset of (voxel v, first channel of 8-channel group grp) in an activation buffer of CG groups
template <int CG>
__device__ __forceinline__ int act_off(int v, int grp) {
    if constexpr (CG == 2) return v * 16 + ((grp ^ ((v >> 2) & 1)) << 3);
    else return v * 8;
}

__device__ __forceinline__ void ldsm_x4(uint32_t a, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n" : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(a));
}
__device__ __forceinline__ void ldsm_x2(uint32_t a, uint32_t& r0, uint32_t& r1) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(a));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t a, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n" : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(a));
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t a, uint32_t& r0, uint32_t& r1) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(a));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Convolution of one tile: acc[m][nt] += in (*) w for the 8 M-fragments of this warp.
// in: activations with CGI 8-channel groups; w: packed weights [NTO*8 rows][ks], row = output
// channel, column k = tap*(8*CGI) + channel (CGI == 1: two taps per 16-wide K step, tap 27
// zero-weighted).
template <int CGI, int NTO>
__device__ __forceinline__ void conv_tile(const __nv_bfloat16* in, const __nv_bfloat16* w, int ks, float (&acc)[8][NTO][4]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = lane >> 3, r = lane & 7;
    int vb[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int mt = warp * 8 + m;
        vb[m] = pad_vox(mt >> 2, (mt & 3) * 2 + (q & 1), r);
#pragma unroll
        for (int nt = 0; nt < NTO; ++nt) acc[m][nt][0] = acc[m][nt][1] = acc[m][nt][2] = acc[m][nt][3] = 0.0f;
    }
    const uint32_t in_s = smem_u32(in);
    const uint32_t wrow = NTO == 2 ? smem_u32(w + ((q >> 1) * 8 + r) * ks + (q & 1) * 8) : smem_u32(w + r * ks + (q & 1) * 8);
    constexpr int kSteps = CGI == 2 ? 27 : 14;
#pragma unroll 1
    for (int step = 0; step < kSteps; ++step) {
        uint32_t b[NTO][2];
        if constexpr (NTO == 2) ldsm_x4(wrow + step * 32, b[0][0], b[0][1], b[1][0], b[1][1]);
        else ldsm_x2(wrow + step * 32, b[0][0], b[0][1]);
        int tap, grp;
        if constexpr (CGI == 2) {
            tap = step;
            grp = q >> 1;
        } else {
            tap = 2 * step + (q >> 1);
            if (tap > 26) tap = 13;  // K padding: zero weights, any finite activation
            grp = 0;
        }
        const int off = tap_off(tap);
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            uint32_t a[4];
            ldsm_x4(in_s + 2 * act_off<CGI>(vb[m] + off, grp), a[0], a[1], a[2], a[3]);
#pragma unroll
            for (int nt = 0; nt < NTO; ++nt) mma_bf16(acc[m][nt], a, b[nt][0], b[nt][1]);
        }
    }
}

// Hidden-layer epilogue: forward out = relu(acc + bias); backward out = acc * (ref > 0).
template <int NTO, bool kBwd>
__device__ __forceinline__ void store_hidden(const float (&acc)[8][NTO][4], __nv_bfloat16* out, const __nv_bfloat16* ref,
                                             const float* bias) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int mt = warp * 8 + m;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const int v = pad_vox(mt >> 2, (mt & 3) * 2 + hh, g);
#pragma unroll
            for (int nt = 0; nt < NTO; ++nt) {
                const int c = nt * 8 + 2 * tq;
                const int e = act_off<NTO>(v, nt) + 2 * tq;
                float x0 = acc[m][nt][2 * hh], x1 = acc[m][nt][2 * hh + 1];
                if constexpr (kBwd) {
                    const __nv_bfloat162 rf = *reinterpret_cast<const __nv_bfloat162*>(ref + e);
                    x0 = __bfloat162float(rf.x) > 0.0f ? x0 : 0.0f;
                    x1 = __bfloat162float(rf.y) > 0.0f ? x1 : 0.0f;
                } else {
                    x0 = fmaxf(__fadd_rn(x0, bias[c]), 0.0f);
                    x1 = fmaxf(__fadd_rn(x1, bias[c + 1]), 0.0f);
                }
                *reinterpret_cast<__nv_bfloat162*>(out + e) = __floats2bfloat162_rn(x0, x1);
            }
        }
    }
}

// Output epilogue (one real output channel): ys[cell] = acc column 0.
__device__ __forceinline__ void store_output(const float (&acc)[8][1][4], float* ys) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tq = lane & 3;
    if (tq != 0) return;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int mt = warp * 8 + m;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) ys[(mt >> 2) * 64 + ((mt & 3) * 2 + hh) * 8 + g] = acc[m][0][2 * hh];
    }
}

// Weight gradient of one tile: gw[n][tap][c] = sum over voxels v of a[v + tap][c] * d[v][n],
// as a GEMM with M = (tap, c), N = n, K = voxels (ldmatrix .trans on both operands).
// a: CGA channel groups; d: NTD groups; only the first nout columns are stored.
template <int CGA, int NTD>
__device__ __forceinline__ void wgrad_tile(const __nv_bfloat16* a, const __nv_bfloat16* d, float* __restrict__ gw, int nout) {
    constexpr int kMT = CGA == 2 ? 27 : 14;
    constexpr int kPerWarp = (kMT + 3) / 4;
    constexpr int kCin = 8 * CGA;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = lane >> 3, r = lane & 7, g = lane >> 2, tq = lane & 3;
    float acc[kPerWarp][NTD][4];
#pragma unroll
    for (int mi = 0; mi < kPerWarp; ++mi)
#pragma unroll
        for (int nt = 0; nt < NTD; ++nt) acc[mi][nt][0] = acc[mi][nt][1] = acc[mi][nt][2] = acc[mi][nt][3] = 0.0f;
    int aoff[kPerWarp], agrp[kPerWarp];
#pragma unroll
    for (int mi = 0; mi < kPerWarp; ++mi) {
        const int mt = warp + 4 * mi;
        int tap;
        if constexpr (CGA == 2) {
            tap = mt;
            agrp[mi] = q & 1;
        } else {
            tap = 2 * mt + (q & 1);
            agrp[mi] = 0;
        }
        if (tap > 26) tap = 13;  // padding rows (not stored)
        aoff[mi] = tap_off(tap);
    }
    const uint32_t a_s = smem_u32(a), d_s = smem_u32(d);
#pragma unroll 1
    for (int ks = 0; ks < 32; ++ks) {
        const int i = ks >> 2, j0 = (ks & 3) * 2;
        uint32_t b[NTD][2];
        if constexpr (NTD == 2) {
            const int v = pad_vox(i, j0 + (q & 1), r);
            ldsm_x4_t(d_s + 2 * act_off<2>(v, q >> 1), b[0][0], b[0][1], b[1][0], b[1][1]);
        } else {
            const int v = pad_vox(i, j0 + (q & 1), r);
            ldsm_x2_t(d_s + 2 * act_off<1>(v, 0), b[0][0], b[0][1]);
        }
        const int vb = pad_vox(i, j0 + (q >> 1), r);
#pragma unroll
        for (int mi = 0; mi < kPerWarp; ++mi) {
            if (warp + 4 * mi >= kMT) continue;
            uint32_t af[4];
            ldsm_x4_t(a_s + 2 * act_off<CGA>(vb + aoff[mi], agrp[mi]), af[0], af[1], af[2], af[3]);
#pragma unroll
            for (int nt = 0; nt < NTD; ++nt) mma_bf16(acc[mi][nt], af, b[nt][0], b[nt][1]);
        }
    }
#pragma unroll
    for (int mi = 0; mi < kPerWarp; ++mi) {
        const int mt = warp + 4 * mi;
        if (mt >= kMT) continue;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            int tap, c;
            if constexpr (CGA == 2) {
                tap = mt;
                c = g + 8 * hh;
            } else {
                tap = 2 * mt + hh;
                c = g;
            }
            if (tap > 26) continue;
#pragma unroll
            for (int nt = 0; nt < NTD; ++nt)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int n = nt * 8 + 2 * tq + e;
                    if (n < nout) gw[(n * 27 + tap) * kCin + c] = acc[mi][nt][2 * hh + e];
                }
        }
    }
}

// bias gradient: db[c] = sum over the tile's voxels of d[v][c] (fixed order)
template <int CG>
__device__ __forceinline__ void bias_grad(const __nv_bfloat16* d, float* red, float* __restrict__ gb) {
    constexpr int H = 8 * CG, kParts = kNetThreads / H;
    const int c = threadIdx.x % H, part = threadIdx.x / H;
    float s = 0.0f;
    for (int cell = part; cell < kCells; cell += kParts) {
        const int v = pad_vox(cell >> 6, (cell >> 3) & 7, cell & 7);
        s += __bfloat162float(d[act_off<CG>(v, c >> 3) + (c & 7)]);
    }
    red[part * H + c] = s;
    __syncthreads();
    if (threadIdx.x < H) {
        float t = 0.0f;
        for (int p = 0; p < kParts; ++p) t += red[p * H + threadIdx.x];
        gb[threadIdx.x] = t;
    }
    __syncthreads();
}

template <int H>
struct NetDims {
    static constexpr int CG = H / 8;
    static constexpr int KS1 = 232;                 // 8 input channels: 28 taps x 8 + 8 (odd number of 16-byte rows)
    static constexpr int KSH = CG == 2 ? 440 : 232;  // H input channels
    static constexpr int F1 = 0, F2 = F1 + H * KS1, F3 = F2 + H * KSH, G3 = F3 + 8 * KSH, G2 = G3 + H * KS1;
    static constexpr int kFwd = G3;      // bf16 elements the forward pass needs
    static constexpr int kPack = G2 + H * KSH;
    // fp32 parameters: W1[H][27][8], b1[H], W2[H][27][H], b2[H], W3[27][H]
    static constexpr int W1 = 0, B1 = W1 + H * 216, W2 = B1 + H, B2 = W2 + H * 27 * H, W3 = B2 + H, kParams = W3 + 27 * H;
    static constexpr int kAct8 = kPadVox * 8, kActH = kPadVox * H;  // bf16 elements of the activation buffers
};

template <int H>
__device__ __forceinline__ void copy_weights(__nv_bfloat16* dst, const __nv_bfloat16* src, int n, float* bias, const float* bsrc) {
    for (int i = threadIdx.x; i < n / 8; i += kNetThreads) reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
    if (threadIdx.x < 2 * H) bias[threadIdx.x] = bsrc[threadIdx.x];
}
// Forward pass over samples; out (z) += (S/D) * f on INTERIOR cells, or, with overwrite, out = (S/D) * f.
template <int H>
__global__ void __launch_bounds__(kNetThreads) k_net_forward(NetIn I, int ns, const __nv_bfloat16* __restrict__ pack,
                                                             const float* __restrict__ bias_g, float* __restrict__ out, int overwrite) {
    using Dm = NetDims<H>;
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* x0 = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* a1 = x0 + Dm::kAct8;
    __nv_bfloat16* a2 = a1 + Dm::kActH;
    __nv_bfloat16* wt = a2 + Dm::kActH;
    float* bias = reinterpret_cast<float*>(wt + Dm::kFwd);
    float* ys = bias + 2 * H;
    float* red = ys + kCells;
    zero_smem(smem, 2 * (Dm::kAct8 + 2 * Dm::kActH));
    copy_weights<H>(wt, pack, Dm::kFwd, bias, bias_g);
    __syncthreads();
    for (int s = blockIdx.x; s < ns; s += gridDim.x) {
        const Staged st = stage_features(I, s, x0, red);
        const int t = I.idx ? I.idx[s] : I.t0 + s;
        if (st.S == 0.0f) {
            if (overwrite) st4(out + (size_t)t * kCells + 4 * threadIdx.x, make_float4(0.f, 0.f, 0.f, 0.f));
            continue;  // uniform over the block
        }
        __syncthreads();
        {
            float acc[8][Dm::CG][4];
            conv_tile<1, Dm::CG>(x0, wt + Dm::F1, Dm::KS1, acc);
            store_hidden<Dm::CG, false>(acc, a1, nullptr, bias);
        }
        __syncthreads();
        {
            float acc[8][Dm::CG][4];
            conv_tile<Dm::CG, Dm::CG>(a1, wt + Dm::F2, Dm::KSH, acc);
            store_hidden<Dm::CG, false>(acc, a2, nullptr, bias + H);
        }
        __syncthreads();
        {
            float acc[8][1][4];
            conv_tile<Dm::CG, 1>(a2, wt + Dm::F3, Dm::KSH, acc);
            store_output(acc, ys);
        }
        __syncthreads();
        const float sc = st.S / st.D;
        float* o = out + (size_t)t * kCells + 4 * threadIdx.x;
        float4 z = overwrite ? make_float4(0.f, 0.f, 0.f, 0.f) : ldcg4(o);
        float zz[4] = {z.x, z.y, z.z, z.w};
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (st.in[u]) zz[u] = __fmaf_rn(sc, ys[4 * threadIdx.x + u], zz[u]);
        st4(o, make_float4(zz[0], zz[1], zz[2], zz[3]));
        __syncthreads();  // ys and x0 are rewritten by the next sample
    }
}

// ---------------------------------------------------------------------------
// Inference on the 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM)
// ---------------------------------------------------------------------------
// Activations are channel-group-major planes: element (voxel v, channel c) of a buffer with
// CG groups sits at ((c >> 3) * kTcVox + v) * 8 + (c & 7), 16 bytes per voxel and group.  In
// the no-swizzle K-major operand layout the 8-voxel rows of the padded grid are core matrices
// (128 contiguous bytes) that follow one another 10 voxels (160 B) apart through the planes
// (the stride-dimension offset): row R = 10 i + j, j = 0..9.  One M = 128 MMA takes 16
// consecutive rows against N output channels for one 16-wide K step, so 5 MMAs (tiles m =
// 0..4, rows 16m..16m+15) cover the tile's 80 rows; the rows j = 8, 9 are border rows of the
// padded grid, computed and never stored.  The two K halves are the two channel groups
// (kTcVox voxels apart) or, with 8 input channels, the next tap (the leading-dimension
// offset).  A tap's shifted operand is therefore only a different start address: no im2col.
// Weights are stored per K step as [K half][n][8] (core matrices of 8 output channels).
// The accumulator of tile m occupies TMEM columns m*N .. m*N+N-1, row r in lane r.
constexpr int kTcTiles = 5;
__device__ int g_net_tc_error;  // set when an MMA completion wait gives up

template <int H>
struct TcDims {
    static constexpr int CG = H / 8;
    static constexpr int S1 = 14, SH = CG == 2 ? 27 : 14;  // K steps of 16
    static constexpr int W1 = 0, W2 = W1 + S1 * 2 * H * 8, W3 = W2 + SH * 2 * H * 8, kW = W3 + SH * 2 * 8 * 8;  // bf16 elements
    static constexpr int kAct = kTcVox * H;
    static constexpr int kCols = H == 16 ? 128 : 64;  // TMEM columns: 5 tiles x N, rounded up to a power of 2
    // shared memory: a1 | x0 and a2 in the same place (x0 is dead once layer 1 has run) | weights
    static constexpr int kActElems = 2 * kAct;
};

// Issue one layer (thread 0): for each i-plane p and K step s, D[p] (+)= A(p, s) B(s).
// CGI: 8-channel groups of the input; N: output columns; steps: K steps of 16.
template <int CGI, int N>
__device__ __forceinline__ void tc_issue_layer(uint32_t in_s, uint32_t w_s, int steps, uint32_t taddr) {
    constexpr uint32_t idesc = (umma_idesc(N) & ~(0x1Fu << 24)) | (8u << 24);  // M = 128
    // descriptors as a base plus the start-address offset in 16-byte units (the low field;
    // shared addresses stay below 256 KB, so nothing carries into the other fields)
    const uint64_t a_base = umma_desc(in_s + (uint32_t)pad_vox(0, 0, 0) * 16u, CGI == 2 ? kTcVox * 16 : 16u, 160u);
    const uint64_t b_base = umma_desc(w_s, N * 16, 128);
#pragma unroll 1
    for (int st = 0; st < steps; ++st) {  // K outer, tiles inner: 5 independent accumulators in flight
        uint64_t a;
        if constexpr (CGI == 2) {
            a = a_base + (uint64_t)(int64_t)tap_off(st);
        } else {  // tap 27: zero weights
            const int t0 = 2 * st;
            const int lbo = t0 + 1 <= 26 ? tap_off(t0 + 1) - tap_off(t0) : 1;
            a = (a_base & ~(0x3FFFull << 16)) + ((uint64_t)lbo << 16) + (uint64_t)(int64_t)tap_off(t0);
        }
        const uint64_t b = b_base + (uint64_t)(st * (2 * N * 8 * 2 / 16));
        const uint32_t acc = st > 0 ? 1u : 0u;
#pragma unroll
        for (int m = 0; m < kTcTiles; ++m) umma_f16(taddr + (uint32_t)(m * N), a + (uint64_t)(m * 160), b, idesc, acc);
    }
}

// voxel of TMEM lane `row` of tile m (-1: a border row of the padded grid, not stored)
__device__ __forceinline__ int tc_tile_voxel(int m, int row) {
    const int R = 16 * m + (row >> 3), i = R / 10, j = R - 10 * i;
    return j < 8 ? pad_vox(i, j, row & 7) : -1;
}

// Hidden-layer epilogue from TMEM: all eight planes' accumulators loaded before one wait, then
// relu(acc + bias) to BF16 into the channel-group-major buffer out (rows 16w..16w+15 of each
// plane, held by lanes 0-15 of warp w).
template <int H>
__device__ __forceinline__ void tc_epilogue_hidden(uint32_t lane_base, int warp, int lane, const float* bias, __nv_bfloat16* out) {
    constexpr int CG = H / 8;
    float v[kTcTiles][H];
#pragma unroll
    for (int m = 0; m < kTcTiles; ++m) {
        if constexpr (H == 16) tmem_ld16(lane_base + m * H, v[m]);
        else tmem_ld8(lane_base + m * H, v[m]);
    }
    tmem_wait_ld();
#pragma unroll
    for (int m = 0; m < kTcTiles; ++m) {
        const int vx = tc_tile_voxel(m, 32 * warp + lane);
        if (vx < 0) continue;
#pragma unroll
        for (int g = 0; g < CG; ++g) {
            __nv_bfloat162 o[4];
#pragma unroll
            for (int e = 0; e < 4; ++e)
                o[e] = __floats2bfloat162_rn(fmaxf(__fadd_rn(v[m][8 * g + 2 * e], bias[8 * g + 2 * e]), 0.0f),
                                             fmaxf(__fadd_rn(v[m][8 * g + 2 * e + 1], bias[8 * g + 2 * e + 1]), 0.0f));
            *reinterpret_cast<uint4*>(out + (g * kTcVox + vx) * 8) = *reinterpret_cast<const uint4*>(o);
        }
    }
}

template <int H>
__global__ void __launch_bounds__(kNetThreads) k_net_forward_tc(NetIn I, int ns, const __nv_bfloat16* __restrict__ pack,
                                                                const float* __restrict__ bias_g, float* __restrict__ out, int overwrite) {
    using Dm = NetDims<H>;
    using Tc = TcDims<H>;
    constexpr int CG = Tc::CG;
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* a1 = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* x0 = a1 + Tc::kAct;
    __nv_bfloat16* a2 = x0;  // group 0 of a2 covers x0 exactly; both keep zero halos
    __nv_bfloat16* wt = a2 + Tc::kAct;
    float* bias = reinterpret_cast<float*>(wt + Tc::kW);
    float* ys = bias + 2 * H;
    float* red = ys + kCells;                                          // 32 floats
    unsigned long long* mbar = reinterpret_cast<unsigned long long*>(red + 32);  // 8-byte aligned
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    zero_smem(smem, 2 * Tc::kActElems);
    // weights: [step][K half][n][8] from the packed [n][k] rows (k = step*16 + half*8 + c)
    for (int e = tid; e < Tc::kW; e += kNetThreads) {
        int base, n_rows, ks, src0, rel = e;
        if (e < Tc::W2) {
            base = Tc::W1, n_rows = H, ks = Dm::KS1, src0 = Dm::F1;
        } else if (e < Tc::W3) {
            base = Tc::W2, n_rows = H, ks = Dm::KSH, src0 = Dm::F2;
        } else {
            base = Tc::W3, n_rows = 8, ks = Dm::KSH, src0 = Dm::F3;
        }
        rel = e - base;
        const int c = rel & 7, n = (rel >> 3) % n_rows, hs = (rel >> 3) / n_rows, half = hs & 1, stp = hs >> 1;
        wt[e] = pack[src0 + n * ks + stp * 16 + half * 8 + c];
    }
    if (tid < 2 * H) bias[tid] = bias_g[tid];
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(Tc::kCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *tslot;
    const uint32_t mb = smem_u32(mbar);
    const uint32_t lane_base = taddr + ((uint32_t)(32 * warp) << 16);
    uint32_t phase = 0;
    bool ok = true;

    // one layer: issue, wait, read the accumulators of this warp's rows
    auto run_layer = [&](auto cgi_tag, auto n_tag, uint32_t in_s, uint32_t w_s, int steps) -> bool {
        constexpr int CGI = decltype(cgi_tag)::value, N = decltype(n_tag)::value;
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            tc_issue_layer<CGI, N>(in_s, w_s, steps, taddr);
            umma_commit(mb);
        }
        const bool done = mbar_wait(mb, phase);
        phase ^= 1u;
        tc_fence_after();
        return __syncthreads_and(done ? 1 : 0) != 0;
    };

    for (int s = blockIdx.x; s < ns && ok; s += gridDim.x) {
        const Staged st = stage_features(I, s, x0, red);
        const int t = I.idx ? I.idx[s] : I.t0 + s;
        if (st.S == 0.0f) {
            if (overwrite) st4(out + (size_t)t * kCells + 4 * tid, make_float4(0.f, 0.f, 0.f, 0.f));
            continue;  // uniform over the block
        }
        // layer 1: x0 (8 channels) -> a1
        ok = run_layer(std::integral_constant<int, 1>{}, std::integral_constant<int, H>{}, smem_u32(x0), smem_u32(wt + Tc::W1), Tc::S1);
        if (!ok) break;
        // x0 doubles as group 0 of a2, whose halo must be zero for layer 3
        if (I.ex.halo || I.ex.nbx) clear_face_halo(x0);
        tc_epilogue_hidden<H>(lane_base, warp, lane, bias, a1);
        // layer 2: a1 -> a2
        ok = run_layer(std::integral_constant<int, CG>{}, std::integral_constant<int, H>{}, smem_u32(a1), smem_u32(wt + Tc::W2), Tc::SH);
        if (!ok) break;
        tc_epilogue_hidden<H>(lane_base, warp, lane, bias + H, a2);
        // layer 3: a2 -> one channel (N = 8, column 0)
        ok = run_layer(std::integral_constant<int, CG>{}, std::integral_constant<int, 8>{}, smem_u32(a2), smem_u32(wt + Tc::W3), Tc::SH);
        if (!ok) break;
        {
            float v[kTcTiles][8];
#pragma unroll
            for (int m = 0; m < kTcTiles; ++m) tmem_ld8(lane_base + m * 8, v[m]);
            tmem_wait_ld();
#pragma unroll
            for (int m = 0; m < kTcTiles; ++m) {
                const int R = 16 * m + ((32 * warp + lane) >> 3), i = R / 10, j = R - 10 * i;
                if (j < 8) ys[i * 64 + j * 8 + (lane & 7)] = v[m][0];
            }
        }
        tc_fence_before();
        __syncthreads();
        const float sc = st.S / st.D;
        float* o = out + (size_t)t * kCells + 4 * tid;
        float4 z = overwrite ? make_float4(0.f, 0.f, 0.f, 0.f) : ldcg4(o);
        float zz[4] = {z.x, z.y, z.z, z.w};
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (st.in[u]) zz[u] = __fmaf_rn(sc, ys[4 * tid + u], zz[u]);
        st4(o, make_float4(zz[0], zz[1], zz[2], zz[3]));
        __syncthreads();  // ys and x0 are rewritten by the next sample
    }
    if (!ok) {
        if (tid == 0) atomicExch(&g_net_tc_error, 1);
        mbar_wait(mb, phase ^ 1u);  // the outstanding phase, bounded
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(Tc::kCols) : "memory");
}

// Forward and backward pass of one batch: per batch slot b (sample idx[b]) the gradient of the
// tile's loss (sum over INTERIOR cells of (f - target * D/S)^2, or its energy form, see below)
// goes to grad[b][kParams] and the loss to loss[b].
template <int H>
__global__ void __launch_bounds__(kNetThreads) k_net_train(NetIn I, int nb, const __nv_bfloat16* __restrict__ pack,
                                                           const float* __restrict__ bias_g, float* __restrict__ grad,
                                                           float* __restrict__ loss, int loss_kind) {
    using Dm = NetDims<H>;
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* x0 = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* dy = x0 + Dm::kAct8;
    __nv_bfloat16* a1 = dy + Dm::kAct8;
    __nv_bfloat16* a2 = a1 + Dm::kActH;  // later dz1
    __nv_bfloat16* dz2 = a2 + Dm::kActH;
    __nv_bfloat16* wt = dz2 + Dm::kActH;
    float* bias = reinterpret_cast<float*>(wt + Dm::kPack);
    float* ys = bias + 2 * H;
    float* red = ys + kCells;  // 128 floats
    zero_smem(smem, 2 * (2 * Dm::kAct8 + 3 * Dm::kActH));
    copy_weights<H>(wt, pack, Dm::kPack, bias, bias_g);
    __syncthreads();
    for (int b = blockIdx.x; b < nb; b += gridDim.x) {
        float* gw = grad + (size_t)b * Dm::kParams;
        const Staged st = stage_features(I, b, x0, red);
        if (st.S == 0.0f) {
            for (int p = threadIdx.x; p < Dm::kParams; p += kNetThreads) gw[p] = 0.0f;
            if (threadIdx.x == 0) loss[b] = 0.0f;
            continue;
        }
        __syncthreads();
        {
            float acc[8][Dm::CG][4];
            conv_tile<1, Dm::CG>(x0, wt + Dm::F1, Dm::KS1, acc);
            store_hidden<Dm::CG, false>(acc, a1, nullptr, bias);
        }
        __syncthreads();
        {
            float acc[8][Dm::CG][4];
            conv_tile<Dm::CG, Dm::CG>(a1, wt + Dm::F2, Dm::KSH, acc);
            store_hidden<Dm::CG, false>(acc, a2, nullptr, bias + H);
        }
        __syncthreads();
        {
            float acc[8][1][4];
            conv_tile<Dm::CG, 1>(a2, wt + Dm::F3, Dm::KSH, acc);
            store_output(acc, ys);
        }
        __syncthreads();
        float g[4];
        const float l = tile_loss_grad(st, ys, loss_kind, g);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int cell = 4 * threadIdx.x + u;
            dy[pad_vox(cell >> 6, (cell >> 3) & 7, cell & 7) * 8] = __float2bfloat16_rn(2.0f * g[u]);
        }
        const float lt = block_sum_f(l, red);  // synchronises: dy is complete
        if (threadIdx.x == 0) loss[b] = lt;
        wgrad_tile<Dm::CG, 1>(a2, dy, gw + Dm::W3, 1);  // W3[tap][c] as [n = 0][tap][c]
        {
            float acc[8][Dm::CG][4];
            conv_tile<1, Dm::CG>(dy, wt + Dm::G3, Dm::KS1, acc);
            store_hidden<Dm::CG, true>(acc, dz2, a2, nullptr);
        }
        __syncthreads();
        wgrad_tile<Dm::CG, Dm::CG>(a1, dz2, gw + Dm::W2, H);
        bias_grad<Dm::CG>(dz2, red, gw + Dm::B2);
        {
            float acc[8][Dm::CG][4];
            conv_tile<Dm::CG, Dm::CG>(dz2, wt + Dm::G2, Dm::KSH, acc);
            store_hidden<Dm::CG, true>(acc, a2, a1, nullptr);  // dz1 over a2
        }
        __syncthreads();
        wgrad_tile<1, Dm::CG>(x0, a2, gw + Dm::W1, H);
        bias_grad<Dm::CG>(a2, red, gw + Dm::B1);
        // bias_grad ends with a barrier: the buffers may be rewritten by the next sample
    }
}

// fp32 parameters -> packed bf16 operands (forward F1..F3, flipped/transposed G3, G2) and biases
template <int H>
__global__ void k_net_pack(const float* __restrict__ p, __nv_bfloat16* __restrict__ pack, float* __restrict__ bias) {
    using Dm = NetDims<H>;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < 2 * H) bias[e] = e < H ? p[Dm::B1 + e] : p[Dm::B2 + e - H];
    if (e >= Dm::kPack) return;
    float v = 0.0f;
    if (e < Dm::F2) {  // F1[n][tap*8 + c]
        const int n = e / Dm::KS1, k = e % Dm::KS1, tap = k / 8, c = k % 8;
        if (tap < 27) v = p[Dm::W1 + (n * 27 + tap) * 8 + c];
    } else if (e < Dm::F3) {  // F2[n][tap*H + c]
        const int n = (e - Dm::F2) / Dm::KSH, k = (e - Dm::F2) % Dm::KSH, tap = k / H, c = k % H;
        if (tap < 27) v = p[Dm::W2 + (n * 27 + tap) * H + c];
    } else if (e < Dm::G3) {  // F3[n][tap*H + c], row 0 only
        const int n = (e - Dm::F3) / Dm::KSH, k = (e - Dm::F3) % Dm::KSH, tap = k / H, c = k % H;
        if (n == 0 && tap < 27) v = p[Dm::W3 + tap * H + c];
    } else if (e < Dm::G2) {  // G3[h][tap'*8 + c] = W3[26 - tap'][h] for c = 0
        const int h = (e - Dm::G3) / Dm::KS1, k = (e - Dm::G3) % Dm::KS1, tap = k / 8, c = k % 8;
        if (c == 0 && tap < 27) v = p[Dm::W3 + (26 - tap) * H + h];
    } else {  // G2[cin][tap'*H + cout] = W2[cout][26 - tap'][cin]
        const int ci = (e - Dm::G2) / Dm::KSH, k = (e - Dm::G2) % Dm::KSH, tap = k / H, co = k % H;
        if (tap < 27) v = p[Dm::W2 + (co * 27 + (26 - tap)) * H + ci];
    }
    pack[e] = __float2bfloat16_rn(v);
}

// Sum the batch's gradients in slot order (scaled), optionally store them, then one Adam step.
__global__ void k_net_reduce_adam(const float* __restrict__ grad, int nb, int np, float scale, float* __restrict__ gout,
                                  float* __restrict__ p, float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2,
                                  float bc1, float bc2, int update) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= np) return;
    float g = 0.0f;
    for (int b = 0; b < nb; ++b) g += grad[(size_t)b * np + e];
    g *= scale;
    if (gout) gout[e] = g;
    if (!update) return;
    const float mm = b1 * m[e] + (1.0f - b1) * g, vv = b2 * v[e] + (1.0f - b2) * g * g;
    m[e] = mm;
    v[e] = vv;
    p[e] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + 1e-8f);
}

template <int H>
size_t forward_smem() {
    using Dm = NetDims<H>;
    return 2 * (size_t)(Dm::kAct8 + 2 * Dm::kActH + Dm::kFwd) + sizeof(float) * (2 * H + kCells + 32);
}
template <int H>
size_t train_smem() {
    using Dm = NetDims<H>;
    return 2 * (size_t)(2 * Dm::kAct8 + 3 * Dm::kActH + Dm::kPack) + sizeof(float) * (2 * H + kCells + kNetThreads);
}

template <int H>
size_t forward_tc_smem() {
    using Tc = TcDims<H>;
    return 2 * (size_t)(Tc::kActElems + Tc::kW) + sizeof(float) * (2 * H + kCells + 32) + 16;
}

int g_fwd_blocks[2] = {0, 0};     // resident forward blocks per SM (H = 8, 16), mma.sync kernel
int g_fwd_tc_blocks[2] = {0, 0};  // the same for the tcgen05 kernel
int g_infer_kind = 0;             // 0: mma.sync inference kernel (measured faster at N = 8), 1: tcgen05

}  // namespace

int net_params(int H) { return H == 32 ? deep_params() : H == 16 ? NetDims<16>::kParams : NetDims<8>::kParams; }
int net_pack_elems(int H) { return H == 32 ? deep_pack_elems() : H == 16 ? NetDims<16>::kPack : NetDims<8>::kPack; }
int net_bias_elems(int H) { return H == 32 ? deep_bias_elems() : 2 * H; }
int net_train_rows(int H, int nb) { return H == 32 ? deep_train_blocks(nb) : nb; }
size_t net_train_scratch_bytes(int H, int nb) { return H == 32 ? deep_scratch_bytes() * (size_t)deep_train_blocks(nb) : 0; }

bool net_init() {
    bool ok = true;
    ok = ok && cudaFuncSetAttribute(k_net_forward<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)forward_smem<8>()) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(k_net_forward<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)forward_smem<16>()) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(k_net_train<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem<8>()) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(k_net_train<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem<16>()) == cudaSuccess;
    if (!ok) return false;
    ok = ok && cudaFuncSetAttribute(k_net_forward_tc<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)forward_tc_smem<8>()) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(k_net_forward_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)forward_tc_smem<16>()) == cudaSuccess;
    if (!ok) return false;
    ok = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_fwd_blocks[0], k_net_forward<8>, kNetThreads, forward_smem<8>()) == cudaSuccess &&
         cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_fwd_blocks[1], k_net_forward<16>, kNetThreads, forward_smem<16>()) == cudaSuccess &&
         cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_fwd_tc_blocks[0], k_net_forward_tc<8>, kNetThreads, forward_tc_smem<8>()) ==
             cudaSuccess &&
         cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_fwd_tc_blocks[1], k_net_forward_tc<16>, kNetThreads, forward_tc_smem<16>()) ==
             cudaSuccess;
    // each resident tcgen05 block holds 64 or 128 of the SM's 512 TMEM columns
    if (g_fwd_tc_blocks[0] > 8) g_fwd_tc_blocks[0] = 8;
    if (g_fwd_tc_blocks[1] > 4) g_fwd_tc_blocks[1] = 4;
    return ok && g_fwd_blocks[0] > 0 && g_fwd_blocks[1] > 0 && g_fwd_tc_blocks[0] > 0 && g_fwd_tc_blocks[1] > 0;
}

static int num_sms() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

void launch_net_pack(int H, const float* params, void* pack, float* bias, cudaStream_t st) {
    if (H == 32) {
        launch_deep_pack(params, pack, bias, st);
        return;
    }
    const int n = net_pack_elems(H);
    note_kernel_launch();
    if (H == 16) k_net_pack<16><<<(n + 255) / 256, 256, 0, st>>>(params, (__nv_bfloat16*)pack, bias);
    else k_net_pack<8><<<(n + 255) / 256, 256, 0, st>>>(params, (__nv_bfloat16*)pack, bias);
}

void launch_net_forward(int H, const float* r, const float* az, const float* diag, const uint8_t* types, const int* idx, int t0, int ns,
                        const void* pack, const float* bias, float* out, bool overwrite, cudaStream_t st, const NetExtra& ex) {
    if (ns <= 0) return;
    if (H == 32) {
        launch_deep_forward(r, az, diag, types, idx, t0, ns, pack, bias, out, overwrite, st, ex);
        return;
    }
    const NetIn I{r, az, diag, types, nullptr, idx, t0, ex};
    if (g_infer_kind == 1) {
        // resident blocks per SM from shared memory (1 KB reserved per block) and TMEM (512 columns)
        int dev = 0, smem_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        const size_t per = (H == 16 ? forward_tc_smem<16>() : forward_tc_smem<8>()) + 1024;
        int per_sm = (int)((size_t)smem_sm / per);
        const int tmem_cap = 512 / (H == 16 ? TcDims<16>::kCols : TcDims<8>::kCols);
        if (per_sm > tmem_cap) per_sm = tmem_cap;
        if (per_sm < 1) per_sm = 1;
        const int cap = num_sms() * per_sm;
        const int blocks = ns < cap ? ns : cap;
        note_kernel_launch();
        if (H == 16)
            k_net_forward_tc<16><<<blocks, kNetThreads, forward_tc_smem<16>(), st>>>(I, ns, (const __nv_bfloat16*)pack, bias, out, overwrite);
        else
            k_net_forward_tc<8><<<blocks, kNetThreads, forward_tc_smem<8>(), st>>>(I, ns, (const __nv_bfloat16*)pack, bias, out, overwrite);
        return;
    }
    const int cap = num_sms() * g_fwd_blocks[H == 16 ? 1 : 0];
    const int blocks = ns < cap ? ns : cap;
    note_kernel_launch();
    if (H == 16)
        k_net_forward<16><<<blocks, kNetThreads, forward_smem<16>(), st>>>(I, ns, (const __nv_bfloat16*)pack, bias, out, overwrite);
    else
        k_net_forward<8><<<blocks, kNetThreads, forward_smem<8>(), st>>>(I, ns, (const __nv_bfloat16*)pack, bias, out, overwrite);
}

void net_set_inference_kind(int kind) { g_infer_kind = kind; }
int net_inference_kind() { return g_infer_kind; }
// 1 if a tcgen05 inference launch gave up waiting for its MMAs since the last call (and clears it)
int net_take_tc_error() {
    int v = 0, z = 0;
    if (cudaMemcpyFromSymbol(&v, g_net_tc_error, sizeof(int)) != cudaSuccess) return -1;
    if (v) cudaMemcpyToSymbol(g_net_tc_error, &z, sizeof(int));
    const int d = deep_take_error();
    return d < 0 ? -1 : (v | d);
}

void launch_net_train(int H, const float* rho, const float* diag, const uint8_t* types, const float* target, const int* idx, int nb,
                      const void* pack, const float* bias, float* grad, float* loss, int loss_kind, cudaStream_t st, const NetExtra& ex,
                      void* scratch) {
    if (nb <= 0) return;
    if (H == 32) {
        launch_deep_train(rho, diag, types, target, idx, nb, pack, bias, grad, loss, loss_kind, st, ex, scratch);
        return;
    }
    const NetIn I{rho, nullptr, diag, types, target, idx, 0, ex};
    const int sms = num_sms();
    const int blocks = nb < sms ? nb : sms;
    note_kernel_launch();
    if (H == 16)
        k_net_train<16><<<blocks, kNetThreads, train_smem<16>(), st>>>(I, nb, (const __nv_bfloat16*)pack, bias, grad, loss, loss_kind);
    else
        k_net_train<8><<<blocks, kNetThreads, train_smem<8>(), st>>>(I, nb, (const __nv_bfloat16*)pack, bias, grad, loss, loss_kind);
}

void launch_net_reduce_adam(const float* grad, int nb, int np, float scale, float* gout, float* p, float* m, float* v, float lr, int step,
                            bool update, cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = update ? 1.0f - (float)std::pow(0.9, step) : 1.0f, bc2 = update ? 1.0f - (float)std::pow(0.999, step) : 1.0f;
    note_kernel_launch();
    k_net_reduce_adam<<<(np + 255) / 256, 256, 0, st>>>(grad, nb, np, scale, gout, p, m, v, lr, b1, b2, bc1, bc2, update ? 1 : 0);
}

}  // namespace cmg
