// The learned finest-level smoother's residual network (hidden = 32) on the 5th-generation
// tensor cores: inference and training (forward and backward) as tcgen05 implicit GEMMs.
//
// network on the 10^3 feature grid of a tile (the same features as the small nets):
//     X0 = relu(conv(x0, W0) + b0)                                  8 -> 32 channels
//     block k = 0..3: H_k = relu(conv(X_k, Wa_k) + ba_k)            32 -> 32
//                     X_k+1 = relu(X_k + conv(H_k, Wb_k) + bb_k)    32 -> 32
//     f = conv(X_4, Wo)                                             32 -> 1
// Every convolution is 3x3x3 over the tile (hidden layers zero-padded at its border), BF16
// operands (weights, x0, X_k, H_k and the back-propagated gradients that enter a
// convolution) and FP32 accumulation in TMEM.
//
// One CTA of 128 threads per SM (194 KB of shared memory) loops over tiles.  Activations
// are channel-group-major planes, element (voxel v, channel c) at ((c >> 3) * kTcVox + v)
// * 8 + (c & 7): 16 bytes per voxel and 8-channel group, the padded 10^3 voxel grid.
//   * A convolution is five M = 128 MMAs per 16-wide K step: K-major A operand straight from
//     the activation buffer (the 8-voxel rows are 128-byte core matrices 160 B apart through
//     the padded grid's planes, 16 of them per MMA, the two border rows of each plane
//     computed and discarded; the K halves are channel groups or, with 8 input channels, the
//     next tap), so a tap's shifted operand is only a start address (no im2col).  Weights
//     per K step as [K half][n][8].  The five tiles' FP32 accumulators (N = 32 columns
//     each) sit side by side in TMEM.
//   * The weights of each convolution (55 KB) stream into one shared buffer with a bulk
//     copy (cp.async.bulk onto an mbarrier) as soon as the previous convolution's MMAs have
//     completed, overlapping the epilogue.
//   * A weight gradient dW[t][n][c] = sum over voxels v of d[v][n] a[v + off(t)][c] is an
//     MMA with K = voxels: both operands MN-major from the same buffers (8 channels of one
//     voxel are 16 contiguous bytes, 8 voxels of a row a 128-byte core matrix, the next
//     row 160 B on: the leading-dimension offset of the no-swizzle MN-major layout; the
//     next channel group one plane on: its stride offset).  With 32 channels M = 64 holds 32
//     real rows (the other 32 read the next 64 KB of shared memory and are never stored);
//     each tap's N = 32 columns accumulate over the tile's 32 K steps, 16 taps per pass of
//     the 512 TMEM columns.
//   * Training keeps x0, X_0..X_3 and H_0..H_3 of the current tile in a per-CTA scratch
//     area in global memory (L2-resident) for the backward pass, and adds each tile's
//     weight and bias gradients to the CTA's own FP32 row of the gradient buffer in a fixed
//     order; the rows are then summed in block order by the Adam kernel.
// Every mbarrier wait is bounded; a wait that gives up sets an error flag that the host
// reads (net_take_tc_error) and the kernel returns after a bounded wait for its copies.
#include <cmath>

#include "net_common.cuh"

namespace cmg {

namespace {

constexpr int kDC = 32;                // hidden channels
constexpr int kDBlk = 4;               // residual blocks
constexpr int kGrpB = kTcVox * 16;     // bytes of one 8-channel group plane
constexpr int kBufB = 4 * kGrpB;       // bytes of a 32-channel activation buffer
// packed bf16 operands [K step][K half][n][8]
constexpr int kWs8 = 14 * 2 * kDC * 8;   // 8 input channels (two taps per K step), N = 32
constexpr int kWs32 = 54 * 2 * kDC * 8;  // 32 input channels (two K steps per tap), N = 32
constexpr int kWsO = 54 * 2 * 8 * 8;     // 32 input channels, N = 8 (the output conv, column 0)
// pack segments: forward F0, FA_k, FB_k, FO; backward (flipped, transposed) GO, GA_k, GB_k
constexpr int kPF0 = 0;
__host__ __device__ constexpr int pFA(int k) { return kWs8 + 2 * k * kWs32; }
__host__ __device__ constexpr int pFB(int k) { return pFA(k) + kWs32; }
constexpr int kPFO = kWs8 + 2 * kDBlk * kWs32;
constexpr int kPGO = kPFO + kWsO;
__host__ __device__ constexpr int pGA(int k) { return kPGO + kWs8 + 2 * k * kWs32; }
__host__ __device__ constexpr int pGB(int k) { return pGA(k) + kWs32; }
constexpr int kDPack = kPGO + kWs8 + 2 * kDBlk * kWs32;
// fp32 parameters: W0[32][27][8], b0[32], per block Wa[32][27][32], ba[32], Wb[32][27][32],
// bb[32], then Wo[27][32]
constexpr int kQW0 = 0, kQB0 = kDC * 216;
constexpr int kQBlk = 2 * kDC * 27 * kDC + 2 * kDC;
__host__ __device__ constexpr int qWa(int k) { return kQB0 + kDC + k * kQBlk; }
__host__ __device__ constexpr int qBa(int k) { return qWa(k) + kDC * 27 * kDC; }
__host__ __device__ constexpr int qWb(int k) { return qBa(k) + kDC; }
__host__ __device__ constexpr int qBb(int k) { return qWb(k) + kDC * 27 * kDC; }
constexpr int kQWO = kQB0 + kDC + kDBlk * kQBlk;
constexpr int kDParams = kQWO + 27 * kDC;
// biases in shared memory: b0, then ba_k, bb_k per block
constexpr int kDBias = (1 + 2 * kDBlk) * kDC;
__host__ __device__ constexpr int bA(int k) { return kDC + 2 * kDC * k; }
__host__ __device__ constexpr int bB(int k) { return bA(k) + kDC; }

// shared memory (bytes): activation buffers P0, P1, weights, then the small arrays
constexpr int kOffP1 = kBufB, kOffW = 2 * kBufB, kOffBias = kOffW + kWs32 * 2;
constexpr int kOffYs = kOffBias + kDBias * 4, kOffRed = kOffYs + kCells * 4, kOffMbar = kOffRed + 128 * 4, kOffSlot = kOffMbar + 32;
// An MN-major A operand of a weight-gradient MMA starts at most 871 voxels into its buffer
// (plus a tap shift of 111) and spans 8 group planes: the allocation covers that from P1.
constexpr int kDWgradSpan = (871 + 111) * 16 + 7 * kGrpB + 160 + 128;
constexpr int kDSmem = (kOffP1 + kDWgradSpan > kOffSlot + 16 ? kOffP1 + kDWgradSpan : kOffSlot + 16) + 128;
static_assert(kOffSlot + 16 <= kDSmem && kDSmem <= 227 * 1024, "residual net: shared memory");
// per-CTA scratch (bytes): x0 (one group plane), X_0..X_3, H_0..H_3, the spilled gradient
__host__ __device__ constexpr size_t kScrX(int k) { return (size_t)kGrpB + (size_t)k * kBufB; }
__host__ __device__ constexpr size_t kScrH(int k) { return (size_t)kGrpB + (size_t)(kDBlk + k) * kBufB; }
constexpr size_t kScrG = (size_t)kGrpB + (size_t)(2 * kDBlk) * kBufB;
constexpr size_t kScrBytes = kScrG + kBufB;

__device__ int g_deep_error;  // set when an mbarrier wait gives up

constexpr int kConvTiles = 5;  // M = 128 tiles of a convolution (rows R = 0..79)
// kind::f16, M = 128, both operands K-major (the convolutions)
__host__ __device__ constexpr uint32_t umma_idesc_m128(int N) { return (umma_idesc(N) & ~(0x1Fu << 24)) | (8u << 24); }
// kind::f16, M = 64, both operands MN-major (the weight-gradient MMAs)
__host__ __device__ constexpr uint32_t umma_idesc_mn(int N) { return umma_idesc(N) | (1u << 15) | (1u << 16); }

__device__ __forceinline__ void bulk_expect(uint32_t mb, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t mb) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst), "l"(src), "r"(bytes),
                 "r"(mb)
                 : "memory");
}
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// Convolution (thread 0): D[tile m] (+)= A(m, step) B(step) for the 5 row tiles.
// CGI = 4: 54 K steps (tap, channel-group pair); CGI = 1: 14 steps of two taps (tap 27 zero).
// M = 128: the 8-voxel rows of the padded grid follow one another 10 voxels (160 B) apart
// through the planes, row R = 10 i + j for j = 0..9, so 16 consecutive rows are one operand;
// tile m holds rows 16m..16m+15, and the rows j = 8, 9 (the border rows of the padded grid)
// are computed and never stored.  80 rows in 5 MMAs instead of 64 in 8 M = 64 MMAs: the
// per-instruction cost of these small MMAs, not their arithmetic, bounds a convolution.
// A descriptor's start address is its low 14 bits in 16-byte units, so each MMA's operand
// descriptor is a base descriptor plus an offset (no field can carry: shared addresses stay
// below 256 KB); the issuing thread spends a couple of instructions per MMA.
template <int CGI, int N>
__device__ __forceinline__ void dc_issue_conv(uint32_t in_s, uint32_t w_s, uint32_t taddr) {
    constexpr int kSteps = CGI == 4 ? 54 : 14;
    constexpr uint32_t idesc = umma_idesc_m128(N);
    const uint64_t a_base = umma_desc(in_s + (uint32_t)pad_vox(0, 0, 0) * 16u, CGI == 4 ? kGrpB : 16u, 160u);
    const uint64_t b_base = umma_desc(w_s, N * 16, 128);
#pragma unroll 1
    for (int st = 0; st < kSteps; ++st) {
        uint64_t a;
        if constexpr (CGI == 4) {
            a = a_base + (uint64_t)(int64_t)((st & 1) * 2 * kTcVox + tap_off(st >> 1));
        } else {  // the leading-dimension offset is the distance to the step's second tap
            const int t0 = 2 * st;
            const int lbo = t0 + 1 <= 26 ? tap_off(t0 + 1) - tap_off(t0) : 1;
            a = (a_base & ~(0x3FFFull << 16)) + ((uint64_t)lbo << 16) + (uint64_t)(int64_t)tap_off(t0);
        }
        const uint64_t b = b_base + (uint64_t)(st * (2 * N * 8 * 2 / 16));
        const uint32_t acc = st > 0 ? 1u : 0u;
#pragma unroll
        for (int m = 0; m < kConvTiles; ++m) umma_f16(taddr + (uint32_t)(m * N), a + (uint64_t)(m * 160), b, idesc, acc);
    }
}

// Weight gradient (thread 0), taps T0..T1-1 into TMEM columns (t - T0) * N: K steps of 16
// voxels (rows j0, j0 + 1 of plane i), the tap's shift on the A (kShiftA) or the B operand.
// The no-swizzle MN-major layout: leading-dimension offset = the K-direction core stride
// (the next 8-voxel row, 160 B), stride offset = the MN-direction one (the next channel
// group's plane).  Start addresses in 16-byte units are voxel indices.
template <int N, bool kShiftA, int T0, int T1>
__device__ __forceinline__ void dc_issue_wgrad(uint32_t a_s, uint32_t b_s, uint32_t taddr) {
    constexpr uint32_t idesc = umma_idesc_mn(N);
    const uint64_t a_base = umma_desc(a_s, 160u, kGrpB), b_base = umma_desc(b_s, 160u, kGrpB);
#pragma unroll 1
    for (int q = 0; q < 32; ++q) {
        const int vb = pad_vox(q >> 2, (q & 3) * 2, 0);
        const uint64_t a = a_base + (uint64_t)vb, b = b_base + (uint64_t)vb;
        const uint32_t acc = q > 0 ? 1u : 0u;
#pragma unroll
        for (int t = T0; t < T1; ++t) {
            const int64_t off = (t / 9 - 1) * 100 + ((t / 3) % 3 - 1) * 10 + (t % 3 - 1);
            umma_f16(taddr + (uint32_t)((t - T0) * N), kShiftA ? a + (uint64_t)off : a, kShiftA ? b : b + (uint64_t)off, idesc, acc);
        }
    }
}

__device__ __forceinline__ void unpack8(uint4 u, float (&f)[8]) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float2 x = __bfloat1622float2(h[e]);
        f[2 * e] = x.x, f[2 * e + 1] = x.y;
    }
}
__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
    uint4 u;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
    for (int e = 0; e < 4; ++e) h[e] = __floats2bfloat162_rn(f[2 * e], f[2 * e + 1]);
    return u;
}

// voxel of TMEM lane `row` of convolution tile m (-1: a border row, not stored)
__device__ __forceinline__ int dc_tile_voxel(int m, int row) {
    const int R = 16 * m + (row >> 3), i = R / 10, j = R - 10 * i;
    return j < 8 ? pad_vox(i, j, row & 7) : -1;
}

// Hidden-layer epilogues: TMEM lane 32 warp + lane of tile m is voxel dc_tile_voxel; the result
// goes to the buffer at dst and, if scr, to the same place in the CTA's scratch.
enum { kEpReluBias, kEpResid, kEpMaskSelf, kEpResidMask };
template <int kOp>
__device__ __forceinline__ void dc_epilogue(uint32_t lane_base, int warp, int lane, unsigned char* dst, const float* bias,
                                            unsigned char* scr, const unsigned char* mask_src) {
#pragma unroll 1
    for (int mt = 0; mt < kConvTiles; ++mt) {
        float v[2][16];
        tmem_ld16(lane_base + (uint32_t)(mt * 32), v[0]);
        tmem_ld16(lane_base + (uint32_t)(mt * 32 + 16), v[1]);
        tmem_wait_ld();
        const int vx = dc_tile_voxel(mt, 32 * warp + lane);
        if (vx < 0) continue;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            uint4* d = reinterpret_cast<uint4*>(dst + g * kGrpB + vx * 16);
            float o[8], old[8], m[8];
            if constexpr (kOp != kEpReluBias) unpack8(*d, old);
            if constexpr (kOp == kEpResidMask) unpack8(__ldcg(reinterpret_cast<const uint4*>(mask_src + g * kGrpB + vx * 16)), m);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const float a = v[g >> 1][(g & 1) * 8 + e];
                const int c = 8 * g + e;
                if constexpr (kOp == kEpReluBias) o[e] = fmaxf(__fadd_rn(a, bias[c]), 0.0f);
                else if constexpr (kOp == kEpResid) o[e] = fmaxf(__fadd_rn(__fadd_rn(a, bias[c]), old[e]), 0.0f);
                else if constexpr (kOp == kEpMaskSelf) o[e] = old[e] > 0.0f ? a : 0.0f;
                else o[e] = m[e] > 0.0f ? __fadd_rn(a, old[e]) : 0.0f;
            }
            const uint4 u = pack8(o);
            *d = u;
            if (scr) *reinterpret_cast<uint4*>(scr + g * kGrpB + vx * 16) = u;
        }
    }
}

// Weight-gradient epilogue: rows 0-31 of the M = 64 accumulator (warp 0 rows 0-15, warp 1 rows
// 16-31, lanes 0-15) added to the CTA's gradient row.  kKind 0: N = 32, gw[(row*27 + t)*32 + n];
// 1: N = 8, gw[(row*27 + t)*8 + n]; 2: N = 8, column 0 only, gw[t*32 + row].
template <int kKind>
__device__ __forceinline__ void dc_wgrad_epilogue(uint32_t lane_base, int warp, int lane, int t0, int t1, float* gw) {
    if (warp >= 2) return;
    const int row = 16 * warp + lane;
#pragma unroll 1
    for (int t = t0; t < t1; ++t) {
        if constexpr (kKind == 0) {
            float v[2][16];
            tmem_ld16(lane_base + (uint32_t)((t - t0) * 32), v[0]);
            tmem_ld16(lane_base + (uint32_t)((t - t0) * 32 + 16), v[1]);
            tmem_wait_ld();
            if (lane < 16) {
                float4* p = reinterpret_cast<float4*>(gw + (row * 27 + t) * 32);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    float4 a = p[i];
                    a.x += v[i >> 2][(i & 3) * 4], a.y += v[i >> 2][(i & 3) * 4 + 1], a.z += v[i >> 2][(i & 3) * 4 + 2],
                        a.w += v[i >> 2][(i & 3) * 4 + 3];
                    p[i] = a;
                }
            }
        } else {
            float v[8];
            tmem_ld8(lane_base + (uint32_t)((t - t0) * 8), v);
            tmem_wait_ld();
            if (lane < 16) {
                if constexpr (kKind == 1) {
                    float4* p = reinterpret_cast<float4*>(gw + (row * 27 + t) * 8);
                    float4 a = p[0], b = p[1];
                    a.x += v[0], a.y += v[1], a.z += v[2], a.w += v[3];
                    b.x += v[4], b.y += v[5], b.z += v[6], b.w += v[7];
                    p[0] = a, p[1] = b;
                } else {
                    gw[t * 32 + row] += v[0];
                }
            }
        }
    }
}

// bias gradient: gb[c] += sum over the tile's 512 voxels of buffer[v][c] (fixed order)
__device__ __forceinline__ void dc_bias_grad(const unsigned char* buf, float* red, float* gb) {
    const int c = threadIdx.x & 31, part = threadIdx.x >> 5;
    const unsigned char* base = buf + (c >> 3) * kGrpB + (c & 7) * 2;
    float s = 0.0f;
    for (int cell = part * 128; cell < part * 128 + 128; ++cell) {
        const int vx = pad_vox(cell >> 6, (cell >> 3) & 7, cell & 7);
        s += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(base + vx * 16));
    }
    red[part * 32 + c] = s;
    __syncthreads();
    if (threadIdx.x < 32) gb[threadIdx.x] += (red[threadIdx.x] + red[32 + threadIdx.x]) + (red[64 + threadIdx.x] + red[96 + threadIdx.x]);
    __syncthreads();
}

// Inference (kTrain false): out (z) += (S/D) f on INTERIOR cells of sample s, or = with overwrite.
// Training: per sample b its loss to loss[b], the gradient summed into gacc[blockIdx.x][kDParams].
template <bool kTrain>
__global__ void __launch_bounds__(kNetThreads, 1) k_net_deep(NetIn I, int ns, const __nv_bfloat16* __restrict__ pack,
                                                             const float* __restrict__ bias_g, float* __restrict__ out, int overwrite,
                                                             float* __restrict__ gacc, float* __restrict__ loss, int loss_kind,
                                                             unsigned char* __restrict__ scratch) {
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* P0 = smem;
    unsigned char* P1 = smem + kOffP1;
    float* bias = reinterpret_cast<float*>(smem + kOffBias);
    float* ys = reinterpret_cast<float*>(smem + kOffYs);
    float* red = reinterpret_cast<float*>(smem + kOffRed);
    const uint32_t mb_mma = smem_u32(smem + kOffMbar), mb_w = mb_mma + 8, mb_a = mb_mma + 16;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kOffSlot);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int kCols = kTrain ? 512 : 256;
    const uint32_t sP0 = smem_u32(P0), sP1 = smem_u32(P1), sW = smem_u32(smem + kOffW);
    unsigned char* scr = kTrain ? scratch + (size_t)blockIdx.x * kScrBytes : nullptr;
    float* gw = kTrain ? gacc + (size_t)blockIdx.x * kDParams : nullptr;

    zero_smem(smem, 2 * kBufB);
    if (tid < kDBias / 4) reinterpret_cast<float4*>(bias)[tid] = reinterpret_cast<const float4*>(bias_g)[tid];
    if constexpr (kTrain)
        for (int i = tid; i < kDParams / 4; i += kNetThreads) reinterpret_cast<float4*>(gw)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb_mma) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb_w) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(kCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *tslot;
    const uint32_t lane_base = taddr + ((uint32_t)(32 * warp) << 16);
    uint32_t ph_mma = 0, ph_w = 0, ph_a = 0;
    bool ok = true, w_pending = false, a_pending = false;

    // weights of one convolution into the shared buffer (thread 0; the buffer must be free)
    auto load_w = [&](int elem0, int elems) {
        if (tid == 0) {
            bulk_expect(mb_w, (uint32_t)elems * 2u);
            bulk_load(sW, pack + elem0, (uint32_t)elems * 2u, mb_w);
        }
        w_pending = true;
    };
    auto wait_w = [&]() -> bool {
        const bool d = mbar_wait(mb_w, ph_w);
        ph_w ^= 1u;
        w_pending = false;
        return d;
    };
    auto wait_a = [&]() -> bool {
        const bool d = mbar_wait(mb_a, ph_a);
        ph_a ^= 1u;
        a_pending = false;
        return d;
    };
    // make the threads' shared and global writes visible to the tensor cores and the bulk
    // copies; also makes a wait's outcome d uniform over the block
    auto publish = [&](bool d) -> bool {
        fence_async_smem();
        if constexpr (kTrain) fence_async_global();
        tc_fence_before();
        const bool r = __syncthreads_and(d ? 1 : 0) != 0;
        tc_fence_after();
        return r;
    };
    // MMAs issued by thread 0 through `issue`, then one commit and a bounded wait
    auto mma_round = [&](auto issue) -> bool {
        if (tid == 0) {
            issue();
            umma_commit(mb_mma);
        }
        const bool d = mbar_wait(mb_mma, ph_mma);
        ph_mma ^= 1u;
        tc_fence_after();
        return __syncthreads_and(d ? 1 : 0) != 0;
    };

    load_w(kPF0, kWs8);
    for (int s = blockIdx.x; s < ns && ok; s += gridDim.x) {
        const Staged st = stage_features(I, s, reinterpret_cast<__nv_bfloat16*>(P1), red);
        const int t = I.idx ? I.idx[s] : I.t0 + s;
        if (st.S == 0.0f) {
            if constexpr (kTrain) {
                if (tid == 0) loss[s] = 0.0f;
            } else if (overwrite) {
                st4(out + (size_t)t * kCells + 4 * tid, make_float4(0.f, 0.f, 0.f, 0.f));
            }
            __syncthreads();
            continue;  // uniform over the block
        }
        __syncthreads();
        if constexpr (kTrain)  // x0 with its border features
            for (int i = tid; i < kGrpB / 16; i += kNetThreads)
                reinterpret_cast<uint4*>(scr)[i] = reinterpret_cast<const uint4*>(P1)[i];
        // ---- forward ----
        ok = publish(wait_w());
        ok = ok && mma_round([&] { dc_issue_conv<1, kDC>(sP1, sW, taddr); });
        if (!ok) break;
        load_w(pFA(0), kWs32);
        clear_face_halo(reinterpret_cast<__nv_bfloat16*>(P1));  // P1 group 0 is a hidden buffer from here on
        dc_epilogue<kEpReluBias>(lane_base, warp, lane, P0, bias, kTrain ? scr + kScrX(0) : nullptr, nullptr);
        for (int k = 0; k < kDBlk && ok; ++k) {
            ok = publish(wait_w());
            ok = ok && mma_round([&] { dc_issue_conv<4, kDC>(sP0, sW, taddr); });
            if (!ok) break;
            load_w(pFB(k), kWs32);
            dc_epilogue<kEpReluBias>(lane_base, warp, lane, P1, bias + bA(k), kTrain ? scr + kScrH(k) : nullptr, nullptr);
            ok = publish(wait_w());
            ok = ok && mma_round([&] { dc_issue_conv<4, kDC>(sP1, sW, taddr); });
            if (!ok) break;
            if (k + 1 < kDBlk) load_w(pFA(k + 1), kWs32);
            else load_w(kPFO, kWsO);
            dc_epilogue<kEpResid>(lane_base, warp, lane, P0, bias + bB(k), (kTrain && k + 1 < kDBlk) ? scr + kScrX(k + 1) : nullptr,
                                  nullptr);
        }
        if (!ok) break;
        ok = publish(wait_w());
        ok = ok && mma_round([&] { dc_issue_conv<4, 8>(sP0, sW, taddr); });
        if (!ok) break;
        if constexpr (kTrain) load_w(kPGO, kWs8);
        else load_w(kPF0, kWs8);  // the next tile's first layer
        {
            float v[8];
            for (int mt = 0; mt < kConvTiles; ++mt) {
                tmem_ld8(lane_base + (uint32_t)(mt * 8), v);
                tmem_wait_ld();
                const int R = 16 * mt + ((32 * warp + lane) >> 3), i = R / 10, j = R - 10 * i;
                if (j < 8) ys[i * 64 + j * 8 + (lane & 7)] = v[0];
            }
        }
        tc_fence_before();
        __syncthreads();
        if constexpr (!kTrain) {
            const float sc = st.S / st.D;
            float* o = out + (size_t)t * kCells + 4 * tid;
            float4 z = overwrite ? make_float4(0.f, 0.f, 0.f, 0.f) : ldcg4(o);
            float zz[4] = {z.x, z.y, z.z, z.w};
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (st.in[u]) zz[u] = __fmaf_rn(sc, ys[4 * tid + u], zz[u]);
            st4(o, make_float4(zz[0], zz[1], zz[2], zz[3]));
            __syncthreads();  // ys and the buffers are rewritten by the next sample
        } else {
            // ---- backward ----
            float g[4];
            const float l = tile_loss_grad(st, ys, loss_kind, g);
            {  // dy (channel 0 = 2 g) over group 0 of P1, which held H_3
                uint4 zero = make_uint4(0, 0, 0, 0);
                for (int i = tid; i < kCells; i += kNetThreads) {
                    const int vx = pad_vox(i >> 6, (i >> 3) & 7, i & 7);
                    *reinterpret_cast<uint4*>(P1 + vx * 16) = zero;
                }
                __syncthreads();
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int cell = 4 * tid + u;
                    *reinterpret_cast<__nv_bfloat16*>(P1 + pad_vox(cell >> 6, (cell >> 3) & 7, cell & 7) * 16) = __float2bfloat16_rn(2.0f * g[u]);
                }
            }
            const float lt = block_sum_f(l, red);
            if (tid == 0) loss[s] = lt;
            ok = publish(wait_w());  // GO
            // dWo (A = X_4 shifted, rows = input channel; B = dy, column 0) and dX_4 = conv(dy, GO)
            ok = ok && mma_round([&] {
                dc_issue_wgrad<8, true, 0, 27>(sP0, sP1, taddr + 256);
                dc_issue_conv<1, kDC>(sP1, sW, taddr);
            });
            if (!ok) break;
            load_w(pGB(kDBlk - 1), kWs32);
            if (tid == 0) {
                bulk_expect(mb_a, kBufB);
                bulk_load(sP1, scr + kScrH(kDBlk - 1), kBufB, mb_a);
            }
            a_pending = true;
            dc_wgrad_epilogue<2>(lane_base + 256, warp, lane, 0, 27, gw + kQWO);
            dc_epilogue<kEpMaskSelf>(lane_base, warp, lane, P0, nullptr, nullptr, nullptr);  // d of block 3's output
            for (int k = kDBlk - 1; k >= 0 && ok; --k) {
                // P0 = d (block k's pre-activation gradient, being loaded for k < 3); P1 <- H_k, W <- GB_k
                const bool da_ok = wait_a();
                ok = publish(wait_w() && da_ok);
                if (!ok) break;
                dc_bias_grad(P0, red, gw + qBb(k));
                ok = mma_round([&] { dc_issue_wgrad<kDC, false, 0, 16>(sP0, sP1, taddr); });
                if (!ok) break;
                dc_wgrad_epilogue<0>(lane_base, warp, lane, 0, 16, gw + qWb(k));
                tc_fence_before();
                __syncthreads();
                tc_fence_after();
                ok = mma_round([&] { dc_issue_wgrad<kDC, false, 16, 27>(sP0, sP1, taddr); });
                if (!ok) break;
                dc_wgrad_epilogue<0>(lane_base, warp, lane, 16, 27, gw + qWb(k));
                tc_fence_before();
                __syncthreads();
                tc_fence_after();
                ok = mma_round([&] { dc_issue_conv<4, kDC>(sP0, sW, taddr); });  // dH_k = conv(d, GB_k)
                if (!ok) break;
                load_w(pGA(k), kWs32);
                dc_epilogue<kEpMaskSelf>(lane_base, warp, lane, P1, nullptr, nullptr, nullptr);  // da = dH_k (H_k > 0)
                __syncthreads();
                dc_bias_grad(P1, red, gw + qBa(k));
                ok = publish(wait_w());
                ok = ok && mma_round([&] { dc_issue_conv<4, kDC>(sP1, sW, taddr); });  // conv(da, GA_k)
                if (!ok) break;
                if (k > 0) load_w(pGB(k - 1), kWs32);
                else load_w(kPF0, kWs8);  // the next tile's first layer
                // d of X_k: (d + conv(da, GA_k)) (X_k > 0), kept in the scratch while X_k is loaded
                dc_epilogue<kEpResidMask>(lane_base, warp, lane, P0, nullptr, scr + kScrG, scr + kScrX(k));
                publish(true);
                if (tid == 0) {
                    bulk_expect(mb_a, kBufB);
                    bulk_load(sP0, scr + kScrX(k), kBufB, mb_a);
                }
                ok = publish(wait_a());
                // dWa_k (A = da, rows = output channel; B = X_k shifted)
                ok = ok && mma_round([&] { dc_issue_wgrad<kDC, false, 0, 16>(sP1, sP0, taddr); });
                if (!ok) break;
                dc_wgrad_epilogue<0>(lane_base, warp, lane, 0, 16, gw + qWa(k));
                tc_fence_before();
                __syncthreads();
                tc_fence_after();
                ok = mma_round([&] { dc_issue_wgrad<kDC, false, 16, 27>(sP1, sP0, taddr); });
                if (!ok) break;
                dc_wgrad_epilogue<0>(lane_base, warp, lane, 16, 27, gw + qWa(k));
                fence_async_smem();
                tc_fence_before();
                __syncthreads();
                tc_fence_after();
                if (tid == 0) {
                    if (k > 0) {
                        bulk_expect(mb_a, 2 * kBufB);
                        bulk_load(sP0, scr + kScrG, kBufB, mb_a);
                        bulk_load(sP1, scr + kScrH(k - 1), kBufB, mb_a);
                    } else {
                        bulk_expect(mb_a, kBufB + kGrpB);
                        bulk_load(sP0, scr + kScrG, kBufB, mb_a);
                        bulk_load(sP1, scr, kGrpB, mb_a);  // x0
                    }
                }
                a_pending = true;
            }
            if (!ok) break;
            // first layer: P0 = d of X_0, P1 group 0 = x0
            ok = publish(wait_a());
            if (!ok) break;
            dc_bias_grad(P0, red, gw + kQB0);
            ok = mma_round([&] { dc_issue_wgrad<8, false, 0, 27>(sP0, sP1, taddr); });
            if (!ok) break;
            dc_wgrad_epilogue<1>(lane_base, warp, lane, 0, 27, gw + kQW0);
            fence_async_smem();
            tc_fence_before();
            __syncthreads();  // the buffers are rewritten by the next sample
            tc_fence_after();
        }
    }
    if (!ok && tid == 0) atomicExch(&g_deep_error, 1);
    // outstanding copies (bounded waits): the next tile's weights, an activation load after an error
    if (w_pending) wait_w();
    if (a_pending) wait_a();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kCols) : "memory");
}

// fp32 parameters -> packed bf16 operands and the bias vector
__global__ void k_net_deep_pack(const float* __restrict__ p, __nv_bfloat16* __restrict__ pack, float* __restrict__ bias) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < kDBias) {
        const int k = (e - kDC) / (2 * kDC), w = (e - kDC) % (2 * kDC);
        bias[e] = e < kDC ? p[kQB0 + e] : (w < kDC ? p[qBa(k) + w] : p[qBb(k) + w - kDC]);
    }
    if (e >= kDPack) return;
    float v = 0.0f;
    if (e < pFA(0)) {  // F0: [step][half][n][c], tap = 2 step + half
        const int s = e / 512, h = (e / 256) & 1, n = (e / 8) % 32, c = e & 7, tap = 2 * s + h;
        if (tap < 27) v = p[kQW0 + (n * 27 + tap) * 8 + c];
    } else if (e < kPFO) {  // FA_k / FB_k: tap = step / 2, input channel (2 (step & 1) + half) 8 + c
        const int seg = (e - pFA(0)) / kWs32, rel = (e - pFA(0)) % kWs32;
        const int s = rel / 512, h = (rel / 256) & 1, n = (rel / 8) % 32, c = rel & 7;
        const int W = (seg & 1) ? qWb(seg >> 1) : qWa(seg >> 1);
        v = p[W + (n * 27 + (s >> 1)) * 32 + (2 * (s & 1) + h) * 8 + c];
    } else if (e < kPGO) {  // FO: N = 8, row 0 = Wo
        const int rel = e - kPFO, s = rel / 128, h = (rel / 64) & 1, n = (rel / 8) % 8, c = rel & 7;
        if (n == 0) v = p[kQWO + (s >> 1) * 32 + (2 * (s & 1) + h) * 8 + c];
    } else if (e < pGA(0)) {  // GO[step][half][n = channel of X_4][c]: Wo[26 - tap][n] for c = 0
        const int rel = e - kPGO, s = rel / 512, h = (rel / 256) & 1, n = (rel / 8) % 32, c = rel & 7, tap = 2 * s + h;
        if (tap < 27 && c == 0) v = p[kQWO + (26 - tap) * 32 + n];
    } else {  // GA_k / GB_k: G[n = input channel][tap'][cout] = W[cout][26 - tap'][n]
        const int seg = (e - pGA(0)) / kWs32, rel = (e - pGA(0)) % kWs32;
        const int s = rel / 512, h = (rel / 256) & 1, n = (rel / 8) % 32, c = rel & 7;
        const int W = (seg & 1) ? qWb(seg >> 1) : qWa(seg >> 1);
        v = p[W + (((2 * (s & 1) + h) * 8 + c) * 27 + (26 - (s >> 1))) * 32 + n];
    }
    pack[e] = __float2bfloat16_rn(v);
}

int g_deep_sms = 0;

}  // namespace

int deep_params() { return kDParams; }
int deep_pack_elems() { return kDPack; }
int deep_bias_elems() { return kDBias; }
size_t deep_scratch_bytes() { return kScrBytes; }

bool deep_init() {
    if (cudaFuncSetAttribute(k_net_deep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDSmem) != cudaSuccess) return false;
    if (cudaFuncSetAttribute(k_net_deep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDSmem) != cudaSuccess) return false;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_deep_sms, cudaDevAttrMultiProcessorCount, dev);
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_net_deep<true>, kNetThreads, kDSmem) != cudaSuccess || per < 1) return false;
    return g_deep_sms > 0;
}

int deep_take_error() {
    int v = 0, z = 0;
    if (cudaMemcpyFromSymbol(&v, g_deep_error, sizeof(int)) != cudaSuccess) return -1;
    if (v) cudaMemcpyToSymbol(g_deep_error, &z, sizeof(int));
    return v;
}

void launch_deep_pack(const float* params, void* pack, float* bias, cudaStream_t st) {
    note_kernel_launch();
    k_net_deep_pack<<<(kDPack + 255) / 256, 256, 0, st>>>(params, (__nv_bfloat16*)pack, bias);
}

void launch_deep_forward(const float* r, const float* az, const float* diag, const uint8_t* types, const int* idx, int t0, int ns,
                         const void* pack, const float* bias, float* out, bool overwrite, cudaStream_t st, const NetExtra& ex) {
    if (ns <= 0) return;
    const NetIn I{r, az, diag, types, nullptr, idx, t0, ex};
    const int blocks = ns < g_deep_sms ? ns : g_deep_sms;
    note_kernel_launch();
    k_net_deep<false><<<blocks, kNetThreads, kDSmem, st>>>(I, ns, (const __nv_bfloat16*)pack, bias, out, overwrite ? 1 : 0, nullptr,
                                                           nullptr, 0, nullptr);
}

int deep_train_blocks(int nb) { return nb < g_deep_sms ? nb : g_deep_sms; }

void launch_deep_train(const float* rho, const float* diag, const uint8_t* types, const float* target, const int* idx, int nb,
                       const void* pack, const float* bias, float* grad, float* loss, int loss_kind, cudaStream_t st, const NetExtra& ex,
                       void* scratch) {
    if (nb <= 0) return;
    const NetIn I{rho, nullptr, diag, types, target, idx, 0, ex};
    note_kernel_launch();
    k_net_deep<true><<<deep_train_blocks(nb), kNetThreads, kDSmem, st>>>(I, nb, (const __nv_bfloat16*)pack, bias, nullptr, 0, grad, loss,
                                                                        loss_kind, (unsigned char*)scratch);
}

}  // namespace cmg
