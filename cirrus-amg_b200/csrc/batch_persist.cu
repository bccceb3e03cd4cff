// Many independent octrees solved by ONE persistent cooperative launch.
//
// The reference has no batched call: its callers loop over AMGSolver::solve
// (src/AMGSolver.h:62, src/AMGSolver.cu:1399-1549), one octree at a time.  Here the
// resident blocks are split into groups (the host's schedule gives their sizes).  A group
// solves the octrees assigned to it, then takes octrees from a shared device work queue
// (ordered largest first), running each octree's whole MG-preconditioned CG solve.  Inside
// a group, work is split by tiles over 128-thread slots (four per block) and the steps of
// the solve are separated by group barriers: a group works like one small GPU, and the
// groups work on different octrees at the same time without waiting for one another.
//
// Every step is the same per-tile code the single solve runs (tiles.cuh), and every
// reduction keeps the single solve's order: one double per LEAF tile (a 128-thread
// block sum), then the partials summed in the fixed order of sum_partials.  Each slot
// of the group sums the partials itself, so every slot holds the same PCG scalars
// without another barrier.  Results therefore equal the single solve's bit for bit.
//
// Barrier waits are bounded: past ~1 s a block records an error flag, every block of
// every group sees it at its next barrier and returns, and the host reports a timeout.
#include "tiles.cuh"

namespace cmg {
namespace {

constexpr int kCtlHead = 0, kCtlError = 1, kCtlGroups = 32;  // per-group words start at 32
constexpr int kCtlStride = 32;                                 // one 128-byte line per group

// PCG scalars of the instance as one slot holds them (written by the slot's thread 0)
struct SlotPcg {
    double gamma, gamma_old, beta, alpha, pAp, rr, rr0, thr, mean, count;
    int iter, done, converged, nonfinite;
};

// Shared memory of a block with NS slots: region A holds either the dense coarse levels
// (the group's first block, between tile steps) or the slots' tile snapshots and residual
// buffers; the tail holds the instance and the slots' scalars, which live across steps.
constexpr int kMaxSlots = 8;
struct __align__(16) BatchTail {
    BatchInst inst;
    SlotPcg pcg[kMaxSlots];
    double red[kMaxSlots][4];
    double bcast[kMaxSlots];
    int q;
};
__host__ __device__ constexpr size_t batch_region_a(int ns) {
    return ((ns * (sizeof(Snap) + sizeof(float) * kCells) > kCoarseSmem ? ns * (sizeof(Snap) + sizeof(float) * kCells) : kCoarseSmem) +
            15) / 16 * 16;
}
template <int NS>
constexpr size_t batch_smem() {
    return batch_region_a(NS) + sizeof(BatchTail);
}
static_assert(sizeof(Snap) % 16 == 0, "snapshots stay 16-byte aligned");

template <int NS>
struct BCtx {
    unsigned char* smem;  // region A, then the tail
    unsigned int* gbar;   // [0] arrivals, [1] generation, [2] queue position of the group's instance
    unsigned int* err;
    int G, grank, slot, tid, gslot, nslot;
    int rbuf;  // which of the instance's two partial buffers the next reduction writes
    SlotSync sync;
    __device__ BatchTail* tl() const { return reinterpret_cast<BatchTail*>(smem + batch_region_a(NS)); }
    __device__ Snap& snap() const { return reinterpret_cast<Snap*>(smem)[slot]; }
    __device__ float* res() const { return reinterpret_cast<float*>(smem + NS * sizeof(Snap)) + slot * kCells; }
    __device__ double* red() const { return tl()->red[slot]; }
    __device__ SlotPcg& pcg() const { return tl()->pcg[slot]; }
};

// the group's barrier; false once any block of the batch has recorded an error
template <class Ctx>
__device__ bool group_sync(const Ctx& C) {
    __syncthreads();
    // a group of one block: the block barrier already orders its threads' global memory
    if (C.G == 1) return *(volatile unsigned int*)C.err == 0;
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = C.gbar + 1;
        const unsigned int g0 = *gen;
        __threadfence();
        if (atomicAdd(C.gbar, 1u) == (unsigned int)C.G - 1) {
            C.gbar[0] = 0;
            __threadfence();
            atomicAdd(C.gbar + 1, 1u);
        } else {
            unsigned int spins = 0;
            while (*gen == g0) {
                if (*(volatile unsigned int*)C.err) break;
                if (++spins > (1u << 24)) {  // ~1 s
                    atomicExch(C.err, 1u);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile unsigned int*)C.err == 0;
}

// block_sum128 of one slot: the same shuffle tree and the same final order
__device__ __forceinline__ double slot_sum128(double v, double* red, const SlotSync& sync, int tid) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) red[tid >> 5] = v;
    sync();
    double r = 0;
    if (tid == 0) r = (red[0] + red[1]) + (red[2] + red[3]);
    sync();
    return r;
}
// sum_partials of one slot, the result on every thread of the slot
template <class Ctx>
__device__ double slot_sum_partials(const Ctx& C, const double* part, int n) {
    double s = 0;
    int i = C.tid;
    for (; i + 7 * 128 < n; i += 8 * 128) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = __ldcg(part + i + u * 128);
#pragma unroll
        for (int u = 0; u < 8; ++u) s += v[u];
    }
    for (; i < n; i += 128) s += __ldcg(part + i);
    const double r = slot_sum128(s, C.red(), C.sync, C.tid);
    if (C.tid == 0) C.tl()->bcast[C.slot] = r;
    C.sync();
    return C.tl()->bcast[C.slot];
}

// The partials of consecutive reductions alternate between two buffers: a slot may
// start writing the next reduction's partials while a slower slot still sums the last.
template <class Ctx>
__device__ __forceinline__ double* next_partials(Ctx& C, const BatchInst& I) {
    double* p = I.partial + (size_t)(C.rbuf & 1) * 2 * (size_t)I.nleaf;
    C.rbuf ^= 1;
    return p;
}

__device__ __forceinline__ float* plane(const BatchInst& I, int c) { return I.g.plane(c); }

// --- the mu-cycle (FASMuCycleStep, src/AMGSolver.cu:1257-1277) by tile steps ---
__device__ int level_sweeps(const BatchInst& I, const BatchArgs& A, int l) {
    return (l == I.top && l >= 3 && I.finest_iters >= 0) ? I.finest_iters : A.level_iters;
}
// GaussSeidelAMG (src/AMGSolver.cu:887-894) on the LEAF and NONLEAF tiles of level l
template <class Ctx>
__device__ bool b_gs(Ctx& C, const BatchInst& I, int l, int iters, int order) {
    const SmoothArgs sa{I.coeff_ch, I.exact, I.om, I.omega};
    float* X = plane(I, 4);
    const float* RHS = plane(I, 1);
    for (int it = 0; it < iters; ++it)
        for (int h = 0; h < 2; ++h) {
            const int color = h ? 1 - order : order;
            for (int t = I.lb[l] + C.gslot; t < I.ab[l]; t += C.nslot) tile_gs(I.g, t, C.tid, X, RHS, color, sa, C.snap(), C.sync);
            if (!group_sync(C)) return false;
        }
    return true;
}
// ResidualAndRestrictAMG128Kernel of level l, then FASSaveSolutionAndUpdateSource on level l-1
template <class Ctx>
__device__ bool b_restrict_save(Ctx& C, const BatchInst& I, int l) {
    float* X = plane(I, 4);
    float* RHS = plane(I, 1);
    for (int t = I.lb[l] + C.gslot; t < I.ab[l]; t += C.nslot)
        tile_restrict(I.g, t, C.tid, X, RHS, I.coeff_ch, I.Rr, C.snap(), C.res(), C.sync);
    if (!group_sync(C)) return false;
    for (int t = I.nlb[l - 1] + C.gslot; t < I.ab[l - 1]; t += C.nslot)
        tile_fas_save(I.g, t, C.tid, X, RHS, plane(I, 3), I.coeff_ch, C.snap(), C.sync);
    return group_sync(C);
}
// FASProlongateAndUpdateAMG128Kernel on every tile of level l
template <class Ctx>
__device__ bool b_prolong(Ctx& C, const BatchInst& I, int l) {
    for (int t = I.lb[l] + C.gslot; t < I.le[l]; t += C.nslot) tile_prolong(I.g, t, C.tid, plane(I, 4), plane(I, 3), I.P);
    return group_sync(C);
}
// levels 0-1 (or the root alone): the dense sub-cycle in the group's first block
template <class Ctx>
__device__ bool b_coarse(Ctx& C, const BatchInst& I, const BatchArgs& A, int top) {
    if (C.grank == 0) {
        const CoarseArgs ca{top, I.coeff_ch, I.mu, A.level_iters, A.coarsest_iters, I.exact, I.om, I.Rr, I.P, I.omega};
        coarse_dense(I.g, ca, plane(I, 4), plane(I, 1), plane(I, 3), C.smem);
    }
    return group_sync(C);
}
// FASMuCycleStep of the finest level with all its recursions, walked without recursion:
// cnt[l] counts the visits of level l-1 still due from the current visit of level l
template <class Ctx>
__device__ bool b_cycle(Ctx& C, const BatchInst& I, const BatchArgs& A) {
    const int top = I.top;
    if (top <= 1) return b_coarse(C, I, A, top);
    int cnt[kBatchMaxLevels];
    int l = top;
    bool down = true;
    for (;;) {
        if (down) {
            if (!b_gs(C, I, l, level_sweeps(I, A, l), 0) || !b_restrict_save(C, I, l)) return false;
            cnt[l] = I.mu;
            if (l - 1 >= 2) {
                if (cnt[l] > 0) {
                    --cnt[l];
                    --l;
                    continue;
                }
            } else {
                for (int r = 0; r < I.mu; ++r)
                    if (!b_coarse(C, I, A, 1)) return false;
            }
        }
        if (!b_prolong(C, I, l) || !b_gs(C, I, l, level_sweeps(I, A, l), 1)) return false;
        if (l == top) return true;
        ++l;
        down = cnt[l] > 0;
        if (down) {
            --cnt[l];
            --l;
        }
    }
}

// --- PCG on the LEAF tiles (src/AMGSolver.cu:1399-1549) ---
// z = 0 on every tile (AMGSolver::FASMuCycle zeroes x first, src/AMGSolver.cu:1283)
template <class Ctx>
__device__ void fill_z(Ctx& C, const BatchInst& I) {
    float* Z = plane(I, 4);
    for (int t = C.gslot; t < I.g.n; t += C.nslot) st4(Z + (size_t)t * kCells + 4 * C.tid, make_float4(0.f, 0.f, 0.f, 0.f));
}
// ReCenterLeafCells (src/PoissonGrid.cu:889-921): the mean's partials, then r -= mean
template <class Ctx>
__device__ bool b_recenter(Ctx& C, const BatchInst& I) {
    const float* R = plane(I, 1);
    double* part = next_partials(C, I);
    double* part2 = part + I.nleaf;
    for (int b = C.gslot; b < I.nleaf; b += C.nslot) {
        const size_t base = (size_t)I.leaf[b] * kCells + 4 * C.tid;
        const float4 r = ldcg4(R + base);
        const uchar4 ty = ldt4(I.g.ctype + base);
        float f = 0.0f;
        int c = 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const bool in = t4get(ty, u) & dInterior;
            const float v = in ? f4get(r, u) : 0.0f;
            f = (u == 0) ? v : __fadd_rn(f, v);
            c += in;
        }
        const double bs = slot_sum128((double)f, C.red(), C.sync, C.tid);
        const double bc = slot_sum128((double)c, C.red(), C.sync, C.tid);
        if (C.tid == 0) {
            part[b] = bs;
            part2[b] = bc;
        }
    }
    if (!group_sync(C)) return false;
    const double sum = slot_sum_partials(C, part, I.nleaf);
    const double cnt = slot_sum_partials(C, part2, I.nleaf);
    const double mean = sum / cnt;
    if (C.tid == 0) {
        C.pcg().mean = mean;
        C.pcg().count = cnt;
    }
    float* Rw = plane(I, 1);
    for (int b = C.gslot; b < I.nleaf; b += C.nslot) {
        const size_t base = (size_t)I.leaf[b] * kCells + 4 * C.tid;
        float4 r = ldcg4(Rw + base);
        const uchar4 ty = ldt4(I.g.ctype + base);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (t4get(ty, u) & dInterior) f4set(r, u, (float)((double)f4get(r, u) - mean));
        st4(Rw + base, r);
    }
    return true;  // the caller's next barrier publishes r
}
// per-LEAF-tile partials of a.b (Dot128Kernel order), then the sum on every slot
template <class Ctx>
__device__ bool b_dot(Ctx& C, const BatchInst& I, const float* Av, const float* Bv, double* out) {
    double* part = next_partials(C, I);
    for (int b = C.gslot; b < I.nleaf; b += C.nslot) {
        const size_t base = (size_t)I.leaf[b] * kCells + 4 * C.tid;
        const double bs = slot_sum128(dot4(ldcg4(Av + base), ldcg4(Bv + base)), C.red(), C.sync, C.tid);
        if (C.tid == 0) part[b] = bs;
    }
    if (!group_sync(C)) return false;
    *out = slot_sum_partials(C, part, I.nleaf);
    return true;
}
// z = M r: zero z (with r recentred first for a pure Neumann problem), then the cycle
template <class Ctx>
__device__ bool b_precond(Ctx& C, const BatchInst& I, const BatchArgs& A) {
    if (A.pure_neumann && !b_recenter(C, I)) return false;
    fill_z(C, I);
    if (!group_sync(C)) return false;
    return b_cycle(C, I, A);
}

template <class Ctx>
__device__ bool solve_instance(Ctx& C, const BatchInst& I, const BatchArgs& A) {
    SlotPcg& P = C.pcg();
    float* X = plane(I, 0);
    float* R = plane(I, 1);
    float* Pp = plane(I, 2);
    float* AP = plane(I, 3);
    float* Z = plane(I, 4);
    if (C.tid == 0) {
        P.gamma = P.gamma_old = P.beta = P.alpha = P.pAp = P.rr = P.rr0 = P.mean = P.count = 0.0;
        P.thr = -1.0;
        P.iter = P.done = P.converged = P.nonfinite = 0;
    }
    C.sync();
    // x = 0 on LEAF tiles; r.r before any recentring (src/AMGSolver.cu:1405-1426)
    for (int b = C.gslot; b < I.nleaf; b += C.nslot) st4(X + (size_t)I.leaf[b] * kCells + 4 * C.tid, make_float4(0.f, 0.f, 0.f, 0.f));
    if (A.sync_stride > 0) {
        double rr0;
        if (!b_dot(C, I, R, R, &rr0)) return false;
        if (C.tid == 0) P.rr0 = rr0;
    }
    if (!b_precond(C, I, A)) return false;
    // p = z; gamma = z.r; the loop gate
    for (int b = C.gslot; b < I.nleaf; b += C.nslot) {
        const size_t base = (size_t)I.leaf[b] * kCells + 4 * C.tid;
        st4(Pp + base, ldcg4(Z + base));
    }
    double d;
    if (!b_dot(C, I, Z, R, &d)) return false;
    if (C.tid == 0) {
        P.gamma = d;
        if (A.sync_stride > 0) {
            const double t = A.tol * A.tol * P.rr0;
            P.thr = t > DBL_MIN ? t : DBL_MIN;
            if (P.rr0 == 0.0) P.done = 1;
        }
        if (P.iter >= A.max_iters) P.done = 1;
    }
    C.sync();
    while (!P.done) {
        // Ap = A p with p.Ap and alpha (src/AMGSolver.cu:1449-1457)
        double* part = next_partials(C, I);
        for (int b = C.gslot; b < I.nleaf; b += C.nslot) {
            const int t = I.leaf[b];
            const Quad Q(t, C.tid);
            Own o;
            load_snap(I.g, t, Pp, I.coeff_ch, LeafHalo{Pp, I.g.ctype}, C.snap(), Q, o, C.sync);
            const Snap& S = C.snap();
            float4 ap;
            ap.x = o.ty.x == dInterior ? own_neg_lap<0>(S, Q, o) : 0.0f;
            ap.y = o.ty.y == dInterior ? own_neg_lap<1>(S, Q, o) : 0.0f;
            ap.z = o.ty.z == dInterior ? own_neg_lap<2>(S, Q, o) : 0.0f;
            ap.w = o.ty.w == dInterior ? own_neg_lap<3>(S, Q, o) : 0.0f;
            st4(AP + Q.base, ap);
            const double bs = slot_sum128(dot4(o.xr, ap), C.red(), C.sync, C.tid);
            if (C.tid == 0) part[b] = bs;
        }
        if (!group_sync(C)) return false;
        const double pap = slot_sum_partials(C, part, I.nleaf);
        if (C.tid == 0) {
            P.pAp = pap;
            P.alpha = P.gamma / pap;
        }
        C.sync();
        // x += alpha p, r -= alpha Ap on INTERIOR cells; r.r and the convergence test
        const float alpha = (float)P.alpha;
        part = next_partials(C, I);
        for (int b = C.gslot; b < I.nleaf; b += C.nslot) {
            const size_t base = (size_t)I.leaf[b] * kCells + 4 * C.tid;
            float4 x = ldcg4(X + base), r = ldcg4(R + base);
            const float4 p = ldcg4(Pp + base), ap = ldcg4(AP + base);
            const uchar4 ty = ldt4(I.g.ctype + base);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (t4get(ty, u) & dInterior) {
                    f4set(x, u, __fmaf_rn(alpha, f4get(p, u), f4get(x, u)));
                    f4set(r, u, __fmaf_rn(-alpha, f4get(ap, u), f4get(r, u)));
                }
            }
            st4(X + base, x);
            st4(R + base, r);
            const double bs = slot_sum128(dot4(r, r), C.red(), C.sync, C.tid);
            if (C.tid == 0) part[b] = bs;
        }
        if (!group_sync(C)) return false;
        const double rr = slot_sum_partials(C, part, I.nleaf);
        if (C.tid == 0) {
            P.rr = rr;
            const int it = ++P.iter;
            const bool bad = !isfinite(rr) || !isfinite(P.alpha);
            const bool conv = A.sync_stride > 0 && (it % A.sync_stride) == 0 && rr < P.thr;
            P.converged = conv;
            P.nonfinite = bad;
            P.done = conv || bad || it >= A.max_iters;
        }
        C.sync();
        if (P.done) break;
        // z = M r; gamma_old, gamma = r.z, beta; p = z + beta p (src/AMGSolver.cu:1500-1536)
        if (!b_precond(C, I, A)) return false;
        if (!b_dot(C, I, R, Z, &d)) return false;
        if (C.tid == 0) {
            P.gamma_old = P.gamma;
            P.gamma = d;
            P.beta = d / P.gamma_old;
        }
        C.sync();
        const float beta = (float)P.beta;
        for (int b = C.gslot; b < I.nleaf; b += C.nslot) {
            const size_t base = (size_t)I.leaf[b] * kCells + 4 * C.tid;
            float4 p = ldcg4(Pp + base);
            const float4 z = ldcg4(Z + base);
            const uchar4 ty = ldt4(I.g.ctype + base);
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (t4get(ty, u) & dInterior) f4set(p, u, __fmaf_rn(beta, f4get(p, u), f4get(z, u)));
            st4(Pp + base, p);
        }
        if (!group_sync(C)) return false;
    }
    return true;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int NS>
__global__ void __launch_bounds__(128 * NS, 1) k_batch_solve(BatchArgs A) {
    extern __shared__ __align__(16) unsigned char smraw[];
    BCtx<NS> C;
    C.smem = smraw;
    C.slot = threadIdx.x >> 7;
    C.tid = threadIdx.x & 127;
    const int group = A.block_group[blockIdx.x];
    const BatchGroup gr = A.groups[group];
    C.G = gr.size;
    C.grank = blockIdx.x - gr.first;
    C.gbar = A.ctl + kCtlGroups + kCtlStride * group;
    C.err = A.ctl + kCtlError;
    C.gslot = C.grank * NS + C.slot;
    C.nslot = gr.size * NS;
    C.sync = SlotSync{1 + C.slot};
    C.rbuf = 0;
    int s = gr.sbegin;
    for (;;) {
        int q;
        if (s < gr.send) {
            q = s++;  // the group's own instances: every block knows them
        } else {
            // the next instance of the shared queue, fetched by the group's first block
            if (C.grank == 0 && threadIdx.x == 0) C.gbar[2] = (unsigned int)A.dyn_begin + atomicAdd(A.ctl + kCtlHead, 1u);
            if (!group_sync(C)) return;
            if (threadIdx.x == 0) C.tl()->q = (int)*(volatile unsigned int*)(C.gbar + 2);
            __syncthreads();
            q = C.tl()->q;
            if (q >= A.n) return;
        }
        const BatchInst* src = A.inst + A.order[q];
        {
            const int* s4 = reinterpret_cast<const int*>(src);
            int* d4 = reinterpret_cast<int*>(&C.tl()->inst);
            for (int w = threadIdx.x; w < (int)(sizeof(BatchInst) / sizeof(int)); w += blockDim.x) d4[w] = s4[w];
        }
        __syncthreads();
        const BatchInst& I = C.tl()->inst;
        const unsigned long long t0 = global_ns();
        const bool ok = solve_instance(C, I, A);
        if (!ok) return;
        if (C.grank == 0 && threadIdx.x == 0) {
            const SlotPcg& P = C.tl()->pcg[0];
            PcgScalars* o = I.s;
            o->gamma = P.gamma;
            o->gamma_old = P.gamma_old;
            o->beta = P.beta;
            o->alpha = P.alpha;
            o->pAp = P.pAp;
            o->rr = P.rr;
            o->rr0 = P.rr0;
            o->thr = P.thr;
            o->tol = A.tol;
            o->mean = P.mean;
            o->count = P.count;
            o->iter = P.iter;
            o->done = P.done;
            o->converged = P.converged;
            o->nonfinite = P.nonfinite;
            o->replaced = 0;
            o->max_iters = A.max_iters;
            o->sync_stride = A.sync_stride;
            I.clock[0] = t0;
            I.clock[1] = global_ns();
            I.clock[2] = (unsigned long long)gr.size;
            I.clock[3] = (unsigned long long)group;
        }
        // the instance copy in shared memory is replaced next: every thread is past its last read
        __syncthreads();
    }
}

}  // namespace

size_t batch_ctl_words(int groups) { return (size_t)kCtlGroups + (size_t)kCtlStride * (size_t)groups; }

template <int NS>
static int resident_of() {
    static int cached = -1, cached_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (cached >= 0 && cached_dev == dev) return cached;
    if (cudaFuncSetAttribute(k_batch_solve<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)batch_smem<NS>()) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_solve<NS>, 128 * NS, batch_smem<NS>()) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 0;
    }
    cached = sms * per_sm;
    cached_dev = dev;
    return cached;
}

bool batch_slots_supported(int slots) { return slots == 4 || slots == 6 || slots == 8; }

int batch_resident_blocks(int slots) {
    switch (slots) {
        case 4: return resident_of<4>();
        case 6: return resident_of<6>();
        case 8: return resident_of<8>();
        default: return 0;
    }
}
size_t batch_smem_bytes(int slots) {
    switch (slots) {
        case 4: return batch_smem<4>();
        case 6: return batch_smem<6>();
        case 8: return batch_smem<8>();
        default: return 0;
    }
}

cudaError_t launch_batch_solve(const BatchArgs& A, int nblocks, int slots, cudaStream_t st) {
    if (!batch_slots_supported(slots) || nblocks <= 0 || A.ngroups <= 0 || nblocks > batch_resident_blocks(slots))
        return cudaErrorInvalidConfiguration;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(128 * slots);
    cfg.dynamicSmemBytes = batch_smem_bytes(slots);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    note_kernel_launch();
    if (slots == 4) return cudaLaunchKernelEx(&cfg, k_batch_solve<4>, A);
    if (slots == 6) return cudaLaunchKernelEx(&cfg, k_batch_solve<6>, A);
    return cudaLaunchKernelEx(&cfg, k_batch_solve<8>, A);
}

}  // namespace cmg
