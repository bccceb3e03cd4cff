// Octree topology built on the device: HADeviceGrid::iterativeRefine with its refineStep
// (src/HAGrid.h:1088-1182), spawnGhostTiles (:856-889) and the canonical tile order and
// index tables of Topology::canonicalize, for the built-in refinement targets.
//
// The reference marks refinement flags on the device but creates tiles, spawns ghosts and
// rebuilds its hash tables on the host, one level at a time.  Here the whole build stays
// in device memory:
//   - tiles live in a pool of records (level | type << 8, tile coordinate), indices handed
//     out by an atomic counter;
//   - an open-addressing hash table maps a tile key to its index; inserts are
//     insert-if-absent by compare-and-swap, so two tiles that spawn the same ghost create
//     it once;
//   - a refinement step runs two kernels per level, finest first: LEAF flags (target above
//     the level, or a flagged GHOST child), then GHOST flags and the refinement of the
//     flagged LEAF tiles, all judged on the tile types as they were when the step began;
//   - the canonical order (level, then LEAF < NONLEAF < GHOST, then Morton code) is one
//     radix sort of 64-bit keys; the face-neighbour, parent and child tables are hash
//     lookups in the sorted order.
// Tile creation order differs from the host builder's, but the sort makes the result the
// same tiles in the same order with the same tables.  The refinement targets are computed
// with explicitly rounded operations in the order of the host's expressions (no
// contraction), so both builders take the same decisions.  The star cases of
// tests/TestGrids.cuh use transcendental functions whose device and host versions may
// differ in the last bit; they are built on the host.
#include <cub/device/device_radix_sort.cuh>

#include <vector>

#include "topo_device.hpp"

namespace cmg {

namespace {

constexpr unsigned long long kEmpty = ~0ull;

__host__ __device__ inline unsigned long long tkey(int level, int i, int j, int k) {
    // Topology::key: 8 bits of level, 18 bits per coordinate offset by 4
    return ((unsigned long long)(level & 0xff) << 56) | ((unsigned long long)((i + 4) & 0x3ffff) << 36) |
           ((unsigned long long)((j + 4) & 0x3ffff) << 18) | (unsigned long long)((k + 4) & 0x3ffff);
}
__device__ inline unsigned hslot(unsigned long long key, unsigned mask) {
    unsigned long long z = key + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return (unsigned)(z ^ (z >> 31)) & mask;
}

struct Tab {
    unsigned long long* hk;
    int* hv;
    unsigned mask;
    int4* rec;  // (level | type << 8, c0, c1, c2)
    int cap;
    int* count;
    int* err;
    __device__ int find(int level, int i, int j, int k) const {
        if (level < 0) return -1;
        const unsigned long long key = tkey(level, i, j, k);
        unsigned h = hslot(key, mask);
        for (unsigned p = 0; p <= mask; ++p, h = (h + 1) & mask) {
            const unsigned long long v = hk[h];
            if (v == key) return hv[h];
            if (v == kEmpty) return -1;
        }
        return -1;
    }
    // insert-if-absent: the index of the tile (new or existing); -1 on overflow
    __device__ int insert(int level, int i, int j, int k, int type, bool* created) const {
        const unsigned long long key = tkey(level, i, j, k);
        unsigned h = hslot(key, mask);
        for (unsigned p = 0; p <= mask; ++p, h = (h + 1) & mask) {
            const unsigned long long prev = atomicCAS(hk + h, kEmpty, key);
            if (prev == kEmpty) {
                const int idx = atomicAdd(count, 1);
                if (idx >= cap) {
                    atomicExch(err, 1);
                    hv[h] = -1;
                    *created = false;
                    return -1;
                }
                rec[idx] = make_int4(level | (type << 8), i, j, k);
                hv[h] = idx;
                *created = true;
                return idx;
            }
            if (prev == key) {
                *created = false;
                return hv[h];
            }
        }
        atomicExch(err, 2);
        *created = false;
        return -1;
    }
};

__device__ inline int rec_level(int4 r) { return r.x & 0xff; }
__device__ inline int rec_type(int4 r) { return (r.x >> 8) & 0xff; }

// ---- refinement targets (topology.cpp case_target), explicitly rounded ----
struct Target {
    int case_id, nprm;
    double prm[kDevTopoMaxParams];
    float h0;
};
__device__ float phi_quarter(float px, float py, float pz) {  // tests/TestGrids.cuh:60-64
    const float dx = __fsub_rn(px, 0.5f), dy = __fsub_rn(py, 0.5f), dz = __fsub_rn(pz, 0.5f);
    return __fsub_rn(__fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz))), 0.25f);
}
__device__ int corners_in_quarter(const float mn[3], const float mx[3], float iso) {
    int cnt = 0;
    for (int d = 0; d < 8; ++d) {
        const float v = phi_quarter((d & 4) ? mx[0] : mn[0], (d & 2) ? mx[1] : mn[1], (d & 1) ? mx[2] : mn[2]);
        if (__fsub_rn(v, iso) < 0.0f) ++cnt;
    }
    return cnt;
}
__device__ double surface_distance(const double mn[3], const double mx[3], const double c[3], double r) {
    double near2 = 0.0, far2 = 0.0;
    for (int d = 0; d < 3; ++d) {
        const double lo = __dsub_rn(mn[d], c[d]), hi = __dsub_rn(mx[d], c[d]);
        const double nd = lo > 0 ? lo : (hi < 0 ? -hi : 0.0);
        const double fd = fmax(fabs(lo), fabs(hi));
        near2 = __dadd_rn(near2, __dmul_rn(nd, nd));
        far2 = __dadd_rn(far2, __dmul_rn(fd, fd));
    }
    const double dn = __dsqrt_rn(near2), df = __dsqrt_rn(far2);
    if (dn <= r && r <= df) return 0.0;
    return r < dn ? __dsub_rn(dn, r) : __dsub_rn(r, df);
}
__device__ int target_of(const Target& T, int level, const int c[3]) {
    const double* prm = T.prm;
    const int min_level = (int)prm[0], max_level = (int)prm[1];
    const float h = __fdiv_rn(T.h0, (float)(1 << level));
    float mn[3], mx[3];
    double dmn[3], dmx[3];
    for (int d = 0; d < 3; ++d) {
        mn[d] = __fmul_rn(__fmul_rn((float)c[d], 8.0f), h);
        mx[d] = __fmul_rn(__fmul_rn((float)(c[d] + 1), 8.0f), h);
        dmn[d] = __dmul_rn(__dmul_rn((double)c[d], 8.0), (double)h);
        dmx[d] = __dmul_rn(__dmul_rn((double)(c[d] + 1), 8.0), (double)h);
    }
    switch (T.case_id) {
    case 0: return max_level;
    case 1: {
        const float e = (float)1e-6;
        bool in = true;
        for (int d = 0; d < 3; ++d)
            if (0.5f < __fsub_rn(mn[d], e) || 0.5f > __fadd_rn(mx[d], e)) in = false;
        return in ? max_level : min_level;
    }
    case 2: {
        const int k = corners_in_quarter(mn, mx, 0.0f);
        return (k == 0 || k == 8) ? min_level : max_level;
    }
    case 3: {
        const int k0 = corners_in_quarter(mn, mx, 0.0f), k1 = corners_in_quarter(mn, mx, 0.01f);
        return (k0 == 8 || k1 == 0) ? min_level : max_level;
    }
    case 6: {
        if (T.nprm < 9) return min_level;
        const double cc[3] = {prm[3], prm[4], prm[5]};
        const double dist = surface_distance(dmn, dmx, cc, prm[6]);
        return dist <= prm[7] ? max_level : (dist <= prm[8] ? (int)prm[2] : min_level);
    }
    case 7: {
        if (T.nprm < 4) return min_level;
        const int ns = (int)prm[3];
        for (int s = 0; s < ns && 7 + 4 * s < T.nprm; ++s) {
            const double cc[3] = {prm[4 + 4 * s], prm[5 + 4 * s], prm[6 + 4 * s]};
            if (surface_distance(dmn, dmx, cc, prm[7 + 4 * s]) <= prm[2]) return max_level;
        }
        return min_level;
    }
    }
    return min_level;
}

// ---- kernels ----
__global__ void k_hash_clear(unsigned long long* hk, int* hv, unsigned n) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        hk[i] = kEmpty;
        hv[i] = -1;
    }
}
// index the first n records (after an upload or the sort)
__global__ void k_hash_fill(Tab T, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int4 r = T.rec[t];
    const unsigned long long key = tkey(rec_level(r), r.y, r.z, r.w);
    unsigned h = hslot(key, T.mask);
    for (unsigned p = 0; p <= T.mask; ++p, h = (h + 1) & T.mask) {
        if (atomicCAS(T.hk + h, kEmpty, key) == kEmpty) {
            T.hv[h] = t;
            return;
        }
    }
    atomicExch(T.err, 2);
}
__global__ void k_snapshot(const int4* rec, int* type0, int* flag, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    type0[t] = rec_type(rec[t]);
    flag[t] = 0;
}
// refineStep, LEAF flags of level L: target above the level, or a flagged GHOST child
__global__ void k_flag_leaf(Tab T, Target tg, const int* type0, int* flag, int nsnap, int L, int maxl, int num_levels) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsnap) return;
    const int4 r = T.rec[t];
    if (rec_level(r) != L || !(type0[t] & kLeaf)) return;
    const int c[3] = {r.y, r.z, r.w};
    bool refine = target_of(tg, L, c) > L;
    if (L < maxl) {
        for (int ci = 0; ci < 8 && !refine; ++ci) {
            const int q = T.find(L + 1, 2 * c[0] + (ci >> 2), 2 * c[1] + ((ci >> 1) & 1), 2 * c[2] + (ci & 1));
            if (q >= 0 && q < nsnap && (type0[q] & kGhost) && flag[q]) refine = true;
        }
    }
    if (L + 1 >= num_levels) refine = false;
    flag[t] = refine ? 1 : 0;
}
// GHOST flags of level L (a flagged LEAF face neighbour) and the refinement of the flagged
// LEAF tiles of level L: the tile becomes NONLEAF, its 8 children LEAF (new or retyped)
__global__ void k_ghost_and_refine(Tab T, const int* type0, int* flag, int nsnap, int L, int* refined, int* maxl) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsnap) return;
    const int4 r = T.rec[t];
    if (rec_level(r) != L) return;
    if (type0[t] == kGhost) {
        bool f = false;
        for (int a = 0; a < 6 && !f; ++a) {
            int n[3] = {r.y, r.z, r.w};
            n[a >> 1] += (a & 1) ? 1 : -1;
            const int q = T.find(L, n[0], n[1], n[2]);
            if (q >= 0 && q < nsnap && (type0[q] & kLeaf) && flag[q]) f = true;
        }
        flag[t] = f ? 1 : 0;
        return;
    }
    if (!(type0[t] & kLeaf) || !flag[t]) return;
    atomicAdd(refined, 1);
    T.rec[t].x = L | (kNonLeaf << 8);
    for (int ci = 0; ci < 8; ++ci) {
        bool created = false;
        const int q = T.insert(L + 1, 2 * r.y + (ci >> 2), 2 * r.z + ((ci >> 1) & 1), 2 * r.w + (ci & 1), kLeaf, &created);
        if (q >= 0 && !created) T.rec[q].x = (L + 1) | (kLeaf << 8);
    }
    atomicMax(maxl, L + 1);
}
// spawnGhostTiles: every empty face neighbour of an active tile at level >= 1 whose parent
// tile is a LEAF becomes a GHOST tile
__global__ void k_spawn_ghosts(Tab T, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int4 r = T.rec[t];
    const int L = rec_level(r);
    if (L < 1 || !(rec_type(r) & (kLeaf | kNonLeaf))) return;
    for (int a = 0; a < 6; ++a) {
        int m[3] = {r.y, r.z, r.w};
        m[a >> 1] += (a & 1) ? 1 : -1;
        if (T.find(L, m[0], m[1], m[2]) >= 0) continue;
        const int p = T.find(L - 1, m[0] >> 1, m[1] >> 1, m[2] >> 1);
        if (p < 0 || !(rec_type(T.rec[p]) & kLeaf)) continue;
        bool created = false;
        T.insert(L, m[0], m[1], m[2], kGhost, &created);
    }
}
// canonical order: level, then tile type (LEAF 1 < NONLEAF 2 < GHOST 4), then Morton code
__device__ unsigned long long morton3(int i, int j, int k) {
    unsigned long long m = 0;
    for (int b = 0; b < 19; ++b) {
        m |= (unsigned long long)((i >> b) & 1) << (3 * b + 2);
        m |= (unsigned long long)((j >> b) & 1) << (3 * b + 1);
        m |= (unsigned long long)((k >> b) & 1) << (3 * b);
    }
    return m;
}
__global__ void k_sort_keys(const int4* rec, unsigned long long* keys, int* idx, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int4 r = rec[t];
    keys[t] = ((unsigned long long)rec_level(r) << 60) | ((unsigned long long)rec_type(r) << 57) | morton3(r.y, r.z, r.w);
    idx[t] = t;
}
__global__ void k_gather(const int4* rec, const int* order, int4* out, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = rec[order[t]];
}
// face neighbours (-x,-y,-z,+x,+y,+z), parent, -1; children dx*4 + dy*2 + dz
__global__ void k_tables(Tab T, int n, int* nb, int* child) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int4 r = T.rec[t];
    const int L = rec_level(r);
    const int c[3] = {r.y, r.z, r.w};
    for (int a = 0; a < 3; ++a) {
        int m[3] = {c[0], c[1], c[2]}, p[3] = {c[0], c[1], c[2]};
        --m[a];
        ++p[a];
        nb[8 * t + a] = T.find(L, m[0], m[1], m[2]);
        nb[8 * t + 3 + a] = T.find(L, p[0], p[1], p[2]);
    }
    nb[8 * t + 6] = T.find(L - 1, c[0] >> 1, c[1] >> 1, c[2] >> 1);
    nb[8 * t + 7] = -1;
    for (int ci = 0; ci < 8; ++ci) child[8 * t + ci] = T.find(L + 1, 2 * c[0] + (ci >> 2), 2 * c[1] + ((ci >> 1) & 1), 2 * c[2] + (ci & 1));
}

// CreateTestGrid's LEAF cell types (tests/TestGrids.cuh:161-167, topology.cpp case_cell_type):
// NEUMANN where all 8 corners of the cell are inside the solid sphere (case 3), else INTERIOR
__global__ void __launch_bounds__(128) k_leaf_case_types(const int4* meta, uint8_t* ctype, const int* leaf, int case_id, float h0) {
    const int t = leaf[blockIdx.x];
    const int4 m = meta[t];
    const int level = m.x & 0xff;
    const float h = __fdiv_rn(h0, (float)(1 << level));
    uint8_t* out = ctype + (size_t)t * 512;
    for (int v = threadIdx.x; v < 512; v += 128) {
        uint8_t ty = kInterior;
        if (case_id == 3) {
            const int l[3] = {v >> 6, (v >> 3) & 7, v & 7}, tc[3] = {m.y, m.z, m.w};
            float mn[3], mx[3];
            for (int d = 0; d < 3; ++d) {
                const int gc = tc[d] * 8 + l[d];
                mn[d] = __fmul_rn((float)gc, h);
                mx[d] = __fmul_rn((float)(gc + 1), h);
            }
            ty = corners_in_quarter(mn, mx, 0.0f) == 8 ? kNeumann : kInterior;
        }
        out[v] = ty;
    }
}

}  // namespace

bool device_cell_types_supported(int case_id) { return case_id >= 0 && case_id <= 7 && case_id != 5; }

cudaError_t device_leaf_cell_types(const int4* meta, uint8_t* ctype, const int* leaf, int nleaf, int case_id, float h0, cudaStream_t st) {
    if (nleaf <= 0) return cudaSuccess;
    k_leaf_case_types<<<nleaf, 128, 0, st>>>(meta, ctype, leaf, case_id, h0);
    return cudaGetLastError();
}

DeviceTopoBuilder::~DeviceTopoBuilder() {
    st = nullptr;  // the owner's stream may be gone; its work has been waited for
    release();
}

void DeviceTopoBuilder::release() {
    for (void* p : {(void*)hk, (void*)hv, (void*)rec, (void*)rec2, (void*)type0, (void*)flag, (void*)keys, (void*)keys2, (void*)idx,
                    (void*)idx2, (void*)nb, (void*)child, (void*)scal, sort_tmp})
        pool_release(p, st);
    hk = nullptr;
    hv = nullptr;
    rec = rec2 = nullptr;
    type0 = flag = idx = idx2 = nb = child = scal = nullptr;
    keys = keys2 = nullptr;
    sort_tmp = nullptr;
    cap = 0;
    hcap = 0;
    sort_tmp_bytes = 0;
}

cudaError_t DeviceTopoBuilder::reserve(int need) {
    if (need <= cap) return cudaSuccess;
    release();
    int c = 1 << 14;
    while (c < need) c <<= 1;
    unsigned h = 1u << 15;
    while (h < 2u * (unsigned)c) h <<= 1;
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = pool_malloc(p, bytes, dev, st);
    };
    A((void**)&hk, sizeof(unsigned long long) * h);
    A((void**)&hv, sizeof(int) * h);
    A((void**)&rec, sizeof(int4) * c);
    A((void**)&rec2, sizeof(int4) * c);
    A((void**)&type0, sizeof(int) * c);
    A((void**)&flag, sizeof(int) * c);
    A((void**)&keys, sizeof(unsigned long long) * c);
    A((void**)&keys2, sizeof(unsigned long long) * c);
    A((void**)&idx, sizeof(int) * c);
    A((void**)&idx2, sizeof(int) * c);
    A((void**)&nb, sizeof(int) * 8 * (size_t)c);
    A((void**)&child, sizeof(int) * 8 * (size_t)c);
    A((void**)&scal, sizeof(int) * 8);
    if (e == cudaSuccess) {
        size_t tb = 0;
        e = cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, idx, idx2, c);
        if (e == cudaSuccess) A(&sort_tmp, tb);
        sort_tmp_bytes = tb;
    }
    if (e != cudaSuccess) {
        release();
        return e;
    }
    cap = c;
    hcap = h;
    return cudaSuccess;
}

bool device_case_supported(int case_id) { return case_id == 0 || case_id == 1 || case_id == 2 || case_id == 3 || case_id == 6 || case_id == 7; }

int device_refine_case(DeviceTopoBuilder& B, Topology& topo, int case_id, const double* params, int nparams, cudaStream_t st, int* steps) {
    if (!device_case_supported(case_id) || nparams < 2 || nparams > kDevTopoMaxParams) return 1;
    const std::vector<TileRec>& cur = topo.tiles();
    int n = (int)cur.size();
    if (n == 0) return 1;
    // scal: [0] count, [1] error, [2] refined in this step, [3] max level
    int need = n < 1024 ? 1024 : 2 * n;
    B.st = st;
    for (;;) {
        if (B.reserve(need) != cudaSuccess) return 2;
        std::vector<int4> h(n);
        int maxl = -1;
        for (int t = 0; t < n; ++t) {
            h[t] = make_int4(cur[t].level | (cur[t].type << 8), cur[t].c[0], cur[t].c[1], cur[t].c[2]);
            maxl = cur[t].level > maxl ? cur[t].level : maxl;
        }
        if (n > 0 && cudaMemcpyAsync(B.rec, h.data(), sizeof(int4) * n, cudaMemcpyHostToDevice, st) != cudaSuccess) return 2;
        int hs[8] = {n, 0, 0, maxl, 0, 0, 0, 0};
        if (cudaMemcpyAsync(B.scal, hs, sizeof(hs), cudaMemcpyHostToDevice, st) != cudaSuccess) return 2;
        Tab T{B.hk, B.hv, B.hcap - 1u, B.rec, B.cap, B.scal, B.scal + 1};
        k_hash_clear<<<(B.hcap + 255) / 256, 256, 0, st>>>(B.hk, B.hv, B.hcap);
        if (n > 0) k_hash_fill<<<(n + 255) / 256, 256, 0, st>>>(T, n);
        Target tg{};
        tg.case_id = case_id;
        tg.nprm = nparams;
        for (int i = 0; i < nparams; ++i) tg.prm[i] = params[i];
        tg.h0 = topo.h0();
        int nsteps = 0, err = 0;
        for (;;) {
            const int nsnap = hs[0];
            const int ms = hs[3];
            k_snapshot<<<(nsnap + 255) / 256, 256, 0, st>>>(B.rec, B.type0, B.flag, nsnap);
            cudaMemsetAsync(B.scal + 2, 0, sizeof(int), st);
            for (int L = ms; L >= 0; --L) {
                k_flag_leaf<<<(nsnap + 255) / 256, 256, 0, st>>>(T, tg, B.type0, B.flag, nsnap, L, ms, topo.num_levels());
                k_ghost_and_refine<<<(nsnap + 255) / 256, 256, 0, st>>>(T, B.type0, B.flag, nsnap, L, B.scal + 2, B.scal + 3);
            }
            if (cudaMemcpyAsync(hs, B.scal, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
                return 2;
            err = hs[1];
            if (err) break;
            const int ncur = hs[0];
            k_spawn_ghosts<<<(ncur + 255) / 256, 256, 0, st>>>(T, ncur);
            if (cudaMemcpyAsync(hs, B.scal, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
                return 2;
            err = hs[1];
            ++nsteps;
            if (err || hs[2] == 0 || nsteps > 64) break;
        }
        if (err == 1) {  // pool full: start over with twice the room
            need = 2 * B.cap;
            continue;
        }
        if (err) return 2;
        // canonical order and tables
        n = hs[0];
        k_sort_keys<<<(n + 255) / 256, 256, 0, st>>>(B.rec, B.keys, B.idx, n);
        size_t tb = B.sort_tmp_bytes;
        if (cub::DeviceRadixSort::SortPairs(B.sort_tmp, tb, B.keys, B.keys2, B.idx, B.idx2, n, 0, 64, st) != cudaSuccess) return 2;
        k_gather<<<(n + 255) / 256, 256, 0, st>>>(B.rec, B.idx2, B.rec2, n);
        Tab S{B.hk, B.hv, B.hcap - 1u, B.rec2, B.cap, B.scal, B.scal + 1};
        k_hash_clear<<<(B.hcap + 255) / 256, 256, 0, st>>>(B.hk, B.hv, B.hcap);
        k_hash_fill<<<(n + 255) / 256, 256, 0, st>>>(S, n);
        k_tables<<<(n + 255) / 256, 256, 0, st>>>(S, n, B.nb, B.child);
        std::vector<int4> hr(n);
        std::vector<int> hnb((size_t)8 * n), hch((size_t)8 * n);
        if (cudaMemcpyAsync(hr.data(), B.rec2, sizeof(int4) * n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(hnb.data(), B.nb, sizeof(int) * 8 * (size_t)n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(hch.data(), B.child, sizeof(int) * 8 * (size_t)n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(hs, B.scal, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
            return 2;
        if (hs[1] || cudaGetLastError() != cudaSuccess) return 2;
        std::vector<TileRec> tiles(n);
        for (int t = 0; t < n; ++t) tiles[t] = TileRec{hr[t].x & 0xff, {hr[t].y, hr[t].z, hr[t].w}, (hr[t].x >> 8) & 0xff};
        topo.adopt(std::move(tiles), std::move(hnb), std::move(hch));
        if (steps) *steps = nsteps;
        return 0;
    }
}

}  // namespace cmg
