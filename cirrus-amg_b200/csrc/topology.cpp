// Host-side octree topology (see topology.hpp).
#include "topology.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <numeric>

namespace cmg {

uint64_t Topology::key(int level, int i, int j, int k) {
    // 18 bits per coordinate (offset by 4 so that -1 neighbours encode), 8 bits of level
    return ((uint64_t)(level & 0xff) << 56) | ((uint64_t)((i + 4) & 0x3ffff) << 36) |
           ((uint64_t)((j + 4) & 0x3ffff) << 18) | (uint64_t)((k + 4) & 0x3ffff);
}

void Topology::ensure_index() const {
    if (!index_stale_) return;
    index_.clear();
    index_.reserve(2 * tiles_.size() + 16);
    for (int t = 0; t < (int)tiles_.size(); ++t) index_.emplace(key(tiles_[t].level, tiles_[t].c[0], tiles_[t].c[1], tiles_[t].c[2]), t);
    index_stale_ = false;
}

int Topology::find(int level, int i, int j, int k) const {
    if (level < 0 || level >= num_levels_) return -1;
    ensure_index();
    auto it = index_.find(key(level, i, j, k));
    return it == index_.end() ? -1 : it->second;
}

int Topology::set(int level, int i, int j, int k, int type) {
    if (level < 0 || level >= num_levels_) return -1;
    ensure_index();
    uint64_t kk = key(level, i, j, k);
    auto it = index_.find(kk);
    if (it != index_.end()) {
        tiles_[it->second].type = type;
        return it->second;
    }
    int idx = (int)tiles_.size();
    tiles_.push_back(TileRec{level, {i, j, k}, type});
    index_.emplace(kk, idx);
    if (level > max_level_) max_level_ = level;
    return idx;
}

void Topology::update_max_level() {
    max_level_ = -1;
    for (const auto& t : tiles_) max_level_ = std::max(max_level_, t.level);
}

// spawnGhostTiles (src/HAGrid.h:856-889): every empty face neighbour of an
// active tile at level >= 1 whose parent tile is a LEAF becomes a GHOST tile.
void Topology::spawn_ghosts() {
    update_max_level();
    static const int dirs[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int level = max_level_; level > 0; --level) {
        const int nsnap = (int)tiles_.size();
        for (int t = 0; t < nsnap; ++t) {
            const TileRec tr = tiles_[t];
            if (tr.level != level || !(tr.type & (kLeaf | kNonLeaf))) continue;
            for (const auto& d : dirs) {
                int n0 = tr.c[0] + d[0], n1 = tr.c[1] + d[1], n2 = tr.c[2] + d[2];
                if (find(level, n0, n1, n2) >= 0) continue;
                int p = find(level - 1, n0 >> 1, n1 >> 1, n2 >> 1);
                if (p >= 0 && (tiles_[p].type & kLeaf)) set(level, n0, n1, n2, kGhost);
            }
        }
    }
    update_max_level();
}

// refineStep (src/HAGrid.h:1088-1170).  Levels are visited finest first.  A
// LEAF is flagged when its target exceeds its level or when one of its GHOST
// children is flagged; a GHOST is flagged when a same-level LEAF neighbour is.
// Flags are computed from the tile types as they were when the step began
// (the device copy of the tree the reference's flag kernels read).
int Topology::refine_step(const TargetFn& target) {
    const int nsnap = (int)tiles_.size();
    std::vector<int> type0(nsnap);
    std::vector<char> flag(nsnap, 0);
    std::vector<std::vector<int>> by_level(num_levels_);
    for (int t = 0; t < nsnap; ++t) {
        type0[t] = tiles_[t].type;
        by_level[tiles_[t].level].push_back(t);
    }
    auto snap_find = [&](int level, int i, int j, int k) {
        int q = find(level, i, j, k);
        return (q >= 0 && q < nsnap) ? q : -1;
    };
    const int maxl = max_level_;
    int total = 0;
    for (int L = maxl; L >= 0; --L) {
        for (int t : by_level[L]) {
            if (!(type0[t] & kLeaf)) continue;
            const TileRec& tr = tiles_[t];
            bool refine = target(L, tr.c[0], tr.c[1], tr.c[2]) > L;
            if (L < maxl) {
                for (int ci = 0; ci < 8 && !refine; ++ci) {
                    int q = snap_find(L + 1, 2 * tr.c[0] + (ci >> 2), 2 * tr.c[1] + ((ci >> 1) & 1), 2 * tr.c[2] + (ci & 1));
                    if (q >= 0 && (type0[q] & kGhost) && flag[q]) refine = true;
                }
            }
            if (L + 1 >= num_levels_) refine = false;
            flag[t] = refine;
        }
        for (int t : by_level[L]) {
            if (type0[t] != kGhost) continue;
            const TileRec& tr = tiles_[t];
            bool f = false;
            for (int a = 0; a < 6 && !f; ++a) {
                int n[3] = {tr.c[0], tr.c[1], tr.c[2]};
                n[a >> 1] += (a & 1) ? 1 : -1;
                int q = snap_find(L, n[0], n[1], n[2]);
                if (q >= 0 && (type0[q] & kLeaf) && flag[q]) f = true;
            }
            flag[t] = f;
        }
        for (int t : by_level[L]) {
            if (!(type0[t] & kLeaf) || !flag[t]) continue;
            ++total;
            tiles_[t].type = kNonLeaf;
            const int c0 = tiles_[t].c[0], c1 = tiles_[t].c[1], c2 = tiles_[t].c[2];
            for (int ci = 0; ci < 8; ++ci) set(L + 1, 2 * c0 + (ci >> 2), 2 * c1 + ((ci >> 1) & 1), 2 * c2 + (ci & 1), kLeaf);
        }
    }
    update_max_level();
    return total;
}

int Topology::iterative_refine(const TargetFn& target) {
    update_max_level();
    int steps = 0;
    for (;;) {
        int cnt = refine_step(target);
        spawn_ghosts();
        ++steps;
        if (cnt == 0 || steps > 64) break;
    }
    return steps;
}

static uint64_t morton3(int i, int j, int k) {
    uint64_t m = 0;
    for (int b = 0; b < 20; ++b) {
        m |= (uint64_t)((i >> b) & 1) << (3 * b + 2);
        m |= (uint64_t)((j >> b) & 1) << (3 * b + 1);
        m |= (uint64_t)((k >> b) & 1) << (3 * b);
    }
    return m;
}

std::vector<int> Topology::canonicalize() {
    const int n = (int)tiles_.size();
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::vector<uint64_t> mk(n);
    for (int t = 0; t < n; ++t) mk[t] = morton3(tiles_[t].c[0], tiles_[t].c[1], tiles_[t].c[2]);
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        const TileRec &x = tiles_[a], &y = tiles_[b];
        if (x.level != y.level) return x.level < y.level;
        if (x.type != y.type) return x.type < y.type;
        return mk[a] < mk[b];
    });
    std::vector<TileRec> sorted(n);
    for (int t = 0; t < n; ++t) sorted[t] = tiles_[order[t]];
    tiles_.swap(sorted);
    index_.clear();
    index_.reserve(2 * n + 16);
    for (int t = 0; t < n; ++t) index_.emplace(key(tiles_[t].level, tiles_[t].c[0], tiles_[t].c[1], tiles_[t].c[2]), t);
    update_max_level();

    nb.assign((size_t)8 * n, -1);
    child.assign((size_t)8 * n, -1);
    for (int t = 0; t < n; ++t) {
        const TileRec& tr = tiles_[t];
        for (int a = 0; a < 3; ++a) {
            int m[3] = {tr.c[0], tr.c[1], tr.c[2]}, p[3] = {tr.c[0], tr.c[1], tr.c[2]};
            --m[a];
            ++p[a];
            nb[8 * t + a] = find(tr.level, m[0], m[1], m[2]);
            nb[8 * t + 3 + a] = find(tr.level, p[0], p[1], p[2]);
        }
        nb[8 * t + 6] = find(tr.level - 1, tr.c[0] >> 1, tr.c[1] >> 1, tr.c[2] >> 1);
        for (int ci = 0; ci < 8; ++ci)
            child[8 * t + ci] = find(tr.level + 1, 2 * tr.c[0] + (ci >> 2), 2 * tr.c[1] + ((ci >> 1) & 1), 2 * tr.c[2] + (ci & 1));
    }
    set_ranges();
    return order;
}

void Topology::adopt(std::vector<TileRec>&& sorted, std::vector<int>&& nb_table, std::vector<int>&& child_table) {
    tiles_ = std::move(sorted);
    nb = std::move(nb_table);
    child = std::move(child_table);
    index_.clear();
    index_stale_ = true;
    update_max_level();
    set_ranges();
}

void Topology::set_ranges() {
    const int n = (int)tiles_.size();
    level_begin.assign(num_levels_, n);
    level_end.assign(num_levels_, n);
    nonleaf_begin.assign(num_levels_, n);
    ghost_begin.assign(num_levels_, n);
    leaf_list.clear();
    for (int L = 0; L < num_levels_; ++L) {
        auto lb = std::lower_bound(tiles_.begin(), tiles_.end(), L, [](const TileRec& r, int l) { return r.level < l; });
        auto le = std::lower_bound(tiles_.begin(), tiles_.end(), L + 1, [](const TileRec& r, int l) { return r.level < l; });
        level_begin[L] = (int)(lb - tiles_.begin());
        level_end[L] = (int)(le - tiles_.begin());
        int nlb = level_end[L], gb = level_end[L];
        for (int t = level_begin[L]; t < level_end[L]; ++t) {
            if (tiles_[t].type != kLeaf && nlb == level_end[L]) nlb = t;
            if (tiles_[t].type == kGhost && gb == level_end[L]) gb = t;
            if (tiles_[t].type == kLeaf) leaf_list.push_back(t);
        }
        if (nlb > gb) nlb = gb;
        nonleaf_begin[L] = nlb;
        ghost_begin[L] = gb;
    }
}

// ---------------------------------------------------------------------------
// built-in targets, float arithmetic as in tests/TestGrids.cuh
// ---------------------------------------------------------------------------
static float phi_sphere_quarter(const float p[3]) {  // TestGrids.cuh:60-64
    float dx = p[0] - 0.5f, dy = p[1] - 0.5f, dz = p[2] - 0.5f;
    return std::sqrt(dx * dx + dy * dy + dz * dz) - 0.25f;
}
static float phi_star(const float p[3]) {  // TestGrids.cuh:97-107
    float x = p[0] - 0.5f, y = p[1] - 0.5f, z = p[2] - 0.5f;
    float r = std::sqrt(x * x + y * y + z * z);
    if (r == 0) return -FLT_MAX;
    float theta = std::acos(z / r);
    float ph = std::atan2(y, x);
    float r0 = (float)(0.237 + 0.079 * std::cos(6 * theta) * std::cos(6 * ph));
    return r - r0;
}
template <class Phi>
static int corners_inside(Phi phi, const float mn[3], const float mx[3], float iso) {
    int cnt = 0;
    for (int d = 0; d < 8; ++d) {
        float p[3] = {(d & 4) ? mx[0] : mn[0], (d & 2) ? mx[1] : mn[1], (d & 1) ? mx[2] : mn[2]};
        if (phi(p) - iso < 0) ++cnt;
    }
    return cnt;
}
static double surface_distance(const double mn[3], const double mx[3], const double c[3], double r) {
    double near2 = 0, far2 = 0;
    for (int d = 0; d < 3; ++d) {
        double lo = mn[d] - c[d], hi = mx[d] - c[d];
        double nd = lo > 0 ? lo : (hi < 0 ? -hi : 0.0);
        double fd = std::max(std::fabs(lo), std::fabs(hi));
        near2 += nd * nd;
        far2 += fd * fd;
    }
    double dn = std::sqrt(near2), df = std::sqrt(far2);
    if (dn <= r && r <= df) return 0;
    return r < dn ? dn - r : r - df;
}

int case_target(int case_id, const double* prm, int nprm, float h0, int level, const int c[3]) {
    const int min_level = (int)prm[0], max_level = (int)prm[1];
    const float h = h0 / (float)(1 << level);
    float mn[3], mx[3];
    double dmn[3], dmx[3];
    for (int d = 0; d < 3; ++d) {
        mn[d] = ((float)c[d] * 8.0f) * h;
        mx[d] = ((float)(c[d] + 1) * 8.0f) * h;
        dmn[d] = c[d] * 8.0 * (double)h;
        dmx[d] = (c[d] + 1) * 8.0 * (double)h;
    }
    switch (case_id) {
    case 0: return max_level;
    case 1: {
        const float e = (float)1e-6;
        bool in = true;
        for (int d = 0; d < 3; ++d)
            if (0.5f < mn[d] - e || 0.5f > mx[d] + e) in = false;
        return in ? max_level : min_level;
    }
    case 2: {
        int k = corners_inside(phi_sphere_quarter, mn, mx, 0.0f);
        return (k == 0 || k == 8) ? min_level : max_level;
    }
    case 3: {
        int k0 = corners_inside(phi_sphere_quarter, mn, mx, 0.0f), k1 = corners_inside(phi_sphere_quarter, mn, mx, 0.01f);
        return (k0 == 8 || k1 == 0) ? min_level : max_level;
    }
    case 4: {
        int k = corners_inside(phi_star, mn, mx, 0.0f);
        return (k == 0 || k == 8) ? min_level : max_level;
    }
    case 5: {
        int k0 = corners_inside(phi_star, mn, mx, 0.0f), k1 = corners_inside(phi_star, mn, mx, 0.01f);
        return (k0 == 8 || k1 == 0) ? min_level : max_level;
    }
    case 6: {
        if (nprm < 9) return min_level;
        const double cc[3] = {prm[3], prm[4], prm[5]};
        double dist = surface_distance(dmn, dmx, cc, prm[6]);
        return dist <= prm[7] ? max_level : (dist <= prm[8] ? (int)prm[2] : min_level);
    }
    case 7: {
        if (nprm < 4) return min_level;
        const int ns = (int)prm[3];
        for (int s = 0; s < ns && 7 + 4 * s < nprm; ++s) {
            const double cc[3] = {prm[4 + 4 * s], prm[5 + 4 * s], prm[6 + 4 * s]};
            if (surface_distance(dmn, dmx, cc, prm[7 + 4 * s]) <= prm[2]) return max_level;
        }
        return min_level;
    }
    }
    return min_level;
}

uint8_t case_cell_type(int case_id, float h0, int level, const int tc[3], int v) {
    if (case_id != 3 && case_id != 5) return kInterior;
    const float h = h0 / (float)(1 << level);
    const int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
    float mn[3], mx[3];
    for (int d = 0; d < 3; ++d) {
        int g = tc[d] * 8 + l[d];
        mn[d] = (float)g * h;
        mx[d] = (float)(g + 1) * h;
    }
    int k = (case_id == 3) ? corners_inside(phi_sphere_quarter, mn, mx, 0.0f) : corners_inside(phi_star, mn, mx, 0.0f);
    return k == 8 ? kNeumann : kInterior;
}

}  // namespace cmg
