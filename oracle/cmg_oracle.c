/*
 * cmg_oracle.c -- CPU oracle (test infrastructure only) for the Cirrus-amg
 * octree MG-preconditioned CG pressure-Poisson solve.
 *
 * This file is the checker the CUDA product is compared against.  It is a
 * restatement in plain C of the reference's algorithm, written from the
 * reference's behaviour; each function names the reference file:line it
 * follows.  Floating-point steps follow the reference's order and its FMA
 * contractions (written here as explicit fmaf) so that a float run of the
 * oracle tracks the reference CUDA solver closely.
 *
 * Layout (oracle-internal): tiles sorted by (level, tile type, Morton code
 * of the tile coordinate); channel c of tile t, cell v at
 * data[(c * n + t) * 512 + v]; cell index v = i*64 + j*8 + k
 * (HAAccessor.h:32-42).
 */
#include "cmg_oracle.h"
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NC 512
/* nearest BF16 (ties to even), as a float: the storage of the mixed-precision cycle's x and
 * rhs on levels >= 3 (finite values) */
static float bf16_round(float v) {
    uint32_t u;
    memcpy(&u, &v, 4);
    u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    memcpy(&v, &u, 4);
    return v;
}
#define XS(g, level, v) (((g)->x_bf16 && (level) >= 3) ? bf16_round(v) : (v))
#define CELL(i, j, k) (((i) << 6) | ((j) << 3) | (k))
#define SX(i, j, k) (((i) + 1) * 100 + ((j) + 1) * 10 + ((k) + 1))

typedef struct {
    int level, c[3];
    int type;
    int flag;
} og_tile;

struct og_grid {
    float h0;
    int num_levels, max_level;
    int n, cap;
    og_tile* t;
    uint64_t* hkeys;
    int* hvals;
    int hcap, hcount;
    int* nbr;    /* [n][6]: 0..2 = -x,-y,-z ; 3..5 = +x,+y,+z  (PoissonTile.h:130) */
    int* parent; /* tile holding the parent cells, level-1 */
    int* child;  /* [n][8], index dx*4+dy*2+dz */
    int nch;
    float* data;
    uint8_t* ctype;
    int ref_mask; /* apply CoarsenOffDiagCoefficientsOneStepKernel's cell-type mask to the stored types */
    int x_bf16;   /* the mixed-precision cycle: x and rhs of levels >= 3 stored in BF16 */
};

/* ------------------------------------------------------------------ */
/* tile registry: open-addressing map (level, i, j, k) -> tile index    */
/* ------------------------------------------------------------------ */
static uint64_t key_of(int level, int i, int j, int k) {
    return ((uint64_t)(level & 0xff) << 56) | ((uint64_t)((i + 4) & 0x3ffff) << 36) |
           ((uint64_t)((j + 4) & 0x3ffff) << 18) | (uint64_t)((k + 4) & 0x3ffff);
}
static uint64_t mix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}
static void map_clear(og_grid* g, int cap) {
    free(g->hkeys); free(g->hvals);
    g->hcap = cap; g->hcount = 0;
    g->hkeys = (uint64_t*)malloc(sizeof(uint64_t) * cap);
    g->hvals = (int*)malloc(sizeof(int) * cap);
    for (int i = 0; i < cap; i++) g->hvals[i] = -1;
}
static int map_find(const og_grid* g, int level, int i, int j, int k) {
    if (level < 0 || level >= g->num_levels) return -1;
    uint64_t key = key_of(level, i, j, k);
    int mask = g->hcap - 1;
    int s = (int)(mix64(key) & (uint64_t)mask);
    while (g->hvals[s] >= 0) {
        if (g->hkeys[s] == key) return g->hvals[s];
        s = (s + 1) & mask;
    }
    return -1;
}
static void map_put(og_grid* g, uint64_t key, int val) {
    int mask = g->hcap - 1;
    int s = (int)(mix64(key) & (uint64_t)mask);
    while (g->hvals[s] >= 0) {
        if (g->hkeys[s] == key) { g->hvals[s] = val; return; }
        s = (s + 1) & mask;
    }
    g->hkeys[s] = key; g->hvals[s] = val; g->hcount++;
}
static void map_rebuild(og_grid* g) {
    int cap = 1024;
    while (cap < 4 * (g->n + 16)) cap <<= 1;
    map_clear(g, cap);
    for (int t = 0; t < g->n; t++) map_put(g, key_of(g->t[t].level, g->t[t].c[0], g->t[t].c[1], g->t[t].c[2]), t);
}
static void free_derived(og_grid* g) {
    free(g->nbr); free(g->parent); free(g->child); free(g->data); free(g->ctype);
    g->nbr = g->parent = g->child = NULL; g->data = NULL; g->ctype = NULL; g->nch = 0;
}

og_grid* og_grid_new(float h0, int num_levels) {
    og_grid* g = (og_grid*)calloc(1, sizeof(og_grid));
    g->h0 = h0; g->num_levels = num_levels; g->max_level = -1;
    g->cap = 64; g->t = (og_tile*)malloc(sizeof(og_tile) * g->cap);
    map_clear(g, 1024);
    return g;
}
void og_grid_free(og_grid* g) {
    if (!g) return;
    free_derived(g); free(g->t); free(g->hkeys); free(g->hvals); free(g);
}
/* HADeviceGrid::setTileHost (HAGrid.h:526): create or retype a tile. */
int og_set_tile(og_grid* g, int level, int i, int j, int k, int type) {
    if (level < 0 || level >= g->num_levels) return -1;
    int idx = map_find(g, level, i, j, k);
    if (idx >= 0) { g->t[idx].type = type; return idx; }
    if (g->n == g->cap) { g->cap *= 2; g->t = (og_tile*)realloc(g->t, sizeof(og_tile) * g->cap); }
    idx = g->n++;
    g->t[idx].level = level; g->t[idx].c[0] = i; g->t[idx].c[1] = j; g->t[idx].c[2] = k;
    g->t[idx].type = type; g->t[idx].flag = 0;
    if (2 * (g->hcount + 1) > g->hcap) map_rebuild(g); else map_put(g, key_of(level, i, j, k), idx);
    return idx;
}
static void compute_max_level(og_grid* g) {
    g->max_level = -1;
    for (int t = 0; t < g->n; t++) if (g->t[t].level > g->max_level) g->max_level = g->t[t].level;
}

/* HADeviceGrid::spawnGhostTiles (HAGrid.h:856-889): an empty same-level
 * face neighbour of an active tile whose parent is a LEAF becomes GHOST. */
static void spawn_ghosts(og_grid* g) {
    compute_max_level(g);
    for (int level = g->max_level; level > 0; level--) {
        int nsnap = g->n;
        for (int t = 0; t < nsnap; t++) {
            if (g->t[t].level != level || !(g->t[t].type & (OG_LEAF | OG_NONLEAF))) continue;
            for (int a = 0; a < 6; a++) {
                int n[3] = {g->t[t].c[0], g->t[t].c[1], g->t[t].c[2]};
                n[a >> 1] += (a & 1) ? 1 : -1;
                if (map_find(g, level, n[0], n[1], n[2]) >= 0) continue;
                int p = map_find(g, level - 1, n[0] >> 1, n[1] >> 1, n[2] >> 1);
                if (p >= 0 && (g->t[p].type & OG_LEAF)) og_set_tile(g, level, n[0], n[1], n[2], OG_GHOST);
            }
        }
    }
    compute_max_level(g);
}

static uint64_t morton3(int i, int j, int k) {
    uint64_t m = 0;
    for (int b = 0; b < 20; b++) {
        m |= (uint64_t)((i >> b) & 1) << (3 * b + 2);
        m |= (uint64_t)((j >> b) & 1) << (3 * b + 1);
        m |= (uint64_t)((k >> b) & 1) << (3 * b);
    }
    return m;
}
static int tile_cmp(const void* a, const void* b) {
    const og_tile* x = (const og_tile*)a;
    const og_tile* y = (const og_tile*)b;
    if (x->level != y->level) return x->level < y->level ? -1 : 1;
    if (x->type != y->type) return x->type < y->type ? -1 : 1;
    uint64_t mx = morton3(x->c[0], x->c[1], x->c[2]), my = morton3(y->c[0], y->c[1], y->c[2]);
    if (mx != my) return mx < my ? -1 : 1;
    return 0;
}
/* Canonical order and the hash-free neighbour/parent/child tables that
 * replace HATileAccessor::findVoxel probes (HAAccessor.h:278) and the
 * per-tile neighbour cache CalculateNeighborTiles (PoissonGrid.cu:139). */
static void finalize(og_grid* g) {
    free_derived(g);
    qsort(g->t, g->n, sizeof(og_tile), tile_cmp);
    map_rebuild(g);
    compute_max_level(g);
    int n = g->n;
    g->nbr = (int*)malloc(sizeof(int) * 6 * (size_t)(n > 0 ? n : 1));
    g->parent = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    g->child = (int*)malloc(sizeof(int) * 8 * (size_t)(n > 0 ? n : 1));
    for (int t = 0; t < n; t++) {
        og_tile* T = &g->t[t];
        for (int a = 0; a < 3; a++) {
            int m[3] = {T->c[0], T->c[1], T->c[2]}, p[3] = {T->c[0], T->c[1], T->c[2]};
            m[a]--; p[a]++;
            g->nbr[t * 6 + a] = map_find(g, T->level, m[0], m[1], m[2]);
            g->nbr[t * 6 + 3 + a] = map_find(g, T->level, p[0], p[1], p[2]);
        }
        g->parent[t] = map_find(g, T->level - 1, T->c[0] >> 1, T->c[1] >> 1, T->c[2] >> 1);
        for (int ci = 0; ci < 8; ci++)
            g->child[t * 8 + ci] = map_find(g, T->level + 1, 2 * T->c[0] + (ci >> 2), 2 * T->c[1] + ((ci >> 1) & 1), 2 * T->c[2] + (ci & 1));
    }
}

/* HADeviceGrid::rebuild (HAGrid.h:892): compress + spawn ghosts. */
int og_rebuild(og_grid* g) {
    spawn_ghosts(g);
    finalize(g);
    return 0;
}

/* ------------------------------------------------------------------ */
/* refinement targets (tests/TestGrids.cuh:7-142) in float arithmetic  */
/* ------------------------------------------------------------------ */
static float voxel_size(const og_grid* g, int level) { return g->h0 / (float)(1 << level); } /* HAAccessor.h:75 */

static float phi_sphere_quarter(const float p[3]) { /* TestGrids.cuh:60-64 */
    float dx = p[0] - 0.5f, dy = p[1] - 0.5f, dz = p[2] - 0.5f;
    return sqrtf(dx * dx + dy * dy + dz * dz) - 0.25f;
}
static float phi_star(const float p[3]) { /* TestGrids.cuh:97-107 */
    float x = p[0] - 0.5f, y = p[1] - 0.5f, z = p[2] - 0.5f;
    float r = sqrtf(x * x + y * y + z * z);
    if (r == 0) return -FLT_MAX;
    float theta = acosf(z / r);
    float ph = atan2f(y, x);
    float r0 = (float)(0.237 + 0.079 * cos(6 * theta) * cos(6 * ph));
    return r - r0;
}
static int corner_count(float (*phi)(const float*), const float mn[3], const float mx[3], float iso) {
    int cnt = 0;
    for (int di = 0; di < 2; di++)
        for (int dj = 0; dj < 2; dj++)
            for (int dk = 0; dk < 2; dk++) {
                float p[3] = {di ? mx[0] : mn[0], dj ? mx[1] : mn[1], dk ? mx[2] : mn[2]};
                if (phi(p) - iso < 0) cnt++;
            }
    return cnt;
}
/* Distance from a tile box to the surface |p - c| = r (0 if the surface
 * crosses the box), in double. */
static double box_sphere_surface_dist(const double mn[3], const double mx[3], const double c[3], double r) {
    double near2 = 0, far2 = 0;
    for (int d = 0; d < 3; d++) {
        double lo = mn[d] - c[d], hi = mx[d] - c[d];
        double nd = (lo > 0) ? lo : (hi < 0 ? -hi : 0);
        double fd = fabs(lo) > fabs(hi) ? fabs(lo) : fabs(hi);
        near2 += nd * nd; far2 += fd * fd;
    }
    double dn = sqrt(near2), df = sqrt(far2);
    if (dn <= r && r <= df) return 0;
    if (r < dn) return dn - r;
    return r - df;
}
static int case_target_at(float h, const int tc[3], int case_id, const double* prm, int nprm) {
    int min_level = (int)prm[0], max_level = (int)prm[1];
    float mn[3], mx[3];
    for (int d = 0; d < 3; d++) { /* HAAccessor.h:123-128 */
        mn[d] = ((float)tc[d] * 8.0f) * h;
        mx[d] = ((float)(tc[d] + 1) * 8.0f) * h;
    }
    switch (case_id) {
    case OG_CASE_UNIFORM: return max_level;
    case OG_CASE_CENTER_POINT: {
        float e = (float)1e-6;
        int in = 1;
        for (int d = 0; d < 3; d++) if (0.5f < mn[d] - e || 0.5f > mx[d] + e) in = 0;
        return in ? max_level : min_level;
    }
    case OG_CASE_SPHERE_EMPTY: {
        int c = corner_count(phi_sphere_quarter, mn, mx, 0.0f);
        return (c == 0 || c == 8) ? min_level : max_level;
    }
    case OG_CASE_SPHERE_SOLID: {
        int c0 = corner_count(phi_sphere_quarter, mn, mx, 0.0f), c1 = corner_count(phi_sphere_quarter, mn, mx, 0.01f);
        return (c0 == 8 || c1 == 0) ? min_level : max_level;
    }
    case OG_CASE_STAR_EMPTY: {
        int c = corner_count(phi_star, mn, mx, 0.0f);
        return (c == 0 || c == 8) ? min_level : max_level;
    }
    case OG_CASE_STAR_SOLID: {
        int c0 = corner_count(phi_star, mn, mx, 0.0f), c1 = corner_count(phi_star, mn, mx, 0.01f);
        return (c0 == 8 || c1 == 0) ? min_level : max_level;
    }
    case OG_CASE_SHELL: {
        /* prm: min_level, max_level, mid_level, cx, cy, cz, r, band_fine, band_mid */
        int mid_level = (int)prm[2];
        double c[3] = {prm[3], prm[4], prm[5]}, r = prm[6], bf = prm[7], bm = prm[8];
        double dmn[3], dmx[3], hd = (double)h;
        for (int d = 0; d < 3; d++) { dmn[d] = tc[d] * 8.0 * hd; dmx[d] = (tc[d] + 1) * 8.0 * hd; }
        double dist = box_sphere_surface_dist(dmn, dmx, c, r);
        return dist <= bf ? max_level : (dist <= bm ? mid_level : min_level);
    }
    case OG_CASE_MULTI_SPHERE: {
        /* prm: min_level, max_level, band, nspheres, then (cx, cy, cz, r) per sphere */
        double band = prm[2];
        int ns = (int)prm[3];
        double dmn[3], dmx[3], hd = (double)h;
        for (int d = 0; d < 3; d++) { dmn[d] = tc[d] * 8.0 * hd; dmx[d] = (tc[d] + 1) * 8.0 * hd; }
        for (int s = 0; s < ns && 4 + 4 * s + 3 < nprm; s++) {
            double c[3] = {prm[4 + 4 * s], prm[5 + 4 * s], prm[6 + 4 * s]};
            if (box_sphere_surface_dist(dmn, dmx, c, prm[7 + 4 * s]) <= band) return max_level;
        }
        return min_level;
    }
    }
    return min_level;
}
static int case_target(const og_grid* g, const og_tile* T, int case_id, const double* prm, int nprm) {
    return case_target_at(voxel_size(g, T->level), T->c, case_id, prm, nprm);
}
/* exported for the reference pin: the target of the tile (level, i, j, k) */
int og_case_target_at(float h0, int case_id, const double* prm, int nprm, int level, int i, int j, int k) {
    int tc[3] = {i, j, k};
    return case_target_at(h0 / (float)(1 << level), tc, case_id, prm, nprm);
}

/* HADeviceGrid::refineStep (HAGrid.h:1088-1170).  Reads see the grid as it
 * was at the start of the step, as the device-side flag kernels do. */
typedef struct {
    int case_id, nprm;
    const double* prm;
    og_target_fn fn;
    void* user;
} target_src;
static int target_of(const og_grid* g, const og_tile* T, const target_src* src) {
    if (src->fn) return src->fn(src->user, T->level, T->c[0], T->c[1], T->c[2]);
    return case_target(g, T, src->case_id, src->prm, src->nprm);
}
static int refine_step(og_grid* g, const target_src* src) {
    int nsnap = g->n, total = 0;
    int* type0 = (int*)malloc(sizeof(int) * (nsnap ? nsnap : 1));
    for (int t = 0; t < nsnap; t++) { type0[t] = g->t[t].type; g->t[t].flag = 0; }
    int maxl = g->max_level;
    for (int L = maxl; L >= 0; L--) {
        for (int t = 0; t < nsnap; t++) {
            og_tile* T = &g->t[t];
            if (T->level != L || !(type0[t] & OG_LEAF)) continue;
            int refine = target_of(g, T, src) > L;
            if (L < maxl) {
                for (int ci = 0; ci < 8; ci++) {
                    int c = map_find(g, L + 1, 2 * T->c[0] + (ci & 1), 2 * T->c[1] + ((ci >> 1) & 1), 2 * T->c[2] + ((ci >> 2) & 1));
                    if (c >= 0 && c < nsnap && (type0[c] & OG_GHOST) && g->t[c].flag) refine = 1;
                }
            }
            if (L + 1 >= g->num_levels) refine = 0;
            T->flag = refine;
        }
        for (int t = 0; t < nsnap; t++) {
            og_tile* T = &g->t[t];
            if (T->level != L || type0[t] != OG_GHOST) continue;
            int f = 0;
            for (int a = 0; a < 6; a++) {
                int n[3] = {T->c[0], T->c[1], T->c[2]};
                n[a >> 1] += (a & 1) ? 1 : -1;
                int q = map_find(g, L, n[0], n[1], n[2]);
                if (q >= 0 && q < nsnap && (type0[q] & OG_LEAF) && g->t[q].flag) f = 1;
            }
            T->flag = f;
        }
        for (int t = 0; t < nsnap; t++) {
            if (g->t[t].level != L || !(type0[t] & OG_LEAF) || !g->t[t].flag) continue;
            total++;
            g->t[t].type = OG_NONLEAF;
            int c0 = g->t[t].c[0], c1 = g->t[t].c[1], c2 = g->t[t].c[2];
            for (int ci = 0; ci < 8; ci++)
                og_set_tile(g, L + 1, 2 * c0 + (ci & 1), 2 * c1 + ((ci >> 1) & 1), 2 * c2 + ((ci >> 2) & 1), OG_LEAF);
        }
    }
    free(type0);
    compute_max_level(g);
    return total;
}

/* HADeviceGrid::iterativeRefine (HAGrid.h:1173-1182) */
static int refine_loop(og_grid* g, const target_src* src) {
    compute_max_level(g);
    int steps = 0;
    while (1) {
        int cnt = refine_step(g, src);
        spawn_ghosts(g);
        steps++;
        if (cnt == 0 || steps > 64) break;
    }
    finalize(g);
    return steps;
}
/* with a built-in target */
int og_refine_case(og_grid* g, int case_id, const double* prm, int nprm) {
    target_src src = {case_id, nprm, prm, NULL, NULL};
    return refine_loop(g, &src);
}
/* with a caller's target function of (level, tile coordinate) */
int og_refine_fn(og_grid* g, og_target_fn fn, void* user) {
    target_src src = {0, 0, NULL, fn, user};
    return refine_loop(g, &src);
}

int og_num_tiles(const og_grid* g) { return g->n; }
int og_max_level(const og_grid* g) { return g->max_level; }
void og_get_tiles(const og_grid* g, int* level, int* ijk, uint8_t* type) {
    for (int t = 0; t < g->n; t++) {
        level[t] = g->t[t].level;
        for (int d = 0; d < 3; d++) ijk[3 * t + d] = g->t[t].c[d];
        type[t] = (uint8_t)g->t[t].type;
    }
}
void og_get_tables(const og_grid* g, int* nbr, int* parent, int* child) {
    memcpy(nbr, g->nbr, sizeof(int) * 6 * g->n);
    memcpy(parent, g->parent, sizeof(int) * g->n);
    memcpy(child, g->child, sizeof(int) * 8 * g->n);
}

int og_alloc_channels(og_grid* g, int nch) {
    free(g->data); free(g->ctype);
    g->nch = nch;
    g->data = (float*)calloc((size_t)nch * g->n * NC, sizeof(float));
    g->ctype = (uint8_t*)calloc((size_t)g->n * NC, 1);
    return (g->data && g->ctype) ? 0 : -1;
}
float* og_channel(og_grid* g, int ch) { return g->data + (size_t)ch * g->n * NC; }
uint8_t* og_cell_types(og_grid* g) { return g->ctype; }
#define CH(g, ch, t) (g->data + ((size_t)(ch) * (g)->n + (t)) * NC)
#define CT(g, t) (g->ctype + (size_t)(t) * NC)

/* CreateTestGrid cell types (TestGrids.cuh:161-167) for LEAF tiles. */
static void leaf_cell_types_at(float h, const int tc[3], int case_id, uint8_t* out) {
    for (int v = 0; v < NC; v++) {
        int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
        uint8_t ty = OG_INTERIOR;
        if (case_id == OG_CASE_SPHERE_SOLID || case_id == OG_CASE_STAR_SOLID) {
            float mn[3], mx[3];
            for (int d = 0; d < 3; d++) { /* HAAccessor.h:132-138 */
                int gc = tc[d] * 8 + l[d];
                mn[d] = (float)gc * h; mx[d] = (float)(gc + 1) * h;
            }
            int c = corner_count(case_id == OG_CASE_SPHERE_SOLID ? phi_sphere_quarter : phi_star, mn, mx, 0.0f);
            ty = (c == 8) ? OG_NEUMANN : OG_INTERIOR;
        }
        out[v] = ty;
    }
}
void og_set_leaf_cell_types_case(og_grid* g, int case_id, const double* prm, int nprm) {
    (void)prm; (void)nprm;
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & OG_LEAF)) continue;
        leaf_cell_types_at(voxel_size(g, g->t[t].level), g->t[t].c, case_id, CT(g, t));
    }
}
/* exported for the reference pin: leaf cell types of the tile (level, i, j, k) */
void og_case_types_at(float h0, int case_id, int level, int i, int j, int k, uint8_t* out512) {
    int tc[3] = {i, j, k};
    leaf_cell_types_at(h0 / (float)(1 << level), tc, case_id, out512);
}

/* ------------------------------------------------------------------ */
/* operator coefficients                                              */
/* ------------------------------------------------------------------ */
/* NegativeLaplacianCoeff (AMGSolver.cu:12-24) */
static float face_coeff(float h, int tt0, int tt1, int c0, int c1) {
    int both_leafs = (tt0 & OG_LEAF) && (tt1 & OG_LEAF);
    int leaf_ghost = ((tt0 & OG_LEAF) && (tt1 & OG_GHOST)) || ((tt0 & OG_GHOST) && (tt1 & OG_LEAF));
    int has_neumann = (c0 & OG_NEUMANN) || (c1 & OG_NEUMANN);
    int has_interior = (c0 & OG_INTERIOR) || (c1 & OG_INTERIOR);
    return ((both_leafs || leaf_ghost) && !has_neumann && has_interior) ? h : 0.0f;
}
/* same-level neighbour cell in direction (axis, sgn): returns tile index (-1 empty) and local cell */
static int nb_cell(const og_grid* g, int t, int v, int axis, int sgn, int* nv) {
    int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
    l[axis] += sgn;
    if (l[axis] >= 0 && l[axis] < 8) { *nv = CELL(l[0], l[1], l[2]); return t; }
    l[axis] &= 7;
    *nv = CELL(l[0], l[1], l[2]);
    return g->nbr[t * 6 + axis + (sgn > 0 ? 3 : 0)];
}
/* parent cell of cell v of tile t: tile g->parent[t] */
static int parent_cell(const og_grid* g, int t, int v) {
    const og_tile* T = &g->t[t];
    int l[3] = {v >> 6, (v >> 3) & 7, v & 7}, p[3];
    for (int d = 0; d < 3; d++) p[d] = ((T->c[d] * 8 + l[d]) >> 1) & 7;
    return CELL(p[0], p[1], p[2]);
}
static void ghost_types_from_parents(og_grid* g) { /* AMGSolver.cu:265-274, MeshCutCell.cu:434-448 */
    for (int t = 0; t < g->n; t++) {
        if (g->t[t].type != OG_GHOST) continue;
        int p = g->parent[t];
        for (int v = 0; v < NC; v++) CT(g, t)[v] = (p >= 0) ? CT(g, p)[parent_cell(g, t, v)] : OG_DIRICHLET;
    }
}

void og_set_reference_mask(og_grid* g, int on) { g->ref_mask = on; }
void og_set_x_bf16(og_grid* g, int on) { g->x_bf16 = on; }

/* PrepareLaplacianSystemFromLeafAndGhostCellTypesAndFaceCoeffs (AMGSolver.cu:89-254) */
void og_prepare_system(og_grid* g, int coeff_ch, float R) {
    /* 1. coarse face coefficient += R * sum of the 4 fine faces, fine levels first
     *    (CoarsenOffDiagCoefficientsOneStepKernel, AMGSolver.cu:27-78).  Every tile
     *    of the fine level takes part (a NONLEAF tile counts as a LEAF of the
     *    subtree cut at its level).  The cell-type mask the reference applies
     *    admits every valid type; NONLEAF cell types are only computed in step 2,
     *    so the mask is taken as open here.  og_set_reference_mask(g, 1) applies
     *    the mask to whatever types the grid holds at this point instead (the
     *    reference reads NONLEAF types there before any write). */
    for (int L = g->max_level; L > 0; L--) {
        for (int t = 0; t < g->n; t++) {
            if (g->t[t].level != L) continue;
            int p = g->parent[t];
            if (p < 0) continue;
            for (int b = 0; b < 64; b++) {
                int fl[3] = {(b >> 4) * 2, ((b >> 2) & 3) * 2, (b & 3) * 2};
                int cv = parent_cell(g, t, CELL(fl[0], fl[1], fl[2]));
                for (int axis = 0; axis < 3; axis++) {
                    float sum = 0;
                    for (int jj = 0; jj < 2; jj++)
                        for (int kk = 0; kk < 2; kk++) {
                            int o[3];
                            o[axis] = 0; o[(axis + 1) % 3] = jj; o[(axis + 2) % 3] = kk; /* rotateCoord, HAAccessor.h:25 */
                            int fv = CELL(fl[0] + o[0], fl[1] + o[1], fl[2] + o[2]);
                            /* the reference masks by the fine cell's stored type
                             * (INTERIOR | DIRICHLET | NEUMANN); with ref_mask off the
                             * mask is open, see the comment above */
                            float fc = CH(g, coeff_ch + axis, t)[fv];
                            if (g->ref_mask && !(CT(g, t)[fv] & (OG_INTERIOR | OG_DIRICHLET | OG_NEUMANN))) fc = 0.0f;
                            sum += fc;
                        }
                    float* cc = &CH(g, coeff_ch + axis, p)[cv];
                    *cc = fmaf(sum, R, *cc);
                }
            }
        }
    }
    /* 2. diagonals and NONLEAF cell types, finest level first */
    for (int L = g->num_levels - 1; L >= 0; L--) {
        for (int t = 0; t < g->n; t++) {
            if (g->t[t].level != L) continue;
            int tt = g->t[t].type;
            float h = voxel_size(g, L);
            float* diag = CH(g, coeff_ch + 3, t);
            if (tt & (OG_LEAF | OG_GHOST)) {
                for (int v = 0; v < NC; v++) {
                    float d = 0;
                    if (CT(g, t)[v] & OG_INTERIOR) {
                        for (int axis = 0; axis < 3; axis++) {
                            d -= CH(g, coeff_ch + axis, t)[v];
                            int nv, q = nb_cell(g, t, v, axis, +1, &nv);
                            float c1 = (q < 0) ? -h : CH(g, coeff_ch + axis, q)[nv];
                            d -= c1;
                        }
                    }
                    diag[v] = d;
                }
            } else {
                for (int v = 0; v < NC; v++) {
                    int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
                    int gc[3];
                    for (int d = 0; d < 3; d++) gc[d] = g->t[t].c[d] * 8 + l[d];
                    int ct[2][2][2];
                    float off[3][2][2][2];
                    float dsum = 0;
                    int interior_cnt = 0;
                    for (int ci = 0; ci < 2; ci++)
                        for (int cj = 0; cj < 2; cj++)
                            for (int ck = 0; ck < 2; ck++) {
                                int cg[3] = {2 * gc[0] + ci, 2 * gc[1] + cj, 2 * gc[2] + ck};
                                int q = g->child[t * 8 + ((cg[0] >> 3) & 1) * 4 + ((cg[1] >> 3) & 1) * 2 + ((cg[2] >> 3) & 1)];
                                if (q >= 0) {
                                    int cv = CELL(cg[0] & 7, cg[1] & 7, cg[2] & 7);
                                    dsum += CH(g, coeff_ch + 3, q)[cv];
                                    interior_cnt += (CT(g, q)[cv] == OG_INTERIOR);
                                    ct[ci][cj][ck] = CT(g, q)[cv];
                                    for (int a = 0; a < 3; a++) off[a][ci][cj][ck] = CH(g, coeff_ch + a, q)[cv];
                                } else {
                                    ct[ci][cj][ck] = OG_DIRICHLET;
                                    for (int a = 0; a < 3; a++) off[a][ci][cj][ck] = 0;
                                }
                            }
                    for (int ci = 0; ci < 2; ci++)
                        for (int cj = 0; cj < 2; cj++)
                            for (int ck = 0; ck < 2; ck++) {
                                if (ct[0][cj][ck] == OG_INTERIOR && ct[1][cj][ck] == OG_INTERIOR) dsum += off[0][1][cj][ck];
                                if (ct[ci][0][ck] == OG_INTERIOR && ct[ci][1][ck] == OG_INTERIOR) dsum += off[1][ci][1][ck];
                                if (ct[ci][cj][0] == OG_INTERIOR && ct[ci][cj][1] == OG_INTERIOR) dsum += off[2][ci][cj][1];
                            }
                    CT(g, t)[v] = interior_cnt > 0 ? OG_INTERIOR : OG_DIRICHLET;
                    diag[v] = dsum * R;
                }
            }
        }
    }
}

/* CoarsenTypesAndAMGCoeffs (AMGSolver.cu:256-318) */
void og_coarsen_types_and_coeffs(og_grid* g, int coeff_ch, float R) {
    ghost_types_from_parents(g);
    for (int t = 0; t < g->n; t++) {
        int tt0 = g->t[t].type;
        float h = voxel_size(g, g->t[t].level);
        for (int v = 0; v < NC; v++) {
            for (int axis = 0; axis < 3; axis++) {
                float c = 0;
                if (tt0 != OG_NONLEAF) {
                    int nv, q = nb_cell(g, t, v, axis, -1, &nv);
                    int tt1 = (q < 0) ? tt0 : g->t[q].type;
                    int ct1 = (q < 0) ? OG_DIRICHLET : CT(g, q)[nv];
                    c = -face_coeff(h, tt0, tt1, CT(g, t)[v], ct1);
                }
                CH(g, coeff_ch + axis, t)[v] = c;
            }
        }
    }
    og_prepare_system(g, coeff_ch, R);
}

/* ------------------------------------------------------------------ */
/* cut cells (cirrus_cutcell/MeshCutCell.cu:262-412, 416-543)          */
/* ------------------------------------------------------------------ */
/* FracInside (MeshCutCell.cu:262-272) */
static float frac_inside(float a, float b) {
    if (a < 0.0f && b < 0.0f) return 0.0f;
    if (a < 0.0f && b >= 0.0f) return b / (b - a);
    if (a >= 0.0f && b < 0.0f) return a / (a - b);
    return 1.0f;
}
/* Marching-squares fluid fraction of a face from its four corner SDFs in
 * cyclic order (FaceFluidRatio, MeshCutCell.cu:305-408): 0 when all corners
 * are inside the solid, 1 when none is; otherwise triangle/trapezoid areas
 * from linear edge crossings, a nonzero result clamped to at least 0.1. */
static float face_fluid_ratio(const float phi[4]) {
    int in[4], nin = 0;
    for (int i = 0; i < 4; i++) { in[i] = phi[i] < 0; nin += in[i]; }
    float ret;
    if (nin == 4) ret = 0.0f;
    else if (nin == 0) ret = 1.0f;
    else if (nin == 3) { /* one fluid corner m: its triangle */
        int m = 0;
        while (in[m]) m++;
        int a = (m + 3) & 3, b = (m + 1) & 3;
        ret = (float)(0.5 * (double)frac_inside(phi[m], phi[a]) * (double)frac_inside(phi[m], phi[b]));
    } else if (nin == 1) { /* one solid corner m: one minus its triangle */
        int m = 0;
        while (!in[m]) m++;
        int a = (m + 1) & 3, b = (m + 3) & 3;
        float e1 = (float)(1.0 - (double)frac_inside(phi[m], phi[a]));
        float e2 = (float)(1.0 - (double)frac_inside(phi[m], phi[b]));
        ret = (float)(1.0 - 0.5 * (double)e1 * (double)e2);
    } else if (in[0] == in[2]) { /* two solid corners on a diagonal: two fluid triangles */
        int f0 = in[0] ? 1 : 0, f1 = f0 + 2;
        double t0 = 0.5 * (double)frac_inside(phi[f0], phi[(f0 + 3) & 3]) * (double)frac_inside(phi[f0], phi[(f0 + 1) & 3]);
        double t1 = 0.5 * (double)frac_inside(phi[f1], phi[(f1 + 3) & 3]) * (double)frac_inside(phi[f1], phi[(f1 + 1) & 3]);
        ret = (float)(t0 + t1);
    } else { /* two adjacent solid corners: a trapezoid from the two crossing edges,
              * summed in float as the reference does (the sign of a zero result follows) */
        float e[2] = {0.0f, 0.0f};
        int ne = 0;
        for (int i = 0; i < 4; i++) {
            if (in[i]) continue;
            int nb = in[(i + 1) & 3] ? ((i + 1) & 3) : ((i + 3) & 3);
            e[ne++] = frac_inside(phi[i], phi[nb]);
        }
        ret = (float)(0.5 * (double)(e[0] + e[1]));
    }
    if (ret < 0.1f && ret != 0.0f) ret = 0.1f;
    return ret;
}
static float sdf_spheres(float px, float py, float pz, int ns, const float* s) {
    float best = FLT_MAX;
    for (int i = 0; i < ns; i++) {
        float dx = px - s[4 * i], dy = py - s[4 * i + 1], dz = pz - s[4 * i + 2];
        float d = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx))) - s[4 * i + 3];
        if (d < best) best = d;
    }
    return best;
}
static float node_sdf(const og_grid* g, int t, int li, int lj, int lk, int ns, const float* s) {
    const og_tile* T = &g->t[t];
    float h = voxel_size(g, T->level);
    return sdf_spheres((float)(T->c[0] * 8 + li) * h, (float)(T->c[1] * 8 + lj) * h, (float)(T->c[2] * 8 + lk) * h, ns, s);
}
/* node SDF of a tile: 9^3 nodes, node (i, j, k) at i*81 + j*9 + k (PoissonTile.h:72) */
static void tile_node_sdf(const og_grid* g, int t, int ns, const float* s, float* nodes) {
    for (int i = 0; i < 9; i++)
        for (int j = 0; j < 9; j++)
            for (int k = 0; k < 9; k++) nodes[i * 81 + j * 9 + k] = node_sdf(g, t, i, j, k, ns, s);
}
/* CellCornerSDFInsideCount (MeshCutCell.cu:239-260): corners of cell (li, lj, lk) below iso */
static int cell_corner_inside_count(const float* nodes, int li, int lj, int lk, float iso) {
    int cnt = 0;
    for (int d = 0; d < 8; d++)
        if (nodes[(li + (d >> 2)) * 81 + (lj + ((d >> 1) & 1)) * 9 + (lk + (d & 1))] - iso < 0) cnt++;
    return cnt;
}
/* exported for the reference pin */
float og_frac_inside(float a, float b) { return frac_inside(a, b); }
void og_face_fluid_ratio(const float* phi4, int n, float* out) {
    for (int i = 0; i < n; i++) out[i] = face_fluid_ratio(phi4 + 4 * i);
}
void og_cell_corner_inside_count(const float* nodes729, float iso, int* out512) {
    for (int v = 0; v < NC; v++) out512[v] = cell_corner_inside_count(nodes729, v >> 6, (v >> 3) & 7, v & 7, iso);
}
/* CreateAMGLaplacianSystemWithSolidCutOnNodeSDF (MeshCutCell.cu:416-543) with
 * the node SDF of a union of spheres evaluated analytically at tile nodes. */
void og_cutcell_sphere_coeffs(og_grid* g, int coeff_ch, float R, int ns, const float* s) {
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & OG_LEAF)) continue;
        float eps = voxel_size(g, g->t[t].level) * 1e-3f; /* SDF_REL_EPS, MeshCutCell.h:8 */
        float nodes[729];
        tile_node_sdf(g, t, ns, s, nodes);
        for (int v = 0; v < NC; v++)
            if (cell_corner_inside_count(nodes, v >> 6, (v >> 3) & 7, v & 7, eps) == 8) CT(g, t)[v] = OG_NEUMANN;
    }
    ghost_types_from_parents(g);
    for (int t = 0; t < g->n; t++) {
        int tt0 = g->t[t].type;
        float h = voxel_size(g, g->t[t].level);
        float nodes[729];
        if (tt0 != OG_NONLEAF) tile_node_sdf(g, t, ns, s, nodes);
        for (int v = 0; v < NC; v++) {
            int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
            for (int axis = 0; axis < 3; axis++) {
                float c = 0; /* NONLEAF: 0 (MeshCutCell.cu:463) */
                if (tt0 != OG_NONLEAF) {
                    c = -0.0f; /* LEAF/GHOST: -coeff, coeff = 0 on an invalid face (MeshCutCell.cu:535) */
                    int nv, q = nb_cell(g, t, v, axis, -1, &nv);
                    int tt1 = (q < 0) ? tt0 : g->t[q].type;
                    int ct1 = (q < 0) ? OG_DIRICHLET : CT(g, q)[nv];
                    if (face_coeff(h, tt0, tt1, CT(g, t)[v], ct1) != 0.0f) {
                        /* face corners in cyclic order (FaceCornerSDFs, MeshCutCell.cu:274-303) */
                        static const int cyc[3][4][3] = {
                            {{0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {0, 1, 0}},
                            {{0, 0, 0}, {0, 0, 1}, {1, 0, 1}, {1, 0, 0}},
                            {{0, 0, 0}, {0, 1, 0}, {1, 1, 0}, {1, 0, 0}}};
                        float phi[4];
                        for (int q4 = 0; q4 < 4; q4++)
                            phi[q4] = nodes[(l[0] + cyc[axis][q4][0]) * 81 + (l[1] + cyc[axis][q4][1]) * 9 + (l[2] + cyc[axis][q4][2])];
                        c = -(h * face_fluid_ratio(phi));
                    }
                }
                CH(g, coeff_ch + axis, t)[v] = c;
            }
        }
    }
    og_prepare_system(g, coeff_ch, R);
}

/* ------------------------------------------------------------------ */
/* matrix-free operator: tile snapshot with a one-cell halo            */
/* (AMGLaplacianTileData + LoadAMGLaplacianTileData, AMGSolver.cu:320-543) */
/* ------------------------------------------------------------------ */
typedef struct {
    float x[1000];
    float c[3][1000]; /* negative-face coefficient of cell (i,j,k); index 8 along the axis = +face of cell 7 */
    float d[NC];
} og_snap;

static void load_snap(const og_grid* g, int t, int x_ch, int coeff_ch, og_snap* S) {
    const float* X = CH(g, x_ch, t);
    const uint8_t* ty = CT(g, t);
    float h = voxel_size(g, g->t[t].level);
    for (int v = 0; v < NC; v++) {
        int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
        S->x[SX(i, j, k)] = (ty[v] == OG_INTERIOR) ? X[v] : 0.0f;
        for (int a = 0; a < 3; a++) S->c[a][SX(i, j, k)] = CH(g, coeff_ch + a, t)[v];
        S->d[v] = CH(g, coeff_ch + 3, t)[v];
    }
    for (int axis = 0; axis < 3; axis++) {
        for (int s = 0; s < 2; s++) {
            int sgn = s ? 1 : -1;
            int q = g->nbr[t * 6 + axis + (s ? 3 : 0)];
            for (int fi = 0; fi < 64; fi++) {
                int a = fi >> 3, b = fi & 7;
                int fl[3], cl[3], nl[3];
                int axk = s ? 8 : -1;
                if (axis == 0) { fl[0] = axk; fl[1] = a; fl[2] = b; }
                else if (axis == 1) { fl[0] = a; fl[1] = axk; fl[2] = b; }
                else { fl[0] = a; fl[1] = b; fl[2] = axk; }
                for (int d = 0; d < 3; d++) { cl[d] = fl[d]; nl[d] = fl[d]; }
                cl[axis] -= sgn;
                nl[axis] = s ? 0 : 7;
                int fx = SX(fl[0], fl[1], fl[2]);
                if (q < 0) {
                    S->x[fx] = 0.0f;
                    if (s) S->c[axis][fx] = h;
                } else if (g->t[q].type & OG_GHOST) {
                    float avg = 0;
                    for (int di = 0; di < 2; di++)
                        for (int dj = 0; dj < 2; dj++)
                            for (int dk = 0; dk < 2; dk++) avg += S->x[SX(cl[0] ^ di, cl[1] ^ dj, cl[2] ^ dk)];
                    avg /= 8;
                    int nv = CELL(nl[0], nl[1], nl[2]);
                    float V1 = CH(g, x_ch, q)[nv];
                    S->x[fx] = (float)((double)S->x[SX(cl[0], cl[1], cl[2])] + 0.5 * (double)(V1 - avg));
                    if (s) S->c[axis][fx] = CH(g, coeff_ch + axis, q)[nv];
                } else {
                    int nv = CELL(nl[0], nl[1], nl[2]);
                    S->x[fx] = (CT(g, q)[nv] == OG_INTERIOR) ? CH(g, x_ch, q)[nv] : 0.0f;
                    if (s) S->c[axis][fx] = CH(g, coeff_ch + axis, q)[nv];
                }
            }
        }
    }
}
/* AMGLaplacianTileData::negativeLap (AMGSolver.cu:346-382) */
static float snap_neg_lap(const og_snap* S, int v) {
    float d = S->d[v];
    if (d == 0) return 0;
    int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
    float sum = S->x[SX(i, j, k)] * d;
    sum = fmaf(S->c[0][SX(i, j, k)], S->x[SX(i - 1, j, k)], sum);
    sum = fmaf(S->c[0][SX(i + 1, j, k)], S->x[SX(i + 1, j, k)], sum);
    sum = fmaf(S->c[1][SX(i, j, k)], S->x[SX(i, j - 1, k)], sum);
    sum = fmaf(S->c[1][SX(i, j + 1, k)], S->x[SX(i, j + 1, k)], sum);
    sum = fmaf(S->c[2][SX(i, j, k)], S->x[SX(i, j, k - 1)], sum);
    sum = fmaf(S->c[2][SX(i, j, k + 1)], S->x[SX(i, j, k + 1)], sum);
    return sum;
}

static int is_active_at(const og_grid* g, int t, int level) { /* subtreeType(level) & LEAF, HATileInfo.h:79 */
    return g->t[t].level == level && (g->t[t].type & (OG_LEAF | OG_NONLEAF));
}

/* PropagateToChildren + AccumulateToParentsOneStep + NegativeLaplacianSameLevelAMG128
 * on LEAF tiles (AMGFullNegativeLaplacianOnLeafs, AMGSolver.cu:589-632). */
static void propagate_ghosts(og_grid* g, int x_ch) {
    /* ghost <- parent value (PoissonGrid.cu:377-405), coarse levels first */
    for (int L = 1; L <= g->max_level; L++)
        for (int t = 0; t < g->n; t++) {
            if (g->t[t].level != L || !(g->t[t].type & OG_GHOST)) continue;
            int p = g->parent[t];
            for (int v = 0; v < NC; v++) {
                if (!(CT(g, t)[v] & (OG_INTERIOR | OG_DIRICHLET | OG_NEUMANN))) continue;
                float val = 0;
                if (p >= 0) {
                    int pv = parent_cell(g, t, v);
                    val = (CT(g, p)[pv] & (OG_INTERIOR | OG_DIRICHLET | OG_NEUMANN)) ? CH(g, x_ch, p)[pv] : 0.0f;
                }
                CH(g, x_ch, t)[v] = val;
            }
        }
}
/* NONLEAF parent <- 1/8 sum of LEAF children, one step (PoissonGrid.cu:408-465) */
static void accumulate_leafs_to_parents(og_grid* g, int x_ch) {
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & OG_LEAF)) continue;
        int p = g->parent[t];
        if (p < 0) continue;
        for (int b = 0; b < 64; b++) {
            int fl[3] = {(b >> 4) * 2, ((b >> 2) & 3) * 2, (b & 3) * 2};
            float sum = 0;
            for (int ii = 0; ii < 2; ii++)
                for (int jj = 0; jj < 2; jj++)
                    for (int kk = 0; kk < 2; kk++) {
                        int v = CELL(fl[0] + ii, fl[1] + jj, fl[2] + kk);
                        sum += (CT(g, t)[v] & (OG_INTERIOR | OG_DIRICHLET | OG_NEUMANN)) ? CH(g, x_ch, t)[v] : 0.0f;
                    }
            CH(g, x_ch, p)[parent_cell(g, t, CELL(fl[0], fl[1], fl[2]))] = sum * 0.125f;
        }
    }
}
static void propagate_and_accumulate(og_grid* g, int x_ch) {
    propagate_ghosts(g, x_ch);
    accumulate_leafs_to_parents(g, x_ch);
}
void og_full_neg_lap_leafs(og_grid* g, int x_ch, int coeff_ch, int ax_ch) {
    propagate_and_accumulate(g, x_ch);
#pragma omp parallel
    {
        og_snap* S = (og_snap*)malloc(sizeof(og_snap));
#pragma omp for schedule(dynamic, 16)
        for (int t = 0; t < g->n; t++) {
            if (!(g->t[t].type & OG_LEAF)) continue;
            load_snap(g, t, x_ch, coeff_ch, S);
            for (int v = 0; v < NC; v++) CH(g, ax_ch, t)[v] = (CT(g, t)[v] == OG_INTERIOR) ? snap_neg_lap(S, v) : 0.0f;
        }
        free(S);
    }
}

/* NegativeLaplacianAndGaussSeidelSameLevelAMG128Kernel (AMGSolver.cu:838-877),
 * GaussSeidelAMG (AMGSolver.cu:887-894): red-black passes over the LEAF and
 * NONLEAF tiles of one level.  Each tile reads a snapshot of itself taken
 * before the pass. */
static void gs_pass(og_grid* g, int level, int color, int x_ch, int coeff_ch, int rhs_ch, double omega) {
    float om = (float)omega;
    int exact = ((double)om == omega);
#pragma omp parallel
    {
        og_snap* S = (og_snap*)malloc(sizeof(og_snap));
#pragma omp for schedule(dynamic, 8)
        for (int t = 0; t < g->n; t++) {
            if (!is_active_at(g, t, level)) continue;
            load_snap(g, t, x_ch, coeff_ch, S);
            float* X = CH(g, x_ch, t);
            const float* B = CH(g, rhs_ch, t);
            for (int v = 0; v < NC; v++) {
                int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
                if (((i + j + k) & 1) != color) continue;
                uint8_t ct = CT(g, t)[v];
                float Ax = snap_neg_lap(S, v);
                float D = S->d[v];
                float delta = (ct & OG_INTERIOR) ? (XS(g, level, B[v]) - Ax) / D : 0.0f;
                float xs = S->x[SX(i, j, k)];
                /* AMGSolver.cu:874: x + delta * omega with omega a double holding a float: the
                 * product is exact in double, the sum rounds to double, then to float */
                X[v] = XS(g, level, exact ? (float)fma((double)delta, (double)om, (double)xs) : (float)((double)xs + (double)delta * omega));
            }
        }
        free(S);
    }
}
void og_gauss_seidel(og_grid* g, int iters, int order, int level, int x_ch, int coeff_ch, int rhs_ch, double omega) {
    for (int it = 0; it < iters; it++) {
        gs_pass(g, level, order, x_ch, coeff_ch, rhs_ch, omega);
        gs_pass(g, level, 1 - order, x_ch, coeff_ch, rhs_ch, omega);
    }
}

/* ResidualAndRestrictAMG128Kernel (AMGSolver.cu:896-960) */
void og_residual_restrict(og_grid* g, int level, int x_ch, int coeff_ch, int rhs_ch, float R_restrict) {
#pragma omp parallel
    {
        og_snap* S = (og_snap*)malloc(sizeof(og_snap));
        float res[NC];
#pragma omp for schedule(dynamic, 8)
        for (int t = 0; t < g->n; t++) {
            if (!is_active_at(g, t, level)) continue;
            int p = g->parent[t];
            load_snap(g, t, x_ch, coeff_ch, S);
            for (int v = 0; v < NC; v++) res[v] = XS(g, level, CH(g, rhs_ch, t)[v]) - snap_neg_lap(S, v);
            if (p < 0) continue;
            for (int b = 0; b < 64; b++) {
                int fl[3] = {(b >> 4) * 2, ((b >> 2) & 3) * 2, (b & 3) * 2};
                float rs = 0, xs = 0;
                for (int ii = 0; ii < 2; ii++)
                    for (int jj = 0; jj < 2; jj++)
                        for (int kk = 0; kk < 2; kk++) {
                            rs += res[CELL(fl[0] + ii, fl[1] + jj, fl[2] + kk)];
                            xs += S->x[SX(fl[0] + ii, fl[1] + jj, fl[2] + kk)];
                        }
                int cv = parent_cell(g, t, CELL(fl[0], fl[1], fl[2]));
                CH(g, rhs_ch, p)[cv] = XS(g, level - 1, rs * R_restrict);
                CH(g, x_ch, p)[cv] = XS(g, level - 1, xs / 8);
            }
        }
        free(S);
    }
}

/* FASSaveSolutionAndUpdateSource128Kernel (AMGSolver.cu:1176-1214), NONLEAF tiles of `level` */
void og_fas_save(og_grid* g, int level, int x_ch, int coeff_ch, int rhs_ch, int x0_ch) {
#pragma omp parallel
    {
        og_snap* S = (og_snap*)malloc(sizeof(og_snap));
        float lap[NC];
#pragma omp for schedule(dynamic, 8)
        for (int t = 0; t < g->n; t++) {
            if (g->t[t].level != level || !(g->t[t].type & OG_NONLEAF)) continue;
            load_snap(g, t, x_ch, coeff_ch, S);
            for (int v = 0; v < NC; v++) lap[v] = snap_neg_lap(S, v);
            for (int v = 0; v < NC; v++) {
                if (CT(g, t)[v] & OG_INTERIOR) {
                    CH(g, rhs_ch, t)[v] = XS(g, level, XS(g, level, CH(g, rhs_ch, t)[v]) + lap[v]);
                    CH(g, x0_ch, t)[v] = CH(g, x_ch, t)[v];
                } else CH(g, rhs_ch, t)[v] = 0.0f;
            }
        }
        free(S);
    }
}

/* FASProlongateAndUpdateAMG128Kernel (AMGSolver.cu:1216-1255): all tiles of `level` */
void og_fas_prolong(og_grid* g, int level, int x_ch, int x0_ch, float P) {
#pragma omp parallel for schedule(dynamic, 8)
    for (int t = 0; t < g->n; t++) {
        if (g->t[t].level != level) continue;
        int p = g->parent[t];
        int ghost = g->t[t].type & OG_GHOST;
        float* X = CH(g, x_ch, t);
        for (int v = 0; v < NC; v++) {
            float cx = 0, cx0 = 0;
            if (p >= 0) {
                int pv = parent_cell(g, t, v);
                cx = CH(g, x_ch, p)[pv];
                cx0 = CH(g, x0_ch, p)[pv];
            }
            int in = CT(g, t)[v] & OG_INTERIOR;
            if (ghost) X[v] = in ? XS(g, level, cx) : 0.0f;
            else X[v] = in ? XS(g, level, fmaf(P, cx - cx0, X[v])) : 0.0f;
        }
    }
}

typedef struct {
    int mu, x_ch, rhs_ch, x0_ch, coeff_ch, level_iters, coarsest_iters;
    double omega;
    float Rr, P;
} mu_args;
/* AMGSolver::FASMuCycleStep (AMGSolver.cu:1257-1277) */
static void fas_step(og_grid* g, int l, const mu_args* A) {
    if (l == 0) {
        og_gauss_seidel(g, A->coarsest_iters / 2, 0, 0, A->x_ch, A->coeff_ch, A->rhs_ch, A->omega);
        og_gauss_seidel(g, A->coarsest_iters / 2, 1, 0, A->x_ch, A->coeff_ch, A->rhs_ch, A->omega);
        return;
    }
    og_gauss_seidel(g, A->level_iters, 0, l, A->x_ch, A->coeff_ch, A->rhs_ch, A->omega);
    og_residual_restrict(g, l, A->x_ch, A->coeff_ch, A->rhs_ch, A->Rr);
    og_fas_save(g, l - 1, A->x_ch, A->coeff_ch, A->rhs_ch, A->x0_ch);
    for (int r = 0; r < A->mu; r++) fas_step(g, l - 1, A);
    og_fas_prolong(g, l, A->x_ch, A->x0_ch, A->P);
    og_gauss_seidel(g, A->level_iters, 1, l, A->x_ch, A->coeff_ch, A->rhs_ch, A->omega);
}
/* AMGSolver::FASMuCycle (AMGSolver.cu:1279-1292) */
void og_fas_mu_cycle(og_grid* g, int mu, int x_ch, int rhs_ch, int x0_ch, int coeff_ch, int level_iters, int coarsest_iters, double omega, float R_restrict, float P) {
    memset(CH(g, x_ch, 0), 0, sizeof(float) * NC * g->n);
    mu_args A = {mu, x_ch, rhs_ch, x0_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict, P};
    fas_step(g, g->max_level, &A);
}

/* ------------------------------------------------------------------ */
/* the cycles nothing in the reference's solve calls                   */
/* ------------------------------------------------------------------ */
/* AMGSolver::VCycle / muCycle start (AMGSolver.cu:1063-1080): x = 0 on every tile, rhs = f on
 * LEAF and NONLEAF tiles, 0 on GHOST tiles */
static void cycle_init(og_grid* g, int x_ch, int f_ch, int rhs_ch) {
    for (int t = 0; t < g->n; t++) {
        int ghost = g->t[t].type & OG_GHOST;
        for (int v = 0; v < NC; v++) {
            CH(g, x_ch, t)[v] = 0.0f;
            CH(g, rhs_ch, t)[v] = ghost ? 0.0f : CH(g, f_ch, t)[v];
        }
    }
}
/* ProlongateAndUpdateAMG128Kernel (AMGSolver.cu:1026-1057), every tile of `level`: GHOST cells
 * take the parent's x, the others add P times it; 0 on cells that are not INTERIOR */
static void prolong_add(og_grid* g, int level, int x_ch, float P) {
#pragma omp parallel for schedule(dynamic, 8)
    for (int t = 0; t < g->n; t++) {
        if (g->t[t].level != level) continue;
        int p = g->parent[t];
        int ghost = g->t[t].type & OG_GHOST;
        float* X = CH(g, x_ch, t);
        for (int v = 0; v < NC; v++) {
            float cx = p >= 0 ? CH(g, x_ch, p)[parent_cell(g, t, v)] : 0.0f;
            int in = CT(g, t)[v] & OG_INTERIOR;
            if (ghost) X[v] = in ? cx : 0.0f;
            else X[v] = in ? fmaf(P, cx, X[v]) : 0.0f;
        }
    }
}
/* DeductFluxOnAbsLeafs128Kernel (AMGSolver.cu:966-992) on the LEAF tiles of `level`: rhs = f
 * - negativeLapOuterNonLeaf (AMGSolver.cu:384-405) on INTERIOR cells, 0 elsewhere.  Only
 * cells of NONLEAF neighbour tiles count; the tile's own cells (LEAF) count 0. */
static void deduct_flux(og_grid* g, int level, int x_ch, int coeff_ch, int f_ch, int rhs_ch) {
#pragma omp parallel
    {
        og_snap* S = (og_snap*)malloc(sizeof(og_snap));
#pragma omp for schedule(dynamic, 8)
        for (int t = 0; t < g->n; t++) {
            if (g->t[t].level != level || !(g->t[t].type & OG_LEAF)) continue;
            load_snap(g, t, x_ch, coeff_ch, S);
            for (int v = 0; v < NC; v++) {
                int c[3] = {v >> 6, (v >> 3) & 7, v & 7};
                float d = S->d[v], s = 0.0f;
                if (d != 0.0f) {
                    s = 0.0f * d;
                    for (int axis = 0; axis < 3; axis++)
                        for (int side = 0; side < 2; side++) {
                            int sgn = side ? 1 : -1;
                            int n[3] = {c[0], c[1], c[2]}, u[3] = {c[0], c[1], c[2]};
                            n[axis] += sgn;
                            u[axis] += side;
                            float x1 = 0.0f;
                            if (n[axis] < 0 || n[axis] > 7) {
                                int q = g->nbr[t * 6 + axis + (side ? 3 : 0)];
                                if (q >= 0 && g->t[q].type == OG_NONLEAF) x1 = S->x[SX(n[0], n[1], n[2])];
                            }
                            s = fmaf(S->c[axis][SX(u[0], u[1], u[2])], x1, s);
                        }
                }
                CH(g, rhs_ch, t)[v] = (CT(g, t)[v] & OG_INTERIOR) ? CH(g, f_ch, t)[v] - s : 0.0f;
            }
        }
        free(S);
    }
}
/* SetLevelZeroAbsTiles128Kernel (AMGSolver.cu:1001-1018): x = 0 on the NONLEAF tiles of `level` */
static void set_zero_nonleaf(og_grid* g, int level, int x_ch) {
    for (int t = 0; t < g->n; t++)
        if (g->t[t].level == level && (g->t[t].type & OG_NONLEAF)) memset(CH(g, x_ch, t), 0, sizeof(float) * NC);
}
typedef struct {
    int rep, x_ch, f_ch, rhs_ch, coeff_ch, level_iters, coarsest_iters;
    double omega;
    float Rr, P;
} cs_args;
/* AMGSolver::muCycleStep (AMGSolver.cu:1130-1149) */
static void mu_step_cs(og_grid* g, int l, const cs_args* A) {
    if (l == 0) {
        og_gauss_seidel(g, A->coarsest_iters / 2, 0, 0, A->x_ch, A->coeff_ch, A->rhs_ch, A->omega);
        og_gauss_seidel(g, A->coarsest_iters / 2, 1, 0, A->x_ch, A->coeff_ch, A->rhs_ch, A->omega);
        return;
    }
    og_gauss_seidel(g, A->level_iters, 0, l, A->x_ch, A->coeff_ch, A->rhs_ch, A->omega);
    og_residual_restrict(g, l, A->x_ch, A->coeff_ch, A->rhs_ch, A->Rr);
    deduct_flux(g, l - 1, A->x_ch, A->coeff_ch, A->f_ch, A->rhs_ch);
    set_zero_nonleaf(g, l - 1, A->x_ch);
    for (int r = 0; r < A->rep; r++) mu_step_cs(g, l - 1, A);
    prolong_add(g, l, A->x_ch, A->P);
    og_gauss_seidel(g, A->level_iters, 1, l, A->x_ch, A->coeff_ch, A->rhs_ch, A->omega);
}
/* AMGSolver::muCycle (AMGSolver.cu:1151-1174) */
void og_mu_cycle(og_grid* g, int repeat_times, int x_ch, int f_ch, int rhs_ch, int coeff_ch, int level_iters, int coarsest_iters, double omega,
                 float R_restrict, float P) {
    cs_args A = {repeat_times, x_ch, f_ch, rhs_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict, P};
    cycle_init(g, x_ch, f_ch, rhs_ch);
    mu_step_cs(g, g->max_level, &A);
}
/* AMGSolver::VCycle (AMGSolver.cu:1060-1128) */
void og_vcycle(og_grid* g, int x_ch, int f_ch, int rhs_ch, int coeff_ch, int level_iters, int coarsest_iters, double omega, float R_restrict,
               float P) {
    cycle_init(g, x_ch, f_ch, rhs_ch);
    for (int l = g->max_level; l > 0; l--) {
        og_gauss_seidel(g, level_iters, 0, l, x_ch, coeff_ch, rhs_ch, omega);
        og_residual_restrict(g, l, x_ch, coeff_ch, rhs_ch, R_restrict);
    }
    og_gauss_seidel(g, coarsest_iters / 2, 0, 0, x_ch, coeff_ch, rhs_ch, omega);
    og_gauss_seidel(g, coarsest_iters / 2, 1, 0, x_ch, coeff_ch, rhs_ch, omega);
    for (int l = 1; l <= g->max_level; l++) {
        prolong_add(g, l, x_ch, P);
        og_gauss_seidel(g, level_iters, 1, l, x_ch, coeff_ch, rhs_ch, omega);
    }
}
/* RestrictSourceToCoarse (AMGSolver.cu:1295-1307): AccumulateToParentsOneStepKernel
 * (PoissonGrid.cu:408-453) on the LEAF and NONLEAF tiles of `level`, INTERIOR cells only,
 * the parent cell set to R times the sum of its 8 children */
static void restrict_source(og_grid* g, int level, int ch, float R) {
    for (int t = 0; t < g->n; t++) {
        if (!is_active_at(g, t, level)) continue;
        int p = g->parent[t];
        if (p < 0) continue;
        for (int b = 0; b < 64; b++) {
            int fl[3] = {(b >> 4) * 2, ((b >> 2) & 3) * 2, (b & 3) * 2};
            float sum = 0;
            for (int ii = 0; ii < 2; ii++)
                for (int jj = 0; jj < 2; jj++)
                    for (int kk = 0; kk < 2; kk++) {
                        int v = CELL(fl[0] + ii, fl[1] + jj, fl[2] + kk);
                        sum += (CT(g, t)[v] & OG_INTERIOR) ? CH(g, ch, t)[v] : 0.0f;
                    }
            CH(g, ch, p)[parent_cell(g, t, CELL(fl[0], fl[1], fl[2]))] = sum * R;
        }
    }
}
/* AMGSolver::FASFCycle (AMGSolver.cu:1358-1387) */
void og_fas_f_cycle(og_grid* g, int mu, int x_ch, int rhs_ch, int x0_ch, int coeff_ch, int level_iters, int coarsest_iters, double omega,
                    float R_restrict, float P) {
    memset(CH(g, x_ch, 0), 0, sizeof(float) * NC * g->n);
    for (int l = g->max_level; l > 0; l--) restrict_source(g, l, rhs_ch, R_restrict);
    og_gauss_seidel(g, coarsest_iters / 2, 0, 0, x_ch, coeff_ch, rhs_ch, omega);
    og_gauss_seidel(g, coarsest_iters / 2, 1, 0, x_ch, coeff_ch, rhs_ch, omega);
    mu_args A = {mu, x_ch, rhs_ch, x0_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict, P};
    for (int l = 1; l <= g->max_level; l++) {
        prolong_add(g, l, x_ch, P);
        fas_step(g, l, &A);
    }
}

/* Dot128Kernel + DeviceReduce (PoissonGrid.cu:156-214): all 512 cells of LEAF
 * tiles, products of each group of four cells summed in float, then double. */
double og_dot(og_grid* g, int a_ch, int b_ch) {
    double* part = (double*)calloc(g->n ? g->n : 1, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & OG_LEAF)) continue;
        const float* A = CH(g, a_ch, t);
        const float* B = CH(g, b_ch, t);
        double s = 0;
        for (int q = 0; q < NC; q += 4) {
            float f = A[q] * B[q];
            f = fmaf(A[q + 1], B[q + 1], f);
            f = fmaf(A[q + 2], B[q + 2], f);
            f = fmaf(A[q + 3], B[q + 3], f);
            s += (double)f;
        }
        part[t] = s;
    }
    double s = 0;
    for (int t = 0; t < g->n; t++) s += part[t];
    free(part);
    return s;
}
/* ReCenterLeafCells (PoissonGrid.cu:889-921): subtract the mean over INTERIOR cells of LEAF tiles */
static void recenter(og_grid* g, int ch) {
    double sum = 0, cnt = 0;
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & OG_LEAF)) continue;
        const float* A = CH(g, ch, t);
        const uint8_t* ty = CT(g, t);
        for (int q = 0; q < NC; q += 4) {
            float f = 0;
            int c = 0;
            for (int u = 0; u < 4; u++) {
                float val = (ty[q + u] & OG_INTERIOR) ? A[q + u] : 0.0f;
                f = (u == 0) ? val : f + val;
                c += (ty[q + u] & OG_INTERIOR) != 0;
            }
            sum += (double)f; cnt += c;
        }
    }
    double mean = sum / cnt;
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & OG_LEAF)) continue;
        float* A = CH(g, ch, t);
        for (int v = 0; v < NC; v++) if (CT(g, t)[v] & OG_INTERIOR) A[v] = (float)((double)A[v] - mean);
    }
}

/* The PCG of AMGSolver::solve (AMGSolver.cu:1399-1549), GMGSolver::solve and
 * CMGSolver::solve, with the operator and the preconditioner passed in.
 * Channels: x 0, b/r 1, p 2, Ap 3 (also the preconditioner's scratch), z 4
 * (PoissonTile.h:13-18).  Returns the iteration count. */
typedef void (*apply_fn)(og_grid* g, const void* ctx, int p_ch, int ap_ch);
typedef void (*precond_fn)(og_grid* g, const void* ctx, int z_ch, int r_ch, int tmp_ch);
static int pcg(og_grid* g, apply_fn apply, precond_fn precond, const void* ctx, int max_iters, double tol, int sync_stride, int pure_neumann,
               double* rel_res) {
    const int X = 0, R = 1, PP = 2, AP = 3, Z = 4;
    double rr0 = 0, thr = 0;
    for (int t = 0; t < g->n; t++) if (g->t[t].type & OG_LEAF) memset(CH(g, X, t), 0, sizeof(float) * NC);
    if (sync_stride > 0) {
        rr0 = og_dot(g, R, R);
        if (rr0 == 0.0) { if (rel_res) *rel_res = 0; return 0; }
        thr = tol * tol * rr0;
        if (thr < DBL_MIN) thr = DBL_MIN;
    }
    if (pure_neumann) recenter(g, R);
    precond(g, ctx, Z, R, AP);
    for (int t = 0; t < g->n; t++) if (g->t[t].type & OG_LEAF) memcpy(CH(g, PP, t), CH(g, Z, t), sizeof(float) * NC);
    double gamma = og_dot(g, Z, R);
    int i;
    for (i = 0; i < max_iters; i++) {
        apply(g, ctx, PP, AP);
        double fp = og_dot(g, PP, AP);
        double alpha = gamma / fp;
        float af = (float)alpha;
        for (int t = 0; t < g->n; t++) {
            if (!(g->t[t].type & OG_LEAF)) continue;
            for (int v = 0; v < NC; v++) {
                if (!(CT(g, t)[v] & OG_INTERIOR)) continue;
                CH(g, X, t)[v] = fmaf(af, CH(g, PP, t)[v], CH(g, X, t)[v]);
                CH(g, R, t)[v] = fmaf(-af, CH(g, AP, t)[v], CH(g, R, t)[v]);
            }
        }
        if (sync_stride > 0 && (i + 1) % sync_stride == 0) {
            double rr = og_dot(g, R, R);
            if (rr < thr) { if (rel_res) *rel_res = sqrt(rr / rr0); return i + 1; }
        }
        if (pure_neumann) recenter(g, R);
        precond(g, ctx, Z, R, AP);
        double gamma_old = gamma;
        gamma = og_dot(g, R, Z);
        double beta = gamma / gamma_old;
        float bf = (float)beta;
        for (int t = 0; t < g->n; t++) {
            if (!(g->t[t].type & OG_LEAF)) continue;
            for (int v = 0; v < NC; v++)
                if (CT(g, t)[v] & OG_INTERIOR) CH(g, PP, t)[v] = fmaf(bf, CH(g, PP, t)[v], CH(g, Z, t)[v]);
        }
    }
    if (sync_stride > 0) {
        double rr = og_dot(g, R, R);
        if (rel_res) *rel_res = sqrt(rr / rr0);
    } else if (rel_res) *rel_res = -1;
    return i;
}

typedef struct {
    int coeff_ch, mu, level_iters, coarsest_iters;
    double omega;
    float Rr, P;
} amg_ctx;
static void amg_apply(og_grid* g, const void* ctx, int p_ch, int ap_ch) {
    og_full_neg_lap_leafs(g, p_ch, ((const amg_ctx*)ctx)->coeff_ch, ap_ch);
}
static void amg_precond(og_grid* g, const void* ctx, int z_ch, int r_ch, int tmp_ch) {
    const amg_ctx* c = (const amg_ctx*)ctx;
    og_fas_mu_cycle(g, c->mu, z_ch, r_ch, tmp_ch, c->coeff_ch, c->level_iters, c->coarsest_iters, c->omega, c->Rr, c->P);
}
int og_amg_solve(og_grid* g, int coeff_ch, double omega, int mu, float Rr, float P, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride, int pure_neumann, double* rel_res) {
    amg_ctx c = {coeff_ch, mu, level_iters, coarsest_iters, omega, Rr, P};
    return pcg(g, amg_apply, amg_precond, &c, max_iters, tol, sync_stride, pure_neumann, rel_res);
}

/* ------------------------------------------------------------------ */
/* right-hand side: face velocity and volume-weighted divergence       */
/* ------------------------------------------------------------------ */
/* Face velocity of a sum of Fourier modes, sampled at the centre of the
 * negative face of every LEAF cell (double arithmetic, stored as float). */
void og_face_velocity_fourier(og_grid* g, int u_ch, int nm, const double* kv, const double* amp, const double* ph) {
    const double two_pi = 6.283185307179586;
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & OG_LEAF)) continue;
        double h = (double)voxel_size(g, g->t[t].level);
        for (int v = 0; v < NC; v++) {
            int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
            for (int axis = 0; axis < 3; axis++) {
                double p[3];
                for (int d = 0; d < 3; d++) p[d] = ((double)(g->t[t].c[d] * 8 + l[d]) + (d == axis ? 0.0 : 0.5)) * h;
                double u = 0;
                for (int m = 0; m < nm; m++) {
                    double arg = two_pi * (kv[3 * m] * p[0] + kv[3 * m + 1] * p[1] + kv[3 * m + 2] * p[2]) + ph[m];
                    u += amp[3 * m + axis] * sin(arg);
                }
                CH(g, u_ch + axis, t)[v] = (float)u;
            }
        }
    }
}
/* AMGVolumeWeightedDivergenceOnLeafs (AMGSolver.cu:790-835) with its
 * PropagateToChildren and AccumulateFacesToParentsOneStep (PoissonGrid.cu:523-586);
 * coeff_ch < 0: AMGVolumeWeightedDivergenceWithoutCoeffOnLeafs (AMGSolver.cu:750-788),
 * the same sum with -u0 h h and u1 h h for the two faces of each axis. */
void og_divergence(og_grid* g, int u_ch, int coeff_ch, int out_ch) {
    const int ALL = OG_INTERIOR | OG_DIRICHLET | OG_NEUMANN;
    for (int axis = 0; axis < 3; axis++)
        for (int L = 1; L <= g->max_level; L++)
            for (int t = 0; t < g->n; t++) {
                if (g->t[t].level != L || !(g->t[t].type & OG_GHOST)) continue;
                int p = g->parent[t];
                for (int v = 0; v < NC; v++) {
                    if (!(CT(g, t)[v] & ALL)) continue;
                    float val = 0;
                    if (p >= 0) {
                        int pv = parent_cell(g, t, v);
                        if (CT(g, p)[pv] & ALL) val = CH(g, u_ch + axis, p)[pv];
                    }
                    CH(g, u_ch + axis, t)[v] = val;
                }
            }
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & OG_LEAF)) continue;
        int p = g->parent[t];
        if (p < 0) continue;
        for (int b = 0; b < 64; b++) {
            int fl[3] = {(b >> 4) * 2, ((b >> 2) & 3) * 2, (b & 3) * 2};
            int cv = parent_cell(g, t, CELL(fl[0], fl[1], fl[2]));
            for (int axis = 0; axis < 3; axis++) {
                float sum = 0;
                for (int jj = 0; jj < 2; jj++)
                    for (int kk = 0; kk < 2; kk++) {
                        int o[3];
                        o[axis] = 0; o[(axis + 1) % 3] = jj; o[(axis + 2) % 3] = kk;
                        int v = CELL(fl[0] + o[0], fl[1] + o[1], fl[2] + o[2]);
                        sum += (CT(g, t)[v] & ALL) ? CH(g, u_ch + axis, t)[v] : 0.0f;
                    }
                CH(g, u_ch + axis, p)[cv] = sum * 0.25f;
            }
        }
    }
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & OG_LEAF)) continue;
        float h = voxel_size(g, g->t[t].level);
        for (int v = 0; v < NC; v++) {
            float sum = 0;
            for (int axis = 0; axis < 3; axis++) {
                for (int s = 0; s < 2; s++) {
                    if (!s) {
                        float u0 = CH(g, u_ch + axis, t)[v];
                        if (coeff_ch < 0) {
                            sum = fmaf(-u0 * h, h, sum); /* AMGSolver.cu:781, sgn = -1 */
                        } else {
                            float c0 = CH(g, coeff_ch + axis, t)[v];
                            sum = fmaf(u0 * c0, h, sum);
                        }
                    } else {
                        int nv, q = nb_cell(g, t, v, axis, +1, &nv);
                        float u1 = 0, c1 = 0;
                        if (q >= 0) {
                            u1 = CH(g, u_ch + axis, q)[nv];
                            if (coeff_ch >= 0) c1 = CH(g, coeff_ch + axis, q)[nv];
                        }
                        if (coeff_ch < 0)
                            sum = fmaf(u1 * h, h, sum); /* AMGSolver.cu:781, sgn = +1 */
                        else
                            sum = fmaf(-u1 * c1, h, sum);
                    }
                }
            }
            CH(g, out_ch, t)[v] = (CT(g, t)[v] & OG_INTERIOR) ? sum : 0.0f;
        }
    }
}

/* AMGAddGradientToFace (src/AMGSolver.cu:634-688): GHOST <- parent and NONLEAF
 * <- mean of LEAF children for x, then on LEAF and GHOST tiles
 * u_axis += (x - x_minus) / h on every face whose fluid ratio -c_axis/h > 0. */
void og_add_gradient_to_face(og_grid* g, int x_ch, int coeff_ch, int u_ch) {
    propagate_and_accumulate(g, x_ch);
#pragma omp parallel
    {
        og_snap* S = (og_snap*)malloc(sizeof(og_snap));
#pragma omp for schedule(dynamic, 8)
        for (int t = 0; t < g->n; t++) {
            if (!(g->t[t].type & (OG_LEAF | OG_GHOST))) continue;
            load_snap(g, t, x_ch, coeff_ch, S);
            float h = voxel_size(g, g->t[t].level);
            for (int v = 0; v < NC; v++) {
                int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
                for (int axis = 0; axis < 3; axis++) {
                    int d[3] = {0, 0, 0};
                    d[axis] = 1;
                    float pu = S->x[SX(i, j, k)], pd = S->x[SX(i - d[0], j - d[1], k - d[2])];
                    float ratio = -S->c[axis][SX(i, j, k)] / h;
                    if (ratio > 0) CH(g, u_ch + axis, t)[v] += (pu - pd) / h;
                }
            }
        }
        free(S);
    }
}

/* ------------------------------------------------------------------ */
/* FP64 CSR assembly of the leaf operator by tracing linear forms      */
/* ------------------------------------------------------------------ */
typedef struct { int col; double v; } og_ent;
typedef struct { og_ent e[512]; int n; } og_row;
static void row_add(og_row* r, int col, double v) {
    if (col < 0 || v == 0.0) return;
    for (int i = 0; i < r->n; i++) if (r->e[i].col == col) { r->e[i].v += v; return; }
    r->e[r->n].col = col; r->e[r->n].v = v; r->n++;
}
static int* g_colmap; /* [n*512] -> unknown index or -1 */
static int col_of(const og_grid* g, int t, int v) {
    if (t < 0 || !(g->t[t].type & OG_LEAF)) return -1;
    return g_colmap[(size_t)t * NC + v];
}
/* value of the (masked) x at a same-level neighbour cell as a linear form, times w */
static void halo_form(const og_grid* g, int t, int v, int axis, int sgn, double w, og_row* r) {
    int nv, q = nb_cell(g, t, v, axis, sgn, &nv);
    if (q < 0) return;
    if (q == t) { if (CT(g, t)[nv] == OG_INTERIOR) row_add(r, col_of(g, t, nv), w); return; }
    int qt = g->t[q].type;
    if (qt & OG_GHOST) {
        /* x_self + 0.5 * (parent value - mean of own 2x2x2 block) */
        int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
        if (CT(g, t)[v] == OG_INTERIOR) row_add(r, col_of(g, t, v), w);
        for (int d = 0; d < 8; d++) {
            int bl[3] = {l[0] ^ (d >> 2), l[1] ^ ((d >> 1) & 1), l[2] ^ (d & 1)};
            int bv = CELL(bl[0], bl[1], bl[2]);
            if (CT(g, t)[bv] == OG_INTERIOR) row_add(r, col_of(g, t, bv), -0.5 * w / 8.0);
        }
        int p = g->parent[q];
        if (p >= 0) row_add(r, col_of(g, p, parent_cell(g, q, nv)), 0.5 * w);
    } else if (qt & OG_LEAF) {
        if (CT(g, q)[nv] == OG_INTERIOR) row_add(r, col_of(g, q, nv), w);
    } else { /* NONLEAF: mean of the 8 children (all in LEAF tiles for a 2:1 graded tree) */
        if (CT(g, q)[nv] != OG_INTERIOR) return;
        int l[3] = {nv >> 6, (nv >> 3) & 7, nv & 7};
        for (int d = 0; d < 8; d++) {
            int cg[3] = {2 * (g->t[q].c[0] * 8 + l[0]) + (d >> 2), 2 * (g->t[q].c[1] * 8 + l[1]) + ((d >> 1) & 1), 2 * (g->t[q].c[2] * 8 + l[2]) + (d & 1)};
            int c = g->child[q * 8 + ((cg[0] >> 3) & 1) * 4 + ((cg[1] >> 3) & 1) * 2 + ((cg[2] >> 3) & 1)];
            if (c < 0) continue;
            row_add(r, col_of(g, c, CELL(cg[0] & 7, cg[1] & 7, cg[2] & 7)), 0.125 * w);
        }
    }
}
static void build_colmap(og_grid* g, int* nrows) {
    free(g_colmap);
    g_colmap = (int*)malloc(sizeof(int) * (size_t)NC * (g->n ? g->n : 1));
    int n = 0;
    for (int t = 0; t < g->n; t++)
        for (int v = 0; v < NC; v++)
            g_colmap[(size_t)t * NC + v] = ((g->t[t].type & OG_LEAF) && CT(g, t)[v] == OG_INTERIOR) ? n++ : -1;
    *nrows = n;
}
static void assemble_row(og_grid* g, int coeff_ch, int t, int v, og_row* r) {
    r->n = 0;
    float d = CH(g, coeff_ch + 3, t)[v];
    if (d == 0) return;
    float h = voxel_size(g, g->t[t].level);
    row_add(r, col_of(g, t, v), d);
    for (int axis = 0; axis < 3; axis++) {
        halo_form(g, t, v, axis, -1, CH(g, coeff_ch + axis, t)[v], r);
        int nv, q = nb_cell(g, t, v, axis, +1, &nv);
        double cp = (q < 0) ? h : CH(g, coeff_ch + axis, q)[nv];
        halo_form(g, t, v, axis, +1, cp, r);
    }
}
int og_assemble_count(og_grid* g, int coeff_ch, int* n_rows, long long* nnz) {
    build_colmap(g, n_rows);
    long long z = 0;
    og_row* r = (og_row*)malloc(sizeof(og_row));
    for (int t = 0; t < g->n; t++)
        for (int v = 0; v < NC; v++)
            if (g_colmap[(size_t)t * NC + v] >= 0) { assemble_row(g, coeff_ch, t, v, r); z += r->n; }
    free(r);
    *nnz = z;
    return 0;
}
static int ent_cmp(const void* a, const void* b) {
    int x = ((const og_ent*)a)->col, y = ((const og_ent*)b)->col;
    return x < y ? -1 : (x > y);
}
int og_assemble(og_grid* g, int coeff_ch, long long* rowptr, int* col, double* val, int* row_tile, int* row_cell) {
    int n;
    build_colmap(g, &n);
    og_row* r = (og_row*)malloc(sizeof(og_row));
    long long z = 0;
    int row = 0;
    rowptr[0] = 0;
    for (int t = 0; t < g->n; t++)
        for (int v = 0; v < NC; v++) {
            if (g_colmap[(size_t)t * NC + v] < 0) continue;
            assemble_row(g, coeff_ch, t, v, r);
            qsort(r->e, r->n, sizeof(og_ent), ent_cmp);
            for (int i = 0; i < r->n; i++) { col[z] = r->e[i].col; val[z] = r->e[i].v; z++; }
            row_tile[row] = t; row_cell[row] = v;
            rowptr[++row] = z;
        }
    free(r);
    return n;
}
int og_csr_matvec(int n, const long long* rp, const int* ci, const double* va, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        double s = 0;
        for (long long z = rp[i]; z < rp[i + 1]; z++) s += va[z] * x[ci[z]];
        y[i] = s;
    }
    return 0;
}
static double vdot(int n, const double* a, const double* b) {
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}
/* Jacobi-preconditioned FP64 CG (method 0) or BiCGSTAB (method 1) on a CSR
 * matrix, stopping at ||b - Ax|| / ||b|| < tol.  CG with a diagonal
 * preconditioner is the algorithm of Eigen's default ConjugateGradient. */
int og_csr_solve(int n, const long long* rp, const int* ci, const double* va, const double* b, double* x, double tol, int max_iters, int method, int* iters_out, double* rel_out) {
    double* dinv = (double*)malloc(sizeof(double) * n);
    double* r = (double*)malloc(sizeof(double) * n);
    double* z = (double*)malloc(sizeof(double) * n);
    double* p = (double*)malloc(sizeof(double) * n);
    double* q = (double*)malloc(sizeof(double) * n);
    double* s = (double*)malloc(sizeof(double) * n);
    double* tv = (double*)malloc(sizeof(double) * n);
    double* rh = (double*)malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++) {
        double d = 0;
        for (long long k = rp[i]; k < rp[i + 1]; k++) if (ci[k] == i) d = va[k];
        dinv[i] = d != 0 ? 1.0 / d : 1.0;
        x[i] = 0;
        r[i] = b[i];
    }
    double bn = sqrt(vdot(n, b, b)), rn = bn;
    int it = 0;
    if (bn == 0) goto done;
    if (method == 0) {
        for (int i = 0; i < n; i++) { z[i] = dinv[i] * r[i]; p[i] = z[i]; }
        double rz = vdot(n, r, z);
        for (it = 0; it < max_iters; it++) {
            og_csr_matvec(n, rp, ci, va, p, q);
            double a = rz / vdot(n, p, q);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; i++) { x[i] += a * p[i]; r[i] -= a * q[i]; z[i] = dinv[i] * r[i]; }
            rn = sqrt(vdot(n, r, r));
            if (rn < tol * bn) { it++; break; }
            double rz2 = vdot(n, r, z), be = rz2 / rz;
            rz = rz2;
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; i++) p[i] = z[i] + be * p[i];
        }
    } else {
        double rho = 1, alpha = 1, omega = 1;
        for (int i = 0; i < n; i++) { rh[i] = r[i]; p[i] = 0; q[i] = 0; }
        for (it = 0; it < max_iters; it++) {
            double rho1 = vdot(n, rh, r);
            double beta = (rho1 / rho) * (alpha / omega);
            rho = rho1;
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; i++) { p[i] = r[i] + beta * (p[i] - omega * q[i]); z[i] = dinv[i] * p[i]; }
            og_csr_matvec(n, rp, ci, va, z, q);
            alpha = rho / vdot(n, rh, q);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; i++) { x[i] += alpha * z[i]; s[i] = r[i] - alpha * q[i]; }
            rn = sqrt(vdot(n, s, s));
            if (rn < tol * bn) { for (int i = 0; i < n; i++) r[i] = s[i]; it++; break; }
            for (int i = 0; i < n; i++) z[i] = dinv[i] * s[i];
            og_csr_matvec(n, rp, ci, va, z, tv);
            omega = vdot(n, tv, s) / vdot(n, tv, tv);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; i++) { x[i] += omega * z[i]; r[i] = s[i] - omega * tv[i]; }
            rn = sqrt(vdot(n, r, r));
            if (rn < tol * bn) { it++; break; }
        }
    }
done:
    og_csr_matvec(n, rp, ci, va, x, q);
    {
        double e = 0;
        for (int i = 0; i < n; i++) e += (b[i] - q[i]) * (b[i] - q[i]);
        if (rel_out) *rel_out = bn > 0 ? sqrt(e) / bn : 0;
    }
    if (iters_out) *iters_out = it;
    free(dinv); free(r); free(z); free(p); free(q); free(s); free(tv); free(rh);
    return 0;
}

/* ------------------------------------------------------------------ */
/* geometric multigrid preconditioners: GMGSolver (src/GMGSolver.cu)    */
/* and CMGSolver (src/CMGSolver.cu), kind OG_GMG / OG_CMG               */
/* ------------------------------------------------------------------ */
typedef struct {
    float x[1000];
    uint8_t ct[1000];
    int tt_own;     /* subtree type of the tile */
    int tt_face[6]; /* subtree type seen across each face (GMG: the tile's own type when empty) */
} og_gsnap;

/* HATileInfo::subtreeType (HATileInfo.h:79-84) */
static int subtree_type(const og_grid* g, int t, int sl) {
    int ty = g->t[t].type;
    return (g->t[t].level == sl && ty == OG_NONLEAF) ? OG_LEAF : ty;
}

/* LoadGMGLaplacianTileData (GMGSolver.cu:81-134) and LoadCMGLaplacianTileData
 * (CMGSolver.cu:59-170): raw x and cell types of the tile and its face halo;
 * an empty neighbour reads x = 0, DIRICHLET; CMG extrapolates across a GHOST
 * neighbour as the AMG loader does. */
static void load_gsnap(const og_grid* g, int kind, int t, int sl, int x_ch, og_gsnap* S) {
    const float* X = CH(g, x_ch, t);
    const uint8_t* ty = CT(g, t);
    S->tt_own = subtree_type(g, t, sl);
    for (int v = 0; v < NC; v++) {
        int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
        S->x[SX(i, j, k)] = X[v];
        S->ct[SX(i, j, k)] = ty[v];
    }
    for (int axis = 0; axis < 3; axis++) {
        for (int s = 0; s < 2; s++) {
            int sgn = s ? 1 : -1;
            int q = g->nbr[t * 6 + axis + (s ? 3 : 0)];
            S->tt_face[axis + 3 * s] = q < 0 ? S->tt_own : subtree_type(g, q, sl);
            for (int fi = 0; fi < 64; fi++) {
                int a = fi >> 3, b = fi & 7;
                int fl[3], cl[3], nl[3];
                int axk = s ? 8 : -1;
                if (axis == 0) { fl[0] = axk; fl[1] = a; fl[2] = b; }
                else if (axis == 1) { fl[0] = a; fl[1] = axk; fl[2] = b; }
                else { fl[0] = a; fl[1] = b; fl[2] = axk; }
                for (int d = 0; d < 3; d++) { cl[d] = fl[d]; nl[d] = fl[d]; }
                cl[axis] -= sgn;
                nl[axis] = s ? 0 : 7;
                int fx = SX(fl[0], fl[1], fl[2]);
                int nv = CELL(nl[0], nl[1], nl[2]);
                if (q < 0) {
                    S->x[fx] = 0.0f;
                    S->ct[fx] = OG_DIRICHLET;
                } else if (kind == OG_CMG && subtree_type(g, q, sl) == OG_GHOST) {
                    float avg = 0;
                    for (int di = 0; di < 2; di++)
                        for (int dj = 0; dj < 2; dj++)
                            for (int dk = 0; dk < 2; dk++) avg += S->x[SX(cl[0] ^ di, cl[1] ^ dj, cl[2] ^ dk)];
                    avg /= 8;
                    float V1 = CH(g, x_ch, q)[nv];
                    S->x[fx] = (float)((double)S->x[SX(cl[0], cl[1], cl[2])] + 0.5 * (double)(V1 - avg));
                    S->ct[fx] = CT(g, q)[nv];
                } else {
                    S->x[fx] = CH(g, x_ch, q)[nv];
                    S->ct[fx] = CT(g, q)[nv];
                }
            }
        }
    }
}

/* NegativeLaplacianCoeff: GMG from the tile types of both sides (GMGSolver.cu:3-31),
 * CMG h unless a side is NEUMANN (CMGSolver.cu:3-7) */
static float geo_coeff(int kind, float h, int tt0, int tt1, int c0, int c1) {
    if ((c0 | c1) & OG_NEUMANN) return 0.0f;
    if (kind == OG_CMG) return h;
    float ooh = 1.0f / h;
    int both = (tt0 & OG_LEAF) && (tt1 & OG_LEAF);
    int lg = ((tt0 & OG_LEAF) && (tt1 & OG_GHOST)) || ((tt0 & OG_GHOST) && (tt1 & OG_LEAF));
    float oodh = both ? ooh : (lg ? (2.0f * ooh) / 3.0f : 0.0f);
    return oodh * ooh;
}
/* GMGLaplacianTileData::negativeLap (GMGSolver.cu:46-66), CMG's (CMGSolver.cu:22-45):
 * sum over -x,+x,-y,+y,-z,+z of coeff * (x0 - x1) (or of coeff for the diagonal);
 * GMG scales by h^3; 0 on cells that are not INTERIOR */
static float gsnap_neg_lap(int kind, const og_gsnap* S, float h, int v, int diag) {
    int l[3] = {v >> 6, (v >> 3) & 7, v & 7};
    int c = SX(l[0], l[1], l[2]);
    int ct0 = S->ct[c];
    float x0 = S->x[c];
    float sum = 0;
    for (int axis = 0; axis < 3; axis++)
        for (int s = 0; s < 2; s++) {
            int sgn = s ? 1 : -1;
            int n[3] = {l[0], l[1], l[2]};
            n[axis] += sgn;
            int inside = n[axis] >= 0 && n[axis] < 8;
            int nc = SX(n[0], n[1], n[2]);
            int tt1 = inside ? S->tt_own : S->tt_face[axis + 3 * s];
            float coeff = geo_coeff(kind, h, S->tt_own, tt1, ct0, S->ct[nc]);
            sum = diag ? sum + coeff : fmaf(coeff, x0 - S->x[nc], sum);
        }
    if (!(ct0 & OG_INTERIOR)) return 0.0f;
    return kind == OG_CMG ? sum : sum * h * h * h;
}

static int geo_level_member(const og_grid* g, int kind, int t, int level, int with_ghosts) {
    if (g->t[t].level != level) return 0;
    int ty = g->t[t].type;
    return (ty & (OG_LEAF | OG_NONLEAF)) || (with_ghosts && kind == OG_GMG && (ty & OG_GHOST));
}

/* GaussSeidelGMG / GaussSeidelCMG (GMGSolver.cu:217-223, CMGSolver.cu:271-276) and their
 * kernels (GMGSolver.cu:173-210, CMGSolver.cu:226-262): x += (b - Ax) / D on INTERIOR cells
 * of one colour, no relaxation factor */
static void geo_gs_pass(og_grid* g, int kind, int level, int color, int x_ch, int rhs_ch) {
    float h = voxel_size(g, level);
#pragma omp parallel
    {
        og_gsnap* S = (og_gsnap*)malloc(sizeof(og_gsnap));
#pragma omp for schedule(dynamic, 16)
        for (int t = 0; t < g->n; t++) {
            if (!geo_level_member(g, kind, t, level, 0)) continue;
            load_gsnap(g, kind, t, level, x_ch, S);
            float* X = CH(g, x_ch, t);
            const float* B = CH(g, rhs_ch, t);
            for (int v = 0; v < NC; v++) {
                int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
                if (((i + j + k) & 1) != color) continue;
                int ct = CT(g, t)[v];
                float Ax = gsnap_neg_lap(kind, S, h, v, 0);
                float D = gsnap_neg_lap(kind, S, h, v, 1);
                float delta = (ct & OG_INTERIOR) ? (B[v] - Ax) / D : 0.0f;
                X[v] = S->x[SX(i, j, k)] + delta;
            }
        }
        free(S);
    }
}
static void geo_gs(og_grid* g, int kind, int iters, int order, int level, int x_ch, int rhs_ch) {
    for (int it = 0; it < iters; it++) {
        geo_gs_pass(g, kind, level, order, x_ch, rhs_ch);
        geo_gs_pass(g, kind, level, 1 - order, x_ch, rhs_ch);
    }
}
void og_geo_gauss_seidel(og_grid* g, int kind, int iters, int order, int level, int x_ch, int rhs_ch) {
    geo_gs(g, kind, iters, order, level, x_ch, rhs_ch);
}

/* ResidualAndRestrict128Kernel (GMGSolver.cu:225-284), ConservativeResidualAndRestrict128Kernel
 * (CMGSolver.cu:278-331): coarse rhs = one_over_alpha * sum of 8 residuals; a GMG GHOST tile
 * adds its sum to its LEAF parent's rhs instead */
static void geo_restrict(og_grid* g, int kind, int level, int x_ch, int rhs_ch, float ooa) {
    float h = voxel_size(g, level);
    og_gsnap* S = (og_gsnap*)malloc(sizeof(og_gsnap));
    float res[NC];
    for (int t = 0; t < g->n; t++) {
        if (!geo_level_member(g, kind, t, level, 1)) continue;
        int p = g->parent[t];
        if (p < 0) continue;
        load_gsnap(g, kind, t, level, x_ch, S);
        for (int v = 0; v < NC; v++) res[v] = CH(g, rhs_ch, t)[v] - gsnap_neg_lap(kind, S, h, v, 0);
        int ghost = g->t[t].type & OG_GHOST;
        for (int b = 0; b < 64; b++) {
            int fl[3] = {(b >> 4) * 2, ((b >> 2) & 3) * 2, (b & 3) * 2};
            float sum = 0;
            for (int ii = 0; ii < 2; ii++)
                for (int jj = 0; jj < 2; jj++)
                    for (int kk = 0; kk < 2; kk++) sum += res[CELL(fl[0] + ii, fl[1] + jj, fl[2] + kk)];
            float* c = &CH(g, rhs_ch, p)[parent_cell(g, t, CELL(fl[0], fl[1], fl[2]))];
            if (ghost) *c = *c + sum;
            else *c = sum * ooa;
        }
    }
    free(S);
}
/* ProlongateAndUpdate128Kernel (GMGSolver.cu:286-316), CMG's (CMGSolver.cu:339-370):
 * x += P * coarse x on INTERIOR cells, GHOST cells take the coarse x, others 0 */
static void geo_prolong(og_grid* g, int kind, int level, int x_ch, float P) {
    for (int t = 0; t < g->n; t++) {
        if (!geo_level_member(g, kind, t, level, 1)) continue;
        int p = g->parent[t];
        int ghost = g->t[t].type & OG_GHOST;
        float* X = CH(g, x_ch, t);
        for (int v = 0; v < NC; v++) {
            float cx = p >= 0 ? CH(g, x_ch, p)[parent_cell(g, t, v)] : 0.0f;
            int in = CT(g, t)[v] & OG_INTERIOR;
            X[v] = ghost ? (in ? cx : 0.0f) : (in ? fmaf(P, cx, X[v]) : 0.0f);
        }
    }
}
/* GMGSolver::VCycle (GMGSolver.cu:324-388), CMGSolver::VCycle (CMGSolver.cu:377-416) */
void og_geo_vcycle(og_grid* g, int kind, int x_ch, int f_ch, int rhs_ch, int level_iters, int coarsest_iters, float ooa, float P) {
    for (int t = 0; t < g->n; t++) {
        memset(CH(g, x_ch, t), 0, sizeof(float) * NC);
        if (g->t[t].type & OG_GHOST) memset(CH(g, rhs_ch, t), 0, sizeof(float) * NC);
        else memcpy(CH(g, rhs_ch, t), CH(g, f_ch, t), sizeof(float) * NC);
    }
    for (int i = g->max_level; i > 0; i--) {
        geo_gs(g, kind, level_iters, 0, i, x_ch, rhs_ch);
        geo_restrict(g, kind, i, x_ch, rhs_ch, ooa);
    }
    geo_gs(g, kind, coarsest_iters / 2, 0, 0, x_ch, rhs_ch);
    geo_gs(g, kind, coarsest_iters / 2, 1, 0, x_ch, rhs_ch);
    for (int i = 1; i <= g->max_level; i++) {
        geo_prolong(g, kind, i, x_ch, P);
        geo_gs(g, kind, level_iters, 1, i, x_ch, rhs_ch);
    }
}

/* FullNegativeLaplacian (GMGSolver.cu:167-171): GHOST x from the parents, the operator on
 * LEAF and GHOST tiles, GHOST results added into their LEAF parents.
 * ConservativeFullNegativeLaplacian (CMGSolver.cu:210-222): GHOST x from the parents,
 * NONLEAF x as the mean of LEAF children, the operator on LEAF tiles. */
void og_geo_full_neg_lap(og_grid* g, int kind, int x_ch, int ax_ch) {
    propagate_ghosts(g, x_ch);
    if (kind == OG_CMG) accumulate_leafs_to_parents(g, x_ch);
#pragma omp parallel
    {
        og_gsnap* S = (og_gsnap*)malloc(sizeof(og_gsnap));
#pragma omp for schedule(dynamic, 16)
        for (int t = 0; t < g->n; t++) {
            int ty = g->t[t].type;
            if (!((ty & OG_LEAF) || (kind == OG_GMG && (ty & OG_GHOST)))) continue;
            float h = voxel_size(g, g->t[t].level);
            load_gsnap(g, kind, t, -1, x_ch, S);
            for (int v = 0; v < NC; v++) CH(g, ax_ch, t)[v] = gsnap_neg_lap(kind, S, h, v, 0);
        }
        free(S);
    }
    if (kind == OG_GMG) {
        for (int t = 0; t < g->n; t++) {
            if (!(g->t[t].type & OG_GHOST)) continue;
            int p = g->parent[t];
            if (p < 0) continue;
            for (int b = 0; b < 64; b++) {
                int fl[3] = {(b >> 4) * 2, ((b >> 2) & 3) * 2, (b & 3) * 2};
                float sum = 0;
                for (int ii = 0; ii < 2; ii++)
                    for (int jj = 0; jj < 2; jj++)
                        for (int kk = 0; kk < 2; kk++) {
                            int v = CELL(fl[0] + ii, fl[1] + jj, fl[2] + kk);
                            sum += (CT(g, t)[v] & (OG_INTERIOR | OG_DIRICHLET | OG_NEUMANN)) ? CH(g, ax_ch, t)[v] : 0.0f;
                        }
                float* c = &CH(g, ax_ch, p)[parent_cell(g, t, CELL(fl[0], fl[1], fl[2]))];
                *c = fmaf(sum, 1.0f, *c);
            }
        }
    }
}

static void geo_apply(og_grid* g, const void* ctx, int p_ch, int ap_ch) {
    const int* c = (const int*)ctx;
    og_geo_full_neg_lap(g, c[0], p_ch, ap_ch);
}
static void geo_precond(og_grid* g, const void* ctx, int z_ch, int r_ch, int tmp_ch) {
    const int* c = (const int*)ctx;
    const float* f = (const float*)(c + 3);
    og_geo_vcycle(g, c[0], z_ch, r_ch, tmp_ch, c[1], c[2], f[0], f[1]);
}
/* GMGSolver::solve (GMGSolver.cu:472-607), CMGSolver::solve (CMGSolver.cu:466-601) */
int og_geo_solve(og_grid* g, int kind, float ooa, float P, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride, int pure_neumann, double* rel_res) {
    int ctx[5] = {kind, level_iters, coarsest_iters, 0, 0};
    memcpy(&ctx[3], &ooa, sizeof(float));
    memcpy(&ctx[4], &P, sizeof(float));
    return pcg(g, geo_apply, geo_precond, ctx, max_iters, tol, sync_stride, pure_neumann, rel_res);
}

/* CalcCellTypesFromLeafs (PoissonGrid.cu:923-977): NONLEAF cells from their active
 * children, finest level first (DIRICHLET before INTERIOR before NEUMANN), then GHOST
 * cells from their parents */
void og_calc_cell_types_from_leafs(og_grid* g) {
    for (int L = g->max_level - 1; L >= 0; L--)
        for (int t = 0; t < g->n; t++) {
            if (g->t[t].level != L || g->t[t].type != OG_NONLEAF) continue;
            for (int v = 0; v < NC; v++) {
                int i = v >> 6, j = (v >> 3) & 7, k = v & 7;
                int c = g->child[t * 8 + ((i >> 2) << 2) + ((j >> 2) << 1) + (k >> 2)];
                int nd = 0, ni = 0;
                if (c >= 0 && (g->t[c].type & (OG_LEAF | OG_NONLEAF))) {
                    int b0 = (i & 3) << 1, b1 = (j & 3) << 1, b2 = (k & 3) << 1;
                    for (int ii = 0; ii < 2; ii++)
                        for (int jj = 0; jj < 2; jj++)
                            for (int kk = 0; kk < 2; kk++) {
                                int ty = CT(g, c)[CELL(b0 + ii, b1 + jj, b2 + kk)];
                                if (ty & OG_DIRICHLET) nd++;
                                else if (ty & OG_INTERIOR) ni++;
                            }
                }
                CT(g, t)[v] = nd > 0 ? OG_DIRICHLET : ni > 0 ? OG_INTERIOR : OG_NEUMANN;
            }
        }
    for (int t = 0; t < g->n; t++) {
        if (g->t[t].type != OG_GHOST) continue;
        int p = g->parent[t];
        for (int v = 0; v < NC; v++) CT(g, t)[v] = p >= 0 ? CT(g, p)[parent_cell(g, t, v)] : OG_DIRICHLET;
    }
}

/* ------------------------------------------------------------------ */
/* stand-alone iterative solvers of the reference's test harness        */
/* ------------------------------------------------------------------ */
/* Dot over the tiles of the given types */
static double dot_types(og_grid* g, int a_ch, int b_ch, int types) {
    double s = 0;
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & types)) continue;
        const float* A = CH(g, a_ch, t);
        const float* B = CH(g, b_ch, t);
        double st = 0;
        for (int q = 0; q < NC; q += 4) {
            float f = A[q] * B[q];
            f = fmaf(A[q + 1], B[q + 1], f);
            f = fmaf(A[q + 2], B[q + 2], f);
            f = fmaf(A[q + 3], B[q + 3], f);
            st += (double)f;
        }
        s += st;
    }
    return s;
}

/* AMGSolver::FASMuCycleSolve (AMGSolver.cu:1311-1356): mu-cycles on x (channel 0) against
 * b (channel 1), channel 2 as the FAS x0 and then the residual b - A x; stops when
 * |r| < tol |b| and returns the iteration index at which it stopped */
int og_fas_mu_cycle_solve(og_grid* g, int coeff_ch, int repeat_times, double omega, float Rr, float P, int max_iters, double tol, int level_iters,
                          int coarsest_iters, double* rel_res) {
    const int X = 0, B = 1, X0 = 2;
    memset(CH(g, X, 0), 0, sizeof(float) * NC * g->n);
    double rhs_norm = sqrt(og_dot(g, B, B));
    double thr = tol * rhs_norm;
    if (thr < DBL_MIN) thr = DBL_MIN;
    mu_args A = {repeat_times, X, B, X0, coeff_ch, level_iters, coarsest_iters, omega, Rr, P};
    double res = rhs_norm;
    int i;
    for (i = 0; i < max_iters; i++) {
        fas_step(g, g->max_level, &A);
        og_full_neg_lap_leafs(g, X, coeff_ch, X0);
        for (int t = 0; t < g->n; t++) {
            if (!(g->t[t].type & OG_LEAF)) continue;
            for (int v = 0; v < NC; v++) CH(g, X0, t)[v] = CH(g, B, t)[v] - CH(g, X0, t)[v];
        }
        res = sqrt(og_dot(g, X0, X0));
        if (res < thr) break;
    }
    if (rel_res) *rel_res = res / rhs_norm;
    return i;
}

/* FullNegativeLaplacian with calc_diag (GMGSolver.cu:167-171): the diagonal of the GMG
 * operator on LEAF and GHOST tiles, GHOST diagonals added into their LEAF parents */
static void gmg_full_diag(og_grid* g, int x_ch, int d_ch) {
    propagate_ghosts(g, x_ch);
    og_gsnap* S = (og_gsnap*)malloc(sizeof(og_gsnap));
    for (int t = 0; t < g->n; t++) {
        int ty = g->t[t].type;
        if (!(ty & (OG_LEAF | OG_GHOST))) continue;
        float h = voxel_size(g, g->t[t].level);
        load_gsnap(g, OG_GMG, t, -1, x_ch, S);
        for (int v = 0; v < NC; v++) CH(g, d_ch, t)[v] = gsnap_neg_lap(OG_GMG, S, h, v, 1);
    }
    free(S);
    for (int t = 0; t < g->n; t++) {
        if (!(g->t[t].type & OG_GHOST)) continue;
        int p = g->parent[t];
        if (p < 0) continue;
        for (int b = 0; b < 64; b++) {
            int fl[3] = {(b >> 4) * 2, ((b >> 2) & 3) * 2, (b & 3) * 2};
            float sum = 0;
            for (int ii = 0; ii < 2; ii++)
                for (int jj = 0; jj < 2; jj++)
                    for (int kk = 0; kk < 2; kk++) {
                        int v = CELL(fl[0] + ii, fl[1] + jj, fl[2] + kk);
                        sum += (CT(g, t)[v] & (OG_INTERIOR | OG_DIRICHLET | OG_NEUMANN)) ? CH(g, d_ch, t)[v] : 0.0f;
                    }
            float* c = &CH(g, d_ch, p)[parent_cell(g, t, CELL(fl[0], fl[1], fl[2]))];
            *c = fmaf(sum, 1.0f, *c);
        }
    }
}
/* GMGSolver::dampedJacobiSolve (GMGSolver.cu:390-470): x += omega r / D on INTERIOR cells
 * of LEAF tiles (x = 0 where D = 0), channels x 0, b 1, r 2, D 3 */
int og_gmg_damped_jacobi_solve(og_grid* g, int max_iters, double tol, float omega, double* rel_res) {
    const int X = 0, B = 1, AX = 2, D = 3;
    memset(CH(g, X, 0), 0, sizeof(float) * NC * g->n);
    double rhs_norm = sqrt(dot_types(g, B, B, OG_LEAF | OG_NONLEAF | OG_GHOST));
    double thr = tol * rhs_norm;
    if (thr < DBL_MIN) thr = DBL_MIN;
    double res = rhs_norm;
    int i;
    for (i = 0; i < max_iters; i++) {
        og_geo_full_neg_lap(g, OG_GMG, X, AX);
        for (int t = 0; t < g->n; t++) {
            if (!(g->t[t].type & OG_LEAF)) continue;
            for (int v = 0; v < NC; v++)
                if (CT(g, t)[v] & OG_INTERIOR) CH(g, AX, t)[v] = CH(g, B, t)[v] - CH(g, AX, t)[v];
        }
        res = sqrt(og_dot(g, AX, AX));
        if (res < thr) break;
        gmg_full_diag(g, X, D);
        for (int t = 0; t < g->n; t++) {
            if (!(g->t[t].type & OG_LEAF)) continue;
            for (int v = 0; v < NC; v++) {
                if (!(CT(g, t)[v] & OG_INTERIOR)) continue;
                float d = CH(g, D, t)[v];
                if (d == 0.0f) CH(g, X, t)[v] = 0.0f;
                else CH(g, X, t)[v] = CH(g, X, t)[v] + (omega * CH(g, AX, t)[v]) / d;
            }
        }
    }
    if (rel_res) *rel_res = res / rhs_norm;
    return i;
}
