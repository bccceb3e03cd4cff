/*
 * ref_harness.cu -- host-side entry points into the reference's own code.
 *
 * TEST INFRASTRUCTURE ONLY.  build_ref.py compiles this file, together with
 * reference headers taken from where they lie and three function definitions
 * cut verbatim out of cirrus_cutcell/MeshCutCell.cu at build time, into
 * oracle/_ref/libcmgref.so.  The tests use it to pin the CPU oracle (and
 * through it the CUDA product) to the reference: the parts of the reference's
 * path that compile and run on a host are run here, unmodified, and compared
 * bit for bit with the restatement.  Nothing in the product loads it.
 *
 * What it exposes (reference file:line in each comment):
 *   - the byte layout of PoissonTile<float,15> and HATileInfo<Tile>
 *     (src/PoissonTile.h:34-39, src/HATileInfo.h:61-95);
 *   - FracInside, FaceFluidRatio, CellCornerSDFInsideCount
 *     (cirrus_cutcell/MeshCutCell.cu:239-412);
 *   - the refinement targets and leaf cell types of the test grids
 *     (tests/TestGrids.cuh:33-150) and the level target of the solver tests'
 *     named grids (tests/SolverTests.cu:17-121);
 *   - PoissonTile::childTile, the data a refined tile hands its children
 *     (src/PoissonTile.h:151-172);
 *   - the header of the 'HAGR' v1 grid blob (src/HAGrid.h:699-708).
 */
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>

#include "PoissonTile.h"
#include "TestGrids.cuh"

/* generated at build time: FracInside, FaceFluidRatio(float x4) and
 * CellCornerSDFInsideCount as they stand in MeshCutCell.cu */
#include "ref_cutcell_extract.inc"
/* generated at build time: SolverTests::SolverTestsLevelTarget */
#include "ref_solvertests_extract.inc"
/* generated at build time: the blob header of HADeviceGrid::dumpBinaryBlob,
 * as ref_hagr::Header */
#include "ref_hagr_extract.inc"

namespace {
HATileAccessor<Tile> host_accessor(float h0) {
    /* only the coordinate half of the accessor is used (mH0); no hash tables */
    return HATileAccessor<Tile>(h0, 0, 0, nullptr, nullptr, nullptr);
}
HATileInfo<Tile> info_of(int level, int ti, int tj, int tk) {
    return HATileInfo<Tile>(LEAF, (uint8_t)level, nullptr, Coord(ti, tj, tk));
}
template <class Case>
int target_of(float h0, int level, int ti, int tj, int tk, int mn, int mx) {
    auto acc = host_accessor(h0);
    auto info = info_of(level, ti, tj, tk);
    return Case::target(acc, info, mn, mx);
}
template <class Case>
int type_of(float h0, int level, int ti, int tj, int tk, int li, int lj, int lk) {
    auto acc = host_accessor(h0);
    auto info = info_of(level, ti, tj, tk);
    return Case::type(acc, info, Coord(li, lj, lk));
}
}  // namespace

extern "C" {

/* out[0..12]: sizeof(Tile), offsetof mData, mNeighbors, mCellType,
 * mIsInterestArea, mIsLockedRefine, mStatus, mSerialIdx, CHNLSIZE,
 * num_channels, sizeof(HATileInfo<Tile>), offsetof HATileInfo::mTilePtr,
 * offsetof HATileInfo::mType.  Returns the number of entries written. */
int cr_layout(long long* out, int n) {
    long long v[] = {
        (long long)sizeof(Tile),
        (long long)offsetof(Tile, mData),
        (long long)offsetof(Tile, mNeighbors),
        (long long)offsetof(Tile, mCellType),
        (long long)offsetof(Tile, mIsInterestArea),
        (long long)offsetof(Tile, mIsLockedRefine),
        (long long)offsetof(Tile, mStatus),
        (long long)offsetof(Tile, mSerialIdx),
        (long long)Tile::CHNLSIZE,
        (long long)Tile::num_channels,
        (long long)sizeof(HATileInfo<Tile>),
        (long long)offsetof(HATileInfo<Tile>, mTilePtr),
        (long long)offsetof(HATileInfo<Tile>, mType),
    };
    int m = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < m && i < n; i++) out[i] = v[i];
    return m;
}

/* MeshCutCell.cu:262-272 */
float cr_frac_inside(float a, float b) { return FracInside(a, b); }

/* MeshCutCell.cu:305-408, over n quadruples */
void cr_face_fluid_ratio(const float* phi4, int n, float* out) {
    for (int i = 0; i < n; i++) out[i] = FaceFluidRatio(phi4[4 * i], phi4[4 * i + 1], phi4[4 * i + 2], phi4[4 * i + 3]);
}

/* MeshCutCell.cu:239-260: node SDF of one tile (9^3 nodes, index i*81+j*9+k)
 * placed in channel `chan` of a reference Tile; counts for all 512 cells. */
void cr_cell_corner_inside_count(const float* nodes729, int chan, float iso, int* out512) {
    std::unique_ptr<Tile> t(new Tile());
    std::memset(t->mData, 0, sizeof(t->mData));
    for (int q = 0; q < 729; q++) t->node(chan, q) = nodes729[q];
    for (int v = 0; v < 512; v++) {
        Coord l = HACoordAccessor<Tile>::localOffsetToCoord((uint32_t)v);
        out512[v] = CellCornerSDFInsideCount(*t, chan, l, iso);
    }
}

/* TestGrids.cuh: case ids as in the oracle (0 uniform, 1 center point,
 * 2 sphere empty, 3 sphere solid, 4 star empty, 5 star solid) */
int cr_case_target(int case_id, float h0, int level, int ti, int tj, int tk, int min_level, int max_level) {
    switch (case_id) {
    case 0: return target_of<UniformGridCase>(h0, level, ti, tj, tk, min_level, max_level);
    case 1: return target_of<CenterPointGridCase>(h0, level, ti, tj, tk, min_level, max_level);
    case 2: return target_of<SphereEmptyGridCase>(h0, level, ti, tj, tk, min_level, max_level);
    case 3: return target_of<SphereSolidGridCase>(h0, level, ti, tj, tk, min_level, max_level);
    case 4: return target_of<StarEmptyGridCase>(h0, level, ti, tj, tk, min_level, max_level);
    case 5: return target_of<StarSolidGridCase>(h0, level, ti, tj, tk, min_level, max_level);
    }
    return -1;
}

/* cell types of a LEAF tile for the same cases, all 512 cells */
int cr_case_types(int case_id, float h0, int level, int ti, int tj, int tk, uint8_t* out512) {
    for (int v = 0; v < 512; v++) {
        Coord l = HACoordAccessor<Tile>::localOffsetToCoord((uint32_t)v);
        int r;
        switch (case_id) {
        case 0: r = type_of<UniformGridCase>(h0, level, ti, tj, tk, l[0], l[1], l[2]); break;
        case 1: r = type_of<CenterPointGridCase>(h0, level, ti, tj, tk, l[0], l[1], l[2]); break;
        case 2: r = type_of<SphereEmptyGridCase>(h0, level, ti, tj, tk, l[0], l[1], l[2]); break;
        case 3: r = type_of<SphereSolidGridCase>(h0, level, ti, tj, tk, l[0], l[1], l[2]); break;
        case 4: r = type_of<StarEmptyGridCase>(h0, level, ti, tj, tk, l[0], l[1], l[2]); break;
        case 5: r = type_of<StarSolidGridCase>(h0, level, ti, tj, tk, l[0], l[1], l[2]); break;
        default: return -1;
        }
        out512[v] = (uint8_t)r;
    }
    return 0;
}

/* SolverTests.cu:17-121, grid ids in the order of tests/TestGridsStr.h */
int cr_solvertests_level_target(int grid_id, float h0, int level, int ti, int tj, int tk) {
    auto acc = host_accessor(h0);
    auto info = info_of(level, ti, tj, tk);
    return SolverTests::SolverTestsLevelTarget(acc, info, (TestGrids)grid_id);
}

/* PoissonTile.h:151-172: parent data (15 channels x 512 cells, then 512
 * types) handed to the child at offset (ox, oy, oz) */
void cr_child_tile(const float* parent_ch, const uint8_t* parent_types, int ox, int oy, int oz, float* child_ch,
                   uint8_t* child_types) {
    std::unique_ptr<Tile> p(new Tile());
    std::memset(p->mData, 0, sizeof(p->mData));
    for (int c = 0; c < Tile::num_channels; c++)
        for (int v = 0; v < 512; v++) (*p)(c, v) = parent_ch[c * 512 + v];
    for (int v = 0; v < 512; v++) p->type(v) = parent_types[v];
    std::unique_ptr<Tile> ch(new Tile(p->childTile(Coord(ox, oy, oz))));
    for (int c = 0; c < Tile::num_channels; c++)
        for (int v = 0; v < 512; v++) child_ch[c * 512 + v] = (*ch)(c, v);
    for (int v = 0; v < 512; v++) child_types[v] = ch->type(v);
}

/* HAGrid.h:699-708 ('HAGR' v1 header) and the record fields of :730-735.
 * out: sizeof(Header), offsetof magic, version, num_levels, max_level,
 * tile_size, coord_size, h0, tile_count, sizeof(Coord), sizeof(Tile). */
int cr_hagr_layout(long long* out, int n) {
    using H = ref_hagr::Header;
    long long v[] = {
        (long long)sizeof(H),
        (long long)offsetof(H, magic),
        (long long)offsetof(H, version),
        (long long)offsetof(H, num_levels),
        (long long)offsetof(H, max_level),
        (long long)offsetof(H, tile_size),
        (long long)offsetof(H, coord_size),
        (long long)offsetof(H, h0),
        (long long)offsetof(H, tile_count),
        (long long)sizeof(Coord),
        (long long)sizeof(Tile),
    };
    int m = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < m && i < n; i++) out[i] = v[i];
    return m;
}

}  // extern "C"
