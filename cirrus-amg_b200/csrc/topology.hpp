// Host-side octree topology: the tile registry of HADeviceGrid (src/HAGrid.h)
// with its refinement and ghost-spawning rules, producing the hash-free
// neighbour / parent / child tables the device kernels index.
#pragma once
#include <cstdint>
#include <functional>
#include <unordered_map>
#include <vector>

namespace cmg {

enum : int { kLeaf = 1, kNonLeaf = 2, kGhost = 4 };
enum : int { kDirichlet = 1, kInterior = 2, kNeumann = 4 };

struct TileRec {
    int level;
    int c[3];
    int type;
};

// Level target of a tile (the argument of HADeviceGrid::iterativeRefine).
using TargetFn = std::function<int(int level, int i, int j, int k)>;

class Topology {
public:
    Topology(float h0, int num_levels) : h0_(h0), num_levels_(num_levels) {}

    float h0() const { return h0_; }
    int num_levels() const { return num_levels_; }
    int max_level() const { return max_level_; }
    int size() const { return (int)tiles_.size(); }
    const std::vector<TileRec>& tiles() const { return tiles_; }

    int find(int level, int i, int j, int k) const;
    int set(int level, int i, int j, int k, int type);  // setTileHost
    void spawn_ghosts();                               // spawnGhostTiles
    int refine_step(const TargetFn& target);           // refineStep
    int iterative_refine(const TargetFn& target);      // iterativeRefine
    // Sort tiles by (level, type, Morton) and build the device tables.
    // Returns, for every tile in the new order, the tile's old index.
    std::vector<int> canonicalize();
    // Take a tile list already in canonical order with its nb / child tables (built
    // elsewhere, e.g. on the device) and derive the level ranges and the LEAF list.
    void adopt(std::vector<TileRec>&& sorted, std::vector<int>&& nb_table, std::vector<int>&& child_table);

    // tables (valid after canonicalize)
    std::vector<int> nb;     // [n][8]: -x,-y,-z,+x,+y,+z, parent, -1
    std::vector<int> child;  // [n][8]: dx*4 + dy*2 + dz
    std::vector<int> level_begin, level_end;      // all tiles of a level
    std::vector<int> nonleaf_begin, ghost_begin;  // type blocks inside a level
    std::vector<int> leaf_list;                   // every LEAF tile

    float voxel_size(int level) const { return h0_ / (float)(1 << level); }

private:
    static uint64_t key(int level, int i, int j, int k);
    void update_max_level();

    float h0_;
    int num_levels_;
    int max_level_ = -1;
    void ensure_index() const;
    void set_ranges();

    std::vector<TileRec> tiles_;
    mutable std::unordered_map<uint64_t, int> index_;
    mutable bool index_stale_ = false;  // adopt() leaves the key index to be rebuilt on first use
};

// Built-in refinement targets and LEAF cell types (tests/TestGrids.cuh).
int case_target(int case_id, const double* prm, int nprm, float h0, int level, const int c[3]);
uint8_t case_cell_type(int case_id, float h0, int level, const int tc[3], int v);

}  // namespace cmg
