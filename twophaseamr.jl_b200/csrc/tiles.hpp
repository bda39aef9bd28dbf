// Haloed block tiles of a CSR level: the per-block data of the two fused
// V-cycle kernels of a level (csrc/tiles.cuh).
//
// A tile is one mesh block (its cells are contiguous in the reference's cell
// order) plus the cells within graph distance 3 of it in the level operator's
// sparsity pattern, listed ring by ring.  The down kernel computes both
// pre-smoothing sweeps, the residual and the restriction of the block's
// coarse cells from the right-hand side on the tile alone (each dependent
// phase shrinks the valid region by one ring); the up kernel computes the
// prolongation and both post-smoothing sweeps of the block from the coarse
// correction on the tile alone.  Halo values are recomputed redundantly in
// each tile instead of being exchanged between launches, which removes four
// of the six grid-wide dependencies a level costs per V-cycle.
#pragma once

#include <cstdint>
#include <vector>

#include "host.hpp"

namespace tpa {

struct TileLevelHost {
    bool ok = false;
    int ntiles = 0;
    int n3max = 0, n2max = 0, n1max = 0;  // largest ring counts (cumulative) over the tiles
    int emax = 0;                         // largest number of local CSR entries of a tile
    int comax = 0;                        // largest number of coarse cells of a tile
    // per tile t, cells cell[cell_off[t] .. cell_off[t + 1]): the block's cells in
    // order (n0 of them), then ring 1, ring 2, ring 3; ring[4 t + r] = cells of
    // rings <= r (ring[4 t] = n0)
    std::vector<int32_t> cell, cell_off, ring;
    std::vector<int32_t> own;  // parallel to cell: the tentative owner (coarse cell) of each tile cell
    // local rows 0 .. n2 - 1 of tile t: entries lrp[lrp_off[t] + k] ..
    // lrp[lrp_off[t] + k + 1] (relative to ent_off[t]) in CSR order; pos is the
    // entry's position in the level CSR, lcol its column as a local cell index
    std::vector<int32_t> lrp, lrp_off, pos, ent_off;
    std::vector<int16_t> lcol;
    // coarse cells whose children lie in tile t: co[co_off[t] ..), and for each
    // the local indices of its first four children (-1: none), in the order of
    // the level's child lists
    std::vector<int32_t> co, co_off;
    std::vector<int16_t> ch;
};

// Tiles of a level with `nblocks` blocks of `cpb` cells, operator A (square,
// sorted columns) and tentative owners `owner` onto `nc` coarse cells.  ok is
// false (and the level keeps the unfused kernels) when a coarse cell's
// children do not all lie in one block, a coarse cell has more than four
// children, or a tile would exceed `max_cells` cells or 32767 local entries.
TileLevelHost build_tiles(const Csr& A, int64_t nblocks, int64_t cpb, const std::vector<int32_t>& owner, int64_t nc,
                          int max_cells);

}  // namespace tpa
