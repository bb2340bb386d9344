// Tiling of the mesh for the fused stage kernel.
//
// Cells are stored in Hilbert order of their barycentres, and consecutive
// runs of at most `tile_cells` cells form compact tiles.  One CTA owns one
// tile.  For its tile it needs the limited gradients of the tile cells and of
// their face neighbours (ring 1), hence the states of ring 2 as well; all of
// these are staged in shared memory, so gradients and face fluxes never go
// to global memory.  Faces on tile borders are evaluated by both adjacent
// tiles (identical arithmetic, so identical results).
#pragma once

#include <stdint.h>

#include <vector>

#include "ccfd_b200.h"

struct TileSet {
    int n_tiles = 0;
    int tile_cells = 0;
    // per tile (size n_tiles + 1 offsets into the concatenated arrays)
    std::vector<int> e_off;      // staged entries E: [tile | ring1 | ring2 | ghosts]
    std::vector<int> counts;     // per tile 4 ints: nT, nG (= nT + ring1), nE_cells, nE
    std::vector<int> e_ref;      // E entry: device cell id, or -1-g for ghost g
    std::vector<int> hs_off;     // per tile offsets into the gradient half-side arrays
    std::vector<int16_t> hs_nbl; // per gradient-cell half-side: local E index of neighbour
    std::vector<int16_t> hs_loc; // per gradient cell: local start of its half-sides (nG + 1 per tile)
    std::vector<int> f_off;      // per tile offsets into the face arrays
    std::vector<int> f_id;       // device id of an interior face, or -1-g for the boundary face of ghost g
    std::vector<int> f_lr;       // packed local indices (owner | neighbour << 16); a boundary
                                 // face's neighbour is the ghost's staged entry
    std::vector<int> f_hs;       // packed local half-side indices (owner | neighbour << 16)
    std::vector<int> u_code;     // per device half-side of a tile cell: 2 * local face + (neighbour ? 1 : 0)
    int max_e = 0, max_g = 0, max_hs = 0, max_f = 0;
};

// device order of cells (device index -> reference cell): Hilbert curve of
// the barycentres
void ccfd_hilbert_order(const ccfd_mesh* m, std::vector<int>& cell_order);

// device order of cells by reverse Cuthill-McKee on the face-neighbour graph
void ccfd_rcm_order(const ccfd_mesh* m, std::vector<int>& cell_order);

// Build the tiles for a mesh whose cells are already in device order.
// cperm: device -> reference cell; cinv: reference -> device cell;
// fdev: reference face -> device interior face id (-1 for boundary faces).
void ccfd_build_tiles(const ccfd_mesh* m, const std::vector<int>& cperm,
                      const std::vector<int>& cinv, const std::vector<int>& fdev, int tile_cells,
                      TileSet& ts);
