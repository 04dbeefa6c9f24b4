// Tile plan of the single-pass (tiled) residual + Jacobian assembly.
//
// The elements are cut into tiles of at most T elements that are compact in
// space (recursive coordinate bisection of the element centroids, each
// connected component of the face graph on its own).  One CTA evaluates one
// tile: the tile's node positions and potentials are staged in shared
// memory, every element's state (gradient, speed, density, centroid) goes
// to shared memory, the upwind walk and the upstream element's state read
// shared memory while they stay inside the tile, and the element residual
// vectors and local matrices are summed in shared memory in the fixed order
// this plan lists.  An output (a residual entry, a diagonal or an
// upper-triangle Jacobian slot) whose contributing elements all lie in one
// tile is written by that tile; any other output is written by each of its
// tiles as a partial sum into a side buffer, and a short combine pass adds
// the partials in tile order.  The local matrices never leave the chip.
//
// Elements are renumbered tile by tile ("internal" ids: tile t owns the
// internal range [eoff[t], eoff[t+1]), ascending user id within a tile);
// `perm` maps internal to user ids and `iperm` back.  Every per-element
// output of the library stays in user order.
#pragma once

#include "internal.cuh"

namespace up3d {

struct TilePlan {
    int32_t T = 0;              // most elements per tile
    int32_t stretch = 1;        // tiles this many times longer along x than across
    int32_t max_edges = 0;      // most distinct element edges of one tile
    int64_t n_tiles = 0;
    int32_t max_nodes = 0;      // most distinct nodes of one tile
    int64_t n_tile_nodes = 0;   // sum over tiles of their distinct nodes
    int64_t n_tile_edges = 0;   // sum over tiles of their distinct element edges
    int64_t n_part = 0;         // partial sums written per evaluation
    int64_t n_cnode = 0;        // node outputs combined from partials (incl. isolated nodes)
    int64_t n_cedge = 0;        // upper slots combined from partials
    double build_s = 0.0;       // host time of the plan build

    DBuf<int32_t> perm;         // (E) internal -> user element
    DBuf<int32_t> iperm;        // (E) user -> internal element
    DBuf<int4> conn;            // (E) global node ids, internal order
    DBuf<int4> fnbr;            // (E) face neighbours as internal ids (-1 boundary)
    DBuf<double4> cen;          // (E) centroids, internal order
    DBuf<double> disp;          // (E, 12) face displacements cen(nbr) - cen(e), internal order
    DBuf<int32_t> eoff;         // (n_tiles + 1) element range of each tile
    DBuf<int32_t> noff;         // (n_tiles + 1) tile-node range of each tile
    DBuf<int32_t> uoff;         // (n_tiles + 1) tile-edge range of each tile
    DBuf<int32_t> tnode;        // (n_tile_nodes) global node of each tile-node, ascending per tile
    DBuf<double4> txyz;         // (n_tile_nodes) its position (x, y, z, 0)
    DBuf<ushort4> lconn;        // (E) tile-local node indices of each element's vertices
    DBuf<int32_t> nent_off;     // (n_tile_nodes + 1)
    DBuf<uint16_t> nent;        // (4E) (local element << 2) | vertex, ascending local element
    DBuf<int2> ndst;            // (n_tile_nodes) {node, diagonal slot} or {-1 - partial, diagonal slot}
    DBuf<int32_t> uent_off;     // (n_tile_edges + 1)
    DBuf<uint16_t> uent;        // (6E) (local element << 3) | pair, ascending local element
    DBuf<int2> udst;            // (n_tile_edges) {slot, transposed slot} or {-1 - partial, 0}
    DBuf<double> part;          // (n_part) partial sums, tile-major
    DBuf<int32_t> cn_off, cn_idx;  // node outputs from partials: first partial of each (R, diagonal) pair
    DBuf<int2> cn_dst;             // {node, diagonal slot or -1}
    DBuf<int32_t> ce_off, ce_idx;  // upper slots from partials, tile order
    DBuf<int2> ce_dst;             // {slot, transposed slot}
};

// Builds (or rebuilds for another tile size or stretch) the mesh's tile
// plan.  Every array is followed by 16 bytes of padding.
void ensure_tiles(up3d_mesh* m, int T, int stretch, cudaStream_t s);

}  // namespace up3d
