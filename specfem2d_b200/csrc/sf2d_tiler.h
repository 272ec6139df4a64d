// Host-side tiler: turns a reference-layout spectral-element mesh (ibool,
// per-element GLL arrays) into the tile-staged device layout.
//
// A tile is a set of up to `tile_elems` elements that one CTA advances per
// time step.  Its points are split into "interior" points (touched only by
// this tile's elements; stored contiguously in device numbering, owned and
// updated by the tile) and "shared" points (touched by several tiles;
// stored after all interior points and finished by a second kernel that
// adds the tiles' partial sums in tile order).  Elements inside a tile are
// greedily coloured so that no two elements of a colour share a point;
// shared-memory assembly then runs colour by colour without atomics.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace sf2d {

constexpr int NGLL = 5;
constexpr int NGLL2 = 25;
constexpr int MAX_COLOURS = 8;

struct TileInfo {
  int elem_base;   // first element slot of the tile (tile-ordered element arrays)
  int nelem;       // elements in the tile
  int n_int;       // interior local points
  int int_begin;   // device id of local point 0
  int n_sh;        // shared local points (local ids n_int .. n_int+n_sh-1)
  int sh_off;      // offset into sh_ids and the partial-sum slots
  int st_off, st_n;    // boundary (Stacey) entries of this tile
  int src_off, src_n;  // source entries of this tile
  int rec_off, rec_n;  // receivers whose element lies in this tile
  int col_end[MAX_COLOURS];  // exclusive end (element index within tile) of each colour
  int ncol;
  int lib_off;     // offset of the tile's local ibool (multiple of 8 entries = 16 bytes)
  int cpl_off, cpl_n;  // fluid-solid coupling entries of this tile (none outside a coupled run)
  int edge_off, edge_n;  // local points on the outer edge of a CPML layer, zeroed every step
  int grp_off, grp_n;    // points that receive boundary, coupling or source terms (one thread each)
};
static_assert(sizeof(TileInfo) == 28 * 4, "TileInfo layout");

struct Tiling {
  int ntiles = 0;
  int nglob = 0;
  int nelem = 0;
  int nshared = 0;       // number of shared points
  int shared_begin = 0;  // device id of the first shared point
  int max_local = 0;     // max local points over tiles
  int max_elems = 0;     // max elements over tiles
  std::vector<TileInfo> tiles;
  std::vector<int> elem_order;        // slot -> original element id
  std::vector<int> elem_tile;         // original element id -> tile
  std::vector<uint16_t> lib;          // lib_off + (slot - elem_base)*25 + q -> local point id
  std::vector<int> dev2glob;          // device id -> original global id
  std::vector<int> glob2dev;          // original global id -> device id
  std::vector<int> sh_ids;            // per tile shared local point -> device id
  std::vector<int> shp_off;           // nshared+1 CSR offsets into shp_slots
  std::vector<int> shp_slots;         // partial-sum slots (sh_off+k) per shared point, tile order
  // global point id -> (tile, local id) lookup used when attaching boundary terms
  int local_id(int tile, int glob) const;
  std::vector<std::vector<std::pair<int, int>>> tile_glob_local;  // per tile sorted (glob, local)
  // tiles of element group k are [group_tile_begin[k], group_tile_begin[k+1])
  std::vector<int> group_tile_begin;
};

// Builds the tiling.  `ibool` is nspec*25 0-based ids in [ispec][j][i]
// order; `centroid_xz` (nspec*2, may be null) orders elements along a Morton
// curve so tiles are compact; without it elements keep their input order.
// `elem_group` (nspec values in [0, ngroups), may be null) keeps elements of
// different groups in different tiles, group 0 first: the elements of a CPML
// layer get tiles (and a kernel variant) of their own.  `group_tile_elems`
// (ngroups values, may be null) sets a tile size per group.
// Returns an empty string on success, else an error message.
std::string build_tiling(int nspec, int nglob, const int *ibool, const double *centroid_xz,
                         int tile_elems, Tiling &out, const int *elem_group = nullptr, int ngroups = 1,
                         const int *group_tile_elems = nullptr);

}  // namespace sf2d
