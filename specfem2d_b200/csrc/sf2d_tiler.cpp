// Host-side tiler (see sf2d_tiler.h).
#include "sf2d_tiler.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace sf2d {

namespace {

uint32_t spread_bits(uint32_t v) {  // 16 -> 32 bits, zeros interleaved
  v &= 0xFFFFu;
  v = (v | (v << 8)) & 0x00FF00FFu;
  v = (v | (v << 4)) & 0x0F0F0F0Fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}

}  // namespace

int Tiling::local_id(int tile, int glob) const {
  const auto &v = tile_glob_local[tile];
  auto it = std::lower_bound(v.begin(), v.end(), std::make_pair(glob, -1));
  if (it == v.end() || it->first != glob) return -1;
  return it->second;
}

std::string build_tiling(int nspec, int nglob, const int *ibool, const double *centroid_xz,
                         int tile_elems, Tiling &T, const int *elem_group, int ngroups,
                         const int *group_tile_elems) {
  if (nspec <= 0 || nglob <= 0 || !ibool) return "empty mesh";
  if (tile_elems < 1 || tile_elems > 256) return "tile_elems must be in [1, 256]";
  if (ngroups < 1 || ngroups > 8) return "ngroups must be in [1, 8]";
  if (group_tile_elems)
    for (int k = 0; k < ngroups; ++k)
      if (group_tile_elems[k] < 1 || group_tile_elems[k] > 256) return "tile_elems must be in [1, 256]";
  for (long long k = 0; k < static_cast<long long>(nspec) * NGLL2; ++k)
    if (ibool[k] < 0 || ibool[k] >= nglob) return "ibool entry out of range";
  if (elem_group)
    for (int e = 0; e < nspec; ++e)
      if (elem_group[e] < 0 || elem_group[e] >= ngroups) return "element group out of range";
  auto group = [&](int e) { return elem_group ? elem_group[e] : 0; };

  // 1. element order along a Morton curve of the centroids (uniform scale)
  std::vector<int> order(nspec);
  std::iota(order.begin(), order.end(), 0);
  if (centroid_xz) {
    double xmin = 1e300, xmax = -1e300, zmin = 1e300, zmax = -1e300;
    for (int e = 0; e < nspec; ++e) {
      xmin = std::min(xmin, centroid_xz[2 * e]);
      xmax = std::max(xmax, centroid_xz[2 * e]);
      zmin = std::min(zmin, centroid_xz[2 * e + 1]);
      zmax = std::max(zmax, centroid_xz[2 * e + 1]);
    }
    const double ext = std::max(std::max(xmax - xmin, zmax - zmin), 1e-30);
    std::vector<uint32_t> code(nspec);
    for (int e = 0; e < nspec; ++e) {
      const uint32_t qx = static_cast<uint32_t>(std::min(65535.0, (centroid_xz[2 * e] - xmin) / ext * 65535.0));
      const uint32_t qz = static_cast<uint32_t>(std::min(65535.0, (centroid_xz[2 * e + 1] - zmin) / ext * 65535.0));
      code[e] = spread_bits(qx) | (spread_bits(qz) << 1);
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return code[a] < code[b]; });
  }
  if (elem_group) std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return group(a) < group(b); });

  // 2. chunk each group into tiles, elements ascending inside each tile
  T = Tiling();
  std::vector<std::vector<int>> tel;
  T.group_tile_begin.assign(ngroups + 1, 0);
  for (int b = 0; b < nspec;) {
    int e = b + 1;
    const int te = group_tile_elems ? group_tile_elems[group(order[b])] : tile_elems;
    while (e < nspec && e - b < te && group(order[e]) == group(order[b])) ++e;
    tel.emplace_back(order.begin() + b, order.begin() + e);
    std::sort(tel.back().begin(), tel.back().end());
    T.group_tile_begin[group(order[b]) + 1] = static_cast<int>(tel.size());
    b = e;
  }
  for (int k = 1; k <= ngroups; ++k) T.group_tile_begin[k] = std::max(T.group_tile_begin[k], T.group_tile_begin[k - 1]);
  const int ntiles = static_cast<int>(tel.size());
  T.ntiles = ntiles;
  T.nglob = nglob;
  T.nelem = nspec;
  T.tiles.assign(ntiles, TileInfo{});
  T.elem_tile.assign(nspec, -1);
  for (int t = 0; t < ntiles; ++t)
    for (int x : tel[t]) T.elem_tile[x] = t;

  // 3. how many tiles touch each point
  std::vector<int> last(nglob, -1), touch(nglob, 0);
  for (int t = 0; t < ntiles; ++t)
    for (int e : tel[t])
      for (int q = 0; q < NGLL2; ++q) {
        const int g = ibool[static_cast<size_t>(e) * NGLL2 + q];
        if (last[g] != t) {
          last[g] = t;
          ++touch[g];
        }
      }
  for (int g = 0; g < nglob; ++g)
    if (touch[g] == 0) return "a global point is not referenced by any element";

  // 4./5. device numbering and local ids
  T.glob2dev.assign(nglob, -1);
  T.dev2glob.assign(nglob, -1);
  T.tile_glob_local.assign(ntiles, {});
  int next_dev = 0;
  std::vector<int> local(nglob, -1);
  std::vector<std::vector<int>> tile_shared_glob(ntiles);
  for (int t = 0; t < ntiles; ++t) {
    TileInfo &ti = T.tiles[t];
    ti.int_begin = next_dev;
    std::vector<int> ints, shs;
    for (int e : tel[t])
      for (int q = 0; q < NGLL2; ++q) {
        const int g = ibool[static_cast<size_t>(e) * NGLL2 + q];
        if (local[g] == -2 - t) continue;  // already seen in this tile
        local[g] = -2 - t;
        (touch[g] == 1 ? ints : shs).push_back(g);
      }
    ti.n_int = static_cast<int>(ints.size());
    ti.n_sh = static_cast<int>(shs.size());
    auto &gl = T.tile_glob_local[t];
    gl.reserve(ints.size() + shs.size());
    for (size_t k = 0; k < ints.size(); ++k) {
      T.glob2dev[ints[k]] = next_dev;
      T.dev2glob[next_dev] = ints[k];
      ++next_dev;
      gl.emplace_back(ints[k], static_cast<int>(k));
    }
    for (size_t k = 0; k < shs.size(); ++k) gl.emplace_back(shs[k], ti.n_int + static_cast<int>(k));
    std::sort(gl.begin(), gl.end());
    tile_shared_glob[t] = std::move(shs);
    T.max_local = std::max(T.max_local, ti.n_int + ti.n_sh);
    T.max_elems = std::max(T.max_elems, static_cast<int>(tel[t].size()));
  }
  if (T.max_local > 65535) return "too many local points in a tile";
  T.shared_begin = next_dev;
  for (int g = 0; g < nglob; ++g)
    if (touch[g] > 1) {
      T.glob2dev[g] = next_dev;
      T.dev2glob[next_dev] = g;
      ++next_dev;
    }
  T.nshared = next_dev - T.shared_begin;

  // shared local -> device id, partial-sum slots
  int sh_total = 0;
  for (int t = 0; t < ntiles; ++t) {
    T.tiles[t].sh_off = sh_total;
    for (int g : tile_shared_glob[t]) T.sh_ids.push_back(T.glob2dev[g]);
    sh_total += T.tiles[t].n_sh;
  }
  std::vector<int> cnt(T.nshared + 1, 0);
  for (int t = 0; t < ntiles; ++t)
    for (int g : tile_shared_glob[t]) ++cnt[T.glob2dev[g] - T.shared_begin + 1];
  T.shp_off.assign(T.nshared + 1, 0);
  for (int s = 0; s < T.nshared; ++s) T.shp_off[s + 1] = T.shp_off[s] + cnt[s + 1];
  T.shp_slots.assign(T.shp_off[T.nshared], -1);
  std::vector<int> fill(T.shp_off.begin(), T.shp_off.end() - 1);
  for (int t = 0; t < ntiles; ++t)  // tile order -> slots sorted by tile
    for (int k = 0; k < T.tiles[t].n_sh; ++k) {
      const int s = T.glob2dev[tile_shared_glob[t][k]] - T.shared_begin;
      T.shp_slots[fill[s]++] = T.tiles[t].sh_off + k;
    }

  // 6. colouring inside each tile, 7. element slots and local ibool
  T.elem_order.reserve(nspec);
  T.lib.reserve(static_cast<size_t>(nspec) * NGLL2);
  std::vector<uint32_t> used;
  for (int t = 0; t < ntiles; ++t) {
    TileInfo &ti = T.tiles[t];
    const int nl = ti.n_int + ti.n_sh;
    used.assign(nl, 0u);
    std::vector<int> colour(tel[t].size(), 0);
    std::vector<int> lid(tel[t].size() * NGLL2);
    for (size_t k = 0; k < tel[t].size(); ++k) {
      const int e = tel[t][k];
      uint32_t m = 0;
      for (int q = 0; q < NGLL2; ++q) {
        const int l = T.local_id(t, ibool[static_cast<size_t>(e) * NGLL2 + q]);
        lid[k * NGLL2 + q] = l;
        m |= used[l];
      }
      int c = 0;
      while (c < MAX_COLOURS && (m >> c) & 1u) ++c;
      if (c == MAX_COLOURS) return "element colouring needs more than 8 colours in a tile";
      colour[k] = c;
      for (int q = 0; q < NGLL2; ++q) used[lid[k * NGLL2 + q]] |= (1u << c);
    }
    std::vector<int> idx(tel[t].size());
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return colour[a] < colour[b]; });
    ti.elem_base = static_cast<int>(T.elem_order.size());
    while (T.lib.size() % 8) T.lib.push_back(0);
    ti.lib_off = static_cast<int>(T.lib.size());
    ti.nelem = static_cast<int>(tel[t].size());
    ti.ncol = 0;
    for (int c = 0; c < MAX_COLOURS; ++c) ti.col_end[c] = 0;
    for (size_t s = 0; s < idx.size(); ++s) {
      const int k = idx[s];
      T.elem_order.push_back(tel[t][k]);
      for (int q = 0; q < NGLL2; ++q) T.lib.push_back(static_cast<uint16_t>(lid[k * NGLL2 + q]));
      ti.col_end[colour[k]] = static_cast<int>(s) + 1;
      ti.ncol = std::max(ti.ncol, colour[k] + 1);
    }
    for (int c = 1; c < ti.ncol; ++c) ti.col_end[c] = std::max(ti.col_end[c], ti.col_end[c - 1]);
  }
  // the kernel copies each tile's local ibool in 16-byte chunks
  while (T.lib.size() % 8) T.lib.push_back(0);
  return "";
}

}  // namespace sf2d

// Host-only diagnostic (declared in include/sf2d_b200.h): builds a tiling and
// checks its invariants without touching the GPU.
extern "C" int sf2d_tiling_stats(int nspec, int nglob, const int *ibool, const double *centroid_xz,
                                 int tile_elems, long long *out8) {
  using namespace sf2d;
  if (!out8) return -1;
  Tiling T;
  const std::string err = build_tiling(nspec, nglob, ibool, centroid_xz, tile_elems, T);
  if (!err.empty()) return -1;
  // every global point has exactly one device id
  std::vector<int> seen(nglob, 0);
  for (int d = 0; d < nglob; ++d) {
    const int g = T.dev2glob[d];
    if (g < 0 || g >= nglob || T.glob2dev[g] != d) return -2;
    ++seen[g];
  }
  for (int g = 0; g < nglob; ++g)
    if (seen[g] != 1) return -2;
  long long max_col = 0, nint = 0;
  for (int t = 0; t < T.ntiles; ++t) {
    const TileInfo &ti = T.tiles[t];
    nint += ti.n_int;
    max_col = std::max<long long>(max_col, ti.ncol);
    // local ibool maps back to the original ibool
    for (int s = ti.elem_base; s < ti.elem_base + ti.nelem; ++s) {
      const int e = T.elem_order[s];
      for (int q = 0; q < NGLL2; ++q) {
        const int l = T.lib[static_cast<size_t>(ti.lib_off) + static_cast<size_t>(s - ti.elem_base) * NGLL2 + q];
        const int g = ibool[static_cast<size_t>(e) * NGLL2 + q];
        const int dev = l < ti.n_int ? ti.int_begin + l : T.sh_ids[ti.sh_off + l - ti.n_int];
        if (T.dev2glob[dev] != g) return -3;
      }
    }
    // no two elements of one colour share a local point
    int cb = 0;
    for (int c = 0; c < ti.ncol; ++c) {
      std::vector<char> mark(ti.n_int + ti.n_sh, 0);
      for (int s = cb; s < ti.col_end[c]; ++s)
        for (int q = 0; q < NGLL2; ++q) {
          const int l = T.lib[static_cast<size_t>(ti.lib_off) + static_cast<size_t>(s) * NGLL2 + q];
          if (mark[l]) return -4;
          mark[l] = 1;
        }
      cb = ti.col_end[c];
    }
    if (cb != ti.nelem) return -5;
  }
  // shared-point slots: each slot used once, slots of a point in tile order
  std::vector<int> used(T.sh_ids.size(), 0);
  for (int s = 0; s < T.nshared; ++s) {
    if (T.shp_off[s + 1] - T.shp_off[s] < 2) return -6;
    for (int k = T.shp_off[s]; k < T.shp_off[s + 1]; ++k) {
      const int slot = T.shp_slots[k];
      if (T.sh_ids[slot] != T.shared_begin + s) return -6;
      if (used[slot]++) return -6;
      if (k > T.shp_off[s] && slot <= T.shp_slots[k - 1]) return -6;
    }
  }
  out8[0] = T.ntiles;
  out8[1] = T.nshared;
  out8[2] = T.max_local;
  out8[3] = T.max_elems;
  out8[4] = max_col;
  out8[5] = nint;
  out8[6] = static_cast<long long>(T.sh_ids.size());
  out8[7] = 0;
  return 0;
}
