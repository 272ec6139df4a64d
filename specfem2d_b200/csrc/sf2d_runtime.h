// Host-side solver object shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "sf2d_b200.h"
#include "sf2d_kernels.cuh"
#include "sf2d_tiler.h"

namespace sf2d {
// Sets the calling thread's last error message and returns `code`.
int fail(int code, const std::string &msg);
const char *last_error();
}  // namespace sf2d

using sf2d::fail;

#define SF2D_CUDA(call)                                                                       \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(e_ == cudaErrorMemoryAllocation ? SF2D_ERR_OOM : SF2D_ERR_CUDA,             \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                        \
  } while (0)

namespace sf2d {

using TileKernel = void (*)(Params, int, int, int);

template <int NT, bool KERN>
TileKernel pick_tile_kernel(bool aniso, bool atten, bool lddrk) {
  if (aniso) {
    if (atten) return lddrk ? k_elastic_tile<NT, true, true, true, KERN> : k_elastic_tile<NT, true, true, false, KERN>;
    return lddrk ? k_elastic_tile<NT, true, false, true, KERN> : k_elastic_tile<NT, true, false, false, KERN>;
  }
  if (atten) return lddrk ? k_elastic_tile<NT, false, true, true, KERN> : k_elastic_tile<NT, false, true, false, KERN>;
  return lddrk ? k_elastic_tile<NT, false, false, true, KERN> : k_elastic_tile<NT, false, false, false, KERN>;
}

// the kernel of a CPML layer's tiles (isotropic, forward); visco: some layer
// elements attenuate (Newmark only)
template <int NT>
inline TileKernel pick_pml_kernel(bool lddrk, bool visco) {
  if (visco) return k_elastic_tile<NT, false, true, false, false, true>;
  return lddrk ? k_elastic_tile<NT, false, false, true, false, true> : k_elastic_tile<NT, false, false, false, false, true>;
}
inline TileKernel pick_pml_kernel(int nt, bool lddrk, bool visco = false) {
  switch (nt) {
    case 128: return pick_pml_kernel<128>(lddrk, visco);
    case 250: return pick_pml_kernel<250>(lddrk, visco);
    case 512: return pick_pml_kernel<512>(lddrk, visco);
    default: return pick_pml_kernel<256>(lddrk, visco);
  }
}

inline TileKernel pick_tile_kernel(int nt, bool aniso, bool atten, bool lddrk, bool kern) {
  switch (nt) {
    case 128: return kern ? pick_tile_kernel<128, true>(aniso, atten, lddrk) : pick_tile_kernel<128, false>(aniso, atten, lddrk);
    case 250: return kern ? pick_tile_kernel<250, true>(aniso, atten, lddrk) : pick_tile_kernel<250, false>(aniso, atten, lddrk);
    case 512: return kern ? pick_tile_kernel<512, true>(aniso, atten, lddrk) : pick_tile_kernel<512, false>(aniso, atten, lddrk);
    default: return kern ? pick_tile_kernel<256, true>(aniso, atten, lddrk) : pick_tile_kernel<256, false>(aniso, atten, lddrk);
  }
}

// Boundary terms of each tile grouped by receiving point, so that one thread
// per point applies them (in parallel over points, in the reference's order at
// each point: Stacey, coupling, sources).  groups: one int4 per point (local
// point, first index into idx, Stacey count | coupling count << 8, source
// count); idx: the point's entries of each type in their list order.  The
// *_local vectors give each entry's tile-local point; tiles' st/cpl/src
// ranges index them.  Sets grp_off / grp_n of every tile.
inline std::string build_boundary_groups(std::vector<TileInfo> &tiles, const std::vector<int> &st_local,
                                         const std::vector<int> &cpl_local, const std::vector<int> &src_local,
                                         std::vector<int4> &groups, std::vector<int> &idx) {
  groups.clear();
  idx.clear();
  std::vector<std::vector<int>> st, cp, sr;
  std::vector<int> pts;
  for (TileInfo &t : tiles) {
    t.grp_off = static_cast<int>(groups.size());
    pts.clear();
    auto add = [&](std::vector<std::vector<int>> &lists, int l, int k) {
      if (static_cast<int>(st.size()) <= l) {
        st.resize(l + 1);
        cp.resize(l + 1);
        sr.resize(l + 1);
      }
      if (st[l].empty() && cp[l].empty() && sr[l].empty()) pts.push_back(l);
      lists[l].push_back(k);
    };
    for (int k = t.st_off; k < t.st_off + t.st_n; ++k) add(st, st_local[k], k);
    for (int k = t.cpl_off; k < t.cpl_off + t.cpl_n; ++k) add(cp, cpl_local[k], k);
    for (int k = t.src_off; k < t.src_off + t.src_n; ++k) add(sr, src_local[k], k);
    std::sort(pts.begin(), pts.end());
    for (int l : pts) {
      if (st[l].size() > 255 || cp[l].size() > 255) return "more than 255 boundary entries at one point";
      groups.push_back(make_int4(l, static_cast<int>(idx.size()),
                                 static_cast<int>(st[l].size() | (cp[l].size() << 8)), static_cast<int>(sr[l].size())));
      for (int k : st[l]) idx.push_back(k);
      for (int k : cp[l]) idx.push_back(k);
      for (int k : sr[l]) idx.push_back(k);
      st[l].clear();
      cp[l].clear();
      sr[l].clear();
    }
    t.grp_n = static_cast<int>(groups.size()) - t.grp_off;
  }
  return "";
}

}  // namespace sf2d

struct sf2d_solver {
  sf2d::Params P{};
  sf2d::Tiling T;
  std::vector<void *> allocs;
  int *d_dev2glob = nullptr;
  float2 *d_stage = nullptr;
  unsigned int *d_norm = nullptr;
  cudaStream_t stream = nullptr;
  size_t smem = 0;
  size_t dev_bytes = 0;
  int nglob = 0, nrec = 0, nstep_total = 0;
  int steps_done = 0;
  int chunk = 32;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  int nt = 256;  // threads per CTA of the tile kernel
  int pml_nt = 256, pml_max_q = 0, pml_max_local = 0;  // the CPML tiles' kernel
  int late_tile0 = 0;  // tiles [late_tile0, pml_tile0) touch points another domain uses
  int nmembers = 0;    // members of a packed batch (sf2d_set_members), 0 = none
  int priority = 0;    // of the solver's streams (0: the default, lowest)

  template <typename T_>
  int alloc(T_ **p, size_t count) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T_);
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), bytes);
    if (e != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? SF2D_ERR_OOM : SF2D_ERR_CUDA,
                  std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(*p);
    dev_bytes += bytes;
    return SF2D_OK;
  }
  template <typename T_>
  int upload(T_ **p, const T_ *host, size_t count) {
    int rc = alloc(p, count);
    if (rc) return rc;
    if (count) SF2D_CUDA(cudaMemcpy(*p, host, count * sizeof(T_), cudaMemcpyHostToDevice));
    return SF2D_OK;
  }
  using TileFn = void (*)(sf2d::Params, int, int, int);
  TileFn tile_fn = nullptr;
  TileFn pml_fn = nullptr;   // tiles [pml_tile0, ntiles) hold the CPML layer's elements
  int pml_tile0 = 0;
  size_t pml_smem = 0;
  size_t npml_q = 0;         // GLL points of the layer's elements
  bool lddrk = false;
  bool kern = false;
  bool atten = false;
  int nstage = 1;
  int nspec = 0;
  int *ctr = nullptr;  // device ints: step, status, step shadow, frame base, kernel frame base
  float *d_stf = nullptr;
  size_t nq = 0;
  // tile-local point of every Stacey and source entry, kept to regroup the
  // boundary terms when coupling entries are added
  std::vector<int> h_st_local, h_src_local;

  // With both tile groups present, the CPML tiles run on a side stream beside
  // the other tiles (the two write disjoint points and slots), joined before
  // the shared-point kernel: their longer latency hides behind the bulk.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int make_side_stream() {
    if (side || !(pml_tile0 > 0 && pml_tile0 < T.ntiles)) return SF2D_OK;
    SF2D_CUDA(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, priority));
    SF2D_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    SF2D_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    return SF2D_OK;
  }
  // parameters of the CPML tiles' kernel: its shared-memory layout is sized
  // by the layer's largest tile
  sf2d::Params pml_params() const {
    sf2d::Params Q = P;
    Q.max_q = pml_max_q;
    Q.max_local = pml_max_local;
    return Q;
  }
  // Tiles [first, ntiles): the plain ones on the solver stream, the CPML ones
  // beside them on the side stream when there is one.  first = late_tile0
  // leaves the early tiles to launch_early.
  // A step kernel on the solver stream with programmatic dependent launch: its
  // CTAs may be scheduled while the previous step kernel drains (each kernel
  // waits for its predecessor's completion before reading, wait_previous_kernel).
  template <typename F, typename... A>
  void launch_pdl(F fn, int grid, int block, size_t smem_bytes, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(static_cast<unsigned>(block));
    cfg.dynamicSmemBytes = smem_bytes;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, fn, args...);
    if (e != cudaSuccess && launch_error == cudaSuccess) launch_error = e;
  }
  cudaError_t launch_error = cudaSuccess;
  void launch_tile(bool record_prev, int stage, int first = 0) {
    const int rp = record_prev ? 1 : 0;
    const int nplain = pml_tile0 - first;
    if (side) {
      cudaEventRecord(ev_fork, stream);
      cudaStreamWaitEvent(side, ev_fork, 0);
      pml_fn<<<T.ntiles - pml_tile0, pml_nt, pml_smem, side>>>(pml_params(), rp, stage, pml_tile0);
      cudaEventRecord(ev_join, side);
      if (nplain > 0) tile_fn<<<nplain, nt, smem, stream>>>(P, rp, stage, first);
      cudaStreamWaitEvent(stream, ev_join, 0);
      return;
    }
    if (nplain > 0) launch_pdl(tile_fn, nplain, nt, smem, P, rp, stage, first);
    if (pml_tile0 < T.ntiles) {
      if (pml_fn)
        pml_fn<<<T.ntiles - pml_tile0, pml_nt, pml_smem, stream>>>(pml_params(), rp, stage, pml_tile0);
      else
        tile_fn<<<T.ntiles - pml_tile0, nt, smem, stream>>>(P, rp, stage, pml_tile0);
    }
  }
  // the early tiles [0, late_tile0) on stream s
  void launch_early(cudaStream_t s, bool record_prev, int stage) {
    if (late_tile0 > 0) tile_fn<<<late_tile0, nt, smem, s>>>(P, record_prev ? 1 : 0, stage, 0);
  }
  // tile-kernel launches of one stage of launch_tile(first)
  int tile_launches(int first) const {
    return (pml_tile0 - first > 0) + (pml_tile0 < T.ntiles);
  }
  void launch_shared(int stage) {
    const int nb = std::max(1, (P.nshared + sf2d::SHARED_NT - 1) / sf2d::SHARED_NT);
    const int last = stage == nstage - 1 ? 1 : 0;
    if (lddrk)
      launch_pdl(sf2d::k_elastic_shared<true, false>, nb, sf2d::SHARED_NT, 0, P, stage, last);
    else if (kern)
      launch_pdl(sf2d::k_elastic_shared<false, true>, nb, sf2d::SHARED_NT, 0, P, stage, last);
    else
      launch_pdl(sf2d::k_elastic_shared<false, false>, nb, sf2d::SHARED_NT, 0, P, stage, last);
  }
  int launch_step(bool record_prev) {
    for (int st = 0; st < nstage; ++st) {
      launch_tile(record_prev && st == 0, st);
      launch_shared(st);
    }
    return SF2D_OK;
  }
  int launch_receivers() {
    if (nrec > 0) launch_pdl(sf2d::k_receivers, (nrec + 127) / 128, 128, 0, P);
    return SF2D_OK;
  }
  int launch_chunk(int n) {
    for (int k = 0; k < n; ++k) launch_step(k > 0);
    launch_receivers();
    if (launch_error != cudaSuccess) {
      const cudaError_t e = launch_error;
      launch_error = cudaSuccess;
      return sf2d::fail(SF2D_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    }
    SF2D_CUDA(cudaGetLastError());
    return SF2D_OK;
  }
  ~sf2d_solver() {
    if (graph) cudaGraphExecDestroy(graph);
    for (void *p : allocs) cudaFree(p);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
  }
};


// Builds a solver; `kern` selects the adjoint variant that accumulates
// sensitivity kernels against forward displacement frames.
// late_elem (may be NULL): per element 1 when another domain reads or writes
// one of its points (fluid-solid coupling); those elements get tiles of their
// own, launched after the other domain's step, and the rest may run beside it
int sf2d_create_solver_internal(const sf2d_elastic_desc *d, bool kern, sf2d_solver **out, const uint8_t *late_elem);

// Zeroes every wavefield, memory variable, kernel sum and counter of a solver.
int sf2d_reset_solver(sf2d_solver *S);
