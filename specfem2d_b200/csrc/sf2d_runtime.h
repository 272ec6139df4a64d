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

// the kernel of a CPML layer's tiles (isotropic, no attenuation, forward)
inline TileKernel pick_pml_kernel(int nt, bool lddrk) {
  switch (nt) {
    case 128: return lddrk ? k_elastic_tile<128, false, false, true, false, true> : k_elastic_tile<128, false, false, false, false, true>;
    case 512: return lddrk ? k_elastic_tile<512, false, false, true, false, true> : k_elastic_tile<512, false, false, false, false, true>;
    default: return lddrk ? k_elastic_tile<256, false, false, true, false, true> : k_elastic_tile<256, false, false, false, false, true>;
  }
}

inline TileKernel pick_tile_kernel(int nt, bool aniso, bool atten, bool lddrk, bool kern) {
  switch (nt) {
    case 128: return kern ? pick_tile_kernel<128, true>(aniso, atten, lddrk) : pick_tile_kernel<128, false>(aniso, atten, lddrk);
    case 512: return kern ? pick_tile_kernel<512, true>(aniso, atten, lddrk) : pick_tile_kernel<512, false>(aniso, atten, lddrk);
    default: return kern ? pick_tile_kernel<256, true>(aniso, atten, lddrk) : pick_tile_kernel<256, false>(aniso, atten, lddrk);
  }
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

  void launch_tile(bool record_prev, int stage) {
    if (pml_tile0 > 0) tile_fn<<<pml_tile0, nt, smem, stream>>>(P, record_prev ? 1 : 0, stage, 0);
    if (pml_tile0 < T.ntiles)
      (pml_fn ? pml_fn : tile_fn)<<<T.ntiles - pml_tile0, nt, pml_fn ? pml_smem : smem, stream>>>(
          P, record_prev ? 1 : 0, stage, pml_tile0);
  }
  void launch_shared(int stage) {
    const int nb = std::max(1, (P.nshared + sf2d::SHARED_NT - 1) / sf2d::SHARED_NT);
    const int last = stage == nstage - 1 ? 1 : 0;
    if (lddrk)
      sf2d::k_elastic_shared<true, false><<<nb, sf2d::SHARED_NT, 0, stream>>>(P, stage, last);
    else if (kern)
      sf2d::k_elastic_shared<false, true><<<nb, sf2d::SHARED_NT, 0, stream>>>(P, stage, last);
    else
      sf2d::k_elastic_shared<false, false><<<nb, sf2d::SHARED_NT, 0, stream>>>(P, stage, last);
  }
  int launch_step(bool record_prev) {
    for (int st = 0; st < nstage; ++st) {
      launch_tile(record_prev && st == 0, st);
      launch_shared(st);
    }
    return SF2D_OK;
  }
  int launch_receivers() {
    if (nrec > 0) sf2d::k_receivers<<<(nrec + 127) / 128, 128, 0, stream>>>(P);
    return SF2D_OK;
  }
  int launch_chunk(int n) {
    for (int k = 0; k < n; ++k) launch_step(k > 0);
    launch_receivers();
    SF2D_CUDA(cudaGetLastError());
    return SF2D_OK;
  }
  ~sf2d_solver() {
    if (graph) cudaGraphExecDestroy(graph);
    for (void *p : allocs) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
};


// Builds a solver; `kern` selects the adjoint variant that accumulates
// sensitivity kernels against forward displacement frames.
int sf2d_create_solver_internal(const sf2d_elastic_desc *d, bool kern, sf2d_solver **out);

// Zeroes every wavefield, memory variable, kernel sum and counter of a solver.
int sf2d_reset_solver(sf2d_solver *S);
