// Host runtime and C ABI of the coupled fluid-solid time step: a fluid
// (acoustic) tile solver and the solid (elastic) tile solver advanced
// together, fluid first, on one stream (iterate_time.F90:183-196).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "sf2d_acoustic.cuh"
#include "sf2d_b200.h"
#include "sf2d_coupled.h"
#include "sf2d_kernels.cuh"
#include "sf2d_runtime.h"
#include "sf2d_tiler.h"

namespace {

using sf2d::AcParams;
using sf2d::NGLL2;
using sf2d::TileInfo;
using sf2d::Tiling;

__global__ void k_gather_f(const float *src, const int *dev2glob, float *dst, int n) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) dst[d] = src[dev2glob[d]];
}
__global__ void k_scatter_f(const float *src, const int *dev2glob, float *dst, int n) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) dst[dev2glob[d]] = src[d];
}
// whole-mesh <-> solid device order (map: device point -> whole-mesh point)
__global__ void k_gather_f2(const float2 *src, const int *map, float2 *dst, int n) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) dst[d] = src[map[d]];
}
__global__ void k_scatter_f2(const float2 *src, const int *map, float2 *dst, int n) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) dst[map[d]] = src[d];
}

using AcTileFn = void (*)(AcParams, int, int, int);

template <bool PML>
AcTileFn pick_ac_tile(int nt, bool lddrk) {
  switch (nt) {
    case 128: return lddrk ? sf2d::k_acoustic_tile<128, true, PML> : sf2d::k_acoustic_tile<128, false, PML>;
    case 250: return lddrk ? sf2d::k_acoustic_tile<250, true, PML> : sf2d::k_acoustic_tile<250, false, PML>;
    case 512: return lddrk ? sf2d::k_acoustic_tile<512, true, PML> : sf2d::k_acoustic_tile<512, false, PML>;
    default: return lddrk ? sf2d::k_acoustic_tile<256, true, PML> : sf2d::k_acoustic_tile<256, false, PML>;
  }
}

// Damping data of one element GLL point p of a descriptor's CPML arrays.
struct PmlAt {
  double kx, kz, ax, az, bx, bz;
};
template <typename Desc>
PmlAt pml_at(const Desc *d, size_t p) {
  PmlAt c;
  c.kx = d->pml_K_x[p];
  c.kz = d->pml_K_z[p];
  c.ax = d->pml_alpha_x[p];
  c.az = d->pml_alpha_z[p];
  c.bx = c.ax + d->pml_d_x[p] / c.kx;
  c.bz = c.az + d->pml_d_z[p] / c.kz;
  return c;
}

}  // namespace

struct sf2d_coupled {
  sf2d_solver *el = nullptr;  // solid sub-solver (owns the stream); none for a fluid-only mesh
  cudaStream_t own_stream = nullptr;  // the stream of a fluid-only run
  cudaStream_t stream() const { return el ? el->stream : own_stream; }
  AcParams A{};
  Tiling T;
  std::vector<void *> allocs;
  int *d_dev2glob = nullptr;
  float *d_stage = nullptr;
  // whole-mesh numbering (sf2d_coupled_set_global_numbering): device point ->
  // whole-mesh point of each domain, and a whole-mesh staging buffer
  int nglob_total = 0;
  int *d_gmap_solid = nullptr, *d_gmap_fluid = nullptr;
  float2 *d_gstage = nullptr;
  int *ctr = nullptr;
  double *seis = nullptr;
  sf2d::CplPml cpl_fluid{}, cpl_solid{};  // coupling entries next to a CPML layer
  AcTileFn tile_fn = nullptr;
  AcTileFn pml_fn = nullptr;  // tiles [pml_tile0, ntiles) hold the fluid CPML layer
  int pml_tile0 = 0;
  size_t pml_smem = 0;
  size_t smem = 0;
  int nt = 256, nstage = 1, nglob = 0, nrec_total = 0, nstep = 0, steps_done = 0;
  size_t npml_q = 0;  // GLL points of the fluid CPML elements
  bool lddrk = false;
  bool adjoint = false;  // an adjoint run: the solid step first (sf2d_coupling_desc.adjoint)
  int chunk = 32;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;

  template <typename T_>
  int alloc(T_ **p, size_t count) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T_);
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), bytes);
    if (e != cudaSuccess)
      return sf2d::fail(e == cudaErrorMemoryAllocation ? SF2D_ERR_OOM : SF2D_ERR_CUDA,
                        std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(*p);
    return SF2D_OK;
  }
  template <typename T_>
  int upload(T_ **p, const T_ *host, size_t count) {
    int rc = alloc(p, count);
    if (rc) return rc;
    if (count) SF2D_CUDA(cudaMemcpy(*p, host, count * sizeof(T_), cudaMemcpyHostToDevice));
    return SF2D_OK;
  }
  // device arrays of one side's CPML coupling entries; `per` memory variables
  // and outputs per entry
  int upload_cpl(sf2d::CplPml &c, const std::vector<int> &pt, const std::vector<double> &coef, int per) {
    int rc = 0;
    c.n = static_cast<int>(pt.size());
    if ((rc = upload_const(&c.point, pt)) || (rc = upload_const(&c.coef, coef))) return rc;
    const size_t n = std::max<size_t>(1, pt.size() * per);
    if ((rc = alloc(&c.rm, n)) || (rc = alloc(&c.out, n))) return rc;
    SF2D_CUDA(cudaMemset(c.rm, 0, sizeof(float) * n));
    SF2D_CUDA(cudaMemset(c.out, 0, sizeof(float) * n));
    if (lddrk) {
      if ((rc = alloc(&c.rm_l, n))) return rc;
      SF2D_CUDA(cudaMemset(c.rm_l, 0, sizeof(float) * n));
    }
    return SF2D_OK;
  }
  template <typename T_>
  int upload_const(const T_ **p, const std::vector<T_> &v) {
    T_ *q = nullptr;
    int rc = upload(&q, v.data(), v.size());
    *p = q;
    return rc;
  }

  // the fluid's CPML tiles beside the others, as the solid's (sf2d_solver::launch_tile)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  void launch_ac_tile(bool record_prev, int stage) {
    const int rp = record_prev ? 1 : 0;
    cudaStream_t s = stream();
    if (side) {
      cudaEventRecord(ev_fork, s);
      cudaStreamWaitEvent(side, ev_fork, 0);
      pml_fn<<<T.ntiles - pml_tile0, nt, pml_smem, side>>>(A, rp, stage, pml_tile0);
      cudaEventRecord(ev_join, side);
      tile_fn<<<pml_tile0, nt, smem, s>>>(A, rp, stage, 0);
      cudaStreamWaitEvent(s, ev_join, 0);
      return;
    }
    if (pml_tile0 > 0) tile_fn<<<pml_tile0, nt, smem, s>>>(A, rp, stage, 0);
    if (pml_tile0 < T.ntiles)
      (pml_fn ? pml_fn : tile_fn)<<<T.ntiles - pml_tile0, nt, pml_fn ? pml_smem : smem, s>>>(A, rp, stage, pml_tile0);
  }
  void launch_ac_shared(int stage) {
    const int nb = std::max(1, (A.nshared + sf2d::SHARED_NT - 1) / sf2d::SHARED_NT);
    const int last = stage == nstage - 1 ? 1 : 0;
    if (lddrk)
      sf2d::k_acoustic_shared<true><<<nb, sf2d::SHARED_NT, 0, stream()>>>(A, stage, last);
    else
      sf2d::k_acoustic_shared<false><<<nb, sf2d::SHARED_NT, 0, stream()>>>(A, stage, last);
  }
  void launch_cpl_fluid(int stage) {
    if (cpl_fluid.n == 0) return;
    const int nb = (cpl_fluid.n + 127) / 128;
    const sf2d::Params &P = el->P;
    if (lddrk)
      sf2d::k_cpl_pml_fluid<true><<<nb, 128, 0, el->stream>>>(cpl_fluid, P.u, P.v, P.a, P.dt, P.dt2o2, A.h_old,
                                                              A.alpha[stage], A.beta[stage]);
    else
      sf2d::k_cpl_pml_fluid<false><<<nb, 128, 0, el->stream>>>(cpl_fluid, P.u, P.v, P.a, P.dt, P.dt2o2, A.h_old,
                                                               0.f, 0.f);
  }
  void launch_cpl_solid(int stage) {
    if (cpl_solid.n == 0) return;
    const int nb = (cpl_solid.n + 127) / 128;
    if (lddrk)
      sf2d::k_cpl_pml_solid<true><<<nb, 128, 0, stream()>>>(cpl_solid, A.p, A.pd, A.pdd, A.pold, A.dt,
                                                              A.alpha[stage], A.beta[stage]);
    else
      sf2d::k_cpl_pml_solid<false><<<nb, 128, 0, stream()>>>(cpl_solid, A.p, A.pd, A.pdd, A.pold, A.dt, 0.f, 0.f);
  }
  // fluid receivers of the step just finished; on the side stream when there is
  // one (they only read fluid fields, which the solid kernels do not touch),
  // joined before the next fluid tile kernel
  cudaEvent_t ev_rec = nullptr, ev_rec_done = nullptr;
  // the solid's early tiles (no coupling point) beside the fluid step
  cudaStream_t early = nullptr;
  cudaEvent_t ev_early_fork = nullptr, ev_early_join = nullptr;
  bool rec_pending = false;
  void launch_ac_receivers() {
    if (A.nrec <= 0) return;
    const int nb = (A.nrec + 127) / 128;
    if (side) {
      cudaEventRecord(ev_rec, stream());
      cudaStreamWaitEvent(side, ev_rec, 0);
      sf2d::k_acoustic_receivers<<<nb, 128, 0, side>>>(A);
      cudaEventRecord(ev_rec_done, side);
      rec_pending = true;
    } else {
      sf2d::k_acoustic_receivers<<<nb, 128, 0, stream()>>>(A);
    }
  }
  void join_ac_receivers() {
    if (rec_pending) cudaStreamWaitEvent(stream(), ev_rec_done, 0);
    rec_pending = false;
  }
  // after a finished fluid step: its chi frame (segment recomputation) and the
  // fluid kernel sums (adjoint sweep), when the run keeps them
  void launch_fluid_post() {
    if (A.pframes) sf2d::k_fluid_frame<<<std::min(1184, (nglob + 255) / 256), 256, 0, stream()>>>(A);
    if (A.kl_ac) sf2d::k_fluid_kernels<<<(A.nslot_q + 127) / 128, 128, 0, stream()>>>(A);
  }
  void launch_step(bool record_prev) {
    if (adjoint) {
      // kernel runs switch the order: the whole solid step, then the fluid step
      // (iterate_time.F90:298-327); Newmark, no CPML, no side streams
      if (el) {
        el->launch_tile(record_prev, 0, 0);
        el->launch_shared(0);
      }
      launch_ac_tile(record_prev, 0);
      launch_ac_shared(0);
      launch_ac_receivers();
      launch_fluid_post();
      return;
    }
    for (int st = 0; st < nstage; ++st) {
      const bool split = el && early && el->late_tile0 > 0;
      if (split) {
        cudaEventRecord(ev_early_fork, stream());
        cudaStreamWaitEvent(early, ev_early_fork, 0);
        el->launch_early(early, record_prev && st == 0, st);
        cudaEventRecord(ev_early_join, early);
      }
      launch_cpl_fluid(st);
      join_ac_receivers();
      launch_ac_tile(record_prev && st == 0, st);
      launch_ac_shared(st);
      if (st == nstage - 1) {
        launch_ac_receivers();
        launch_fluid_post();
      }
      launch_cpl_solid(st);
      if (el) {
        el->launch_tile(record_prev && st == 0, st, split ? el->late_tile0 : 0);
        if (split) cudaStreamWaitEvent(stream(), ev_early_join, 0);
        el->launch_shared(st);
      }
    }
  }
  int launch_chunk(int n) {
    for (int k = 0; k < n; ++k) launch_step(k > 0);
    join_ac_receivers();
    if (el) el->launch_receivers();
    SF2D_CUDA(cudaGetLastError());
    return SF2D_OK;
  }
  ~sf2d_coupled() {
    if (graph) cudaGraphExecDestroy(graph);
    if (el) sf2d_destroy(el);
    for (void *p : allocs) cudaFree(p);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_rec) cudaEventDestroy(ev_rec);
    if (ev_rec_done) cudaEventDestroy(ev_rec_done);
    if (ev_early_fork) cudaEventDestroy(ev_early_fork);
    if (ev_early_join) cudaEventDestroy(ev_early_join);
    if (early) cudaStreamDestroy(early);
    if (side) cudaStreamDestroy(side);
    if (own_stream) cudaStreamDestroy(own_stream);
  }
};

extern "C" int sf2d_coupled_create(const sf2d_elastic_desc *eld, const sf2d_acoustic_desc *ad,
                                   const sf2d_coupling_desc *cp, sf2d_coupled **out) {
  using namespace sf2d;
  if (!eld || !ad || !cp || !out) return fail(SF2D_ERR_INVALID, "null argument");
  *out = nullptr;
  if (ad->nspec <= 0 || ad->nglob <= 0 || !ad->ibool || !ad->xix || !ad->xiz || !ad->gammax || !ad->gammaz ||
      !ad->jacobian || !ad->rhostore || !ad->kappastore || !ad->rmass_inverse)
    return fail(SF2D_ERR_INVALID, "missing fluid mesh arrays");
  if (ad->nfree < 0 || ad->nstacey < 0 || ad->nsrc < 0 || ad->nrec < 0 || cp->ncpl_ac < 0 || cp->ncpl_el < 0)
    return fail(SF2D_ERR_INVALID, "negative count");
  if (cp->nrec_total != eld->nrec + ad->nrec) return fail(SF2D_ERR_INVALID, "receiver counts do not add up");
  if (cp->seismotype < 1 || cp->seismotype > 6 || cp->seismotype == 5)
    return fail(SF2D_ERR_INVALID, "seismotype must be 1 to 4 or 6");
  if (cp->seismotype == 4 && eld->nrec > 0)
    return fail(SF2D_ERR_INVALID, "pressure receivers must lie in fluid elements");
  for (int k = 0; k < ad->nrec; ++k)
    if (!ad->rec_global || ad->rec_global[k] < 0 || ad->rec_global[k] >= cp->nrec_total)
      return fail(SF2D_ERR_INVALID, "fluid receiver index out of range");
  for (int k = 0; k < eld->nrec; ++k)
    if (!cp->el_rec_global || cp->el_rec_global[k] < 0 || cp->el_rec_global[k] >= cp->nrec_total)
      return fail(SF2D_ERR_INVALID, "solid receiver index out of range");
  for (long long k = 0; k < static_cast<long long>(ad->nspec) * NGLL2; ++k)
    if (ad->ibool[k] < 0 || ad->ibool[k] >= ad->nglob) return fail(SF2D_ERR_INVALID, "fluid ibool out of range");
  for (int k = 0; k < cp->ncpl_ac; ++k)
    if (cp->cpl_ac_point[k] < 0 || cp->cpl_ac_point[k] >= ad->nglob || cp->cpl_ac_el_point[k] < 0 ||
        cp->cpl_ac_el_point[k] >= eld->nglob)
      return fail(SF2D_ERR_INVALID, "coupling point out of range");
  for (int k = 0; k < cp->ncpl_el; ++k)
    if (cp->cpl_el_point[k] < 0 || cp->cpl_el_point[k] >= eld->nglob || cp->cpl_el_ac_point[k] < 0 ||
        cp->cpl_el_ac_point[k] >= ad->nglob)
      return fail(SF2D_ERR_INVALID, "coupling point out of range");
  for (int k = 0; k < ad->nstacey; ++k)
    if (ad->st_iglob[k] < 0 || ad->st_iglob[k] >= ad->nglob) return fail(SF2D_ERR_INVALID, "fluid Stacey point out of range");
  for (int k = 0; k < ad->nfree; ++k)
    if (ad->free_iglob[k] < 0 || ad->free_iglob[k] >= ad->nglob) return fail(SF2D_ERR_INVALID, "free-surface point out of range");
  for (int k = 0; k < ad->nsrc; ++k)
    if (ad->src_ispec[k] < 0 || ad->src_ispec[k] >= ad->nspec) return fail(SF2D_ERR_INVALID, "fluid source element out of range");
  for (int k = 0; k < ad->nrec; ++k)
    if (ad->rec_ispec[k] < 0 || ad->rec_ispec[k] >= ad->nspec) return fail(SF2D_ERR_INVALID, "fluid receiver element out of range");
  const bool pml_ac = ad->pml_region != nullptr, pml_el = eld->pml_region != nullptr;
  const bool adjoint = cp->adjoint != 0;
  if (adjoint && (pml_ac || pml_el)) return fail(SF2D_ERR_INVALID, "adjoint runs are implemented without CPML layers");
  if (adjoint && eld->time_scheme == 2) return fail(SF2D_ERR_INVALID, "adjoint runs are implemented for Newmark");
  std::vector<int> group;
  if (pml_ac) {
    if (!ad->pml_K_x || !ad->pml_K_z || !ad->pml_d_x || !ad->pml_d_z || !ad->pml_alpha_x || !ad->pml_alpha_z ||
        !(ad->pml_dt > 0.0))
      return fail(SF2D_ERR_INVALID, "missing fluid CPML arrays");
    if (ad->nstacey > 0) return fail(SF2D_ERR_INVALID, "CPML layers and Stacey conditions exclude each other");
    if (ad->npml_edge < 0 || (ad->npml_edge > 0 && !ad->pml_edge_iglob))
      return fail(SF2D_ERR_INVALID, "bad fluid CPML edge list");
    for (int k = 0; k < ad->npml_edge; ++k)
      if (ad->pml_edge_iglob[k] < 0 || ad->pml_edge_iglob[k] >= ad->nglob)
        return fail(SF2D_ERR_INVALID, "fluid CPML edge point out of range");
    group.assign(ad->nspec, 0);
    for (int e = 0; e < ad->nspec; ++e) {
      if (ad->pml_region[e] < 0 || ad->pml_region[e] > 3) return fail(SF2D_ERR_INVALID, "CPML region must be 0 to 3");
      group[e] = ad->pml_region[e] > 0 ? 1 : 0;
    }
  }
  if (pml_ac || pml_el) {
    if ((cp->ncpl_ac > 0 && !cp->cpl_ac_el_elpt) || (cp->ncpl_el > 0 && !cp->cpl_el_ac_elpt))
      return fail(SF2D_ERR_INVALID, "coupling entries need their element points with CPML layers");
    for (int k = 0; k < cp->ncpl_ac; ++k)
      if (cp->cpl_ac_el_elpt[k] < 0 || cp->cpl_ac_el_elpt[k] >= eld->nspec * NGLL2)
        return fail(SF2D_ERR_INVALID, "coupling element point out of range");
    for (int k = 0; k < cp->ncpl_el; ++k)
      if (cp->cpl_el_ac_elpt[k] < 0 || cp->cpl_el_ac_elpt[k] >= ad->nspec * NGLL2)
        return fail(SF2D_ERR_INVALID, "coupling element point out of range");
  }

  auto *C = new sf2d_coupled();
  std::unique_ptr<sf2d_coupled> guard(C);
  C->adjoint = adjoint;
  // the solid sub-solver; its receivers are renumbered into the run's list below.
  // A solid description with nspec = 0 makes a fluid-only run: only its time
  // stepping members (nstep, deltat..., time_scheme, nstage, alpha/beta_lddrk,
  // threads_per_block) and the GLL arrays (hprime, hprimewgll, wxgll, wzgll) are read.
  const bool fluid_only = eld->nspec == 0;
  sf2d_solver *S = nullptr;
  const int scheme = eld->time_scheme == 0 ? 1 : eld->time_scheme;
  if (fluid_only) {
    if (cp->ncpl_ac > 0 || cp->ncpl_el > 0 || eld->nrec > 0 || eld->nsrc > 0)
      return fail(SF2D_ERR_INVALID, "a fluid-only run has no coupling, solid source or solid receiver");
    if (!eld->hprime || !eld->hprimewgll || !eld->wxgll || !eld->wzgll) return fail(SF2D_ERR_INVALID, "missing GLL arrays");
    if (scheme != 1 && scheme != 2) return fail(SF2D_ERR_INVALID, "time_scheme must be 1 (Newmark) or 2 (LDDRK)");
    if (scheme == 2 && (!eld->alpha_lddrk || !eld->beta_lddrk)) return fail(SF2D_ERR_INVALID, "LDDRK needs alpha/beta");
    C->lddrk = scheme == 2;
    C->nstage = C->lddrk ? 6 : 1;
    C->nt = eld->threads_per_block > 0 ? eld->threads_per_block : 256;
    if (C->nt != 128 && C->nt != 250 && C->nt != 256 && C->nt != 512)
      return fail(SF2D_ERR_INVALID, "threads_per_block must be 128, 250, 256 or 512");
    SF2D_CUDA(cudaStreamCreateWithFlags(&C->own_stream, cudaStreamNonBlocking));
  } else {
    sf2d_elastic_desc e2 = *eld;
    if (e2.seismotype == 4 || e2.seismotype == 6 || e2.seismotype == 0) e2.seismotype = 1;
    // solid elements touching a coupling point get tiles of their own (late
    // tiles, after the fluid step); the others never touch a point the fluid
    // reads or a fluid value, so they run beside the fluid step
    if (eld->nglob <= 0 || !eld->ibool || (cp->ncpl_el > 0 && !cp->cpl_el_point) ||
        (cp->ncpl_ac > 0 && !cp->cpl_ac_el_point))
      return fail(SF2D_ERR_INVALID, "missing solid mesh or coupling points");
    std::vector<uint8_t> cpl_pt(eld->nglob, 0), late(eld->nspec, 0);
    for (int k = 0; k < cp->ncpl_el; ++k) {
      const int g = cp->cpl_el_point[k];
      if (g < 0 || g >= eld->nglob) return fail(SF2D_ERR_INVALID, "solid coupling point out of range");
      cpl_pt[g] = 1;
    }
    for (int k = 0; k < cp->ncpl_ac; ++k) {
      const int g = cp->cpl_ac_el_point[k];
      if (g < 0 || g >= eld->nglob) return fail(SF2D_ERR_INVALID, "solid coupling point out of range");
      cpl_pt[g] = 1;
    }
    for (int e = 0; e < eld->nspec; ++e)
      for (int q = 0; q < NGLL2; ++q) {
        const int g = eld->ibool[static_cast<size_t>(e) * NGLL2 + q];
        if (g >= 0 && g < eld->nglob && cpl_pt[g]) late[e] = 1;
      }
    // an adjoint run's solid accumulates the sensitivity kernels
    if (int rc = sf2d_create_solver_internal(&e2, adjoint, &C->el, late.data())) return rc;
    S = C->el;
    if (cp->seismotype == 6) S->P.seismotype = 6;  // potential receivers in the solid record zero
    C->lddrk = S->lddrk;
    C->nstage = S->nstage;
    C->nt = S->nt;
  }
  if (ad->nsrc > 0 && eld->nstage != C->nstage) return fail(SF2D_ERR_INVALID, "stf must hold one value per step and stage");
  if (ad->threads_per_block > 0) {
    C->nt = ad->threads_per_block;
    if (C->nt != 128 && C->nt != 250 && C->nt != 256 && C->nt != 512)
      return fail(SF2D_ERR_INVALID, "threads_per_block must be 128, 250, 256 or 512");
  }
  C->nstep = eld->nstep;
  C->nrec_total = cp->nrec_total;
  int rc = 0;

  // ---- fluid tiling and per-slot data
  const int te = ad->tile_elems > 0 ? ad->tile_elems : 32;
  // the fluid layer's tiles are a quarter of the size: there are few of them
  // (one wave), so the shorter per-tile latency sets the layer kernel's time
  const int group_te[2] = {te, std::max(4, te / 4)};
  std::string err = build_tiling(ad->nspec, ad->nglob, ad->ibool, ad->centroid_xz, te, C->T,
                                 pml_ac ? group.data() : nullptr, pml_ac ? 2 : 1, pml_ac ? group_te : nullptr);
  if (!err.empty()) return fail(SF2D_ERR_INVALID, "fluid tiling: " + err);
  const Tiling &T = C->T;
  C->pml_tile0 = pml_ac ? T.group_tile_begin[1] : T.ntiles;
  const int pml_slot0 = C->pml_tile0 < T.ntiles ? T.tiles[C->pml_tile0].elem_base : ad->nspec;
  const size_t nq = static_cast<size_t>(ad->nspec) * NGLL2;
  std::vector<float4> geo(nq);
  std::vector<float> fac(nq);
  for (int s = 0; s < ad->nspec; ++s) {
    const size_t src = static_cast<size_t>(T.elem_order[s]) * NGLL2;
    for (int q = 0; q < NGLL2; ++q) {
      geo[s * NGLL2 + q] = make_float4(ad->xix[src + q], ad->xiz[src + q], ad->gammax[src + q], ad->gammaz[src + q]);
      fac[s * NGLL2 + q] = ad->jacobian[src + q] / ad->rhostore[src + q];  // deriv(6) = J / rho in FP32
    }
  }
  std::vector<float> rmass(ad->nglob);
  std::vector<uint8_t> fmask(ad->nglob, 0);
  for (int g = 0; g < ad->nglob; ++g) rmass[g] = ad->rmass_inverse[T.dev2glob[g]];
  for (int k = 0; k < ad->nfree; ++k) fmask[T.glob2dev[ad->free_iglob[k]]] |= AC_FREE;
  std::vector<int> pml_set_idx;
  std::vector<PmlSet> pml_sets;
  std::vector<float> pml_jk;
  if (pml_ac) {
    for (int k = 0; k < ad->npml_edge; ++k) fmask[T.glob2dev[ad->pml_edge_iglob[k]]] |= AC_EDGE;
    pml_build_sets(ad, T.elem_order, pml_slot0, ad->nspec - pml_slot0, ad->pml_dt, pml_sets, pml_set_idx);
    for (int s = pml_slot0; s < ad->nspec; ++s)
      for (int q = 0; q < NGLL2; ++q) {
        const size_t p = static_cast<size_t>(T.elem_order[s]) * NGLL2 + q;
        pml_jk.push_back(ad->jacobian[p] / ad->kappastore[p]);  // fac = J / kappa in FP32
      }
  }
  const size_t npml_q = static_cast<size_t>(ad->nspec - pml_slot0) * NGLL2;
  // a boundary or coupling point goes to the tile of the first element holding it
  std::vector<int> glob_tile(ad->nglob, -1);
  for (int e = 0; e < ad->nspec; ++e)
    for (int q = 0; q < NGLL2; ++q) {
      const int g = ad->ibool[static_cast<size_t>(e) * NGLL2 + q];
      if (glob_tile[g] < 0) glob_tile[g] = T.elem_tile[e];
    }
  std::vector<TileInfo> tiles = T.tiles;
  std::vector<std::vector<int>> st_t(T.ntiles), cpl_t(T.ntiles), src_t(T.ntiles), rec_t(T.ntiles);
  for (int k = 0; k < ad->nstacey; ++k) st_t[glob_tile[ad->st_iglob[k]]].push_back(k);
  for (int k = 0; k < cp->ncpl_ac; ++k) cpl_t[glob_tile[cp->cpl_ac_point[k]]].push_back(k);
  for (int k = 0; k < ad->nsrc; ++k) src_t[T.elem_tile[ad->src_ispec[k]]].push_back(k);
  for (int k = 0; k < ad->nrec; ++k) rec_t[T.elem_tile[ad->rec_ispec[k]]].push_back(k);
  std::vector<int> st_local, cpl_local, cpl_src, cpl_pml_pt, src_local, src_id, rec_id, rec_dev;
  std::vector<double> cpl_pml_coef;
  std::vector<float2> st_wr, src_sk;
  std::vector<float4> cpl_nw, rec_geo;
  std::vector<float> rec_rho;
  std::vector<double> rec_h;
  for (int t = 0; t < T.ntiles; ++t) {
    tiles[t].st_off = static_cast<int>(st_local.size());
    for (int k : st_t[t]) {
      st_local.push_back(T.local_id(t, ad->st_iglob[k]));
      st_wr.push_back(make_float2(ad->st_w[k], ad->st_rho_vp[k]));
    }
    tiles[t].st_n = static_cast<int>(st_local.size()) - tiles[t].st_off;
    tiles[t].cpl_off = static_cast<int>(cpl_local.size());
    for (int k : cpl_t[t]) {
      cpl_local.push_back(T.local_id(t, cp->cpl_ac_point[k]));
      cpl_src.push_back(S->T.glob2dev[cp->cpl_ac_el_point[k]]);  // entries exist only with a solid
      cpl_nw.push_back(make_float4(cp->cpl_ac_nx[k], cp->cpl_ac_nz[k], cp->cpl_ac_w[k], 0.f));
      const int q = pml_el ? cp->cpl_ac_el_elpt[k] : -1;
      const int region = q >= 0 ? eld->pml_region[q / NGLL2] : 0;
      if (region <= 0) continue;
      // solid element in the layer: strain coefficients of lik_parameter_computation,
      // 13 form for X-only, 31 form for Z-only (compute_coupling_acoustic_el.f90:113-134)
      if (region == CPML_XZ)
        return fail(SF2D_ERR_INVALID, "a fluid-solid boundary in a CPML corner region is not supported");
      const PmlAt c = pml_at(eld, static_cast<size_t>(q));
      const bool x_only = region == CPML_X_ONLY;
      const PmlLik L = x_only ? pml_lik(c.kx, c.bx, c.ax, c.kz, c.bz, c.az, region, true)
                              : pml_lik(c.kz, c.bz, c.az, c.kx, c.bx, c.ax, region, false);
      const double bb = x_only ? c.ax : c.az;
      const PmlConv cv = pml_conv(bb, eld->pml_dt);
      cpl_pml_pt.push_back(cpl_src.back());
      cpl_src.back() = ~static_cast<int>(cpl_pml_pt.size() - 1);
      for (double x : {L.A0, L.A1, cv.c0, cv.c1, cv.c2, bb}) cpl_pml_coef.push_back(x);
    }
    tiles[t].cpl_n = static_cast<int>(cpl_local.size()) - tiles[t].cpl_off;
    tiles[t].src_off = static_cast<int>(src_local.size());
    for (int k : src_t[t])
      for (int q = 0; q < NGLL2; ++q) {
        const size_t p = static_cast<size_t>(ad->src_ispec[k]) * NGLL2 + q;
        src_local.push_back(T.local_id(t, ad->ibool[p]));
        src_id.push_back(k);
        // an adjoint source adds (xir gammar) s to chi_dot_dot, without 1/kappa
        // (compute_add_sources_acoustic.f90:247-290): divided by 1 here
        src_sk.push_back(make_float2(ad->sourcearrays[static_cast<size_t>(k) * NGLL2 + q],
                                     adjoint ? 1.f : ad->kappastore[p]));
      }
    tiles[t].src_n = static_cast<int>(src_local.size()) - tiles[t].src_off;
    tiles[t].rec_off = static_cast<int>(rec_id.size());
    for (int k : rec_t[t]) {
      rec_id.push_back(ad->rec_global[k]);
      for (int q = 0; q < NGLL2; ++q) {
        const size_t p = static_cast<size_t>(ad->rec_ispec[k]) * NGLL2 + q;
        rec_dev.push_back(T.glob2dev[ad->ibool[p]]);
        rec_geo.push_back(make_float4(ad->xix[p], ad->xiz[p], ad->gammax[p], ad->gammaz[p]));
        rec_rho.push_back(ad->rhostore[p]);
      }
      for (int i = 0; i < 5; ++i) rec_h.push_back(ad->hxir[k * 5 + i]);
      for (int j = 0; j < 5; ++j) rec_h.push_back(ad->hgammar[k * 5 + j]);
    }
    tiles[t].rec_n = static_cast<int>(rec_id.size()) - tiles[t].rec_off;
  }
  for (const TileInfo &t : tiles)
    if (t.rec_n > C->nt) return fail(SF2D_ERR_INVALID, "more fluid receivers in one tile than threads per CTA");
  std::vector<int> slot_pos(T.shp_slots.size());
  for (size_t k = 0; k < T.shp_slots.size(); ++k) slot_pos[T.shp_slots[k]] = static_cast<int>(k);
  // per tile: the local points on the free surface or a layer's outer edge, with their bits
  std::vector<int> edge_local;
  for (int t = 0; t < T.ntiles; ++t) {
    tiles[t].edge_off = static_cast<int>(edge_local.size());
    for (const auto &gl : T.tile_glob_local[t]) {
      const uint8_t m = fmask[T.glob2dev[gl.first]];
      if (m) edge_local.push_back(gl.second | (static_cast<int>(m) << 16));
    }
    tiles[t].edge_n = static_cast<int>(edge_local.size()) - tiles[t].edge_off;
  }
  std::vector<int4> bgroups;
  std::vector<int> bnd_idx;
  err = build_boundary_groups(tiles, st_local, cpl_local, src_local, bgroups, bnd_idx);
  if (!err.empty()) return fail(SF2D_ERR_INVALID, err);

  AcParams &A = C->A;
  C->nglob = ad->nglob;
  float *p, *pd, *pdd;
  if ((rc = C->alloc(&p, ad->nglob)) || (rc = C->alloc(&pd, ad->nglob)) || (rc = C->alloc(&pdd, ad->nglob))) return rc;
  SF2D_CUDA(cudaMemset(p, 0, sizeof(float) * ad->nglob));
  SF2D_CUDA(cudaMemset(pd, 0, sizeof(float) * ad->nglob));
  SF2D_CUDA(cudaMemset(pdd, 0, sizeof(float) * ad->nglob));
  A.p = p;
  A.pd = pd;
  A.pdd = pdd;
  if (C->lddrk) {
    float *pl, *pdl;
    if ((rc = C->alloc(&pl, ad->nglob)) || (rc = C->alloc(&pdl, ad->nglob))) return rc;
    SF2D_CUDA(cudaMemset(pl, 0, sizeof(float) * ad->nglob));
    SF2D_CUDA(cudaMemset(pdl, 0, sizeof(float) * ad->nglob));
    A.pL = pl;
    A.pdL = pdl;
    for (int k = 0; k < 6; ++k) {
      A.alpha[k] = eld->alpha_lddrk[k];
      A.beta[k] = eld->beta_lddrk[k];
    }
  }
  if ((rc = C->upload_const(&A.rmass, rmass)) || (rc = C->upload_const(&A.free_mask, fmask)) ||
      (rc = C->upload_const(&A.tiles, tiles)) || (rc = C->upload_const(&A.lib, T.lib)) ||
      (rc = C->upload_const(&A.bgroups, bgroups)) || (rc = C->upload_const(&A.bnd_idx, bnd_idx)) ||
      (rc = C->upload_const(&A.geo, geo)) || (rc = C->upload_const(&A.fac, fac)) ||
      (rc = C->upload_const(&A.sh_ids, T.sh_ids)) || (rc = C->upload_const(&A.shp_off, T.shp_off)) ||
      (rc = C->upload_const(&A.slot_pos, slot_pos)) || (rc = C->upload_const(&A.st_local, st_local)) ||
      (rc = C->upload_const(&A.edge_local, edge_local)) ||
      (rc = C->upload_const(&A.st_wr, st_wr)) || (rc = C->upload_const(&A.cpl_local, cpl_local)) ||
      (rc = C->upload_const(&A.cpl_src, cpl_src)) || (rc = C->upload_const(&A.cpl_nw, cpl_nw)) ||
      (rc = C->upload_const(&A.src_local, src_local)) || (rc = C->upload_const(&A.src_id, src_id)) ||
      (rc = C->upload_const(&A.src_sk, src_sk)) || (rc = C->upload_const(&A.rec_id, rec_id)) ||
      (rc = C->upload_const(&A.rec_dev, rec_dev)) || (rc = C->upload_const(&A.rec_h, rec_h)) ||
      (rc = C->upload_const(&A.rec_geo, rec_geo)) || (rc = C->upload_const(&A.rec_rho, rec_rho)))
    return rc;
  if (pml_ac || pml_el) {
    if ((rc = C->upload_cpl(C->cpl_fluid, cpl_pml_pt, cpl_pml_coef, 2))) return rc;
    A.cpl_pml_u = reinterpret_cast<const float2 *>(C->cpl_fluid.out);
  }
  if (pml_ac) {
    if ((rc = C->upload_const(&A.pml_sets, pml_sets)) || (rc = C->upload_const(&A.pml_set_idx, pml_set_idx)) ||
        (rc = C->upload_const(&A.pml_jk, pml_jk)))
      return rc;
    for (int l = 0; l < (C->lddrk ? 2 : 1); ++l) {
      float2 *r = nullptr;
      if ((rc = C->alloc(&r, npml_q * 3))) return rc;
      SF2D_CUDA(cudaMemset(r, 0, sizeof(float2) * std::max<size_t>(1, npml_q * 3)));
      (l ? A.pml_rm_l : A.pml_rm) = r;
    }
    if (!C->lddrk) {
      if ((rc = C->alloc(&A.pold, ad->nglob))) return rc;
      SF2D_CUDA(cudaMemset(A.pold, 0, sizeof(float) * ad->nglob));
    }
    A.pml_slot0 = pml_slot0;
    A.DT = ad->pml_dt;
    C->npml_q = npml_q;
  }
  A.h_old = static_cast<double>(eld->deltatsquareover2) / 2.0;
  float *partial;
  if ((rc = C->alloc(&partial, T.sh_ids.size()))) return rc;
  A.partial = partial;
  std::vector<float> stf(static_cast<size_t>(ad->nsrc) * eld->nstep * C->nstage);
  if (ad->nsrc) {
    if (!ad->stf || !ad->sourcearrays) return fail(SF2D_ERR_INVALID, "missing fluid source arrays");
    std::memcpy(stf.data(), ad->stf, stf.size() * sizeof(float));
  }
  if ((rc = C->upload_const(&A.stf, stf))) return rc;
  const size_t nseis = static_cast<size_t>(cp->nrec_total) * eld->nstep * 2;
  if ((rc = C->alloc(&C->seis, nseis))) return rc;
  SF2D_CUDA(cudaMemset(C->seis, 0, sizeof(double) * std::max<size_t>(1, nseis)));
  A.seis = C->seis;
  // step, step shadow, status, -, chi frame base, kernel frame base
  if ((rc = C->alloc(&C->ctr, 8))) return rc;
  SF2D_CUDA(cudaMemset(C->ctr, 0, 8 * sizeof(int)));
  A.d_step = C->ctr;
  A.d_step_b = C->ctr + 1;
  A.d_status = C->ctr + 2;
  A.pframe_base = C->ctr + 4;
  A.kp_base = C->ctr + 5;
  A.adjoint = adjoint ? 1 : 0;
  A.nglob_ac = ad->nglob;
  if (S) {
    A.u_el = S->P.u;
    A.v_el = S->P.v;
    A.a_el = S->P.a;
  }
  A.nstep_stf = eld->nstep;
  A.nstage = C->nstage;
  A.nstep_seis = eld->nstep;
  A.seismotype = cp->seismotype;
  A.use_trick = cp->use_trick;
  A.nrec = ad->nrec;
  A.cosrot = cp->cosrot;
  A.sinrot = cp->sinrot;
  A.dt = eld->deltat;
  A.dto2 = eld->deltatover2;
  A.dt2o2 = eld->deltatsquareover2;
  A.shared_begin = T.shared_begin;
  A.nshared = T.nshared;
  A.max_q = T.max_elems * NGLL2;
  A.max_local = T.max_local;
  for (int k = 0; k < 25; ++k) {
    A.hconst[k] = eld->hprime[k];
    A.hconst[25 + k] = eld->hprimewgll[k];
  }
  for (int k = 0; k < 5; ++k) {
    A.hconst[50 + k] = eld->wxgll[k];
    A.hconst[55 + k] = eld->wzgll[k];
  }
  if ((rc = C->upload(&C->d_dev2glob, T.dev2glob.data(), T.dev2glob.size()))) return rc;
  if ((rc = C->alloc(&C->d_stage, ad->nglob))) return rc;
  C->smem = ac_smem_layout(A.max_q, A.max_local).total;
  if (C->smem > 220 * 1024) return fail(SF2D_ERR_INVALID, "fluid tile too large for shared memory");
  C->tile_fn = pick_ac_tile<false>(C->nt, C->lddrk);
  if (pml_ac) {
    C->pml_fn = pick_ac_tile<true>(C->nt, C->lddrk);
    C->pml_smem = ac_smem_layout(A.max_q, A.max_local, true).total;
    if (C->pml_smem > 220 * 1024) return fail(SF2D_ERR_INVALID, "fluid tile too large for shared memory");
    if (C->pml_tile0 > 0 && C->pml_tile0 < T.ntiles) {
      SF2D_CUDA(cudaStreamCreateWithPriority(&C->side, cudaStreamNonBlocking, C->el ? C->el->priority : 0));
      SF2D_CUDA(cudaEventCreateWithFlags(&C->ev_fork, cudaEventDisableTiming));
      SF2D_CUDA(cudaEventCreateWithFlags(&C->ev_join, cudaEventDisableTiming));
      SF2D_CUDA(cudaEventCreateWithFlags(&C->ev_rec, cudaEventDisableTiming));
      SF2D_CUDA(cudaEventCreateWithFlags(&C->ev_rec_done, cudaEventDisableTiming));
    }
  }
  if (C->el && C->el->late_tile0 > 0 && !adjoint) {
    int least = 0, greatest = 0;
    SF2D_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    SF2D_CUDA(cudaStreamCreateWithPriority(&C->early, cudaStreamNonBlocking, least));
    SF2D_CUDA(cudaEventCreateWithFlags(&C->ev_early_fork, cudaEventDisableTiming));
    SF2D_CUDA(cudaEventCreateWithFlags(&C->ev_early_join, cudaEventDisableTiming));
  }
  {
    // the limit belongs to the kernel: only ever raise it (see the solid solver)
    static std::mutex attr_mutex;
    std::lock_guard<std::mutex> lock(attr_mutex);
    const std::pair<AcTileFn, size_t> fns[2] = {{C->tile_fn, C->smem}, {C->pml_fn, C->pml_smem}};
    for (const auto &fs : fns) {
      if (!fs.first) continue;
      cudaFuncAttributes fa;
      SF2D_CUDA(cudaFuncGetAttributes(&fa, fs.first));
      if (fa.maxDynamicSharedSizeBytes < static_cast<int>(fs.second))
        SF2D_CUDA(cudaFuncSetAttribute(fs.first, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(fs.second)));
    }
  }

  // ---- solid side: receivers into the run's list, coupling entries per tile
  if (fluid_only) {
    SF2D_CUDA(cudaDeviceSynchronize());
    *out = guard.release();
    return SF2D_OK;
  }
  if (S->nrec > 0) {
    std::vector<int> ids(S->nrec);
    SF2D_CUDA(cudaMemcpy(ids.data(), S->P.rec_id, sizeof(int) * S->nrec, cudaMemcpyDeviceToHost));
    for (int &k : ids) k = cp->el_rec_global[k];
    SF2D_CUDA(cudaMemcpy(const_cast<int *>(S->P.rec_id), ids.data(), sizeof(int) * S->nrec, cudaMemcpyHostToDevice));
  }
  S->P.seis = C->seis;
  {
    std::vector<TileInfo> et(S->T.ntiles);
    SF2D_CUDA(cudaMemcpy(et.data(), S->P.tiles, sizeof(TileInfo) * et.size(), cudaMemcpyDeviceToHost));
    std::vector<int> eg_tile(eld->nglob, -1);
    for (int e = 0; e < eld->nspec; ++e)
      for (int q = 0; q < NGLL2; ++q) {
        const int g = eld->ibool[static_cast<size_t>(e) * NGLL2 + q];
        if (eg_tile[g] < 0) eg_tile[g] = S->T.elem_tile[e];
      }
    std::vector<std::vector<int>> by_t(S->T.ntiles);
    for (int k = 0; k < cp->ncpl_el; ++k) {
      const int t = eg_tile[cp->cpl_el_point[k]];
      if (t < S->late_tile0) return fail(SF2D_ERR_INVALID, "coupling entry in an early tile");
      by_t[t].push_back(k);
    }
    std::vector<int> e_local, e_src, e_pt;
    std::vector<float4> e_nw;
    std::vector<double> e_coef;
    for (int t = 0; t < S->T.ntiles; ++t) {
      et[t].cpl_off = static_cast<int>(e_local.size());
      for (int k : by_t[t]) {
        e_local.push_back(S->T.local_id(t, cp->cpl_el_point[k]));
        e_src.push_back(T.glob2dev[cp->cpl_el_ac_point[k]]);
        e_nw.push_back(make_float4(cp->cpl_el_nx[k], cp->cpl_el_nz[k], cp->cpl_el_w[k], 0.f));
        const int q = pml_ac ? cp->cpl_el_ac_elpt[k] : -1;
        const int region = q >= 0 ? ad->pml_region[q / NGLL2] : 0;
        if (region <= 0) continue;
        // fluid element in the layer: coefficients of l_parameter_computation
        // (compute_coupling_viscoelastic_ac.f90:105-123), pole alpha_x
        const PmlAt c = pml_at(ad, static_cast<size_t>(q));
        const PmlL L = pml_l(c.kx, c.bx, c.ax, c.kz, c.bz, c.az, region);
        const PmlConv cv = pml_conv(c.ax, ad->pml_dt);
        e_pt.push_back(e_src.back());
        e_src.back() = ~static_cast<int>(e_pt.size() - 1);
        for (double x : {L.A0, L.A1, L.A2, L.A3, cv.c0, cv.c1, cv.c2, c.ax}) e_coef.push_back(x);
      }
      et[t].cpl_n = static_cast<int>(e_local.size()) - et[t].cpl_off;
    }
    if (pml_ac || pml_el) {
      if ((rc = C->upload_cpl(C->cpl_solid, e_pt, e_coef, 1))) return rc;
      S->P.cpl_pml_p = C->cpl_solid.out;
      if (C->cpl_solid.n > 0 && !C->lddrk && !A.pold)
        return fail(SF2D_ERR_INVALID, "CPML coupling entries without a fluid CPML layer");
    }
    // the solid's boundary terms regrouped with the coupling entries
    std::vector<int4> eg;
    std::vector<int> ei;
    err = build_boundary_groups(et, S->h_st_local, e_local, S->h_src_local, eg, ei);
    if (!err.empty()) return fail(SF2D_ERR_INVALID, err);
    if ((rc = C->upload_const(&S->P.bgroups, eg)) || (rc = C->upload_const(&S->P.bnd_idx, ei))) return rc;
    SF2D_CUDA(cudaMemcpy(const_cast<TileInfo *>(S->P.tiles), et.data(), sizeof(TileInfo) * et.size(),
                         cudaMemcpyHostToDevice));
    if ((rc = C->upload_const(&S->P.cpl_local, e_local)) || (rc = C->upload_const(&S->P.cpl_src, e_src)) ||
        (rc = C->upload_const(&S->P.cpl_nw, e_nw)))
      return rc;
    S->P.pdd_ac = A.pdd;
    S->P.p_ac = A.p;
    S->P.pd_ac = A.pd;
    S->P.cpl_adjoint = adjoint ? 1 : 0;
  }
  SF2D_CUDA(cudaDeviceSynchronize());
  *out = guard.release();
  return SF2D_OK;
}

extern "C" int sf2d_coupled_prepare(sf2d_coupled *C) {
  using namespace sf2d;
  if (!C) return fail(SF2D_ERR_INVALID, "null solver");
  const int K = C->chunk;
  if (C->graph && C->graph_steps == K) return SF2D_OK;
  if (C->graph) cudaGraphExecDestroy(C->graph);
  C->graph = nullptr;
  cudaStream_t st = C->stream();
  cudaGraph_t g;
  SF2D_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  C->launch_chunk(K);
  SF2D_CUDA(cudaStreamEndCapture(st, &g));
  // the captured kernels keep their streams' priorities
  cudaError_t e = cudaGraphInstantiate(&C->graph, g, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(SF2D_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  SF2D_CUDA(cudaGraphUpload(C->graph, st));
  SF2D_CUDA(cudaStreamSynchronize(st));
  C->graph_steps = K;
  return SF2D_OK;
}

extern "C" int sf2d_coupled_enqueue(sf2d_coupled *C, int nstep) {
  using namespace sf2d;
  if (!C || nstep < 0) return fail(SF2D_ERR_INVALID, "bad arguments");
  sf2d_solver *S = C->el;
  cudaStream_t st = C->stream();
  const int K = C->chunk;
  int done = 0;
  if (nstep >= K) {
    if (int rc = sf2d_coupled_prepare(C)) return rc;
    for (; done + K <= nstep; done += K) SF2D_CUDA(cudaGraphLaunch(C->graph, st));
  }
  if (done < nstep)
    if (int rc = C->launch_chunk(nstep - done)) return rc;
  C->steps_done += nstep;
  if (S) S->steps_done += nstep;
  return SF2D_OK;
}

extern "C" int sf2d_coupled_synchronize(sf2d_coupled *C) {
  using namespace sf2d;
  if (!C) return fail(SF2D_ERR_INVALID, "null solver");
  sf2d_solver *S = C->el;
  SF2D_CUDA(cudaStreamSynchronize(C->stream()));
  int status[2] = {0, 0};
  if (S) SF2D_CUDA(cudaMemcpy(&status[0], S->P.d_status, sizeof(int), cudaMemcpyDeviceToHost));
  SF2D_CUDA(cudaMemcpy(&status[1], C->A.d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (status[0] || status[1]) return fail(SF2D_ERR_UNSTABLE, "wavefield blew up (NaN or |field| > 1e25)");
  return SF2D_OK;
}

extern "C" int sf2d_coupled_run(sf2d_coupled *C, int nstep, double *seismograms) {
  using namespace sf2d;
  if (!C || nstep < 0) return fail(SF2D_ERR_INVALID, "bad arguments");
  const int it0 = C->steps_done;
  if (seismograms && it0 + nstep > C->nstep) return fail(SF2D_ERR_INVALID, "run exceeds the seismogram buffer length");
  if (int rc = sf2d_coupled_enqueue(C, nstep)) return rc;
  if (int rc = sf2d_coupled_synchronize(C)) return rc;
  if (seismograms && C->nrec_total && nstep) {
    SF2D_CUDA(cudaMemcpy2D(seismograms, sizeof(double) * 2 * nstep, C->seis + static_cast<size_t>(it0) * 2,
                           sizeof(double) * 2 * C->nstep, sizeof(double) * 2 * nstep, C->nrec_total,
                           cudaMemcpyDeviceToHost));
  }
  return SF2D_OK;
}

extern "C" int sf2d_coupled_copy_seismograms(sf2d_coupled *C, int it0, int n, double *out) {
  using namespace sf2d;
  if (!C || !out || it0 < 0 || n < 0 || it0 + n > C->nstep) return fail(SF2D_ERR_INVALID, "bad arguments");
  SF2D_CUDA(cudaStreamSynchronize(C->stream()));
  if (C->nrec_total && n)
    SF2D_CUDA(cudaMemcpy2D(out, sizeof(double) * 2 * n, C->seis + static_cast<size_t>(it0) * 2,
                           sizeof(double) * 2 * C->nstep, sizeof(double) * 2 * n, C->nrec_total,
                           cudaMemcpyDeviceToHost));
  return SF2D_OK;
}

extern "C" int sf2d_coupled_get_fields(sf2d_coupled *C, float *displ, float *veloc, float *accel, float *pot,
                                       float *pot_dot, float *pot_dot_dot) {
  using namespace sf2d;
  if (!C) return fail(SF2D_ERR_INVALID, "null solver");
  if (C->el)
    if (int rc = sf2d_get_fields(C->el, displ, veloc, accel)) return rc;
  const float *src[3] = {C->A.p, C->A.pd, C->A.pdd};
  float *dst[3] = {pot, pot_dot, pot_dot_dot};
  const int n = C->nglob;
  cudaStream_t s = C->stream();
  for (int k = 0; k < 3; ++k) {
    if (!dst[k]) continue;
    k_scatter_f<<<(n + 255) / 256, 256, 0, s>>>(src[k], C->d_dev2glob, C->d_stage, n);
    SF2D_CUDA(cudaGetLastError());
    SF2D_CUDA(cudaMemcpyAsync(dst[k], C->d_stage, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    SF2D_CUDA(cudaStreamSynchronize(s));
  }
  return SF2D_OK;
}

extern "C" int sf2d_coupled_set_fields(sf2d_coupled *C, const float *displ, const float *veloc, const float *accel,
                                       const float *pot, const float *pot_dot, const float *pot_dot_dot) {
  using namespace sf2d;
  if (!C) return fail(SF2D_ERR_INVALID, "null solver");
  if (C->el)
    if (int rc = sf2d_set_fields(C->el, displ, veloc, accel)) return rc;
  float *dst[3] = {C->A.p, C->A.pd, C->A.pdd};
  const float *src[3] = {pot, pot_dot, pot_dot_dot};
  const int n = C->nglob;
  cudaStream_t s = C->stream();
  for (int k = 0; k < 3; ++k) {
    if (!src[k]) {
      SF2D_CUDA(cudaMemsetAsync(dst[k], 0, sizeof(float) * n, s));
      continue;
    }
    SF2D_CUDA(cudaMemcpyAsync(C->d_stage, src[k], sizeof(float) * n, cudaMemcpyHostToDevice, s));
    k_gather_f<<<(n + 255) / 256, 256, 0, s>>>(C->d_stage, C->d_dev2glob, dst[k], n);
    SF2D_CUDA(cudaGetLastError());
  }
  SF2D_CUDA(cudaStreamSynchronize(s));
  return SF2D_OK;
}

extern "C" int sf2d_coupled_set_global_numbering(sf2d_coupled *C, int nglob_total, const int *solid_points,
                                                  const int *fluid_points) {
  using namespace sf2d;
  if (!C || nglob_total <= 0 || !fluid_points || (C->el && !solid_points))
    return fail(SF2D_ERR_INVALID, "bad arguments");
  if (C->d_gstage) return fail(SF2D_ERR_INVALID, "global numbering already set");
  std::vector<int> gf(C->nglob), gs;
  for (int d = 0; d < C->nglob; ++d) {
    const int g = fluid_points[C->T.dev2glob[d]];
    if (g < 0 || g >= nglob_total) return fail(SF2D_ERR_INVALID, "fluid point outside the mesh numbering");
    gf[d] = g;
  }
  if (C->el) {
    const sf2d_solver *S = C->el;
    gs.resize(S->nglob);
    for (int d = 0; d < S->nglob; ++d) {
      const int g = solid_points[S->T.dev2glob[d]];
      if (g < 0 || g >= nglob_total) return fail(SF2D_ERR_INVALID, "solid point outside the mesh numbering");
      gs[d] = g;
    }
  }
  int rc;
  if ((rc = C->upload(&C->d_gmap_fluid, gf.data(), gf.size()))) return rc;
  if (C->el && (rc = C->upload(&C->d_gmap_solid, gs.data(), gs.size()))) return rc;
  if ((rc = C->alloc(&C->d_gstage, static_cast<size_t>(nglob_total)))) return rc;
  C->nglob_total = nglob_total;
  return SF2D_OK;
}

extern "C" int sf2d_coupled_set_fields_global(sf2d_coupled *C, const float *displ, const float *veloc,
                                              const float *accel, const float *pot, const float *pot_dot,
                                              const float *pot_dot_dot) {
  using namespace sf2d;
  if (!C) return fail(SF2D_ERR_INVALID, "null solver");
  if (!C->d_gstage) return fail(SF2D_ERR_INVALID, "no whole-mesh numbering (sf2d_coupled_set_global_numbering)");
  const size_t nt = static_cast<size_t>(C->nglob_total);
  cudaStream_t s = C->stream();
  if (C->el) {
    sf2d_solver *S = C->el;
    float2 *dst[3] = {S->P.u, S->P.v, S->P.a};
    const float *src[3] = {displ, veloc, accel};
    const int n = S->nglob;
    for (int k = 0; k < 3; ++k) {
      if (!src[k]) {
        SF2D_CUDA(cudaMemsetAsync(dst[k], 0, sizeof(float2) * n, s));
        continue;
      }
      SF2D_CUDA(cudaMemcpyAsync(C->d_gstage, src[k], sizeof(float2) * nt, cudaMemcpyHostToDevice, s));
      k_gather_f2<<<(n + 255) / 256, 256, 0, s>>>(C->d_gstage, C->d_gmap_solid, dst[k], n);
      SF2D_CUDA(cudaGetLastError());
    }
  }
  float *dst[3] = {C->A.p, C->A.pd, C->A.pdd};
  const float *src[3] = {pot, pot_dot, pot_dot_dot};
  const int n = C->nglob;
  float *stage = reinterpret_cast<float *>(C->d_gstage);
  for (int k = 0; k < 3; ++k) {
    if (!src[k]) {
      SF2D_CUDA(cudaMemsetAsync(dst[k], 0, sizeof(float) * n, s));
      continue;
    }
    SF2D_CUDA(cudaMemcpyAsync(stage, src[k], sizeof(float) * nt, cudaMemcpyHostToDevice, s));
    k_gather_f<<<(n + 255) / 256, 256, 0, s>>>(stage, C->d_gmap_fluid, dst[k], n);
    SF2D_CUDA(cudaGetLastError());
  }
  SF2D_CUDA(cudaStreamSynchronize(s));
  return SF2D_OK;
}

extern "C" int sf2d_coupled_get_fields_global(sf2d_coupled *C, float *displ, float *veloc, float *accel, float *pot,
                                              float *pot_dot, float *pot_dot_dot) {
  using namespace sf2d;
  if (!C) return fail(SF2D_ERR_INVALID, "null solver");
  if (!C->d_gstage) return fail(SF2D_ERR_INVALID, "no whole-mesh numbering (sf2d_coupled_set_global_numbering)");
  const size_t nt = static_cast<size_t>(C->nglob_total);
  cudaStream_t s = C->stream();
  float *hdst[6] = {displ, veloc, accel, pot, pot_dot, pot_dot_dot};
  for (int k = 0; k < 6; ++k) {
    if (!hdst[k]) continue;
    const bool solid = k < 3;
    // points outside the domain read zero
    SF2D_CUDA(cudaMemsetAsync(C->d_gstage, 0, (solid ? sizeof(float2) : sizeof(float)) * nt, s));
    if (solid && C->el) {
      const float2 *src[3] = {C->el->P.u, C->el->P.v, C->el->P.a};
      const int n = C->el->nglob;
      k_scatter_f2<<<(n + 255) / 256, 256, 0, s>>>(src[k], C->d_gmap_solid, C->d_gstage, n);
    } else if (!solid) {
      const float *src[3] = {C->A.p, C->A.pd, C->A.pdd};
      const int n = C->nglob;
      k_scatter_f<<<(n + 255) / 256, 256, 0, s>>>(src[k - 3], C->d_gmap_fluid, reinterpret_cast<float *>(C->d_gstage),
                                                   n);
    }
    SF2D_CUDA(cudaGetLastError());
    SF2D_CUDA(cudaMemcpyAsync(hdst[k], C->d_gstage, (solid ? sizeof(float2) : sizeof(float)) * nt,
                              cudaMemcpyDeviceToHost, s));
  }
  SF2D_CUDA(cudaStreamSynchronize(s));
  return SF2D_OK;
}

extern "C" int sf2d_coupled_time_kernels(sf2d_coupled *C, int nstep, float *ms) {
  using namespace sf2d;
  if (!C || nstep <= 0 || !ms) return fail(SF2D_ERR_INVALID, "bad arguments");
  sf2d_solver *S = C->el;
  cudaStream_t str = C->stream();
  cudaEvent_t ev[5];
  for (auto &e : ev) SF2D_CUDA(cudaEventCreate(&e));
  double acc[4] = {0, 0, 0, 0};
  for (int k = 0; k < nstep; ++k)
    for (int st = 0; st < C->nstage; ++st) {
      const bool rp = k > 0 && st == 0;
      SF2D_CUDA(cudaEventRecord(ev[0], str));
      C->launch_cpl_fluid(st);
      C->launch_ac_tile(rp, st);
      SF2D_CUDA(cudaEventRecord(ev[1], str));
      C->launch_ac_shared(st);
      if (st == C->nstage - 1 && C->A.nrec > 0)  // the step's fluid receivers, on the timed stream
        sf2d::k_acoustic_receivers<<<(C->A.nrec + 127) / 128, 128, 0, str>>>(C->A);
      SF2D_CUDA(cudaEventRecord(ev[2], str));
      C->launch_cpl_solid(st);
      if (S) S->launch_tile(rp, st);
      SF2D_CUDA(cudaEventRecord(ev[3], str));
      if (S) S->launch_shared(st);
      SF2D_CUDA(cudaEventRecord(ev[4], str));
      SF2D_CUDA(cudaEventSynchronize(ev[4]));
      for (int q = 0; q < 4; ++q) {
        float t = 0.f;
        SF2D_CUDA(cudaEventElapsedTime(&t, ev[q], ev[q + 1]));
        acc[q] += t;
      }
    }
  SF2D_CUDA(cudaGetLastError());
  if (S) S->launch_receivers();
  SF2D_CUDA(cudaStreamSynchronize(str));
  C->steps_done += nstep;
  if (S) S->steps_done += nstep;
  for (auto &e : ev) cudaEventDestroy(e);
  const double launches = static_cast<double>(nstep) * C->nstage;
  for (int q = 0; q < 4; ++q) ms[q] = static_cast<float>(acc[q] / launches);
  ms[4] = static_cast<float>((acc[0] + acc[1] + acc[2] + acc[3]) / nstep);
  return SF2D_OK;
}

extern "C" int sf2d_coupled_layout_info(sf2d_coupled *C, long long *info) {
  using namespace sf2d;
  if (!C || !info) return fail(SF2D_ERR_INVALID, "bad arguments");
  info[0] = C->T.ntiles;
  info[1] = C->T.nshared;
  info[2] = C->A.max_local;
  info[3] = static_cast<long long>(C->smem);
  info[4] = C->T.nglob - C->T.nshared;
  info[5] = static_cast<long long>(C->T.sh_ids.size());
  return SF2D_OK;
}

extern "C" int sf2d_coupled_solid_layout_info(sf2d_coupled *C, long long *info8) {
  using namespace sf2d;
  if (!C) return fail(SF2D_ERR_INVALID, "null solver");
  if (!C->el) return fail(SF2D_ERR_INVALID, "a fluid-only run has no solid layout");
  return sf2d_layout_info(C->el, info8);
}

extern "C" int sf2d_coupled_launch_count(sf2d_coupled *C, int nstep, long long *launches) {
  using namespace sf2d;
  if (!C || !launches || nstep < 0) return fail(SF2D_ERR_INVALID, "bad arguments");
  const sf2d_solver *S = C->el;
  long long per_stage = (C->cpl_fluid.n > 0) + (C->pml_tile0 > 0) + (C->pml_tile0 < C->T.ntiles) + 1 +
                        (C->cpl_solid.n > 0);
  if (S) per_stage += (C->early ? S->tile_launches(S->late_tile0) + (S->late_tile0 > 0) : S->tile_launches(0)) + 1;
  const long long chunks = nstep / C->chunk + (nstep % C->chunk ? 1 : 0);
  *launches = per_stage * C->nstage * nstep + (C->A.nrec > 0 ? nstep : 0) + (S && S->nrec > 0 ? chunks : 0) +
              ((C->A.pframes != nullptr) + (C->A.kl_ac != nullptr)) * static_cast<long long>(nstep);
  return SF2D_OK;
}

extern "C" int sf2d_coupled_get_stream(sf2d_coupled *C, void **stream) {
  using namespace sf2d;
  if (!C || !stream) return fail(SF2D_ERR_INVALID, "bad arguments");
  *stream = static_cast<void *>(C->stream());
  return SF2D_OK;
}

extern "C" int sf2d_coupled_destroy(sf2d_coupled *C) {
  delete C;
  return SF2D_OK;
}

// ---------------------------------------------------------------------------
// Kernel run of a coupled mesh (sf2d_coupled_fwi_*): the solid path's scheme
// (sf2d_fwi.cu) over both domains.  The forward solver writes solid
// displacement frames (its tile kernels) and fluid chi frames (k_fluid_frame)
// while a segment is recomputed; the adjoint solver (adjoint = 1) reads them
// in its solid tile kernels and in k_fluid_kernels.

namespace {

// Zeroes the fields, kernel sums, seismograms and step counters of a coupled
// solver (frame bases are left to the caller).
int coupled_reset(sf2d_coupled *C) {
  cudaStream_t s = C->stream();
  if (C->el)
    if (int rc = sf2d_reset_solver(C->el)) return rc;
  const size_t n = static_cast<size_t>(C->nglob);
  SF2D_CUDA(cudaMemsetAsync(C->A.p, 0, sizeof(float) * n, s));
  SF2D_CUDA(cudaMemsetAsync(C->A.pd, 0, sizeof(float) * n, s));
  SF2D_CUDA(cudaMemsetAsync(C->A.pdd, 0, sizeof(float) * n, s));
  if (C->A.kl_ac) SF2D_CUDA(cudaMemsetAsync(C->A.kl_ac, 0, sizeof(float2) * C->A.nslot_q, s));
  const size_t nseis = static_cast<size_t>(C->nrec_total) * C->nstep * 2;
  if (nseis) SF2D_CUDA(cudaMemsetAsync(C->seis, 0, sizeof(double) * nseis, s));
  SF2D_CUDA(cudaMemsetAsync(C->ctr, 0, 3 * sizeof(int), s));
  C->steps_done = 0;
  return SF2D_OK;
}

int put_ctr(int *ctr, int idx, int value, cudaStream_t s) {
  // pageable source: staged at call time, ordered on the stream
  SF2D_CUDA(cudaMemcpyAsync(ctr + idx, &value, sizeof(int), cudaMemcpyHostToDevice, s));
  return SF2D_OK;
}

constexpr int NO_FRAMES = 1 << 30;  // a frame base no step reaches

}  // namespace

struct sf2d_coupled_fwi {
  sf2d_coupled *fwd = nullptr, *adj = nullptr;
  int nstep = 0, K = 0, nseg = 0, nrec_total = 0, ng_s = 0, ng_f = 0, nspec_s = 0, nspec_f = 0;
  float dt = 0.f;
  float2 *sframes = nullptr, *ckpt_s = nullptr;  // solid: K frames; nseg * 3 * ng_s (u, v, a)
  float *pframes = nullptr, *ckpt_f = nullptr;   // fluid: K frames; nseg * 3 * ng_f (chi, chi_dot, chi_dot_dot)
  std::vector<int> ibool_s, el_rec, ac_rec;      // solid ibool; run receiver index of each solid / fluid receiver
  std::vector<float> rho_s, kappa_s, mu_s;
  std::vector<void *> allocs;
  cudaEvent_t ev_fwd = nullptr, ev_adj = nullptr;
  ~sf2d_coupled_fwi() {
    if (fwd) cudaStreamSynchronize(fwd->stream());
    if (adj) cudaStreamSynchronize(adj->stream());
    if (ev_fwd) cudaEventDestroy(ev_fwd);
    if (ev_adj) cudaEventDestroy(ev_adj);
    for (void *p : allocs) cudaFree(p);
    delete adj;
    delete fwd;
  }
  template <typename T_>
  int alloc(T_ **p, size_t count) {
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(T_));
    if (e != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? SF2D_ERR_OOM : SF2D_ERR_CUDA,
                  std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(*p);
    return SF2D_OK;
  }
};

extern "C" int sf2d_coupled_fwi_create(const sf2d_elastic_desc *eld, const sf2d_acoustic_desc *ad,
                                       const sf2d_coupling_desc *cp, const float *solid_rhostore,
                                       const float *solid_kappastore, int checkpoint_every, sf2d_coupled_fwi **out) {
  using namespace sf2d;
  if (!eld || !ad || !cp || !out) return fail(SF2D_ERR_INVALID, "null argument");
  *out = nullptr;
  if (checkpoint_every < 1) return fail(SF2D_ERR_INVALID, "checkpoint_every must be >= 1");
  if (eld->time_scheme == 2) return fail(SF2D_ERR_INVALID, "the kernel run is implemented for Newmark");
  if (cp->adjoint) return fail(SF2D_ERR_INVALID, "pass the forward coupling description");
  if (cp->nrec_total < 1 || eld->nstep < 1) return fail(SF2D_ERR_INVALID, "the kernel run needs receivers and steps");
  const bool solid = eld->nspec > 0;
  if (solid && (!solid_rhostore || !solid_kappastore || !eld->mustore))
    return fail(SF2D_ERR_INVALID, "missing solid rho / kappa / mu");
  auto F = std::make_unique<sf2d_coupled_fwi>();
  sf2d_coupled *fw = nullptr;
  if (int rc = sf2d_coupled_create(eld, ad, cp, &fw)) return rc;
  F->fwd = fw;
  const int nstep = eld->nstep;
  // adjoint problem: one pseudo-source per solid receiver component and per
  // fluid receiver, weighted by the receiver's Lagrange products (FP32)
  sf2d_elastic_desc ed = *eld;
  std::vector<int> s_ispec;
  std::vector<float> s_arr, s_stf;
  if (solid) {
    const int nr = eld->nrec;
    s_ispec.resize(2 * nr);
    s_arr.assign(static_cast<size_t>(2 * nr) * 50, 0.f);
    s_stf.assign(static_cast<size_t>(std::max(1, 2 * nr)) * nstep, 0.f);
    for (int r = 0; r < nr; ++r)
      for (int c = 0; c < 2; ++c) {
        s_ispec[2 * r + c] = eld->rec_ispec[r];
        for (int j = 0; j < 5; ++j)
          for (int i = 0; i < 5; ++i)
            s_arr[(static_cast<size_t>(2 * r + c) * 25 + j * 5 + i) * 2 + c] =
                static_cast<float>(eld->hxir[r * 5 + i]) * static_cast<float>(eld->hgammar[r * 5 + j]);
      }
    ed.nsrc = 2 * nr;
    ed.src_ispec = s_ispec.data();
    ed.sourcearrays = s_arr.data();
    ed.stf = s_stf.data();
    ed.nstage = 1;
  }
  sf2d_acoustic_desc a2 = *ad;
  const int nrf = ad->nrec;
  std::vector<float> f_arr(static_cast<size_t>(nrf) * 25), f_stf(static_cast<size_t>(std::max(1, nrf)) * nstep, 0.f);
  for (int r = 0; r < nrf; ++r)
    for (int j = 0; j < 5; ++j)
      for (int i = 0; i < 5; ++i)
        f_arr[static_cast<size_t>(r) * 25 + j * 5 + i] =
            static_cast<float>(ad->hxir[r * 5 + i]) * static_cast<float>(ad->hgammar[r * 5 + j]);
  a2.nsrc = nrf;
  a2.src_ispec = ad->rec_ispec;
  a2.sourcearrays = f_arr.data();
  a2.stf = f_stf.data();
  sf2d_coupling_desc c2 = *cp;
  c2.adjoint = 1;
  sf2d_coupled *aj = nullptr;
  if (int rc = sf2d_coupled_create(&ed, &a2, &c2, &aj)) return rc;
  F->adj = aj;
  F->nstep = nstep;
  F->K = checkpoint_every;
  F->nseg = (nstep + checkpoint_every - 1) / checkpoint_every;
  F->nrec_total = cp->nrec_total;
  F->ng_f = ad->nglob;
  F->nspec_f = ad->nspec;
  F->dt = eld->deltat;
  F->ac_rec.assign(ad->rec_global, ad->rec_global + nrf);
  if (solid) {
    F->ng_s = eld->nglob;
    F->nspec_s = eld->nspec;
    const size_t nl = static_cast<size_t>(eld->nspec) * 25;
    F->ibool_s.assign(eld->ibool, eld->ibool + nl);
    F->rho_s.assign(solid_rhostore, solid_rhostore + nl);
    F->kappa_s.assign(solid_kappastore, solid_kappastore + nl);
    F->mu_s.assign(eld->mustore, eld->mustore + nl);
    F->el_rec.assign(cp->el_rec_global, cp->el_rec_global + eld->nrec);
  }
  int rc = 0;
  const size_t K = static_cast<size_t>(F->K);
  if ((rc = F->alloc(&F->pframes, K * F->ng_f)) || (rc = F->alloc(&F->ckpt_f, static_cast<size_t>(F->nseg) * 3 * F->ng_f)))
    return rc;
  if (solid && ((rc = F->alloc(&F->sframes, K * F->ng_s)) ||
                (rc = F->alloc(&F->ckpt_s, static_cast<size_t>(F->nseg) * 3 * F->ng_s))))
    return rc;
  // fluid kernel accumulation: per element point (slot order) its point, rho, kappa
  {
    const Tiling &T = aj->T;
    const size_t nq = static_cast<size_t>(ad->nspec) * 25;
    std::vector<int> sib(nq);
    std::vector<float2> rk(nq);
    for (int sl = 0; sl < ad->nspec; ++sl)
      for (int q = 0; q < 25; ++q) {
        const size_t p = static_cast<size_t>(T.elem_order[sl]) * 25 + q;
        sib[static_cast<size_t>(sl) * 25 + q] = T.glob2dev[ad->ibool[p]];
        rk[static_cast<size_t>(sl) * 25 + q] = make_float2(ad->rhostore[p], ad->kappastore[p]);
      }
    AcParams &A = aj->A;
    if ((rc = aj->upload_const(&A.slot_ibool, sib)) || (rc = aj->upload_const(&A.slot_rk, rk)) ||
        (rc = aj->alloc(&A.kl_ac, nq)))
      return rc;
    SF2D_CUDA(cudaMemset(A.kl_ac, 0, sizeof(float2) * std::max<size_t>(nq, 1)));
    A.nslot_q = static_cast<int>(nq);
    A.kpframes = F->pframes;
    A.npframes = F->K;
    // the forward solver's fluid tiling is the adjoint one's (same mesh, same options)
    fw->A.pframes = F->pframes;
    fw->A.npframes = F->K;
  }
  if (solid) {
    fw->el->P.frames = F->sframes;
    fw->el->P.nframes = F->K;
    aj->el->P.kframes = F->sframes;
  }
  SF2D_CUDA(cudaEventCreateWithFlags(&F->ev_fwd, cudaEventDisableTiming));
  SF2D_CUDA(cudaEventCreateWithFlags(&F->ev_adj, cudaEventDisableTiming));
  if ((rc = put_ctr(fw->ctr, 4, NO_FRAMES, fw->stream()))) return rc;
  if (solid && (rc = put_ctr(fw->el->ctr, 3, NO_FRAMES, fw->stream()))) return rc;
  SF2D_CUDA(cudaStreamSynchronize(fw->stream()));
  *out = F.release();
  return SF2D_OK;
}

extern "C" int sf2d_coupled_fwi_forward(sf2d_coupled_fwi *F, double *seismograms) {
  using namespace sf2d;
  if (!F) return fail(SF2D_ERR_INVALID, "null handle");
  sf2d_coupled *C = F->fwd;
  cudaStream_t s = C->stream();
  int rc = coupled_reset(C);
  if (rc) return rc;
  if ((rc = put_ctr(C->ctr, 4, NO_FRAMES, s))) return rc;
  if (C->el && (rc = put_ctr(C->el->ctr, 3, NO_FRAMES, s))) return rc;
  const size_t ns = static_cast<size_t>(F->ng_s), nf = static_cast<size_t>(F->ng_f);
  for (int seg = 0; seg < F->nseg; ++seg) {
    if (C->el) {
      float2 *ck = F->ckpt_s + static_cast<size_t>(seg) * 3 * ns;
      const sf2d::Params &P = C->el->P;
      SF2D_CUDA(cudaMemcpyAsync(ck, P.u, sizeof(float2) * ns, cudaMemcpyDeviceToDevice, s));
      SF2D_CUDA(cudaMemcpyAsync(ck + ns, P.v, sizeof(float2) * ns, cudaMemcpyDeviceToDevice, s));
      SF2D_CUDA(cudaMemcpyAsync(ck + 2 * ns, P.a, sizeof(float2) * ns, cudaMemcpyDeviceToDevice, s));
    }
    float *cf = F->ckpt_f + static_cast<size_t>(seg) * 3 * nf;
    SF2D_CUDA(cudaMemcpyAsync(cf, C->A.p, sizeof(float) * nf, cudaMemcpyDeviceToDevice, s));
    SF2D_CUDA(cudaMemcpyAsync(cf + nf, C->A.pd, sizeof(float) * nf, cudaMemcpyDeviceToDevice, s));
    SF2D_CUDA(cudaMemcpyAsync(cf + 2 * nf, C->A.pdd, sizeof(float) * nf, cudaMemcpyDeviceToDevice, s));
    if ((rc = sf2d_coupled_enqueue(C, std::min(F->K, F->nstep - seg * F->K)))) return rc;
  }
  const int st = sf2d_coupled_synchronize(C);
  if (st && st != SF2D_ERR_UNSTABLE) return st;
  if (seismograms)
    SF2D_CUDA(cudaMemcpy(seismograms, C->seis, sizeof(double) * F->nrec_total * F->nstep * 2, cudaMemcpyDeviceToHost));
  return st;
}

extern "C" int sf2d_coupled_fwi_backward(sf2d_coupled_fwi *F, const float *adj_src, float *rho_kl, float *kappa_kl,
                                         float *mu_kl, float *rho_ac_kl, float *kappa_ac_kl) {
  using namespace sf2d;
  if (!F || !adj_src || !rho_ac_kl || !kappa_ac_kl) return fail(SF2D_ERR_INVALID, "null argument");
  sf2d_coupled *A = F->adj, *C = F->fwd;
  const bool solid = A->el != nullptr;
  if (solid && (!rho_kl || !kappa_kl || !mu_kl)) return fail(SF2D_ERR_INVALID, "null solid kernel array");
  const int nstep = F->nstep;
  cudaStream_t sa = A->stream(), sf = C->stream();
  // time-reversed adjoint sources of the pseudo-sources
  if (solid) {
    const int nr = static_cast<int>(F->el_rec.size());
    std::vector<float> stf(static_cast<size_t>(2 * nr) * nstep);
    for (int r = 0; r < nr; ++r)
      for (int c = 0; c < 2; ++c)
        for (int it = 0; it < nstep; ++it)
          stf[static_cast<size_t>(2 * r + c) * nstep + it] =
              adj_src[(static_cast<size_t>(F->el_rec[r]) * nstep + (nstep - 1 - it)) * 2 + c];
    if (nr) SF2D_CUDA(cudaMemcpy(A->el->d_stf, stf.data(), sizeof(float) * stf.size(), cudaMemcpyHostToDevice));
  }
  {
    const int nr = static_cast<int>(F->ac_rec.size());
    std::vector<float> stf(static_cast<size_t>(nr) * nstep);
    for (int r = 0; r < nr; ++r)
      for (int it = 0; it < nstep; ++it)
        stf[static_cast<size_t>(r) * nstep + it] = adj_src[(static_cast<size_t>(F->ac_rec[r]) * nstep + (nstep - 1 - it)) * 2];
    if (nr)
      SF2D_CUDA(cudaMemcpy(const_cast<float *>(A->A.stf), stf.data(), sizeof(float) * stf.size(), cudaMemcpyHostToDevice));
  }
  int rc = coupled_reset(A);
  if (rc) return rc;
  const size_t ns = static_cast<size_t>(F->ng_s), nf = static_cast<size_t>(F->ng_f);
  for (int seg = F->nseg - 1; seg >= 0; --seg) {
    const int s0 = seg * F->K;
    const int n = std::min(F->K, nstep - s0);
    // recompute the forward segment once the adjoint sweep no longer reads the frames
    SF2D_CUDA(cudaStreamWaitEvent(sf, F->ev_adj, 0));
    if (solid) {
      const float2 *ck = F->ckpt_s + static_cast<size_t>(seg) * 3 * ns;
      const sf2d::Params &P = C->el->P;
      SF2D_CUDA(cudaMemcpyAsync(P.u, ck, sizeof(float2) * ns, cudaMemcpyDeviceToDevice, sf));
      SF2D_CUDA(cudaMemcpyAsync(P.v, ck + ns, sizeof(float2) * ns, cudaMemcpyDeviceToDevice, sf));
      SF2D_CUDA(cudaMemcpyAsync(P.a, ck + 2 * ns, sizeof(float2) * ns, cudaMemcpyDeviceToDevice, sf));
      if ((rc = put_ctr(C->el->ctr, 0, s0, sf)) || (rc = put_ctr(C->el->ctr, 3, s0, sf))) return rc;
    }
    const float *cf = F->ckpt_f + static_cast<size_t>(seg) * 3 * nf;
    SF2D_CUDA(cudaMemcpyAsync(C->A.p, cf, sizeof(float) * nf, cudaMemcpyDeviceToDevice, sf));
    SF2D_CUDA(cudaMemcpyAsync(C->A.pd, cf + nf, sizeof(float) * nf, cudaMemcpyDeviceToDevice, sf));
    SF2D_CUDA(cudaMemcpyAsync(C->A.pdd, cf + 2 * nf, sizeof(float) * nf, cudaMemcpyDeviceToDevice, sf));
    if ((rc = put_ctr(C->ctr, 0, s0, sf)) || (rc = put_ctr(C->ctr, 4, s0, sf))) return rc;
    if ((rc = sf2d_coupled_enqueue(C, n))) return rc;
    SF2D_CUDA(cudaEventRecord(F->ev_fwd, sf));
    // adjoint steps nstep-s0-n .. nstep-s0-1 pair with frames n-1 .. 0
    SF2D_CUDA(cudaStreamWaitEvent(sa, F->ev_fwd, 0));
    if (solid && (rc = put_ctr(A->el->ctr, 4, nstep - 1 - s0, sa))) return rc;
    if ((rc = put_ctr(A->ctr, 5, nstep - 1 - s0, sa))) return rc;
    if ((rc = sf2d_coupled_enqueue(A, n))) return rc;
    SF2D_CUDA(cudaEventRecord(F->ev_adj, sa));
  }
  SF2D_CUDA(cudaStreamSynchronize(sf));
  const int st = sf2d_coupled_synchronize(A);
  if (st && st != SF2D_ERR_UNSTABLE) return st;
  if ((rc = put_ctr(C->ctr, 4, NO_FRAMES, sf))) return rc;
  if (solid && (rc = put_ctr(C->el->ctr, 3, NO_FRAMES, sf))) return rc;
  // solid kernel sums back to the sub-mesh layout with save_kernels_elastic's scaling
  if (solid) {
    const sf2d_solver *S = A->el;
    std::vector<float2> kmu(S->nq);
    std::vector<float> rg(ns);
    SF2D_CUDA(cudaMemcpy(kmu.data(), S->P.kmu_kl, sizeof(float2) * S->nq, cudaMemcpyDeviceToHost));
    SF2D_CUDA(cudaMemcpy(rg.data(), S->P.rho_kl_glob, sizeof(float) * ns, cudaMemcpyDeviceToHost));
    const sf2d::Tiling &T = S->T;
    const float dt = F->dt;
    for (int sl = 0; sl < F->nspec_s; ++sl) {
      const int e = T.elem_order[sl];
      for (int q = 0; q < 25; ++q) {
        const size_t p = static_cast<size_t>(e) * 25 + q;
        const float rsum = rg[T.glob2dev[F->ibool_s[p]]];
        const float2 km = kmu[static_cast<size_t>(sl) * 25 + q];
        rho_kl[p] = -F->rho_s[p] * dt * rsum;
        mu_kl[p] = -2.f * F->mu_s[p] * dt * km.y;
        kappa_kl[p] = -F->kappa_s[p] * dt * km.x;
      }
    }
  }
  // fluid sums (deltat and 1/rho, 1/kappa already in) back to element order
  {
    std::vector<float2> kl(A->A.nslot_q);
    SF2D_CUDA(cudaMemcpy(kl.data(), A->A.kl_ac, sizeof(float2) * kl.size(), cudaMemcpyDeviceToHost));
    const sf2d::Tiling &T = A->T;
    for (int sl = 0; sl < F->nspec_f; ++sl) {
      const size_t e = static_cast<size_t>(T.elem_order[sl]);
      for (int q = 0; q < 25; ++q) {
        rho_ac_kl[e * 25 + q] = kl[static_cast<size_t>(sl) * 25 + q].x;
        kappa_ac_kl[e * 25 + q] = kl[static_cast<size_t>(sl) * 25 + q].y;
      }
    }
  }
  return st;
}

extern "C" int sf2d_coupled_fwi_adjoint_seismograms(sf2d_coupled_fwi *F, double *seismograms) {
  using namespace sf2d;
  if (!F || !seismograms) return fail(SF2D_ERR_INVALID, "null argument");
  SF2D_CUDA(cudaStreamSynchronize(F->adj->stream()));
  SF2D_CUDA(cudaMemcpy(seismograms, F->adj->seis, sizeof(double) * F->nrec_total * F->nstep * 2,
                       cudaMemcpyDeviceToHost));
  return SF2D_OK;
}

extern "C" int sf2d_coupled_fwi_kernel_sums(sf2d_coupled_fwi *F, float *rho_kl, float *kappa_kl, float *mu_kl) {
  using namespace sf2d;
  if (!F || !rho_kl || !kappa_kl || !mu_kl) return fail(SF2D_ERR_INVALID, "null argument");
  if (!F->adj->el) return fail(SF2D_ERR_INVALID, "the mesh has no solid element");
  const sf2d_solver *S = F->adj->el;
  SF2D_CUDA(cudaStreamSynchronize(F->adj->stream()));
  std::vector<float2> kmu(S->nq);
  std::vector<float> rg(F->ng_s);
  SF2D_CUDA(cudaMemcpy(kmu.data(), S->P.kmu_kl, sizeof(float2) * S->nq, cudaMemcpyDeviceToHost));
  SF2D_CUDA(cudaMemcpy(rg.data(), S->P.rho_kl_glob, sizeof(float) * F->ng_s, cudaMemcpyDeviceToHost));
  const sf2d::Tiling &T = S->T;
  for (int sl = 0; sl < F->nspec_s; ++sl) {
    const int e = T.elem_order[sl];
    for (int q = 0; q < 25; ++q) {
      const size_t p = static_cast<size_t>(e) * 25 + q;
      const float2 km = kmu[static_cast<size_t>(sl) * 25 + q];
      rho_kl[p] = rg[T.glob2dev[F->ibool_s[p]]];
      kappa_kl[p] = km.x;
      mu_kl[p] = km.y;
    }
  }
  return SF2D_OK;
}

extern "C" int sf2d_coupled_fwi_adjoint_run(sf2d_coupled_fwi *F, sf2d_coupled **adj) {
  if (!F || !adj) return sf2d::fail(SF2D_ERR_INVALID, "null argument");
  *adj = F->adj;
  return SF2D_OK;
}

extern "C" int sf2d_coupled_fwi_destroy(sf2d_coupled_fwi *F) {
  delete F;
  return SF2D_OK;
}
