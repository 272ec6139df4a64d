// Misfit gradient of the elastic Newmark path: forward run with segment
// checkpoints, then an adjoint sweep that recomputes each forward segment
// from its checkpoint (displacement frames written by the step kernels) and
// advances the adjoint wavefield over it while the step kernels accumulate
// the sensitivity kernels.  Follows the reference's undo-attenuation scheme
// (src/specfem2D/iterate_time_undoatt.F90:193-601): adjoint step it is paired
// with forward step NSTEP - it + 1, adjoint sources are the time-reversed
// residuals injected at the receivers (compute_add_sources_viscoelastic.f90:
// 351-405), kernels are scaled as save_adjoint_kernels.f90:134-141.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "sf2d_b200.h"
#include "sf2d_runtime.h"

struct sf2d_fwi {
  sf2d_solver *fwd = nullptr, *adj = nullptr;
  int nstep = 0, K = 0, nseg = 0, nglob = 0, nspec = 0, nrec = 0;
  float dt = 0.f;
  float2 *frames = nullptr;
  float2 *aframes = nullptr;  // forward accelerations, with the approximate Hessian
  float2 *ckpt = nullptr;     // nseg * 3 * nglob (u, v, a)
  float4 *ckpt_att = nullptr; // nseg * 3 * nq (memory variables and old strains)
  std::vector<int> ibool;
  std::vector<float> rho, kappa, mu;
  std::vector<void *> allocs;
  cudaEvent_t ev_fwd = nullptr, ev_adj = nullptr;
  ~sf2d_fwi() {
    if (fwd) cudaStreamSynchronize(fwd->stream);
    if (adj) cudaStreamSynchronize(adj->stream);
    if (ev_fwd) cudaEventDestroy(ev_fwd);
    if (ev_adj) cudaEventDestroy(ev_adj);
    for (void *p : allocs) cudaFree(p);
    sf2d_destroy(adj);
    sf2d_destroy(fwd);
  }
};

static int set_ctr(sf2d_solver *S, int idx, int value) {
  // pageable source: staged at call time, ordered on the stream
  SF2D_CUDA(cudaMemcpyAsync(S->ctr + idx, &value, sizeof(int), cudaMemcpyHostToDevice, S->stream));
  return SF2D_OK;
}

extern "C" int sf2d_fwi_create(const sf2d_elastic_desc *d, const float *rhostore, const float *kappastore,
                               int checkpoint_every, sf2d_fwi **out) {
  if (!d || !out || !rhostore || !kappastore) return fail(SF2D_ERR_INVALID, "null argument");
  *out = nullptr;
  if (checkpoint_every < 1) return fail(SF2D_ERR_INVALID, "checkpoint_every must be >= 1");
  if (d->time_scheme == 2) return fail(SF2D_ERR_INVALID, "the gradient is implemented for Newmark");
  if (d->nrec < 1 || d->nstep < 1) return fail(SF2D_ERR_INVALID, "the gradient needs receivers and steps");
  auto F = std::make_unique<sf2d_fwi>();
  int rc = sf2d_create_solver_internal(d, false, &F->fwd, nullptr);
  if (rc) return rc;
  // adjoint problem: the same medium, one pseudo-source per receiver component
  // whose weights are the receiver's Lagrange products (formed in FP32)
  const int nrec = d->nrec, nstep = d->nstep;
  std::vector<int> a_ispec(2 * nrec);
  std::vector<float> a_arr(static_cast<size_t>(2 * nrec) * 50, 0.f), a_stf(static_cast<size_t>(2 * nrec) * nstep, 0.f);
  for (int r = 0; r < nrec; ++r)
    for (int c = 0; c < 2; ++c) {
      a_ispec[2 * r + c] = d->rec_ispec[r];
      for (int j = 0; j < 5; ++j)
        for (int i = 0; i < 5; ++i) {
          const float h = static_cast<float>(d->hxir[r * 5 + i]) * static_cast<float>(d->hgammar[r * 5 + j]);
          a_arr[(static_cast<size_t>(2 * r + c) * 25 + j * 5 + i) * 2 + c] = h;
        }
    }
  sf2d_elastic_desc ad = *d;
  ad.nsrc = 2 * nrec;
  ad.src_ispec = a_ispec.data();
  ad.sourcearrays = a_arr.data();
  ad.stf = a_stf.data();
  ad.nstage = 1;
  // the adjoint field is recorded at the receivers too (write_seismograms.F90
  // records the adjoint wavefield in a kernel run)
  rc = sf2d_create_solver_internal(&ad, true, &F->adj, nullptr);
  if (rc) return rc;
  F->nstep = nstep;
  F->K = checkpoint_every;
  F->nseg = (nstep + checkpoint_every - 1) / checkpoint_every;
  F->nglob = d->nglob;
  F->nspec = d->nspec;
  F->nrec = nrec;
  F->dt = d->deltat;
  const size_t nl = static_cast<size_t>(d->nspec) * 25;
  F->ibool.assign(d->ibool, d->ibool + nl);
  F->rho.assign(rhostore, rhostore + nl);
  F->kappa.assign(kappastore, kappastore + nl);
  F->mu.assign(d->mustore, d->mustore + nl);
  auto dev_alloc = [&](void **p, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? SF2D_ERR_OOM : SF2D_ERR_CUDA,
                  std::string("cudaMalloc: ") + cudaGetErrorString(e));
    F->allocs.push_back(*p);
    return SF2D_OK;
  };
  const size_t ng = static_cast<size_t>(d->nglob);
  if ((rc = dev_alloc(reinterpret_cast<void **>(&F->frames), sizeof(float2) * ng * F->K))) return rc;
  if ((rc = dev_alloc(reinterpret_cast<void **>(&F->ckpt), sizeof(float2) * ng * 3 * F->nseg))) return rc;
  if (F->fwd->atten &&
      (rc = dev_alloc(reinterpret_cast<void **>(&F->ckpt_att), sizeof(float4) * F->fwd->nq * 3 * F->nseg)))
    return rc;
  SF2D_CUDA(cudaEventCreateWithFlags(&F->ev_fwd, cudaEventDisableTiming));
  SF2D_CUDA(cudaEventCreateWithFlags(&F->ev_adj, cudaEventDisableTiming));
  // frames are written only while the frame base is in range
  F->fwd->P.frames = F->frames;
  F->fwd->P.nframes = F->K;
  F->adj->P.kframes = F->frames;
  if ((rc = set_ctr(F->fwd, 3, 1 << 30))) return rc;
  SF2D_CUDA(cudaStreamSynchronize(F->fwd->stream));
  *out = F.release();
  return SF2D_OK;
}

extern "C" int sf2d_fwi_forward(sf2d_fwi *F, double *seismograms) {
  if (!F) return fail(SF2D_ERR_INVALID, "null handle");
  sf2d_solver *S = F->fwd;
  int rc = sf2d_reset_solver(S);
  if (rc) return rc;
  if ((rc = set_ctr(S, 3, 1 << 30))) return rc;
  const size_t ng = static_cast<size_t>(F->nglob);
  for (int seg = 0; seg < F->nseg; ++seg) {
    float2 *ck = F->ckpt + static_cast<size_t>(seg) * 3 * ng;
    SF2D_CUDA(cudaMemcpyAsync(ck, S->P.u, sizeof(float2) * ng, cudaMemcpyDeviceToDevice, S->stream));
    SF2D_CUDA(cudaMemcpyAsync(ck + ng, S->P.v, sizeof(float2) * ng, cudaMemcpyDeviceToDevice, S->stream));
    SF2D_CUDA(cudaMemcpyAsync(ck + 2 * ng, S->P.a, sizeof(float2) * ng, cudaMemcpyDeviceToDevice, S->stream));
    if (F->ckpt_att)
      SF2D_CUDA(cudaMemcpyAsync(F->ckpt_att + static_cast<size_t>(seg) * 3 * S->nq, S->P.att_state,
                                sizeof(float4) * 3 * S->nq, cudaMemcpyDeviceToDevice, S->stream));
    const int n = std::min(F->K, F->nstep - seg * F->K);
    if ((rc = sf2d_enqueue(S, n))) return rc;
  }
  const int st = sf2d_synchronize(S, 0.0);
  if (st && st != SF2D_ERR_UNSTABLE) return st;
  if (seismograms) {
    S->steps_done = 0;  // the seismogram buffer holds steps 0 .. nstep-1
    if ((rc = sf2d_copy_seismograms(S, 0, F->nstep, seismograms))) return rc;
  }
  return st;
}

extern "C" int sf2d_fwi_backward(sf2d_fwi *F, const float *adj_src, float *rho_kl, float *kappa_kl, float *mu_kl) {
  if (!F || !adj_src || !rho_kl || !kappa_kl || !mu_kl) return fail(SF2D_ERR_INVALID, "null argument");
  sf2d_solver *A = F->adj, *S = F->fwd;
  const int nstep = F->nstep, nrec = F->nrec;
  // time-reversed adjoint source per pseudo-source (2 per receiver)
  std::vector<float> stf(static_cast<size_t>(2 * nrec) * nstep);
  for (int r = 0; r < nrec; ++r)
    for (int c = 0; c < 2; ++c)
      for (int it = 0; it < nstep; ++it)
        stf[static_cast<size_t>(2 * r + c) * nstep + it] = adj_src[(static_cast<size_t>(r) * nstep + (nstep - 1 - it)) * 2 + c];
  SF2D_CUDA(cudaMemcpyAsync(A->d_stf, stf.data(), sizeof(float) * stf.size(), cudaMemcpyHostToDevice, A->stream));
  int rc = sf2d_reset_solver(A);
  if (rc) return rc;
  const size_t ng = static_cast<size_t>(F->nglob);
  std::vector<int> bases(static_cast<size_t>(2 * F->nseg));
  for (int seg = F->nseg - 1; seg >= 0; --seg) {
    const int s0 = seg * F->K;
    const int n = std::min(F->K, nstep - s0);
    // recompute the forward segment once the adjoint sweep no longer reads the frames
    SF2D_CUDA(cudaStreamWaitEvent(S->stream, F->ev_adj, 0));
    const float2 *ck = F->ckpt + static_cast<size_t>(seg) * 3 * ng;
    SF2D_CUDA(cudaMemcpyAsync(S->P.u, ck, sizeof(float2) * ng, cudaMemcpyDeviceToDevice, S->stream));
    SF2D_CUDA(cudaMemcpyAsync(S->P.v, ck + ng, sizeof(float2) * ng, cudaMemcpyDeviceToDevice, S->stream));
    SF2D_CUDA(cudaMemcpyAsync(S->P.a, ck + 2 * ng, sizeof(float2) * ng, cudaMemcpyDeviceToDevice, S->stream));
    if (F->ckpt_att)
      SF2D_CUDA(cudaMemcpyAsync(S->P.att_state, F->ckpt_att + static_cast<size_t>(seg) * 3 * S->nq,
                                sizeof(float4) * 3 * S->nq, cudaMemcpyDeviceToDevice, S->stream));
    if ((rc = set_ctr(S, 0, s0)) || (rc = set_ctr(S, 3, s0))) return rc;
    if ((rc = sf2d_enqueue(S, n))) return rc;
    SF2D_CUDA(cudaEventRecord(F->ev_fwd, S->stream));
    // adjoint steps nstep-s0-n .. nstep-s0-1 pair with frames n-1 .. 0
    SF2D_CUDA(cudaStreamWaitEvent(A->stream, F->ev_fwd, 0));
    if ((rc = set_ctr(A, 4, nstep - 1 - s0))) return rc;
    if ((rc = sf2d_enqueue(A, n))) return rc;
    SF2D_CUDA(cudaEventRecord(F->ev_adj, A->stream));
  }
  SF2D_CUDA(cudaStreamSynchronize(S->stream));
  const int st = sf2d_synchronize(A, 0.0);
  if (st && st != SF2D_ERR_UNSTABLE) return st;
  if ((rc = set_ctr(S, 3, 1 << 30))) return rc;
  // kernel sums back to the reference layout, then save_kernels_elastic scaling
  std::vector<float2> kmu(A->nq);
  std::vector<float> rg(ng);
  SF2D_CUDA(cudaMemcpy(kmu.data(), A->P.kmu_kl, sizeof(float2) * A->nq, cudaMemcpyDeviceToHost));
  SF2D_CUDA(cudaMemcpy(rg.data(), A->P.rho_kl_glob, sizeof(float) * ng, cudaMemcpyDeviceToHost));
  const sf2d::Tiling &T = A->T;
  const float dt = F->dt;
  for (int sl = 0; sl < F->nspec; ++sl) {
    const int e = T.elem_order[sl];
    for (int q = 0; q < 25; ++q) {
      const size_t p = static_cast<size_t>(e) * 25 + q;
      const float rsum = rg[T.glob2dev[F->ibool[p]]];
      const float2 km = kmu[static_cast<size_t>(sl) * 25 + q];
      rho_kl[p] = -F->rho[p] * dt * rsum;
      mu_kl[p] = -2.f * F->mu[p] * dt * km.y;
      kappa_kl[p] = -F->kappa[p] * dt * km.x;
    }
  }
  return st;
}

extern "C" int sf2d_fwi_enable_hessian(sf2d_fwi *F) {
  if (!F) return fail(SF2D_ERR_INVALID, "null handle");
  if (F->aframes) return SF2D_OK;
  const size_t ng = static_cast<size_t>(F->nglob);
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&F->aframes), sizeof(float2) * ng * F->K);
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? SF2D_ERR_OOM : SF2D_ERR_CUDA, "cudaMalloc (acceleration frames)");
  F->allocs.push_back(F->aframes);
  float2 *hess = nullptr;
  e = cudaMalloc(reinterpret_cast<void **>(&hess), sizeof(float2) * std::max<size_t>(ng, 1));
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? SF2D_ERR_OOM : SF2D_ERR_CUDA, "cudaMalloc (Hessian sums)");
  F->allocs.push_back(hess);
  F->fwd->P.aframes = F->aframes;
  F->adj->P.kaframes = F->aframes;
  F->adj->P.hess_glob = hess;
  // step graphs captured before hold the old parameters
  for (sf2d_solver *S : {F->fwd, F->adj})
    if (S->graph) {
      cudaGraphExecDestroy(S->graph);
      S->graph = nullptr;
    }
  return SF2D_OK;
}

extern "C" int sf2d_fwi_hessian(sf2d_fwi *F, float *hess1, float *hess2) {
  if (!F || !hess1 || !hess2) return fail(SF2D_ERR_INVALID, "null argument");
  sf2d_solver *A = F->adj;
  if (!A->P.hess_glob) return fail(SF2D_ERR_INVALID, "the Hessian was not enabled (sf2d_fwi_enable_hessian)");
  SF2D_CUDA(cudaStreamSynchronize(A->stream));
  std::vector<float2> h(F->nglob);
  SF2D_CUDA(cudaMemcpy(h.data(), A->P.hess_glob, sizeof(float2) * h.size(), cudaMemcpyDeviceToHost));
  const sf2d::Tiling &T = A->T;
  const size_t nl = static_cast<size_t>(F->nspec) * 25;
  for (size_t p = 0; p < nl; ++p) {
    const float2 v = h[T.glob2dev[F->ibool[p]]];
    hess1[p] = v.x * F->dt;
    hess2[p] = v.y * F->dt;
  }
  return SF2D_OK;
}

extern "C" int sf2d_fwi_adjoint_seismograms(sf2d_fwi *F, double *seismograms) {
  if (!F || !seismograms) return fail(SF2D_ERR_INVALID, "null argument");
  return sf2d_copy_seismograms(F->adj, 0, F->nstep, seismograms);
}

extern "C" int sf2d_fwi_kernel_sums(sf2d_fwi *F, float *rho_kl, float *kappa_kl, float *mu_kl) {
  if (!F || !rho_kl || !kappa_kl || !mu_kl) return fail(SF2D_ERR_INVALID, "null argument");
  const sf2d_solver *A = F->adj;
  SF2D_CUDA(cudaStreamSynchronize(A->stream));
  const size_t ng = static_cast<size_t>(F->nglob);
  std::vector<float2> kmu(A->nq);
  std::vector<float> rg(ng);
  SF2D_CUDA(cudaMemcpy(kmu.data(), A->P.kmu_kl, sizeof(float2) * A->nq, cudaMemcpyDeviceToHost));
  SF2D_CUDA(cudaMemcpy(rg.data(), A->P.rho_kl_glob, sizeof(float) * ng, cudaMemcpyDeviceToHost));
  const sf2d::Tiling &T = A->T;
  for (int sl = 0; sl < F->nspec; ++sl) {
    const int e = T.elem_order[sl];
    for (int q = 0; q < 25; ++q) {
      const size_t p = static_cast<size_t>(e) * 25 + q;
      const float2 km = kmu[static_cast<size_t>(sl) * 25 + q];
      rho_kl[p] = rg[T.glob2dev[F->ibool[p]]];
      kappa_kl[p] = km.x;
      mu_kl[p] = km.y;
    }
  }
  return SF2D_OK;
}

extern "C" int sf2d_fwi_adjoint_fields(sf2d_fwi *F, float *displ, float *veloc, float *accel) {
  if (!F) return fail(SF2D_ERR_INVALID, "null handle");
  return sf2d_get_fields(F->adj, displ, veloc, accel);
}

extern "C" int sf2d_fwi_destroy(sf2d_fwi *F) {
  delete F;
  return SF2D_OK;
}
