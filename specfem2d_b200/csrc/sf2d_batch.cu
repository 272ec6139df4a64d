// Batches of shots and models: one packed mesh, one launch per step for all
// members (the GPU counterpart of NUMBER_OF_SIMULTANEOUS_RUNS,
// src/shared/parallel.F90:40-50, 1714).  Host code only: the members are
// concatenated into one sf2d_elastic_desc and run by the ordinary solver or
// gradient pair, whose tile kernels need no change because no tile mixes
// members.

#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "sf2d_runtime.h"

namespace {

constexpr int NQ = 25;
constexpr double kShift = 1.0e8;  // metres between consecutive members' element centres along x

template <typename T>
void append(std::vector<T> &dst, const T *src, size_t n) {
  if (n) dst.insert(dst.end(), src, src + n);
}

}  // namespace

struct sf2d_batch {
  sf2d_elastic_desc d{};  // the packed description (points into the vectors below)
  std::vector<int> ibool, st_iglob, src_ispec, rec_ispec, aniso_flag, elem_member;
  std::vector<float> xix, xiz, gammax, gammaz, lambda, mu, rmass, st_nx, st_nz, st_w, st_rvp, st_rvs, srcarr, stf;
  std::vector<float> c[6], att[8], rho, kappa;
  std::vector<double> centroid, hxir, hgammar;
  std::vector<int> member_model, model_elem_off;  // model of each member; elements of each model
  std::vector<long long> member_elem_off;
  int nmembers = 0, nmodels = 0, nrec = 0;
  sf2d_solver *S = nullptr;
  sf2d_fwi *F = nullptr;
  ~sf2d_batch() {
    if (S) sf2d_destroy(S);
    if (F) sf2d_fwi_destroy(F);
  }
};

extern "C" int sf2d_batch_create(const sf2d_elastic_desc *models, int nmodels, const sf2d_shot *shots, int nshots,
                                 const float *const *rhostore, const float *const *kappastore, int checkpoint_every,
                                 sf2d_batch **out) {
  using sf2d::fail;
  if (!models || nmodels < 1 || nshots < 0 || (nshots > 0 && !shots) || !out || checkpoint_every < 0)
    return fail(SF2D_ERR_INVALID, "sf2d_batch_create: bad arguments");
  *out = nullptr;
  const sf2d_elastic_desc &m0 = models[0];
  const bool kern = checkpoint_every > 0;
  if (kern && (!rhostore || !kappastore)) return fail(SF2D_ERR_INVALID, "a gradient batch needs rhostore and kappastore");
  const bool aniso = m0.ispec_is_anisotropic != nullptr, att_nm = m0.att_a1 != nullptr,
             att_lr = m0.att_itau1 != nullptr;
  for (int k = 0; k < nmodels; ++k) {
    const sf2d_elastic_desc &m = models[k];
    if (m.nstep != m0.nstep || m.deltat != m0.deltat || m.time_scheme != m0.time_scheme || m.nstage != m0.nstage)
      return fail(SF2D_ERR_INVALID, "batch models must share nstep, the time step and the time scheme");
    if (m.seismotype != m0.seismotype || m.cosrot != m0.cosrot || m.sinrot != m0.sinrot)
      return fail(SF2D_ERR_INVALID, "batch models must share the seismogram type and the receiver rotation");
    if ((m.ispec_is_anisotropic != nullptr) != aniso || (m.att_a1 != nullptr) != att_nm ||
        (m.att_itau1 != nullptr) != att_lr)
      return fail(SF2D_ERR_INVALID, "batch models must share their physics (anisotropy, attenuation)");
    if (m.pml_region) return fail(SF2D_ERR_INVALID, "CPML layers are not packed into batches");
    if (!m.centroid_xz) return fail(SF2D_ERR_INVALID, "batch models need element centres (centroid_xz)");
    if (m.nspec < 1 || m.nglob < 1 || !m.ibool) return fail(SF2D_ERR_INVALID, "empty batch model");
    if (kern && (!rhostore[k] || !kappastore[k])) return fail(SF2D_ERR_INVALID, "missing rhostore/kappastore");
  }
  if (kern && m0.time_scheme == 2) return fail(SF2D_ERR_INVALID, "gradient batches are Newmark only");
  const int nmem = nshots > 0 ? nshots : nmodels;
  for (int s = 0; s < nshots; ++s) {
    if (shots[s].model < 0 || shots[s].model >= nmodels) return fail(SF2D_ERR_INVALID, "shot model out of range");
    const sf2d_elastic_desc &m = models[shots[s].model];
    if (shots[s].nsrc < 0 || (shots[s].nsrc > 0 && (!shots[s].src_ispec || !shots[s].sourcearrays || !shots[s].stf)))
      return fail(SF2D_ERR_INVALID, "bad shot sources");
    for (int k = 0; k < shots[s].nsrc; ++k)
      if (shots[s].src_ispec[k] < 0 || shots[s].src_ispec[k] >= m.nspec)
        return fail(SF2D_ERR_INVALID, "shot source element out of range");
  }
  std::unique_ptr<sf2d_batch> B(new sf2d_batch());
  B->nmembers = nmem;
  B->nmodels = nmodels;
  B->model_elem_off.assign(nmodels + 1, 0);
  for (int k = 0; k < nmodels; ++k) B->model_elem_off[k + 1] = B->model_elem_off[k] + models[k].nspec;
  const int nstage = m0.nstage > 0 ? m0.nstage : 1;
  long long eoff = 0, goff = 0;
  B->member_elem_off.push_back(0);
  for (int mi = 0; mi < nmem; ++mi) {
    const int mk = nshots > 0 ? shots[mi].model : mi;
    const sf2d_elastic_desc &m = models[mk];
    B->member_model.push_back(mk);
    const size_t nl = static_cast<size_t>(m.nspec) * NQ;
    if (eoff + m.nspec > 2147483647LL || goff + m.nglob > 2147483647LL)
      return fail(SF2D_ERR_INVALID, "batch larger than 2^31 elements or points");
    for (size_t p = 0; p < nl; ++p) B->ibool.push_back(m.ibool[p] + static_cast<int>(goff));
    append(B->xix, m.xix, nl);
    append(B->xiz, m.xiz, nl);
    append(B->gammax, m.gammax, nl);
    append(B->gammaz, m.gammaz, nl);
    append(B->lambda, m.lambdastore, nl);
    append(B->mu, m.mustore, nl);
    append(B->rmass, m.rmass_inverse, 2 * static_cast<size_t>(m.nglob));
    for (int e = 0; e < m.nspec; ++e) {
      B->centroid.push_back(m.centroid_xz[2 * e] + kShift * mi);
      B->centroid.push_back(m.centroid_xz[2 * e + 1]);
      B->elem_member.push_back(mi);
    }
    for (int k = 0; k < m.nstacey; ++k) B->st_iglob.push_back(m.st_iglob[k] + static_cast<int>(goff));
    append(B->st_nx, m.st_nx, m.nstacey);
    append(B->st_nz, m.st_nz, m.nstacey);
    append(B->st_w, m.st_w, m.nstacey);
    append(B->st_rvp, m.st_rho_vp, m.nstacey);
    append(B->st_rvs, m.st_rho_vs, m.nstacey);
    // sources: the shot's, or the model's own
    const int nsrc = nshots > 0 ? shots[mi].nsrc : m.nsrc;
    const int *sis = nshots > 0 ? shots[mi].src_ispec : m.src_ispec;
    const float *sar = nshots > 0 ? shots[mi].sourcearrays : m.sourcearrays;
    const float *stf = nshots > 0 ? shots[mi].stf : m.stf;
    for (int k = 0; k < nsrc; ++k) B->src_ispec.push_back(sis[k] + static_cast<int>(eoff));
    append(B->srcarr, sar, static_cast<size_t>(nsrc) * NQ * 2);
    append(B->stf, stf, static_cast<size_t>(nsrc) * m0.nstep * nstage);
    for (int r = 0; r < m.nrec; ++r) B->rec_ispec.push_back(m.rec_ispec[r] + static_cast<int>(eoff));
    append(B->hxir, m.hxir, static_cast<size_t>(m.nrec) * 5);
    append(B->hgammar, m.hgammar, static_cast<size_t>(m.nrec) * 5);
    B->nrec += m.nrec;
    if (aniso) {
      append(B->aniso_flag, m.ispec_is_anisotropic, m.nspec);
      const float *cs[6] = {m.c11, m.c13, m.c15, m.c33, m.c35, m.c55};
      for (int k = 0; k < 6; ++k) append(B->c[k], cs[k], nl);
    }
    const float *as[8] = {m.att_a1, m.att_b1, m.att_a2, m.att_b2, m.att_itau1, m.att_phi1, m.att_itau2, m.att_phi2};
    for (int k = 0; k < 8; ++k)
      if (as[k]) append(B->att[k], as[k], nl * 3);
    if (kern) {
      append(B->rho, rhostore[mk], nl);
      append(B->kappa, kappastore[mk], nl);
    }
    eoff += m.nspec;
    goff += m.nglob;
    B->member_elem_off.push_back(eoff);
  }
  sf2d_elastic_desc &d = B->d;
  d = m0;  // time stepping, GLL tables, tile options
  // no CPML member: none of the layer's arrays of the first model carries over
  d.pml_region = nullptr;
  d.pml_K_x = d.pml_K_z = d.pml_d_x = d.pml_d_z = d.pml_alpha_x = d.pml_alpha_z = nullptr;
  d.rhostore = d.jacobian = nullptr;
  d.npml_edge = 0;
  d.pml_edge_iglob = nullptr;
  d.pml_visco = nullptr;
  d.att_teps1 = d.att_teps2 = d.att_mu1 = d.att_mu2 = nullptr;
  d.nspec = static_cast<int>(eoff);
  d.nglob = static_cast<int>(goff);
  d.ibool = B->ibool.data();
  d.xix = B->xix.data();
  d.xiz = B->xiz.data();
  d.gammax = B->gammax.data();
  d.gammaz = B->gammaz.data();
  d.lambdastore = B->lambda.data();
  d.mustore = B->mu.data();
  d.rmass_inverse = B->rmass.data();
  d.centroid_xz = B->centroid.data();
  d.nstacey = static_cast<int>(B->st_iglob.size());
  d.st_iglob = B->st_iglob.data();
  d.st_nx = B->st_nx.data();
  d.st_nz = B->st_nz.data();
  d.st_w = B->st_w.data();
  d.st_rho_vp = B->st_rvp.data();
  d.st_rho_vs = B->st_rvs.data();
  d.nsrc = static_cast<int>(B->src_ispec.size());
  d.src_ispec = B->src_ispec.data();
  d.sourcearrays = B->srcarr.data();
  d.stf = B->stf.data();
  d.nrec = B->nrec;
  d.rec_ispec = B->rec_ispec.data();
  d.hxir = B->hxir.data();
  d.hgammar = B->hgammar.data();
  if (aniso) {
    d.ispec_is_anisotropic = B->aniso_flag.data();
    d.c11 = B->c[0].data();
    d.c13 = B->c[1].data();
    d.c15 = B->c[2].data();
    d.c33 = B->c[3].data();
    d.c35 = B->c[4].data();
    d.c55 = B->c[5].data();
  }
  const float **ad[8] = {&d.att_a1, &d.att_b1, &d.att_a2, &d.att_b2, &d.att_itau1, &d.att_phi1, &d.att_itau2,
                         &d.att_phi2};
  for (int k = 0; k < 8; ++k) *ad[k] = B->att[k].empty() ? nullptr : B->att[k].data();
  int rc;
  if (kern) {
    rc = sf2d_fwi_create(&d, B->rho.data(), B->kappa.data(), checkpoint_every, &B->F);
  } else {
    rc = sf2d_elastic_create(&d, &B->S);
    if (!rc) rc = sf2d_set_members(B->S, B->elem_member.data(), nmem);
  }
  if (rc) return rc;
  *out = B.release();
  return SF2D_OK;
}

extern "C" int sf2d_batch_info(sf2d_batch *b, long long *info4) {
  if (!b || !info4) return sf2d::fail(SF2D_ERR_INVALID, "null argument");
  info4[0] = b->nmembers;
  info4[1] = b->d.nspec;
  info4[2] = b->d.nglob;
  info4[3] = b->nrec;
  return SF2D_OK;
}

extern "C" int sf2d_batch_run_forward(sf2d_batch *b, double *seismograms) {
  if (!b) return sf2d::fail(SF2D_ERR_INVALID, "null batch");
  if (b->F) return sf2d_fwi_forward(b->F, seismograms);
  int rc = sf2d_reset_solver(b->S);
  if (!rc) rc = sf2d_set_members(b->S, b->elem_member.data(), b->nmembers);  // clears the statuses
  if (rc) return rc;
  return sf2d_run(b->S, b->d.nstep, seismograms);
}

extern "C" int sf2d_batch_run_adjoint(sf2d_batch *b, const float *adj_src, float *rho_kl, float *kappa_kl,
                                      float *mu_kl) {
  if (!b || !adj_src || !rho_kl || !kappa_kl || !mu_kl) return sf2d::fail(SF2D_ERR_INVALID, "null argument");
  if (!b->F) return sf2d::fail(SF2D_ERR_INVALID, "a forward batch has no adjoint run");
  const size_t nl = static_cast<size_t>(b->d.nspec) * NQ;
  std::vector<float> rk(nl), kk(nl), mk(nl);
  const int st = sf2d_fwi_backward(b->F, adj_src, rk.data(), kk.data(), mk.data());
  if (st && st != SF2D_ERR_UNSTABLE) return st;
  // each member's kernels into its model's arrays, summed over the model's shots
  const size_t nm = static_cast<size_t>(b->model_elem_off[b->nmodels]) * NQ;
  std::memset(rho_kl, 0, sizeof(float) * nm);
  std::memset(kappa_kl, 0, sizeof(float) * nm);
  std::memset(mu_kl, 0, sizeof(float) * nm);
  for (int mi = 0; mi < b->nmembers; ++mi) {
    const size_t src = static_cast<size_t>(b->member_elem_off[mi]) * NQ;
    const size_t dst = static_cast<size_t>(b->model_elem_off[b->member_model[mi]]) * NQ;
    const size_t n = static_cast<size_t>(b->member_elem_off[mi + 1] - b->member_elem_off[mi]) * NQ;
    for (size_t p = 0; p < n; ++p) {
      rho_kl[dst + p] += rk[src + p];
      kappa_kl[dst + p] += kk[src + p];
      mu_kl[dst + p] += mk[src + p];
    }
  }
  return st;
}

extern "C" int sf2d_batch_member_status(sf2d_batch *b, int *status) {
  if (!b || !status) return sf2d::fail(SF2D_ERR_INVALID, "null argument");
  if (!b->S) return sf2d::fail(SF2D_ERR_INVALID, "member status is kept by forward batches");
  return sf2d_member_status(b->S, status);
}

extern "C" int sf2d_batch_destroy(sf2d_batch *b) {
  delete b;
  return SF2D_OK;
}
