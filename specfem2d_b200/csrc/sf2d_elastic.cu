// Host runtime and C ABI of the elastic time-marching path (see
// sf2d_kernels.cuh for the device side and include/sf2d_b200.h for the API).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "sf2d_b200.h"
#include "sf2d_kernels.cuh"
#include "sf2d_tiler.h"

#include "sf2d_runtime.h"

namespace sf2d {
namespace {
thread_local std::string g_err;
}  // namespace
int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}
const char *last_error() { return g_err.c_str(); }
}  // namespace sf2d

extern "C" const char *sf2d_last_error(void) { return sf2d::last_error(); }

int sf2d_create_solver_internal(const sf2d_elastic_desc *d, bool kern, sf2d_solver **out, const uint8_t *late_elem) {
  using namespace sf2d;
  if (!d || !out) return fail(SF2D_ERR_INVALID, "null argument");
  *out = nullptr;
  if (d->nspec <= 0 || d->nglob <= 0 || !d->ibool || !d->xix || !d->xiz || !d->gammax || !d->gammaz ||
      !d->lambdastore || !d->mustore || !d->rmass_inverse || !d->hprime || !d->hprimewgll || !d->wxgll ||
      !d->wzgll)
    return fail(SF2D_ERR_INVALID, "missing mesh arrays");
  if (d->nstacey < 0 || d->nsrc < 0 || d->nrec < 0 || d->nstep < 0)
    return fail(SF2D_ERR_INVALID, "negative count");
  if (d->nsrc > 0 && (!d->src_ispec || !d->sourcearrays || !d->stf))
    return fail(SF2D_ERR_INVALID, "missing source arrays");
  if (d->nrec > 0 && (!d->rec_ispec || !d->hxir || !d->hgammar))
    return fail(SF2D_ERR_INVALID, "missing receiver arrays");
  if (d->nstacey > 0 && (!d->st_iglob || !d->st_nx || !d->st_nz || !d->st_w || !d->st_rho_vp || !d->st_rho_vs))
    return fail(SF2D_ERR_INVALID, "missing Stacey arrays");
  if (d->seismotype < 1 || d->seismotype > 3) return fail(SF2D_ERR_INVALID, "seismotype must be 1, 2 or 3");
  const int scheme = d->time_scheme == 0 ? 1 : d->time_scheme;
  if (scheme != 1 && scheme != 2) return fail(SF2D_ERR_INVALID, "time_scheme must be 1 (Newmark) or 2 (LDDRK)");
  const bool lddrk = scheme == 2;
  const int nstage = lddrk ? 6 : 1;
  if (lddrk && (!d->alpha_lddrk || !d->beta_lddrk)) return fail(SF2D_ERR_INVALID, "LDDRK needs alpha/beta");
  if (d->nsrc > 0 && d->nstage != nstage)
    return fail(SF2D_ERR_INVALID, "stf must hold one value per time step and stage");
  const bool aniso = d->ispec_is_anisotropic != nullptr;
  if (aniso && (!d->c11 || !d->c13 || !d->c15 || !d->c33 || !d->c35 || !d->c55))
    return fail(SF2D_ERR_INVALID, "missing anisotropic coefficients");
  const bool atten = lddrk ? (d->att_itau1 != nullptr) : (d->att_a1 != nullptr);
  if (atten && !lddrk && (!d->att_b1 || !d->att_a2 || !d->att_b2))
    return fail(SF2D_ERR_INVALID, "missing Newmark attenuation coefficients");
  if (atten && lddrk && (!d->att_phi1 || !d->att_itau2 || !d->att_phi2))
    return fail(SF2D_ERR_INVALID, "missing LDDRK attenuation coefficients");
  const bool pml = d->pml_region != nullptr;
  bool pml_visco = false;  // some layer elements attenuate
  std::vector<int> group;
  if (pml) {
    if (!d->pml_K_x || !d->pml_K_z || !d->pml_d_x || !d->pml_d_z || !d->pml_alpha_x || !d->pml_alpha_z ||
        !d->rhostore || !d->jacobian || !(d->pml_dt > 0.0))
      return fail(SF2D_ERR_INVALID, "missing CPML arrays");
    if (kern) return fail(SF2D_ERR_INVALID, "CPML layers are not part of the adjoint sweep");
    if (d->nstacey > 0) return fail(SF2D_ERR_INVALID, "CPML layers and Stacey conditions exclude each other");
    if (atten && lddrk)
      return fail(SF2D_ERR_INVALID, "CPML layers in an attenuating medium need Newmark time stepping");
    if (d->pml_visco && !atten) return fail(SF2D_ERR_INVALID, "pml_visco needs the attenuation coefficients");
    if (d->pml_visco && (!d->att_itau1 || !d->att_itau2 || !d->att_phi1 || !d->att_phi2 || !d->att_teps1 ||
                         !d->att_teps2 || !d->att_mu1 || !d->att_mu2))
      return fail(SF2D_ERR_INVALID, "missing Zener parameters of the attenuating CPML layer");
    if (d->npml_edge < 0 || (d->npml_edge > 0 && !d->pml_edge_iglob))
      return fail(SF2D_ERR_INVALID, "bad CPML edge list");
    for (int k = 0; k < d->npml_edge; ++k)
      if (d->pml_edge_iglob[k] < 0 || d->pml_edge_iglob[k] >= d->nglob)
        return fail(SF2D_ERR_INVALID, "CPML edge point out of range");
    group.assign(d->nspec, 0);
    for (int e = 0; e < d->nspec; ++e) {
      const int r = d->pml_region[e];
      if (r < 0 || r > 3) return fail(SF2D_ERR_INVALID, "CPML region must be 0 to 3");
      if (r > 0 && aniso && d->ispec_is_anisotropic[e]) return fail(SF2D_ERR_INVALID, "anisotropic element in a CPML layer");
      group[e] = r > 0 ? 2 : 0;
      if (r > 0 && d->pml_visco && d->pml_visco[e]) pml_visco = true;
    }
  }
  // tile groups: 0 early (no point another domain reads or writes), 1 late
  // (elements in late_elem: fluid-solid coupling), 2 CPML layer; the early
  // tiles of a coupled step may run beside the fluid step
  if (late_elem) {
    if (group.empty()) group.assign(d->nspec, 0);
    for (int e = 0; e < d->nspec; ++e)
      if (group[e] == 0 && late_elem[e]) group[e] = 1;
  }
  const bool grouped = !group.empty();

  auto *S = new sf2d_solver();
  std::unique_ptr<sf2d_solver> guard(S);
  const int te = d->tile_elems > 0 ? d->tile_elems : 64;
  const int group_te[3] = {te, te, d->pml_tile_elems > 0 ? d->pml_tile_elems : te};
  std::string err = build_tiling(d->nspec, d->nglob, d->ibool, d->centroid_xz, te, S->T,
                                 grouped ? group.data() : nullptr, grouped ? 3 : 1, grouped ? group_te : nullptr);
  if (!err.empty()) return fail(SF2D_ERR_INVALID, "tiling: " + err);
  const Tiling &T = S->T;
  S->late_tile0 = late_elem ? T.group_tile_begin[1] : 0;
  for (int k = 0; k < d->nsrc; ++k)
    if (d->src_ispec[k] < 0 || d->src_ispec[k] >= d->nspec) return fail(SF2D_ERR_INVALID, "source element out of range");
  for (int k = 0; k < d->nrec; ++k)
    if (d->rec_ispec[k] < 0 || d->rec_ispec[k] >= d->nspec) return fail(SF2D_ERR_INVALID, "receiver element out of range");
  for (int k = 0; k < d->nstacey; ++k)
    if (d->st_iglob[k] < 0 || d->st_iglob[k] >= d->nglob) return fail(SF2D_ERR_INVALID, "Stacey point out of range");

  // per-slot element data
  const size_t nq = static_cast<size_t>(d->nspec) * NGLL2;
  std::vector<float4> geo(nq);
  std::vector<float2> mat(nq);
  for (int s = 0; s < d->nspec; ++s) {
    const size_t src = static_cast<size_t>(T.elem_order[s]) * NGLL2;
    for (int q = 0; q < NGLL2; ++q) {
      geo[s * NGLL2 + q] = make_float4(d->xix[src + q], d->xiz[src + q], d->gammax[src + q], d->gammaz[src + q]);
      mat[s * NGLL2 + q] = make_float2(d->lambdastore[src + q], d->mustore[src + q]);
    }
  }
  // anisotropic blocks, in slot order
  std::vector<int> aniso_idx;
  std::vector<float4> c4;
  std::vector<float2> c2;
  if (aniso) {
    aniso_idx.assign(d->nspec, -1);
    int na = 0;
    for (int s = 0; s < d->nspec; ++s) {
      const int e = T.elem_order[s];
      if (!d->ispec_is_anisotropic[e]) continue;
      aniso_idx[s] = na++;
      const size_t src = static_cast<size_t>(e) * NGLL2;
      for (int q = 0; q < NGLL2; ++q) {
        c4.push_back(make_float4(d->c11[src + q], d->c13[src + q], d->c15[src + q], d->c33[src + q]));
        c2.push_back(make_float2(d->c35[src + q], d->c55[src + q]));
      }
    }
  }
  // attenuation coefficients: 3 float4 per element point, slot order
  std::vector<float4> att_coef;
  if (atten) {
    att_coef.resize(nq * 3);
    const float *k0 = lddrk ? d->att_itau1 : d->att_a1, *k1 = lddrk ? d->att_itau2 : d->att_a2;
    const float *k2 = lddrk ? d->att_phi1 : d->att_b1, *k3 = lddrk ? d->att_phi2 : d->att_b2;
    for (int s = 0; s < d->nspec; ++s) {
      const size_t src = static_cast<size_t>(T.elem_order[s]) * NGLL2;
      for (int q = 0; q < NGLL2; ++q)
        for (int l = 0; l < 3; ++l) {
          const size_t o = (src + q) * 3 + l;
          att_coef[(static_cast<size_t>(s) * NGLL2 + q) * 3 + l] = make_float4(k0[o], k1[o], k2[o], k3[o]);
        }
    }
  }
  std::vector<float2> rmass(d->nglob);
  for (int g = 0; g < d->nglob; ++g) {
    const int o = T.dev2glob[g];
    rmass[g] = make_float2(d->rmass_inverse[2 * o], d->rmass_inverse[2 * o + 1]);
  }
  // boundary entries grouped by tile, reference order inside a tile
  std::vector<TileInfo> tiles = T.tiles;
  std::vector<std::vector<int>> st_by_tile(T.ntiles), src_by_tile(T.ntiles), rec_by_tile(T.ntiles);
  // a Stacey point belongs to the tile of any element containing it; pick the first
  std::vector<int> glob_tile(d->nglob, -1);
  for (int e = 0; e < d->nspec; ++e)
    for (int q = 0; q < NGLL2; ++q) {
      const int g = d->ibool[static_cast<size_t>(e) * NGLL2 + q];
      if (glob_tile[g] < 0) glob_tile[g] = T.elem_tile[e];
    }
  for (int k = 0; k < d->nstacey; ++k) st_by_tile[glob_tile[d->st_iglob[k]]].push_back(k);
  for (int k = 0; k < d->nsrc; ++k) src_by_tile[T.elem_tile[d->src_ispec[k]]].push_back(k);
  for (int k = 0; k < d->nrec; ++k) rec_by_tile[T.elem_tile[d->rec_ispec[k]]].push_back(k);
  std::vector<int> st_local, src_local, src_id, rec_id, rec_dev;
  std::vector<float4> st_nw;
  std::vector<float2> st_rho, src_arr;
  std::vector<double> rec_h;
  for (int t = 0; t < T.ntiles; ++t) {
    tiles[t].st_off = static_cast<int>(st_local.size());
    for (int k : st_by_tile[t]) {
      st_local.push_back(T.local_id(t, d->st_iglob[k]));
      st_nw.push_back(make_float4(d->st_nx[k], d->st_nz[k], d->st_w[k], 0.f));
      st_rho.push_back(make_float2(d->st_rho_vp[k], d->st_rho_vs[k]));
    }
    tiles[t].st_n = static_cast<int>(st_local.size()) - tiles[t].st_off;
    tiles[t].src_off = static_cast<int>(src_local.size());
    for (int k : src_by_tile[t])
      for (int q = 0; q < NGLL2; ++q) {
        const int g = d->ibool[static_cast<size_t>(d->src_ispec[k]) * NGLL2 + q];
        src_local.push_back(T.local_id(t, g));
        src_id.push_back(k);
        src_arr.push_back(make_float2(d->sourcearrays[(static_cast<size_t>(k) * NGLL2 + q) * 2],
                                      d->sourcearrays[(static_cast<size_t>(k) * NGLL2 + q) * 2 + 1]));
      }
    tiles[t].src_n = static_cast<int>(src_local.size()) - tiles[t].src_off;
    tiles[t].rec_off = static_cast<int>(rec_id.size());
    for (int k : rec_by_tile[t]) {
      rec_id.push_back(k);
      for (int q = 0; q < NGLL2; ++q)
        rec_dev.push_back(T.glob2dev[d->ibool[static_cast<size_t>(d->rec_ispec[k]) * NGLL2 + q]]);
      for (int i = 0; i < 5; ++i) rec_h.push_back(d->hxir[k * 5 + i]);
      for (int j = 0; j < 5; ++j) rec_h.push_back(d->hgammar[k * 5 + j]);
    }
    tiles[t].rec_n = static_cast<int>(rec_id.size()) - tiles[t].rec_off;
  }
  // CPML layer: element slots [pml_slot0, nspec) (the last tiles), per-point
  // damping data, the outer edge as per-tile local lists and a shared-point mask
  S->pml_tile0 = grouped ? T.group_tile_begin[2] : T.ntiles;
  const int pml_slot0 = S->pml_tile0 < T.ntiles ? T.tiles[S->pml_tile0].elem_base : d->nspec;
  std::vector<int> pml_set_idx, edge_local, pml_vset_idx;
  std::vector<PmlSet> pml_sets;
  std::vector<PmlVisco> pml_vsets;
  std::vector<float> pml_rhoj;
  std::vector<uint8_t> sh_edge;
  if (pml) {
    pml_build_sets(d, T.elem_order, pml_slot0, d->nspec - pml_slot0, d->pml_dt, pml_sets, pml_set_idx);
    if (pml_visco)
      pml_build_visco_sets(d, T.elem_order, pml_slot0, d->nspec - pml_slot0, d->pml_dt, pml_vsets, pml_vset_idx);
    for (int s = pml_slot0; s < d->nspec; ++s)
      for (int q = 0; q < NGLL2; ++q) {
        const size_t p = static_cast<size_t>(T.elem_order[s]) * NGLL2 + q;
        pml_rhoj.push_back(d->rhostore[p] * d->jacobian[p]);
      }
    std::vector<uint8_t> on_edge(d->nglob, 0);
    for (int k = 0; k < d->npml_edge; ++k) on_edge[d->pml_edge_iglob[k]] = 1;
    for (int t = 0; t < T.ntiles; ++t) {
      tiles[t].edge_off = static_cast<int>(edge_local.size());
      for (const auto &gl : T.tile_glob_local[t])
        if (on_edge[gl.first]) edge_local.push_back(gl.second);
      tiles[t].edge_n = static_cast<int>(edge_local.size()) - tiles[t].edge_off;
    }
    sh_edge.assign(std::max(T.nshared, 1), 0);
    for (int s = 0; s < T.nshared; ++s) sh_edge[s] = on_edge[T.dev2glob[T.shared_begin + s]];
  }
  S->npml_q = static_cast<size_t>(d->nspec - pml_slot0) * NGLL2;
  std::vector<int4> bgroups;
  std::vector<int> bnd_idx;
  err = build_boundary_groups(tiles, st_local, {}, src_local, bgroups, bnd_idx);
  if (!err.empty()) return fail(SF2D_ERR_INVALID, err);
  S->h_st_local = st_local;
  S->h_src_local = src_local;

  // a solver split for a coupled step runs its streams at the highest
  // priority: the other domain's step, on the critical path, shares them, and
  // the early tiles beside it take the lowest
  if (late_elem) {
    int least = 0, greatest = 0;
    SF2D_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    S->priority = greatest;
  }
  SF2D_CUDA(cudaStreamCreateWithPriority(&S->stream, cudaStreamNonBlocking, S->priority));
  Params &P = S->P;
  int rc = 0;
  float2 *u, *v, *a;
  if ((rc = S->alloc(&u, d->nglob)) || (rc = S->alloc(&v, d->nglob)) || (rc = S->alloc(&a, d->nglob))) return rc;
  P.u = u;
  P.v = v;
  P.a = a;
  SF2D_CUDA(cudaMemset(u, 0, sizeof(float2) * d->nglob));
  SF2D_CUDA(cudaMemset(v, 0, sizeof(float2) * d->nglob));
  SF2D_CUDA(cudaMemset(a, 0, sizeof(float2) * d->nglob));
#define UP(field, type, vec) \
  do {                        \
    type *p_ = nullptr;       \
    if ((rc = S->upload(&p_, vec.data(), vec.size()))) return rc; \
    P.field = p_;             \
  } while (0)
  UP(rmass, float2, rmass);
  UP(tiles, TileInfo, tiles);
  UP(lib, uint16_t, T.lib);
  UP(geo, float4, geo);
  UP(mat, float2, mat);
  UP(sh_ids, int, T.sh_ids);
  UP(shp_off, int, T.shp_off);
  {
    std::vector<int> slot_pos(T.shp_slots.size());
    for (size_t k = 0; k < T.shp_slots.size(); ++k) slot_pos[T.shp_slots[k]] = static_cast<int>(k);
    UP(slot_pos, int, slot_pos);
  }
  UP(bgroups, int4, bgroups);
  UP(bnd_idx, int, bnd_idx);
  UP(st_local, int, st_local);
  UP(st_nw, float4, st_nw);
  UP(st_rho, float2, st_rho);
  UP(src_local, int, src_local);
  UP(src_id, int, src_id);
  UP(src_arr, float2, src_arr);
  UP(rec_id, int, rec_id);
  UP(rec_dev, int, rec_dev);
  UP(rec_h, double, rec_h);
  if (aniso) {
    UP(aniso_idx, int, aniso_idx);
    UP(c4, float4, c4);
    UP(c2, float2, c2);
  }
  if (atten) {
    UP(att_coef, float4, att_coef);
    float4 *st = nullptr;
    if ((rc = S->alloc(&st, nq * 3))) return rc;
    SF2D_CUDA(cudaMemset(st, 0, sizeof(float4) * nq * 3));
    P.att_state = st;
    if (lddrk) {
      float4 *stl = nullptr;
      if ((rc = S->alloc(&stl, nq * 3))) return rc;
      SF2D_CUDA(cudaMemset(stl, 0, sizeof(float4) * nq * 3));
      P.att_state_l = stl;
    }
  }
  if (lddrk) {
    float2 *ul, *vl;
    if ((rc = S->alloc(&ul, d->nglob)) || (rc = S->alloc(&vl, d->nglob))) return rc;
    SF2D_CUDA(cudaMemset(ul, 0, sizeof(float2) * d->nglob));
    SF2D_CUDA(cudaMemset(vl, 0, sizeof(float2) * d->nglob));
    P.uL = ul;
    P.vL = vl;
    for (int k = 0; k < 6; ++k) {
      P.alpha[k] = d->alpha_lddrk[k];
      P.beta[k] = d->beta_lddrk[k];
    }
  }
  if (pml) {
    UP(pml_sets, PmlSet, pml_sets);
    UP(pml_set_idx, int, pml_set_idx);
    UP(pml_rhoj, float, pml_rhoj);
    UP(edge_local, int, edge_local);
    UP(sh_edge, uint8_t, sh_edge);
    float4 *rm = nullptr;
    if ((rc = S->alloc(&rm, S->npml_q * 3))) return rc;
    SF2D_CUDA(cudaMemset(rm, 0, sizeof(float4) * std::max<size_t>(1, S->npml_q * 3)));
    P.pml_rm = rm;
    if (lddrk) {
      float4 *rml = nullptr;
      if ((rc = S->alloc(&rml, S->npml_q * 3))) return rc;
      SF2D_CUDA(cudaMemset(rml, 0, sizeof(float4) * std::max<size_t>(1, S->npml_q * 3)));
      P.pml_rm_l = rml;
    }
    if (pml_visco) {
      UP(pml_vsets, PmlVisco, pml_vsets);
      UP(pml_vset_idx, int, pml_vset_idx);
      float2 *vm = nullptr;
      if ((rc = S->alloc(&vm, S->npml_q * 9))) return rc;
      SF2D_CUDA(cudaMemset(vm, 0, sizeof(float2) * std::max<size_t>(1, S->npml_q * 9)));
      P.pml_vm = vm;
    }
    P.pml_slot0 = pml_slot0;
    P.DT = d->pml_dt;
    P.h_old = static_cast<double>(d->deltatsquareover2) / 2.0;
  }
#undef UP
  float2 *partial;
  if ((rc = S->alloc(&partial, T.sh_ids.size()))) return rc;
  P.partial = partial;
  std::vector<float> stf(static_cast<size_t>(d->nsrc) * d->nstep * nstage);
  if (d->nsrc) std::memcpy(stf.data(), d->stf, stf.size() * sizeof(float));
  float *d_stf;
  if ((rc = S->upload(&d_stf, stf.data(), stf.size()))) return rc;
  P.stf = d_stf;
  S->d_stf = d_stf;
  double *seis;
  if ((rc = S->alloc(&seis, static_cast<size_t>(d->nrec) * d->nstep * 2))) return rc;
  P.seis = seis;
  if (d->nrec && d->nstep) SF2D_CUDA(cudaMemset(seis, 0, sizeof(double) * d->nrec * d->nstep * 2));
  int *ctr;
  if ((rc = S->alloc(&ctr, 8))) return rc;
  SF2D_CUDA(cudaMemset(ctr, 0, 8 * sizeof(int)));
  P.d_step = ctr;
  P.d_status = ctr + 1;
  P.d_step_b = ctr + 2;
  P.frame_base = ctr + 3;
  P.kern_base = ctr + 4;
  P.nglob = d->nglob;
  S->ctr = ctr;
  S->kern = kern;
  S->atten = atten;
  S->nspec = d->nspec;
  S->nq = nq;
  if (kern) {
    float2 *kmu;
    float *rg;
    if ((rc = S->alloc(&kmu, nq)) || (rc = S->alloc(&rg, d->nglob))) return rc;
    SF2D_CUDA(cudaMemset(kmu, 0, sizeof(float2) * nq));
    SF2D_CUDA(cudaMemset(rg, 0, sizeof(float) * d->nglob));
    P.kmu_kl = kmu;
    P.rho_kl_glob = rg;
  }
  if ((rc = S->upload(&S->d_dev2glob, T.dev2glob.data(), T.dev2glob.size()))) return rc;
  if ((rc = S->alloc(&S->d_stage, d->nglob))) return rc;
  if ((rc = S->alloc(&S->d_norm, 1))) return rc;
  P.nstep_stf = d->nstep;
  P.nstage = nstage;
  P.nstep_seis = d->nstep;
  P.seismotype = d->seismotype;
  P.nrec = d->nrec;
  P.cosrot = d->cosrot;
  P.sinrot = d->sinrot;
  P.dt = d->deltat;
  P.dto2 = d->deltatover2;
  P.dt2o2 = d->deltatsquareover2;
  P.shared_begin = T.shared_begin;
  P.nshared = T.nshared;
  P.max_q = T.max_elems * NGLL2;
  P.max_local = T.max_local;
  for (int k = 0; k < 25; ++k) {
    P.hconst[k] = d->hprime[k];
    P.hconst[25 + k] = d->hprimewgll[k];
  }
  for (int k = 0; k < 5; ++k) {
    P.hconst[50 + k] = d->wxgll[k];
    P.hconst[55 + k] = d->wzgll[k];
  }
  S->smem = tile_smem_layout(P.max_q, P.max_local, kern).total;
  if (S->smem > 220 * 1024) return fail(SF2D_ERR_INVALID, "tile too large for shared memory");
  S->nt = d->threads_per_block > 0 ? d->threads_per_block : 256;
  if (S->nt != 128 && S->nt != 250 && S->nt != 256 && S->nt != 512)
    return fail(SF2D_ERR_INVALID, "threads_per_block must be 128, 250, 256 or 512");
  S->pml_nt = d->pml_threads_per_block > 0 ? d->pml_threads_per_block : S->nt;
  if (S->pml_nt != 128 && S->pml_nt != 250 && S->pml_nt != 256 && S->pml_nt != 512)
    return fail(SF2D_ERR_INVALID, "pml_threads_per_block must be 128, 250, 256 or 512");
  if (d->nrec > 0) {
    for (int t = 0; t < T.ntiles; ++t)
      if (tiles[t].rec_n > (t < S->pml_tile0 ? S->nt : S->pml_nt))
        return fail(SF2D_ERR_INVALID, "more receivers in one tile than threads per CTA");
  }
  S->tile_fn = pick_tile_kernel(S->nt, aniso, atten, lddrk, kern);
  if (pml) {
    // the layer's tiles may be smaller than the others: their kernel gets its
    // own shared-memory layout (the largest layer tile's)
    int pe = 0, pl = 0;
    for (int t = S->pml_tile0; t < T.ntiles; ++t) {
      pe = std::max(pe, tiles[t].nelem);
      pl = std::max(pl, tiles[t].n_int + tiles[t].n_sh);
    }
    S->pml_max_q = pe * NGLL2;
    S->pml_max_local = pl;
    S->pml_fn = pick_pml_kernel(S->pml_nt, lddrk, pml_visco);
    S->pml_smem = tile_smem_layout(S->pml_max_q, S->pml_max_local, false, true).total;
    if (S->pml_smem > 220 * 1024) return fail(SF2D_ERR_INVALID, "tile too large for shared memory");
  }
  S->lddrk = lddrk;
  S->nstage = nstage;
  if ((rc = S->make_side_stream())) return rc;
  {
    // The limit is a property of the kernel, shared by every solver in the
    // process: only ever raise it, or a later solver with smaller tiles would
    // make the launches of an earlier one with larger tiles fail.
    static std::mutex attr_mutex;
    std::lock_guard<std::mutex> lock(attr_mutex);
    const std::pair<TileKernel, size_t> fns[2] = {{S->tile_fn, S->smem}, {S->pml_fn, S->pml_smem}};
    for (const auto &fs : fns) {
      if (!fs.first) continue;
      cudaFuncAttributes fa;
      SF2D_CUDA(cudaFuncGetAttributes(&fa, fs.first));
      if (fa.maxDynamicSharedSizeBytes < static_cast<int>(fs.second))
        SF2D_CUDA(cudaFuncSetAttribute(fs.first, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(fs.second)));
    }
  }
  S->nglob = d->nglob;
  S->nrec = d->nrec;
  S->nstep_total = d->nstep;
  SF2D_CUDA(cudaStreamSynchronize(S->stream));
  *out = guard.release();
  return SF2D_OK;
}

extern "C" int sf2d_initialize_device(int rank, int *ndevices) {
  if (rank < 0) return fail(SF2D_ERR_INVALID, "rank must be >= 0");
  int n = 0;
  const cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) return fail(SF2D_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  if (n == 0) return fail(SF2D_ERR_CUDA, "there is no CUDA device");
  const int dev = rank % n;
  SF2D_CUDA(cudaSetDevice(dev));
  int got = -1;
  SF2D_CUDA(cudaGetDevice(&got));
  if (got != dev) return fail(SF2D_ERR_CUDA, "device id conflict after cudaSetDevice");
  if (ndevices) *ndevices = n;
  return SF2D_OK;
}

extern "C" int sf2d_elastic_create(const sf2d_elastic_desc *d, sf2d_solver **out) {
  return sf2d_create_solver_internal(d, false, out, nullptr);
}

extern "C" int sf2d_set_fields(sf2d_solver *S, const float *displ, const float *veloc, const float *accel) {
  if (!S) return fail(SF2D_ERR_INVALID, "null solver");
  float2 *dst[3] = {S->P.u, S->P.v, S->P.a};
  const float *src[3] = {displ, veloc, accel};
  const int n = S->nglob;
  for (int k = 0; k < 3; ++k) {
    if (!src[k]) {
      SF2D_CUDA(cudaMemsetAsync(dst[k], 0, sizeof(float2) * n, S->stream));
      continue;
    }
    SF2D_CUDA(cudaMemcpyAsync(S->d_stage, src[k], sizeof(float2) * n, cudaMemcpyHostToDevice, S->stream));
    sf2d::k_permute_in<<<(n + 255) / 256, 256, 0, S->stream>>>(S->d_stage, S->d_dev2glob, dst[k], n);
    SF2D_CUDA(cudaGetLastError());
  }
  SF2D_CUDA(cudaStreamSynchronize(S->stream));
  return SF2D_OK;
}

extern "C" int sf2d_get_fields(sf2d_solver *S, float *displ, float *veloc, float *accel) {
  if (!S) return fail(SF2D_ERR_INVALID, "null solver");
  const float2 *srcs[3] = {S->P.u, S->P.v, S->P.a};
  float *dst[3] = {displ, veloc, accel};
  const int n = S->nglob;
  for (int k = 0; k < 3; ++k) {
    if (!dst[k]) continue;
    sf2d::k_permute_out<<<(n + 255) / 256, 256, 0, S->stream>>>(srcs[k], S->d_dev2glob, S->d_stage, n);
    SF2D_CUDA(cudaGetLastError());
    SF2D_CUDA(cudaMemcpyAsync(dst[k], S->d_stage, sizeof(float2) * n, cudaMemcpyDeviceToHost, S->stream));
    SF2D_CUDA(cudaStreamSynchronize(S->stream));
  }
  return SF2D_OK;
}

extern "C" int sf2d_prepare(sf2d_solver *S) {
  if (!S) return fail(SF2D_ERR_INVALID, "null solver");
  const int K = S->chunk;
  if (S->graph && S->graph_steps == K) return SF2D_OK;
  if (S->graph) cudaGraphExecDestroy(S->graph);
  S->graph = nullptr;
  // capture records the chunk's launches without running them
  cudaGraph_t g;
  SF2D_CUDA(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
  S->launch_chunk(K);
  SF2D_CUDA(cudaStreamEndCapture(S->stream, &g));
  cudaError_t e = cudaGraphInstantiate(&S->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(SF2D_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  SF2D_CUDA(cudaGraphUpload(S->graph, S->stream));
  SF2D_CUDA(cudaStreamSynchronize(S->stream));
  S->graph_steps = K;
  return SF2D_OK;
}

extern "C" int sf2d_enqueue(sf2d_solver *S, int nstep) {
  if (!S || nstep < 0) return fail(SF2D_ERR_INVALID, "bad arguments");
  const int K = S->chunk;
  int done = 0;
  if (nstep >= K) {
    if (int rc = sf2d_prepare(S)) return rc;
    for (; done + K <= nstep; done += K) SF2D_CUDA(cudaGraphLaunch(S->graph, S->stream));
  }
  if (done < nstep) {
    int rc = S->launch_chunk(nstep - done);
    if (rc) return rc;
  }
  S->steps_done += nstep;
  return SF2D_OK;
}

extern "C" int sf2d_synchronize(sf2d_solver *S, double timeout_s) {
  if (!S) return fail(SF2D_ERR_INVALID, "null solver");
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(S->stream);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return fail(SF2D_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
    if (timeout_s > 0 &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_s)
      return fail(SF2D_ERR_TIMEOUT, "the time loop did not finish within the timeout (the steps keep running)");
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  int status = 0;
  SF2D_CUDA(cudaMemcpy(&status, S->P.d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (status) return fail(SF2D_ERR_UNSTABLE, "wavefield blew up (NaN or |u| > 1e25)");
  return SF2D_OK;
}

extern "C" int sf2d_set_members(sf2d_solver *S, const int *elem_member, int nmembers) {
  if (!S || !elem_member || nmembers < 1) return fail(SF2D_ERR_INVALID, "bad arguments");
  const sf2d::Tiling &T = S->T;
  std::vector<int> tm(T.ntiles), sm(T.nshared, -1);
  for (int t = 0; t < T.ntiles; ++t) {
    const sf2d::TileInfo &ti = T.tiles[t];
    int m = -1;
    for (int k = 0; k < ti.nelem; ++k) {
      const int e = T.elem_order[ti.elem_base + k];
      const int me = elem_member[e];
      if (me < 0 || me >= nmembers) return fail(SF2D_ERR_INVALID, "member id out of range");
      if (m >= 0 && me != m) return fail(SF2D_ERR_INVALID, "a tile holds elements of two members");
      m = me;
    }
    tm[t] = m;
    for (int k = 0; k < ti.n_sh; ++k) {
      const int s = T.sh_ids[ti.sh_off + k] - T.shared_begin;
      if (sm[s] >= 0 && sm[s] != m) return fail(SF2D_ERR_INVALID, "two members share a point");
      sm[s] = m;
    }
  }
  if (!S->P.member_status) {
    int *d_tm = nullptr, *d_sm = nullptr, *d_st = nullptr;
    if (int rc = S->alloc(&d_tm, tm.size())) return rc;
    if (int rc = S->alloc(&d_sm, sm.size())) return rc;
    if (int rc = S->alloc(&d_st, static_cast<size_t>(nmembers))) return rc;
    S->P.tile_member = d_tm;
    S->P.shared_member = d_sm;
    S->P.member_status = d_st;
    S->nmembers = nmembers;
  } else if (nmembers != S->nmembers) {
    return fail(SF2D_ERR_INVALID, "the member count is fixed by the first sf2d_set_members");
  }
  SF2D_CUDA(cudaMemcpy(const_cast<int *>(S->P.tile_member), tm.data(), sizeof(int) * tm.size(), cudaMemcpyHostToDevice));
  if (!sm.empty())
    SF2D_CUDA(cudaMemcpy(const_cast<int *>(S->P.shared_member), sm.data(), sizeof(int) * sm.size(),
                         cudaMemcpyHostToDevice));
  SF2D_CUDA(cudaMemset(S->P.member_status, 0, sizeof(int) * nmembers));
  // graphs captured before hold the old parameters
  if (S->graph) {
    cudaGraphExecDestroy(S->graph);
    S->graph = nullptr;
  }
  return SF2D_OK;
}

extern "C" int sf2d_member_status(sf2d_solver *S, int *status) {
  if (!S || !status) return fail(SF2D_ERR_INVALID, "bad arguments");
  if (!S->P.member_status) return fail(SF2D_ERR_INVALID, "no members: call sf2d_set_members first");
  SF2D_CUDA(cudaMemcpyAsync(status, S->P.member_status, sizeof(int) * S->nmembers, cudaMemcpyDeviceToHost, S->stream));
  SF2D_CUDA(cudaStreamSynchronize(S->stream));
  return SF2D_OK;
}

extern "C" int sf2d_copy_seismograms(sf2d_solver *S, int it0, int nstep, double *out) {
  if (!S || !out || it0 < 0 || nstep < 0 || it0 + nstep > S->nstep_total)
    return fail(SF2D_ERR_INVALID, "bad seismogram range");
  if (S->nrec == 0 || nstep == 0) return SF2D_OK;
  SF2D_CUDA(cudaMemcpy2DAsync(out, sizeof(double) * 2 * nstep, S->P.seis + static_cast<size_t>(it0) * 2,
                              sizeof(double) * 2 * S->nstep_total, sizeof(double) * 2 * nstep, S->nrec,
                              cudaMemcpyDeviceToHost, S->stream));
  SF2D_CUDA(cudaStreamSynchronize(S->stream));
  return SF2D_OK;
}

extern "C" int sf2d_run(sf2d_solver *S, int nstep, double *seismograms) {
  if (!S) return fail(SF2D_ERR_INVALID, "null solver");
  const int it0 = S->steps_done;
  if (seismograms && it0 + nstep > S->nstep_total)
    return fail(SF2D_ERR_INVALID, "run exceeds the seismogram buffer length");
  int rc = sf2d_enqueue(S, nstep);
  if (rc) return rc;
  const int st = sf2d_synchronize(S, 0.0);
  if (st && st != SF2D_ERR_UNSTABLE) return st;
  if (seismograms) {
    rc = sf2d_copy_seismograms(S, it0, nstep, seismograms);
    if (rc) return rc;
  }
  return st;
}

extern "C" int sf2d_get_norm(sf2d_solver *S, float *max_norm) {
  if (!S || !max_norm) return fail(SF2D_ERR_INVALID, "bad arguments");
  SF2D_CUDA(cudaMemsetAsync(S->d_norm, 0, sizeof(unsigned int), S->stream));
  sf2d::k_max_norm<<<256, 256, 0, S->stream>>>(S->P.u, S->nglob, S->d_norm);
  SF2D_CUDA(cudaGetLastError());
  unsigned int bits = 0;
  SF2D_CUDA(cudaMemcpyAsync(&bits, S->d_norm, sizeof(bits), cudaMemcpyDeviceToHost, S->stream));
  SF2D_CUDA(cudaStreamSynchronize(S->stream));
  std::memcpy(max_norm, &bits, sizeof(float));
  return SF2D_OK;
}

extern "C" int sf2d_step_index(sf2d_solver *S, int *it) {
  if (!S || !it) return fail(SF2D_ERR_INVALID, "bad arguments");
  *it = S->steps_done;
  return SF2D_OK;
}

extern "C" int sf2d_get_stream(sf2d_solver *S, void **stream) {
  if (!S || !stream) return fail(SF2D_ERR_INVALID, "bad arguments");
  *stream = S->stream;
  return SF2D_OK;
}

extern "C" int sf2d_time_kernels(sf2d_solver *S, int nstep, float *ms) {
  if (!S || !ms || nstep <= 0) return fail(SF2D_ERR_INVALID, "bad arguments");
  const int ns = S->nstage;
  std::vector<cudaEvent_t> ev(static_cast<size_t>(3) * nstep * ns);
  for (auto &e : ev) SF2D_CUDA(cudaEventCreate(&e));
  for (int k = 0; k < nstep; ++k)
    for (int st = 0; st < ns; ++st) {
      const size_t b = (static_cast<size_t>(k) * ns + st) * 3;
      SF2D_CUDA(cudaEventRecord(ev[b], S->stream));
      S->launch_tile(k > 0 && st == 0, st);
      SF2D_CUDA(cudaEventRecord(ev[b + 1], S->stream));
      S->launch_shared(st);
      SF2D_CUDA(cudaEventRecord(ev[b + 2], S->stream));
    }
  S->launch_receivers();
  SF2D_CUDA(cudaGetLastError());
  SF2D_CUDA(cudaStreamSynchronize(S->stream));
  double a = 0, bsum = 0;
  for (size_t k = 0; k < ev.size(); k += 3) {
    float x = 0, y = 0;
    cudaEventElapsedTime(&x, ev[k], ev[k + 1]);
    cudaEventElapsedTime(&y, ev[k + 1], ev[k + 2]);
    a += x;
    bsum += y;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  S->steps_done += nstep;
  const double nl = static_cast<double>(nstep) * ns;
  ms[0] = static_cast<float>(a / nl);
  ms[1] = static_cast<float>(bsum / nl);
  ms[2] = static_cast<float>((a + bsum) / nstep);
  return SF2D_OK;
}

extern "C" int sf2d_layout_info(sf2d_solver *S, long long *info) {
  if (!S || !info) return fail(SF2D_ERR_INVALID, "bad arguments");
  info[0] = S->T.ntiles;
  info[1] = S->T.nshared;
  info[2] = S->T.max_local;
  info[3] = S->T.max_elems;
  info[4] = static_cast<long long>(S->dev_bytes);
  info[5] = static_cast<long long>(S->smem);
  info[6] = S->nt;
  info[7] = static_cast<long long>(S->T.sh_ids.size());
  return SF2D_OK;
}

extern "C" int sf2d_launch_count(sf2d_solver *S, int nstep, long long *launches) {
  if (!S || !launches || nstep < 0) return fail(SF2D_ERR_INVALID, "bad arguments");
  const long long per_stage = S->tile_launches(0) + 1;
  const long long chunks = nstep / S->chunk + (nstep % S->chunk ? 1 : 0);
  *launches = per_stage * S->nstage * nstep + (S->nrec > 0 ? chunks : 0);
  return SF2D_OK;
}

extern "C" int sf2d_destroy(sf2d_solver *S) {
  if (!S) return SF2D_OK;
  cudaStreamSynchronize(S->stream);
  delete S;
  return SF2D_OK;
}

int sf2d_reset_solver(sf2d_solver *S) {
  const sf2d::Params &P = S->P;
  const size_t ng = static_cast<size_t>(S->nglob);
  SF2D_CUDA(cudaMemsetAsync(P.u, 0, sizeof(float2) * ng, S->stream));
  SF2D_CUDA(cudaMemsetAsync(P.v, 0, sizeof(float2) * ng, S->stream));
  SF2D_CUDA(cudaMemsetAsync(P.a, 0, sizeof(float2) * ng, S->stream));
  if (P.uL) SF2D_CUDA(cudaMemsetAsync(P.uL, 0, sizeof(float2) * ng, S->stream));
  if (P.vL) SF2D_CUDA(cudaMemsetAsync(P.vL, 0, sizeof(float2) * ng, S->stream));
  if (P.att_state) SF2D_CUDA(cudaMemsetAsync(P.att_state, 0, sizeof(float4) * S->nq * 3, S->stream));
  if (P.att_state_l) SF2D_CUDA(cudaMemsetAsync(P.att_state_l, 0, sizeof(float4) * S->nq * 3, S->stream));
  if (P.kmu_kl) SF2D_CUDA(cudaMemsetAsync(P.kmu_kl, 0, sizeof(float2) * S->nq, S->stream));
  if (P.rho_kl_glob) SF2D_CUDA(cudaMemsetAsync(P.rho_kl_glob, 0, sizeof(float) * ng, S->stream));
  if (P.hess_glob) SF2D_CUDA(cudaMemsetAsync(P.hess_glob, 0, sizeof(float2) * ng, S->stream));
  if (P.pml_rm) SF2D_CUDA(cudaMemsetAsync(P.pml_rm, 0, sizeof(float4) * S->npml_q * 3, S->stream));
  if (P.pml_rm_l) SF2D_CUDA(cudaMemsetAsync(P.pml_rm_l, 0, sizeof(float4) * S->npml_q * 3, S->stream));
  if (P.pml_vm) SF2D_CUDA(cudaMemsetAsync(P.pml_vm, 0, sizeof(float2) * S->npml_q * 9, S->stream));
  if (S->nrec && S->nstep_total)
    SF2D_CUDA(cudaMemsetAsync(P.seis, 0, sizeof(double) * S->nrec * S->nstep_total * 2, S->stream));
  SF2D_CUDA(cudaMemsetAsync(S->ctr, 0, 3 * sizeof(int), S->stream));
  S->steps_done = 0;
  return SF2D_OK;
}
