// Device side of the tile-staged acoustic (fluid) time step, NGLL = 5.
//
// The fluid is solved for the scalar potential chi with u = grad(chi) / rho
// and pressure p = -chi_dot_dot (compute_forces_viscoacoustic.f90:34-417).
// It uses the same tiling as the solid (sf2d_tiler.h) over the fluid
// elements, with its own device numbering of the fluid points.  One CTA per
// tile and time step (or LDDRK stage):
//   1. cp.async of local ibool, geometry, J/rho and chi, chi_dot,
//      chi_dot_dot of the tile's points into shared memory;
//   2. Newmark predictor (update_displacement_Newmark.F90:353-402) or a
//      cleared accumulator (LDDRK), free-surface points zeroed
//      (enforce_acoustic_free_surface.f90:35-96);
//   3. one thread, in reference order: Stacey chi_dd -= chi_d w / (rho vp)
//      (compute_stacey_acoustic.f90:78-180), the solid's normal displacement
//      chi_dd += w (u . n) (compute_coupling_acoustic_el.f90:60-283, with the
//      solid's predicted displacement formed here from its u, v, a), the
//      pressure sources chi_dd += s stf / kappa (compute_add_sources_acoustic.f90:49-75);
//   4. per GLL point: gradient through hprime, mapping, J/rho weak-form terms
//      (compute_forces_viscoacoustic.f90:105-238);
//   5. weighted transpose contraction with hprimewgll assembled colour by
//      colour (:306-322);
//   6. interior points: chi_dd *= rmass_inverse, corrector or LDDRK update
//      (update_displacement_Newmark.F90:631-662, update_displacement_LDDRK.F90:88-115),
//      free-surface zeroing, write-back; shared points: partial sums.
// A second kernel finishes the shared points in tile order.  The fluid step
// runs before the solid step, which then reads the new chi_dot_dot on the
// coupling edges (iterate_time.F90:183-196).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "sf2d_kernels.cuh"
#include "sf2d_tiler.h"

namespace sf2d {

struct AcParams {
  float *p, *pd, *pdd;        // chi, chi_dot, chi_dot_dot (fluid device order)
  float *pL, *pdL;            // LDDRK auxiliary fields
  const float *rmass;         // rmass_inverse_acoustic
  const uint8_t *free_mask;   // 1 on free-surface points
  const TileInfo *tiles;
  const uint16_t *lib;
  const float4 *geo;          // xix, xiz, gammax, gammaz (tile slot order)
  const float *fac;           // jacobian / rho formed in FP32
  const int *sh_ids;
  float *partial;
  const int *shp_off, *shp_slots;
  const int *st_local;
  const float2 *st_wr;        // Stacey weight (jacobian1D * w), rho * vp
  // coupling (fluid side): tile-local point, solid device point, (nx, nz, w, 0)
  const int *cpl_local, *cpl_src;
  const float4 *cpl_nw;
  const float2 *u_el, *v_el, *a_el;  // solid fields of the previous step (or stage)
  const int *src_local, *src_id;
  const float2 *src_sk;       // sourcearray value (hlagrange) and kappa per source point
  const float *stf;           // [isrc][it][stage]
  // receivers in fluid elements
  const int *rec_id, *rec_dev;
  const double *rec_h;        // hxir[5], hgammar[5]
  const float4 *rec_geo;      // 25 per receiver: xix, xiz, gammax, gammaz
  const float *rec_rho;       // 25 per receiver
  double *seis;               // [irec][it][2] for all receivers of the run
  int *d_step, *d_step_b;
  int *d_status;
  int nstep_stf, nstage, nstep_seis, seismotype, use_trick, nrec;
  double cosrot, sinrot;
  float dt, dto2, dt2o2;
  float alpha[6], beta[6];
  int shared_begin, nshared;
  int max_q, max_local;
  float hconst[60];           // hprime[25], hprimewgll[25], wxgll[5], wzgll[5]
};

// Shared-memory regions of one fluid tile, 16-byte aligned.
struct AcSmem {
  size_t geo, fac, p, pd, acc, h, lib, total;
};
__host__ __device__ inline AcSmem ac_smem_layout(int max_q, int max_local) {
  AcSmem L;
  size_t o = 0;
  L.geo = o;
  o = align16(o + static_cast<size_t>(max_q) * sizeof(float4));
  L.fac = o;
  o = align16(o + static_cast<size_t>(max_q) * sizeof(float));
  L.p = o;
  o = align16(o + static_cast<size_t>(max_local) * sizeof(float));
  L.pd = o;
  o = align16(o + static_cast<size_t>(max_local) * sizeof(float));
  L.acc = o;
  o = align16(o + static_cast<size_t>(max_local) * sizeof(float));
  L.h = o;
  o = align16(o + 64 * sizeof(float));
  L.lib = o;
  o = align16(o + static_cast<size_t>((max_q + 7) / 8 * 8) * sizeof(uint16_t));
  L.total = o;
  return L;
}

__device__ __forceinline__ void cp_async4(void *s, const void *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}

// Receiver in a fluid element (write_seismograms.F90:75-150): pressure
// -chi_dot_dot (or -chi with USE_TRICK_FOR_BETTER_PRESSURE) for seismotype 4
// (compute_pressure.f90:542-572); otherwise grad(field) / rho formed in double
// and stored in FP32 per GLL point (compute_vector_field.f90:143-207), then
// interpolated and rotated.
__device__ __forceinline__ void record_receiver_ac(const AcParams &A, int r, int step) {
  if (step < 0 || step >= A.nstep_seis) return;
  const int *dev = A.rec_dev + 25 * r;
  const double *h = A.rec_h + 10 * r;
  double vx = 0.0, vz = 0.0;
  double *out = A.seis + (static_cast<size_t>(A.rec_id[r]) * A.nstep_seis + step) * 2;
  if (A.seismotype == 4) {
    const float *f = A.use_trick ? A.p : A.pdd;
    for (int j = 0; j < 5; ++j)
      for (int i = 0; i < 5; ++i) {
        const double hl = static_cast<double>(static_cast<float>(h[i]) * static_cast<float>(h[5 + j]));
        vx += static_cast<double>(-f[dev[j * 5 + i]]) * hl;
      }
    out[0] = vx;
    out[1] = 0.0;
    return;
  }
  const float *f = A.seismotype == 2 ? A.pd : (A.seismotype == 3 ? A.pdd : A.p);
  for (int j = 0; j < 5; ++j)
    for (int i = 0; i < 5; ++i) {
      double t1 = 0.0, t2 = 0.0;
      for (int k = 0; k < 5; ++k) {
        t1 += static_cast<double>(f[dev[j * 5 + k]]) * static_cast<double>(A.hconst[5 * i + k]);
        t2 += static_cast<double>(f[dev[k * 5 + i]]) * static_cast<double>(A.hconst[5 * j + k]);
      }
      const float4 g = A.rec_geo[25 * r + j * 5 + i];
      const double rho = A.rec_rho[25 * r + j * 5 + i];
      const float fx = static_cast<float>((t1 * static_cast<double>(g.x) + t2 * static_cast<double>(g.z)) / rho);
      const float fz = static_cast<float>((t1 * static_cast<double>(g.y) + t2 * static_cast<double>(g.w)) / rho);
      const double hl = static_cast<double>(static_cast<float>(h[i]) * static_cast<float>(h[5 + j]));
      vx += static_cast<double>(fx) * hl;
      vz += static_cast<double>(fz) * hl;
    }
  out[0] = A.cosrot * vx + A.sinrot * vz;
  out[1] = -A.sinrot * vx + A.cosrot * vz;
}

template <int NT, bool LDDRK>
__global__ void __launch_bounds__(NT) k_acoustic_tile(const AcParams A, int record_prev, int stage) {
  extern __shared__ __align__(16) unsigned char smem[];
  const TileInfo &ti = A.tiles[blockIdx.x];
  const int tid = threadIdx.x;
  const int n_int = ti.n_int;
  const int n_sh = ti.n_sh;
  const int nl = n_int + n_sh;
  const int nq = ti.nelem * 25;
  const int ebase = ti.elem_base * 25;
  const int int_begin = ti.int_begin;
  const AcSmem L = ac_smem_layout(A.max_q, A.max_local);
  float4 *s_geo = reinterpret_cast<float4 *>(smem + L.geo);
  float *s_fac = reinterpret_cast<float *>(smem + L.fac);
  float *s_p = reinterpret_cast<float *>(smem + L.p);
  float *s_pd = reinterpret_cast<float *>(smem + L.pd);
  float *s_acc = reinterpret_cast<float *>(smem + L.acc);
  float *s_h = reinterpret_cast<float *>(smem + L.h);
  uint16_t *s_lib = reinterpret_cast<uint16_t *>(smem + L.lib);

  const int step = *A.d_step;
  if (blockIdx.x == 0 && tid == 0) *A.d_step_b = step;
  if (record_prev && tid < ti.rec_n) record_receiver_ac(A, ti.rec_off + tid, step - 1);

  // 1. loads
  {
    const uint4 *glib = reinterpret_cast<const uint4 *>(A.lib + ti.lib_off);
    const int nlib16 = (nq + 7) / 8;
    for (int k = tid; k < nlib16; k += NT) cp_async16(s_lib + 8 * k, glib + k);
    for (int f = tid; f < nq; f += NT) {
      cp_async16(s_geo + f, A.geo + ebase + f);
      cp_async4(s_fac + f, A.fac + ebase + f);
    }
    for (int l = tid; l < n_int; l += NT) {
      const int g = int_begin + l;
      cp_async4(s_p + l, A.p + g);
      cp_async4(s_pd + l, A.pd + g);
      if (!LDDRK) cp_async4(s_acc + l, A.pdd + g);
    }
    for (int k = tid; k < n_sh; k += NT) {
      const int g = A.sh_ids[ti.sh_off + k];
      cp_async4(s_p + n_int + k, A.p + g);
      cp_async4(s_pd + n_int + k, A.pd + g);
      if (!LDDRK) cp_async4(s_acc + n_int + k, A.pdd + g);
    }
    if (tid < 60) s_h[tid] = A.hconst[tid];
    cp_async_wait_all();
  }
  __syncthreads();

  // 2. predictor (or cleared accumulator), free surface
  const float dt = A.dt, dto2 = A.dto2, dt2o2 = A.dt2o2;
  for (int l = tid; l < nl; l += NT) {
    const int g = l < n_int ? int_begin + l : A.sh_ids[ti.sh_off + l - n_int];
    float p = s_p[l], pd = s_pd[l];
    if (!LDDRK) {
      const float pdd = s_acc[l];
      p = newmark_displ(p, pd, pdd, dt, dt2o2);
      pd = newmark_veloc(pd, pdd, dto2);
    }
    if (A.free_mask[g]) {
      p = 0.f;
      pd = 0.f;
    }
    s_p[l] = p;
    s_pd[l] = pd;
    s_acc[l] = 0.f;
  }
  __syncthreads();

  // 3. boundary terms, coupling and sources in reference order, one thread
  if (tid == 0) {
    for (int q = ti.st_off; q < ti.st_off + ti.st_n; ++q) {
      const int l = A.st_local[q];
      const float2 wr = A.st_wr[q];
      s_acc[l] = s_acc[l] - s_pd[l] * wr.x / wr.y;
    }
    for (int q = ti.cpl_off; q < ti.cpl_off + ti.cpl_n; ++q) {
      const int l = A.cpl_local[q];
      const int ge = A.cpl_src[q];
      const float4 nw = A.cpl_nw[q];
      float2 u = A.u_el[ge];
      if (!LDDRK) {
        const float2 v = A.v_el[ge], a = A.a_el[ge];
        u.x = newmark_displ(u.x, v.x, a.x, dt, dt2o2);
        u.y = newmark_displ(u.y, v.y, a.y, dt, dt2o2);
      }
      const float displ_n = u.x * nw.x + u.y * nw.y;
      s_acc[l] = s_acc[l] + nw.z * displ_n;
    }
    for (int q = ti.src_off; q < ti.src_off + ti.src_n; ++q) {
      const int l = A.src_local[q];
      const float f = step < A.nstep_stf
                          ? A.stf[(static_cast<size_t>(A.src_id[q]) * A.nstep_stf + step) * A.nstage + stage]
                          : 0.f;
      const float2 sk = A.src_sk[q];
      s_acc[l] = s_acc[l] + sk.x * f / sk.y;
    }
  }

  // 4. element pass 1: gradient of chi and the J/rho weak-form terms
  for (int f = tid; f < nq; f += NT) {
    const int e = f / 25;
    const int q = f - 25 * e;
    const int j = q / 5;
    const int i = q - 5 * j;
    const uint16_t *le = s_lib + 25 * e;
    float dxi = 0.f, dgam = 0.f;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      dxi += s_p[le[5 * j + k]] * s_h[5 * i + k];
      dgam += s_p[le[5 * k + i]] * s_h[5 * j + k];
    }
    const float4 g4 = s_geo[f];
    const float dxl = dxi * g4.x + dgam * g4.z;
    const float dzl = dxi * g4.y + dgam * g4.w;
    const float fac = s_fac[f];
    s_geo[f] = make_float4(fac * (g4.x * dxl + g4.y * dzl), fac * (g4.z * dxl + g4.w * dzl), 0.f, 0.f);
  }
  __syncthreads();

  // 5. weighted transpose contraction, colour by colour
  int cb = 0;
  for (int c = 0; c < ti.ncol; ++c) {
    const int ce = ti.col_end[c] * 25;
    for (int f = cb + tid; f < ce; f += NT) {
      const int e = f / 25;
      const int q = f - 25 * e;
      const int j = q / 5;
      const int i = q - 5 * j;
      const float4 *te = s_geo + 25 * e;
      float s1 = 0.f, s2 = 0.f;
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        s1 += te[5 * j + k].x * s_h[25 + 5 * k + i];
        s2 += te[5 * k + i].y * s_h[25 + 5 * k + j];
      }
      const int l = s_lib[f];
      s_acc[l] = s_acc[l] - (s_h[55 + j] * s1 + s_h[50 + i] * s2);
    }
    cb = ce;
    __syncthreads();
  }

  // 6. mass, corrector or LDDRK update, free surface, write-back
  bool bad = false;
  for (int l = tid; l < nl; l += NT) {
    const float acc = s_acc[l];
    if (l < n_int) {
      const int g = int_begin + l;
      float pdd = acc * A.rmass[g];
      float pd = s_pd[l], p = s_p[l];
      if (!LDDRK) {
        pd = newmark_veloc(pd, pdd, dto2);
      } else {
        const float al = A.alpha[stage], be = A.beta[stage];
        float pdl = A.pdL[g], pl = A.pL[g];
        pdl = al * pdl + dt * pdd;
        pl = al * pl + dt * pd;
        pd = pd + be * pdl;
        p = p + be * pl;
        A.pdL[g] = pdl;
        A.pL[g] = pl;
      }
      if (A.free_mask[g]) {
        p = 0.f;
        pd = 0.f;
        pdd = 0.f;
      }
      A.p[g] = p;
      A.pd[g] = pd;
      A.pdd[g] = pdd;
      bad |= !(fabsf(p) < 1e25f);
    } else {
      A.partial[ti.sh_off + l - n_int] = acc;
    }
  }
  if (bad) *A.d_status = 1;
}

template <bool LDDRK>
__global__ void __launch_bounds__(SHARED_NT) k_acoustic_shared(const AcParams A, int stage, int last_stage) {
  const int s = blockIdx.x * SHARED_NT + threadIdx.x;
  const int step = *A.d_step_b;
  if (s < A.nshared) {
    const int g = A.shared_begin + s;
    float p = A.p[g], pd = A.pd[g];
    if (!LDDRK) {
      const float pdd0 = A.pdd[g];
      p = newmark_displ(p, pd, pdd0, A.dt, A.dt2o2);
      pd = newmark_veloc(pd, pdd0, A.dto2);
    }
    const bool fs = A.free_mask[g] != 0;
    if (fs) {
      p = 0.f;
      pd = 0.f;
    }
    float acc = 0.f;
    for (int k = A.shp_off[s]; k < A.shp_off[s + 1]; ++k) acc += A.partial[A.shp_slots[k]];
    float pdd = acc * A.rmass[g];
    if (!LDDRK) {
      pd = newmark_veloc(pd, pdd, A.dto2);
    } else {
      const float al = A.alpha[stage], be = A.beta[stage];
      float pdl = A.pdL[g], pl = A.pL[g];
      pdl = al * pdl + A.dt * pdd;
      pl = al * pl + A.dt * pd;
      pd = pd + be * pdl;
      p = p + be * pl;
      A.pdL[g] = pdl;
      A.pL[g] = pl;
    }
    if (fs) {
      p = 0.f;
      pd = 0.f;
      pdd = 0.f;
    }
    A.p[g] = p;
    A.pd[g] = pd;
    A.pdd[g] = pdd;
    if (!(fabsf(p) < 1e25f)) *A.d_status = 1;
  }
  if (last_stage && blockIdx.x == 0 && threadIdx.x == 0) *A.d_step = step + 1;
}

// records the step before *d_step for every fluid receiver
static __global__ void k_acoustic_receivers(const AcParams A) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < A.nrec) record_receiver_ac(A, r, *A.d_step - 1);
}

}  // namespace sf2d
