// Device side of the tile-staged acoustic (fluid) time step, NGLL = 5.
//
// The fluid is solved for the scalar potential chi with u = grad(chi) / rho
// and pressure p = -chi_dot_dot (compute_forces_viscoacoustic.f90:34-417).
// It uses the same tiling as the solid (sf2d_tiler.h) over the fluid
// elements, with its own device numbering of the fluid points.  One CTA per
// tile and time step (or LDDRK stage):
//   1. cp.async of local ibool and chi, chi_dot, chi_dot_dot of the tile's
//      points into shared memory (geometry and J/rho are read from global
//      memory where they are used);
//   2. Newmark predictor (update_displacement_Newmark.F90:353-402) or a
//      cleared accumulator (LDDRK), free-surface points zeroed
//      (enforce_acoustic_free_surface.f90:35-96);
//   3. one thread per receiving point, in the reference's order at that
//      point: Stacey chi_dd -= chi_d w / (rho vp)
//      (compute_stacey_acoustic.f90:78-180), the solid's normal displacement
//      chi_dd += w (u . n) (compute_coupling_acoustic_el.f90:60-283, with the
//      solid's predicted displacement formed here from its u, v, a), the
//      pressure sources chi_dd += s stf / kappa (compute_add_sources_acoustic.f90:49-75);
//   4. derivative lines through hprime (one thread per element row or
//      column), per GLL point the mapping and J/rho weak-form terms
//      (compute_forces_viscoacoustic.f90:105-238), weighted transpose lines
//      with hprimewgll (:306-322);
//   5. assembly colour by colour;
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
  const int *shp_off, *slot_pos;  // point-major partial sums, as in the solid kernels
  const int *edge_local;      // per tile (edge_off, edge_n): local point | free_mask bits << 16
  const int4 *bgroups;        // per tile (grp_off, grp_n): point, first idx, Stacey | coupling << 8, sources
  const int *bnd_idx;         // entries of each group
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
  // CPML: elements of slots >= pml_slot0 lie in the layer (see Params)
  int pml_slot0;
  const PmlSet *pml_sets;     // coefficient sets of the layer
  const int *pml_set_idx;     // per PML point: its set
  const float *pml_jk;        // jacobian / kappa per PML point
  float2 *pml_rm;             // 3 per PML point: dchi_dx memory (1, 2), dchi_dz memory (1, 2), chi memory (1, 2)
  float2 *pml_rm_l;           // LDDRK copies
  float *pold;                // mid-step chi of this step for the solid's coupling terms (Newmark + CPML)
  double DT, h_old;
  // fluid-side coupling entries whose solid element lies in a CPML layer have
  // cpl_src = ~k: the displacement they see is formed before this kernel (k_cpl_pml_fluid)
  const float2 *cpl_pml_u;    // per layer entry k: the displacement to apply
  // adjoint run (SIMULATION_TYPE 3): the solid step runs first and the fluid
  // takes minus the solid's acceleration of this step as its coupling
  // displacement (compute_coupling_acoustic_el.f90:89-95)
  int adjoint;
  // segment recomputation: chi frames written after every step, frame = step - *pframe_base;
  // npframes frames (written by a forward run, read by an adjoint run)
  float *pframes;
  const int *pframe_base;
  int npframes;
  // adjoint sweep with kernel accumulation: forward chi frame = *kp_base - step;
  // per element point (slot order) its fluid point, rho and kappa, and the
  // sums of 1/rho grad(chi_adj) . grad(chi) dt and 1/kappa chi_adj_dd chi dt
  const float *kpframes;
  const int *kp_base;
  const int *slot_ibool;
  const float2 *slot_rk;
  float2 *kl_ac;
  int nslot_q, nglob_ac;
};

// Scalar line helpers of the fluid kernel (as line_derivs / line_weighted of
// the solid kernel): out[m] = sum_k f_k hprime[m][k]; in place
// t[m] = sum_k t_k hprimewgll[k][m]; constant-bank coefficients.
__device__ __forceinline__ void line_derivs_ac(const AcParams &A, const float *fld, const uint16_t *le, int st,
                                               float *out) {
  float in[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) in[k] = fld[le[st * k]];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    float d = 0.f;
#pragma unroll
    for (int k = 0; k < 5; ++k) d += in[k] * A.hconst[5 * m + k];
    out[st * m] = d;
  }
}
__device__ __forceinline__ void line_weighted_ac(const AcParams &A, float *buf, int st) {
  float in[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) in[k] = buf[st * k];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    float d = 0.f;
#pragma unroll
    for (int k = 0; k < 5; ++k) d += in[k] * A.hconst[25 + 5 * k + m];
    buf[st * m] = d;
  }
}

// free_mask bits: free surface, outer edge of a CPML layer; both zero chi,
// chi_dot and chi_dot_dot before and after the forces
constexpr uint8_t AC_FREE = 1, AC_EDGE = 2;

// Shared-memory regions of one fluid tile, 16-byte aligned (pold and pml only
// in CPML tiles).
struct AcSmem {
  size_t p, pd, acc, h, lib, mask, d1, d2, pold, od1, od2, pml, total;
};
__host__ __device__ inline AcSmem ac_smem_layout(int max_q, int max_local, bool pml = false) {
  AcSmem L;
  size_t o = 0;
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
  L.mask = o;  // uint8 per local point: free surface / layer edge bits
  o = align16(o + static_cast<size_t>(max_local));
  const size_t qb = align16(static_cast<size_t>(max_q) * sizeof(float));
  L.d1 = o;
  o += qb;
  L.d2 = o;
  o += qb;
  L.pold = o;
  if (pml) o = align16(o + static_cast<size_t>(max_local) * sizeof(float));
  L.od1 = o;
  if (pml) o += qb;
  L.od2 = o;
  if (pml) o += qb;
  L.pml = o;
  if (pml) o += qb;
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
  if (A.seismotype == 6) {
    // the potential itself (write_seismograms.F90:149-170)
    for (int j = 0; j < 5; ++j)
      for (int i = 0; i < 5; ++i) {
        const double hl = static_cast<double>(static_cast<float>(h[i]) * static_cast<float>(h[5 + j]));
        vx += static_cast<double>(A.p[dev[j * 5 + i]]) * hl;
      }
    out[0] = vx;
    out[1] = 0.0;
    return;
  }
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

// PML: the tiles of a CPML layer: mid-step chi + dt^2/4 chi_dot_dot, the
// gradient and potential memory variables, the modified gradient and the
// extra terms (pml_compute_memory_variables.f90:42-224,
// pml_compute_accel_contribution.f90:42-180).  Tiles [tile0, tile0 + gridDim.x).
template <int NT, bool LDDRK, bool PML = false>
__global__ void __launch_bounds__(NT, PML ? 768 / NT : 1536 / NT)
    k_acoustic_tile(const AcParams A, int record_prev, int stage, int tile0) {
  extern __shared__ __align__(16) unsigned char smem[];
  const TileInfo &ti = A.tiles[tile0 + blockIdx.x];
  const int tid = threadIdx.x;
  const int n_int = ti.n_int;
  const int n_sh = ti.n_sh;
  const int nl = n_int + n_sh;
  const int nq = ti.nelem * 25;
  const int ebase = ti.elem_base * 25;
  const int int_begin = ti.int_begin;
  const AcSmem L = ac_smem_layout(A.max_q, A.max_local, PML);
  float *s_pold = reinterpret_cast<float *>(smem + L.pold);
  float *s_pml = reinterpret_cast<float *>(smem + L.pml);
  float *s_d1 = reinterpret_cast<float *>(smem + L.d1);
  uint8_t *s_mask = reinterpret_cast<uint8_t *>(smem + L.mask);
  float *s_d2 = reinterpret_cast<float *>(smem + L.d2);
  float *s_od1 = reinterpret_cast<float *>(smem + L.od1);
  float *s_od2 = reinterpret_cast<float *>(smem + L.od2);
  float *s_p = reinterpret_cast<float *>(smem + L.p);
  float *s_pd = reinterpret_cast<float *>(smem + L.pd);
  float *s_acc = reinterpret_cast<float *>(smem + L.acc);
  float *s_h = reinterpret_cast<float *>(smem + L.h);
  uint16_t *s_lib = reinterpret_cast<uint16_t *>(smem + L.lib);

  const int step = *A.d_step;
  if (blockIdx.x == 0 && tid == 0) *A.d_step_b = step;
  // fluid receivers are recorded by k_acoustic_receivers after each step: their
  // double-precision gradient would hold registers through the whole tile
  (void)record_prev;

  // 1. loads
  {
    const uint4 *glib = reinterpret_cast<const uint4 *>(A.lib + ti.lib_off);
    const int nlib16 = (nq + 7) / 8;
    for (int k = tid; k < nlib16; k += NT) cp_async16(s_lib + 8 * k, glib + k);
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

  // 2. predictor (or cleared accumulator); then the tile's free-surface and
  //    layer-edge points (a per-tile list: no per-point mask loads) are zeroed
  //    and flagged for step 6
  const float dt = A.dt, dto2 = A.dto2, dt2o2 = A.dt2o2;
  for (int l = tid; l < nl; l += NT) {
    float p = s_p[l], pd = s_pd[l];
    if (!LDDRK) {
      const float pdd = s_acc[l];
      // mid-step potential (update_displacement_Newmark.F90:374-380)
      if (PML) s_pold[l] = static_cast<float>(static_cast<double>(p) + A.h_old * static_cast<double>(pdd));
      p = newmark_displ(p, pd, pdd, dt, dt2o2);
      pd = newmark_veloc(pd, pdd, dto2);
    }
    s_p[l] = p;
    s_pd[l] = pd;
    s_acc[l] = 0.f;
    s_mask[l] = 0;
  }
  __syncthreads();
  if (ti.edge_n > 0) {
    for (int k = tid; k < ti.edge_n; k += NT) {
      const int v = A.edge_local[ti.edge_off + k];
      const int l = v & 0xFFFF;
      const uint8_t m = static_cast<uint8_t>(v >> 16);
      s_p[l] = 0.f;
      s_pd[l] = 0.f;
      if (PML && !LDDRK && (m & AC_EDGE)) s_pold[l] = 0.f;  // the layer's edge (pml_boundary_acoustic)
      s_mask[l] = m;
    }
    __syncthreads();
  }

  // 3. boundary terms, coupling and sources: one thread per receiving point,
  //    in the reference's order at that point
  for (int gi = tid; gi < ti.grp_n; gi += NT) {
    const int4 g = A.bgroups[ti.grp_off + gi];
    const int l = g.x;
    const int *ix = A.bnd_idx + g.y;
    float acc = s_acc[l];
    const int nst = g.z & 255, ncp = g.z >> 8;
    for (int k = 0; k < nst; ++k) {
      const float2 wr = A.st_wr[ix[k]];
      acc = acc - s_pd[l] * wr.x / wr.y;
    }
    ix += nst;
    // the solid's normal displacement; a negative source names the CPML entry
    // ~src, whose displacement k_cpl_pml_fluid formed
    for (int k = 0; k < ncp; ++k) {
      const int q = ix[k];
      const int ge = A.cpl_src[q];
      const float4 nw = A.cpl_nw[q];
      float2 u;
      if (ge >= 0 && A.adjoint) {
        const float2 a = A.a_el[ge];
        u = make_float2(-a.x, -a.y);
      } else if (ge >= 0) {
        u = A.u_el[ge];
        if (!LDDRK) {
          const float2 v = A.v_el[ge], a = A.a_el[ge];
          u.x = newmark_displ(u.x, v.x, a.x, dt, dt2o2);
          u.y = newmark_displ(u.y, v.y, a.y, dt, dt2o2);
        }
      } else {
        u = A.cpl_pml_u[~ge];
      }
      const float displ_n = u.x * nw.x + u.y * nw.y;
      acc = acc + nw.z * displ_n;
    }
    ix += ncp;
    for (int k = 0; k < g.w; ++k) {
      const int q = ix[k];
      const float f = step < A.nstep_stf
                          ? A.stf[(static_cast<size_t>(A.src_id[q]) * A.nstep_stf + step) * A.nstage + stage]
                          : 0.f;
      const float2 sk = A.src_sk[q];
      acc = acc + sk.x * f / sk.y;
    }
    s_acc[l] = acc;
  }

  // the first point's geometry and J/rho are requested now (see the solid kernel)
  float4 g_next = make_float4(0.f, 0.f, 0.f, 0.f);
  float fac_next = 0.f;
  if (tid < nq) {
    g_next = __ldg(A.geo + ebase + tid);
    fac_next = __ldg(A.fac + ebase + tid);
  }

  // 4a. derivative lines: one thread per element row (xi) or column (gamma),
  //     hprime from the kernel's constant bank (see the solid kernel)
  const int nlines = 10 * ti.nelem;
  for (int t = tid, el = tid / 10; t < nlines; t += NT, el += NT / 10) {
    // with NT a multiple of 10 every thread keeps one line position r
    const int e = NT % 10 == 0 ? el : t / 10;
    const int r = NT % 10 == 0 ? tid % 10 : t - 10 * e;
    const int a0 = r < 5 ? 5 * r : r - 5;
    const int st = r < 5 ? 1 : 5;
    const uint16_t *le = s_lib + 25 * e + a0;
    const int o = 25 * e + a0;
    line_derivs_ac(A, s_p, le, st, (r < 5 ? s_d1 : s_d2) + o);
    if (PML && !LDDRK) line_derivs_ac(A, s_pold, le, st, (r < 5 ? s_od1 : s_od2) + o);
  }
  __syncthreads();

  // 4b. per GLL point: mapping and the J/rho weak-form terms (t1, t2 overwrite
  //     the derivatives), the layer's memory variables in CPML tiles
  constexpr bool FIXQ = NT % 25 == 0;  // every thread keeps one GLL position
  const int q0 = tid % 25, j0 = q0 / 5, i0 = q0 - 5 * j0;
  for (int f = tid, ef = tid / 25; f < nq; f += NT, ef += NT / 25) {
    const int e = FIXQ ? ef : f / 25;
    const int q = FIXQ ? q0 : f - 25 * e;
    const int j = FIXQ ? j0 : q / 5;
    const int i = FIXQ ? i0 : q - 5 * j;
    const uint16_t *le = s_lib + 25 * e;
    const float dxi = s_d1[f], dgam = s_d2[f];
    // geometry from global memory, the next point's requested before this one is computed
    const float4 g4 = g_next;
    const float fac = fac_next;
    if (f + NT < nq) {
      g_next = __ldg(A.geo + ebase + f + NT);
      fac_next = __ldg(A.fac + ebase + f + NT);
    }
    float dxl = dxi * g4.x + dgam * g4.z;
    float dzl = dxi * g4.y + dgam * g4.w;
    if (PML) {
      const int ps = ebase + f - 25 * A.pml_slot0;
      const PmlSet &c = A.pml_sets[A.pml_set_idx[ps]];
      float dxl_o = 0.f, dzl_o = 0.f;
      if (!LDDRK) {
        const float oxi = s_od1[f], og = s_od2[f];
        dxl_o = oxi * g4.x + og * g4.z;
        dzl_o = oxi * g4.y + og * g4.w;
      }
      const PmlConv &cax = c.cax, &caz = c.caz, &cbx = c.cbx, &cbz = c.cbz;
      const PmlLik &zx = c.zx, &xz = c.xz;  // poles (alpha_z, beta_x) and (alpha_x, beta_z)
      float2 rx = A.pml_rm[3 * ps], rz = A.pml_rm[3 * ps + 1], rp = A.pml_rm[3 * ps + 2];
      float2 lx = make_float2(0.f, 0.f), lz = lx, lp = lx;
      if (LDDRK) {
        lx = A.pml_rm_l[3 * ps];
        lz = A.pml_rm_l[3 * ps + 1];
        lp = A.pml_rm_l[3 * ps + 2];
      }
      const float al = A.alpha[stage], be = A.beta[stage];
      pml_update<LDDRK>(rx.x, lx.x, caz, c.az, dxl, dxl_o, al, be, dt);
      pml_update<LDDRK>(rx.y, lx.y, cbx, c.bx, dxl, dxl_o, al, be, dt);
      pml_update<LDDRK>(rz.x, lz.x, cax, c.ax, dzl, dzl_o, al, be, dt);
      pml_update<LDDRK>(rz.y, lz.y, cbz, c.bz, dzl, dzl_o, al, be, dt);
      dxl = static_cast<float>(zx.A0 * dxl + zx.A1 * rx.x + zx.A2 * rx.y);
      dzl = static_cast<float>(xz.A0 * dzl + xz.A1 * rz.x + xz.A2 * rz.y);
      // the layer's terms at this point (pml_compute_accel_contribution.f90:42-180)
      const PmlL &Lc = c.l;  // poles alpha_x, alpha_z
      const int lq = le[q];
      const float pq = s_p[lq], pdq = s_pd[lq];
      const float po = LDDRK ? 0.f : s_pold[lq];
      pml_update<LDDRK>(rp.x, lp.x, cax, c.ax, pq, po, al, be, dt);
      pml_update<LDDRK>(rp.y, lp.y, caz, c.az, pq, po, al, be, dt);
      const float wwf = s_h[50 + i] * s_h[55 + j] * A.pml_jk[ps];
      s_pml[f] = static_cast<float>(static_cast<double>(wwf) *
                                    (Lc.A1 * pdq + Lc.A2 * pq + Lc.A3 * rp.x + Lc.A4 * rp.y));
      A.pml_rm[3 * ps] = rx;
      A.pml_rm[3 * ps + 1] = rz;
      A.pml_rm[3 * ps + 2] = rp;
      if (LDDRK) {
        A.pml_rm_l[3 * ps] = lx;
        A.pml_rm_l[3 * ps + 1] = lz;
        A.pml_rm_l[3 * ps + 2] = lp;
      }
    }
    s_d1[f] = fac * (g4.x * dxl + g4.y * dzl);
    s_d2[f] = fac * (g4.z * dxl + g4.w * dzl);
  }
  __syncthreads();

  // 4c. weighted transpose lines, in place
  for (int t = tid, el = tid / 10; t < nlines; t += NT, el += NT / 10) {
    // with NT a multiple of 10 every thread keeps one line position r
    const int e = NT % 10 == 0 ? el : t / 10;
    const int r = NT % 10 == 0 ? tid % 10 : t - 10 * e;
    const int a0 = r < 5 ? 5 * r : r - 5;
    line_weighted_ac(A, (r < 5 ? s_d1 : s_d2) + 25 * e + a0, r < 5 ? 1 : 5);
  }
  __syncthreads();

  // 5. assembly, colour by colour: chi_dd -= wz * row term + wx * column term
  int cb = 0;
  for (int c = 0; c < ti.ncol; ++c) {
    const int ce = ti.col_end[c] * 25;
    for (int f = cb + tid, ef = (cb + tid) / 25; f < ce; f += NT, ef += NT / 25) {  // cb: a multiple of 25
      const int e = FIXQ ? ef : f / 25;
      const int q = FIXQ ? q0 : f - 25 * e;
      const int j = FIXQ ? j0 : q / 5;
      const int i = FIXQ ? i0 : q - 5 * j;
      const int l = s_lib[f];
      float acc = s_acc[l] - (s_h[55 + j] * s_d1[f] + s_h[50 + i] * s_d2[f]);
      if (PML) acc = acc - s_pml[f];
      s_acc[l] = acc;
    }
    cb = ce;
    __syncthreads();
  }

  // 6. mass, corrector or LDDRK update, free surface, write-back (each
  //    point's rmass, mask or slot requested one iteration ahead)
  bool bad = false;
  float rm_next = 0.f;
  int sp_next = 0;
  if (tid < n_int)
    rm_next = A.rmass[int_begin + tid];
  else if (tid < nl)
    sp_next = A.slot_pos[ti.sh_off + tid - n_int];
  for (int l = tid; l < nl; l += NT) {
    const float acc = s_acc[l];
    const float rm = rm_next;
    const uint8_t fm = s_mask[l];
    const int sp = sp_next;
    if (l + NT < n_int) {
      rm_next = A.rmass[int_begin + l + NT];
    } else if (l + NT < nl) {
      sp_next = A.slot_pos[ti.sh_off + l + NT - n_int];
    }
    if (l < n_int) {
      const int g = int_begin + l;
      float pdd = acc * rm;
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
      if (fm) {
        p = 0.f;
        pd = 0.f;
        pdd = 0.f;
      }
      A.p[g] = p;
      A.pd[g] = pd;
      A.pdd[g] = pdd;
      if (PML && !LDDRK && A.pold) A.pold[g] = s_pold[l];
      bad |= !(fabsf(p) < 1e25f);
    } else {
      A.partial[sp] = acc;
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
    const uint8_t m = A.free_mask[g];
    if (!LDDRK) {
      const float pdd0 = A.pdd[g];
      if (A.pold)
        A.pold[g] = (m & AC_EDGE) ? 0.f
                                  : static_cast<float>(static_cast<double>(p) + A.h_old * static_cast<double>(pdd0));
      p = newmark_displ(p, pd, pdd0, A.dt, A.dt2o2);
      pd = newmark_veloc(pd, pdd0, A.dto2);
    }
    const bool fs = m != 0;
    if (fs) {
      p = 0.f;
      pd = 0.f;
    }
    float acc = 0.f;
    for (int k = A.shp_off[s]; k < A.shp_off[s + 1]; ++k) acc += A.partial[k];
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

// Coupling entries next to a CPML layer, one thread per entry, once per step
// or LDDRK stage.  Both memory variables advance here, so the tile kernels
// only read the result.
struct CplPml {
  int n;              // layer entries
  const int *point;   // fluid side: solid device point; solid side: fluid device point
  const double *coef; // fluid side 6 per entry: A0, A1, c0, c1, c2, bb; solid side 8: A0..A3, c0, c1, c2, bb
  float *rm, *rm_l;   // fluid side 2 per entry (x, z), solid side 1
  float *out;         // fluid side float2 displacement, solid side pressure
};

// Fluid side (compute_coupling_acoustic_el.f90:111-160): the solid's predicted
// displacement u as A0 u + A1 r, r the memory variable of u driven by the
// mid-step displacement u0 + dt^2/4 a0 (Newmark), for a solid element in a layer.
template <bool LDDRK>
__global__ void k_cpl_pml_fluid(const CplPml C, const float2 *u_el, const float2 *v_el, const float2 *a_el, float dt,
                                float dt2o2, double h_old, float al, float be) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= C.n) return;
  const int ge = C.point[k];
  const float2 u0 = u_el[ge];
  float2 u = u0, uo = make_float2(0.f, 0.f);
  if (!LDDRK) {
    const float2 v = v_el[ge], a0 = a_el[ge];
    u.x = newmark_displ(u0.x, v.x, a0.x, dt, dt2o2);
    u.y = newmark_displ(u0.y, v.y, a0.y, dt, dt2o2);
    uo = make_float2(static_cast<float>(static_cast<double>(u0.x) + h_old * static_cast<double>(a0.x)),
                     static_cast<float>(static_cast<double>(u0.y) + h_old * static_cast<double>(a0.y)));
  }
  const double *c = C.coef + 6 * k;
  const PmlConv cv{c[2], c[3], c[4]};
  float2 rf = make_float2(C.rm[2 * k], C.rm[2 * k + 1]);
  float2 rfl = LDDRK ? make_float2(C.rm_l[2 * k], C.rm_l[2 * k + 1]) : make_float2(0.f, 0.f);
  pml_update<LDDRK>(rf.x, rfl.x, cv, c[5], u.x, uo.x, al, be, dt);
  pml_update<LDDRK>(rf.y, rfl.y, cv, c[5], u.y, uo.y, al, be, dt);
  C.rm[2 * k] = rf.x;
  C.rm[2 * k + 1] = rf.y;
  if (LDDRK) {
    C.rm_l[2 * k] = rfl.x;
    C.rm_l[2 * k + 1] = rfl.y;
  }
  C.out[2 * k] = static_cast<float>(c[0] * static_cast<double>(u.x) + c[1] * static_cast<double>(rf.x));
  C.out[2 * k + 1] = static_cast<float>(c[0] * static_cast<double>(u.y) + c[1] * static_cast<double>(rf.y));
}

// Solid side (compute_coupling_viscoelastic_ac.f90:105-150): the pressure
// -(A0 chi_dd + A1 chi_d + A2 chi + A3 r) of a fluid element in a layer, r the
// memory variable of chi driven by the mid-step chi (Newmark); runs after the
// fluid step, before the solid tile kernel.
template <bool LDDRK>
__global__ void k_cpl_pml_solid(const CplPml C, const float *p, const float *pd, const float *pdd, const float *pold,
                                float dt, float al, float be) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= C.n) return;
  const int ga = C.point[k];
  const double *c = C.coef + 8 * k;
  const PmlConv cv{c[4], c[5], c[6]};
  float r = C.rm[k];
  float rl = LDDRK ? C.rm_l[k] : 0.f;
  const float pot = p[ga];
  pml_update<LDDRK>(r, rl, cv, c[7], pot, LDDRK ? 0.f : pold[ga], al, be, dt);
  C.rm[k] = r;
  if (LDDRK) C.rm_l[k] = rl;
  C.out[k] = static_cast<float>(-(c[0] * static_cast<double>(pdd[ga]) + c[1] * static_cast<double>(pd[ga]) +
                                  c[2] * static_cast<double>(pot) + c[3] * static_cast<double>(r)));
}

// records the step before *d_step for every fluid receiver (launched after the
// last stage of every step)
static __global__ void k_acoustic_receivers(const AcParams A) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < A.nrec) record_receiver_ac(A, r, *A.d_step - 1);
}

// After a finished step (*d_step already advanced): chi into its frame when the
// frame lies in [0, npframes).
static __global__ void k_fluid_frame(const AcParams A) {
  const int fi = (*A.d_step - 1) - *A.pframe_base;
  if (fi < 0 || fi >= A.npframes) return;
  float *dst = A.pframes + static_cast<size_t>(fi) * A.nglob_ac;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < A.nglob_ac; g += gridDim.x * blockDim.x) dst[g] = A.p[g];
}

// compute_kernels_ac (compute_kernels.f90:293-449; the GPU form,
// compute_kernels_acoustic_cuda in src/gpu/compute_kernels_cuda.cu), after a
// finished adjoint step: at every fluid element point the gradients of the
// adjoint chi and of the forward chi of the paired frame (derivative lines in
// FP32, the mapping applied in double and stored in FP32), and
//   sum.x += 1/rho (grad chi_adj . grad chi) dt,  sum.y += 1/kappa chi_adj_dd chi dt.
static __global__ void k_fluid_kernels(const AcParams A) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= A.nslot_q) return;
  const int fi = *A.kp_base - (*A.d_step - 1);
  if (fi < 0 || fi >= A.npframes) return;  // no paired frame: nothing accumulates
  const float *b = A.kpframes + static_cast<size_t>(fi) * A.nglob_ac;
  const int e0 = q - q % 25, i = q % 5, j = (q % 25) / 5;
  float t1 = 0.f, t2 = 0.f, b1 = 0.f, b2 = 0.f;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const int gr = A.slot_ibool[e0 + j * 5 + k], gc = A.slot_ibool[e0 + k * 5 + i];
    t1 = t1 + A.p[gr] * A.hconst[5 * i + k];
    b1 = b1 + b[gr] * A.hconst[5 * i + k];
    t2 = t2 + A.p[gc] * A.hconst[5 * j + k];
    b2 = b2 + b[gc] * A.hconst[5 * j + k];
  }
  const float4 gm = A.geo[q];
  const float ax = static_cast<float>(static_cast<double>(t1) * gm.x + static_cast<double>(t2) * gm.z);
  const float az = static_cast<float>(static_cast<double>(t1) * gm.y + static_cast<double>(t2) * gm.w);
  const float bx = static_cast<float>(static_cast<double>(b1) * gm.x + static_cast<double>(b2) * gm.z);
  const float bz = static_cast<float>(static_cast<double>(b1) * gm.y + static_cast<double>(b2) * gm.w);
  const int g = A.slot_ibool[q];
  const float2 rk = A.slot_rk[q];
  float2 s = A.kl_ac[q];
  s.x = s.x + 1.f / rk.x * (ax * bx + az * bz) * A.dt;
  s.y = s.y + 1.f / rk.y * A.pdd[g] * b[g] * A.dt;
  A.kl_ac[q] = s;
}

}  // namespace sf2d
