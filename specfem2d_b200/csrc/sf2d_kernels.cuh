// Device side of the tile-staged elastic time step (NGLL = 5).
//
// One CTA advances one tile of elements by one Newmark step or one LDDRK
// stage:
//   1. cp.async of the tile's local ibool and the fields of all its points
//      straight into shared memory (geometry and material are read from
//      global memory where they are used);
//   2. Newmark predictor u' = u + dt v + dt^2/2 a, v' = v + dt/2 a
//      (update_displacement_Newmark.F90:408-454) in shared memory, or a
//      cleared accumulator for an LDDRK stage (iterate_time.F90:167-181);
//   3. Stacey traction on the (predicted) velocity, fluid pressure and
//      sources, one thread per receiving point in the reference's order at
//      that point (compute_stacey_elastic.f90:160-335,
//      compute_add_sources_viscoelastic.f90:36-101);
//   4. derivative lines (one thread per element row or column: the 5x5
//      contraction with hprime, mxm_4comp_singleA :810-883), then per GLL
//      point the Jacobian mapping, isotropic (lambda, mu as
//      compute_forces_viscoelastic.F90:286-294 forms them) or anisotropic
//      stress (:372-445, in double as the reference), 3-SLS memory variables
//      and their stress correction (compute_attenuation_viscoelastic.f90:36-236,
//      :481-503), weak-form terms (:669-675), then the weighted transpose
//      lines with hprimewgll (:760-782);
//   5. assembly into the shared accumulator colour by colour (no two elements
//      of a colour share a point: no atomics);
//   6. interior points: a *= rmass_inverse, then the Newmark corrector
//      (update_displacement_Newmark.F90:564-589) or the LDDRK update
//      (update_displacement_LDDRK.F90:55-79), write-back; shared points: the
//      tile's partial sum goes to its slot.
// A second kernel finishes shared points, adding the partial sums in tile
// order.  Results are bit-identical from run to run.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "sf2d_pml.cuh"
#include "sf2d_tiler.h"

namespace sf2d {

struct Params {
  float2 *u, *v, *a;
  float2 *uL, *vL;  // LDDRK auxiliary fields
  const float2 *rmass;
  const TileInfo *tiles;
  const uint16_t *lib;
  const float4 *geo;   // xix, xiz, gammax, gammaz per element GLL point (tile slot order)
  const float2 *mat;   // lambda, mu (lambda = rho*cp*cp - 2*mu in FP32, as the CPU solver forms it)
  const int *aniso_idx;  // per element slot: index of its anisotropic block, -1 when isotropic
  const float4 *c4;      // c11, c13, c15, c33 per point of anisotropic elements
  const float2 *c2;      // c35, c55
  const float4 *att_coef;  // 3 per element point: Newmark {A1, A2, B1, B2}[sls], LDDRK {1/tau1, 1/tau2, phi1, phi2}[sls]
  float4 *att_state;       // 3 per element point: {e1[0..2], e11[0]}, {e11[1..2], e13[0..1]}, {e13[2], old strains}
  float4 *att_state_l;     // LDDRK: e1_LDDRK, e11_LDDRK, e13_LDDRK with the same packing
  const int *sh_ids;
  float2 *partial;
  // shared-point partial sums, point-major: the slots of shared point s are
  // [shp_off[s], shp_off[s+1]) in tile order; slot_pos maps a tile's shared
  // local point (sh_off + k) to its slot
  const int *shp_off, *slot_pos;
  const int4 *bgroups;    // per tile (grp_off, grp_n): point, first idx, Stacey | coupling << 8, sources
  const int *bnd_idx;     // entries of each group
  const int *st_local;
  const float4 *st_nw;    // nx, nz, weight, 0
  const float2 *st_rho;   // rho*vp, rho*vs
  const int *src_local, *src_id;
  const float2 *src_arr;
  const float *stf;       // [isrc][it][stage]
  const int *rec_id, *rec_dev;
  const double *rec_h;    // 10 per receiver: hxir[5], hgammar[5]
  double *seis;           // [irec][it][2]
  int *d_step, *d_status;
  // packed batches: the member (independent sub-mesh) of every tile and shared
  // point, and one status word per member (1 = its field blew up, masked)
  const int *tile_member, *shared_member;
  int *member_status;
  int *d_step_b;          // copy of *d_step written by the tile kernel, read by the shared-point kernel
  // segment recomputation: displacement frames written after every step, frame = step - *frame_base
  float2 *frames;
  const int *frame_base;
  int nframes, nglob;
  // forward acceleration frames (approximate Hessian), written beside the displacement frames
  float2 *aframes;
  // adjoint sweep with kernel accumulation: forward frame = *kern_base - step
  const float2 *kframes;
  const float2 *kaframes;  // forward acceleration frames read by the adjoint sweep (Hessian), or null
  float2 *hess_glob;       // per device point: sums of |b_a|^2 and a_adj . b_a (Hessian), or null
  const int *kern_base;
  float2 *kmu_kl;         // per element point (slot order): kappa and mu integrand sums
  float *rho_kl_glob;     // per device point: rho integrand sum
  // fluid-solid coupling (solid side): tile-local point, fluid device point, (nx, nz, w, 0)
  const int *cpl_local, *cpl_src;
  const float4 *cpl_nw;
  const float *pdd_ac;    // chi_dot_dot of the fluid, fluid device order
  // adjoint run (SIMULATION_TYPE 3, solid step first): the pressure term is the
  // fluid's predicted chi of this step, formed from chi, chi_dot, chi_dot_dot
  // (compute_coupling_viscoelastic_ac.f90:89-93)
  const float *p_ac, *pd_ac;
  int cpl_adjoint;
  // CPML: elements of slots >= pml_slot0 lie in the layer, "PML points" are
  // their GLL points in slot order (index (slot - pml_slot0) * 25 + q)
  int pml_slot0;
  const PmlSet *pml_sets;  // coefficient sets of the layer
  const int *pml_set_idx;  // per PML point: its set
  const float *pml_rhoj;  // rho * jacobian per PML point
  float4 *pml_rm;         // 3 per PML point: strain memory zx (dux_dx 1,2, duz_dx 1,2), xz (dux_dz, duz_dz),
                          // displacement memory (x 1, z 1, x 2, z 2)
  float4 *pml_rm_l;       // LDDRK copies
  const int *edge_local;  // per tile (edge_off, edge_n): local points on the layer's outer edge
  const uint8_t *sh_edge; // per shared point: 1 on the outer edge
  double DT, h_old;       // DT, and deltatsquareover2 / 2 for the mid-step field
  // solid-side coupling entries whose fluid element lies in a CPML layer have
  // cpl_src = ~k: their pressure is formed before this kernel (k_cpl_pml_solid)
  const float *cpl_pml_p; // per layer entry k: the pressure to apply
  // CPML in attenuating solids (Newmark): per PML point its viscoelastic set,
  // -1 in elastic layer elements; 9 memory variables per PML point, per SLS
  // (bulk dux_dx, duz_dz), (shear dux_dx, duz_dz), (shear dux_dz, duz_dx)
  const PmlVisco *pml_vsets;
  const int *pml_vset_idx;
  float2 *pml_vm;
  int nstep_stf, nstage, nstep_seis, seismotype, nrec;
  double cosrot, sinrot;
  float dt, dto2, dt2o2;
  float alpha[6], beta[6];
  int shared_begin, nshared;
  int max_q, max_local;
  float hconst[60];  // hprime[25], hprimewgll[25], wxgll[5], wzgll[5]
};

constexpr int SHARED_NT = 256;

// Newmark predictor u + dt v + dt^2/2 a and v + dt/2 a in the reference's
// operation order with every product and sum rounded (no contraction), so
// that every kernel that forms the predicted field of a point (the tile and
// shared-point kernels, and the fluid side of the coupling, which needs the
// solid's predicted displacement before the solid kernels run) gets the
// same bits (update_displacement_Newmark.F90:353-454).
__device__ __forceinline__ float newmark_displ(float u, float v, float a, float dt, float dt2o2) {
  return __fadd_rn(__fadd_rn(u, __fmul_rn(dt, v)), __fmul_rn(dt2o2, a));
}
__device__ __forceinline__ float newmark_veloc(float v, float a, float dto2) { return __fadd_rn(v, __fmul_rn(dto2, a)); }

__device__ __forceinline__ void record_receiver(const Params &P, int r, int step) {
  if (step < 0 || step >= P.nstep_seis) return;
  if (P.seismotype == 6) {
    // a potential receiver in a solid records nothing (write_seismograms.F90:149-170)
    double *out = P.seis + (static_cast<size_t>(P.rec_id[r]) * P.nstep_seis + step) * 2;
    out[0] = 0.0;
    out[1] = 0.0;
    return;
  }
  const float2 *field = P.seismotype == 2 ? P.v : (P.seismotype == 3 ? P.a : P.u);
  const int *dev = P.rec_dev + 25 * r;
  const double *h = P.rec_h + 10 * r;
  double vx = 0.0, vz = 0.0;
  for (int j = 0; j < 5; ++j)
    for (int i = 0; i < 5; ++i) {
      const float2 f = field[dev[j * 5 + i]];
      // xir_store_loc and gammar_store_loc are CUSTOM_REAL: the product is formed in FP32
      const double hl = static_cast<double>(static_cast<float>(h[i]) * static_cast<float>(h[5 + j]));
      vx += static_cast<double>(f.x) * hl;
      vz += static_cast<double>(f.y) * hl;
    }
  double *out = P.seis + (static_cast<size_t>(P.rec_id[r]) * P.nstep_seis + step) * 2;
  out[0] = P.cosrot * vx + P.sinrot * vz;
  out[1] = -P.sinrot * vx + P.cosrot * vz;
}

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async8(void *s, const void *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async16(void *s, const void *g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// Programmatic dependent launch (sm_90 and later): a step kernel launched with
// the programmatic-serialization attribute may be scheduled while the kernel
// before it in the stream still runs; griddepcontrol.wait then blocks until
// that kernel has completed and its writes are visible, so every read of the
// previous kernel's results comes after it.  launch_dependents lets the next
// kernel be scheduled once all of this kernel's CTAs have started (the short
// shared-point and receiver kernels call it, so the next step's tiles start as
// they drain).  Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void wait_previous_kernel() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void allow_next_kernel() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// Shared-memory layout of one tile (sizes from the largest tile); every region
// starts on a 16-byte boundary, as 16-byte cp.async destinations require:
//   u, v, acc float2[max_local]  (old u, v, a -> predicted u, v and the accumulator)
//   h    float[64]      hprime, hprimewgll, wxgll, wzgll
//   lib  uint16[max_q rounded up to 8]
//   d1, d2 float2[max_q]  xi / gamma derivatives, then the weak-form terms t1, t2,
//        then their weighted transposes
//   b    float2[max_local], bd1, bd2 float2[max_q]  forward frame and its
//        derivatives (adjoint sweep with kernels)
//   uold float2[max_local], od1, od2, pml float2[max_q]  mid-step displacement,
//        its derivatives and the layer's acceleration terms (CPML tiles)
struct TileSmem {
  size_t u, v, acc, h, lib, d1, d2, b, bd1, bd2, uold, od1, od2, pml, total;
};
__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~static_cast<size_t>(15); }
__host__ __device__ inline TileSmem tile_smem_layout(int max_q, int max_local, bool kern = false, bool pml = false) {
  TileSmem L;
  size_t o = 0;
  L.u = o;
  o = align16(o + static_cast<size_t>(max_local) * sizeof(float2));
  L.v = o;
  o = align16(o + static_cast<size_t>(max_local) * sizeof(float2));
  L.acc = o;
  o = align16(o + static_cast<size_t>(max_local) * sizeof(float2));
  L.h = o;
  o = align16(o + 64 * sizeof(float));
  L.lib = o;
  o = align16(o + static_cast<size_t>((max_q + 7) / 8 * 8) * sizeof(uint16_t));
  const size_t qb = align16(static_cast<size_t>(max_q) * sizeof(float2));
  const size_t lb = align16(static_cast<size_t>(max_local) * sizeof(float2));
  L.d1 = o;
  o += qb;
  L.d2 = o;
  o += qb;
  L.b = o;
  if (kern) o += lb;
  L.bd1 = o;
  if (kern) o += qb;
  L.bd2 = o;
  if (kern) o += qb;
  L.uold = o;
  if (pml) o += lb;
  L.od1 = o;
  if (pml) o += qb;
  L.od2 = o;
  if (pml) o += qb;
  L.pml = o;
  if (pml) o += qb;
  L.total = o;
  return L;
}

// Memory-variable update of one element point (Newmark recursive convolution or
// LDDRK ADE stage); returns the sums of e1, e11, e13 over the SLS.
template <bool LDDRK>
__device__ __forceinline__ void attenuation_point(const Params &P, size_t pa, float dux_dxl, float dux_dzl,
                                                  float duz_dxl, float duz_dzl, int stage, float &e1s,
                                                  float &e11s, float &e13s) {
  const float4 c0 = P.att_coef[pa], c1 = P.att_coef[pa + 1], c2 = P.att_coef[pa + 2];
  float4 s0 = P.att_state[pa], s1 = P.att_state[pa + 1], s2 = P.att_state[pa + 2];
  float e1[3] = {s0.x, s0.y, s0.z}, e11[3] = {s0.w, s1.x, s1.y}, e13[3] = {s1.z, s1.w, s2.x};
  const float4 cc[3] = {c0, c1, c2};
  const float theta_n = dux_dxl + duz_dzl;
  if (!LDDRK) {
    const float old_xx = s2.y, old_zz = s2.z, old_xz = s2.w;
    const float theta_n1 = old_xx + old_zz;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      float a = cc[s].x;
      e1[s] = a * a * e1[s] + cc[s].z * (theta_n + a * theta_n1);
      a = cc[s].y;
      e11[s] = a * a * e11[s] + cc[s].w * (dux_dxl - theta_n / 2.f + a * (old_xx - theta_n1 / 2.f));
      e13[s] = a * a * e13[s] + cc[s].w * (dux_dzl + duz_dxl + a * old_xz);
    }
    s2.y = dux_dxl;
    s2.z = duz_dzl;
    s2.w = dux_dzl + duz_dxl;
  } else {
    float4 l0 = P.att_state_l[pa], l1 = P.att_state_l[pa + 1], l2 = P.att_state_l[pa + 2];
    float e1l[3] = {l0.x, l0.y, l0.z}, e11l[3] = {l0.w, l1.x, l1.y}, e13l[3] = {l1.z, l1.w, l2.x};
    const float al = P.alpha[stage], be = P.beta[stage];
    const double dt = static_cast<double>(P.dt);
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const double itau1 = cc[s].x, itau2 = cc[s].y;
      const float phi1 = cc[s].z, phi2 = cc[s].w;
      // 1/tau_sigma is a double in the reference: these products are double there too
      e1l[s] = static_cast<float>(static_cast<double>(al * e1l[s]) +
                                  dt * (static_cast<double>(theta_n * phi1) - static_cast<double>(e1[s]) * itau1));
      e1[s] = e1[s] + be * e1l[s];
      e11l[s] = static_cast<float>(static_cast<double>(al * e11l[s] + P.dt * ((dux_dxl - theta_n / 2.f) * phi2)) -
                                   dt * (static_cast<double>(e11[s]) * itau2));
      e11[s] = e11[s] + be * e11l[s];
      e13l[s] = static_cast<float>(static_cast<double>(al * e13l[s] + P.dt * ((dux_dzl + duz_dxl) * phi2)) -
                                   dt * (static_cast<double>(e13[s]) * itau2));
      e13[s] = e13[s] + be * e13l[s];
    }
    P.att_state_l[pa] = make_float4(e1l[0], e1l[1], e1l[2], e11l[0]);
    P.att_state_l[pa + 1] = make_float4(e11l[1], e11l[2], e13l[0], e13l[1]);
    P.att_state_l[pa + 2] = make_float4(e13l[2], 0.f, 0.f, 0.f);
  }
  P.att_state[pa] = make_float4(e1[0], e1[1], e1[2], e11[0]);
  P.att_state[pa + 1] = make_float4(e11[1], e11[2], e13[0], e13[1]);
  P.att_state[pa + 2] = make_float4(e13[2], s2.y, s2.z, s2.w);
  e1s = e1[0] + e1[1] + e1[2];
  e11s = e11[0] + e11[1] + e11[2];
  e13s = e13[0] + e13[1] + e13[2];
}

// Sensitivity-kernel integrands at one element point (compute_kernels.f90:75-292):
// strains of the adjoint field (a_*) and of the forward frame (b_*) with the mapping
// derivatives used in double, as the reference declares them.
__device__ __forceinline__ void kernel_point(float dux_dxi, float duz_dxi, float dux_dg, float duz_dg, float bdux_dxi,
                                             float bduz_dxi, float bdux_dg, float bduz_dg, float4 g4, float &kap,
                                             float &muk) {
  const double xixl = g4.x, xizl = g4.y, gammaxl = g4.z, gammazl = g4.w;
  const float dux_dxl = static_cast<float>(dux_dxi * xixl + dux_dg * gammaxl);
  const float dux_dzl = static_cast<float>(dux_dxi * xizl + dux_dg * gammazl);
  const float duz_dxl = static_cast<float>(duz_dxi * xixl + duz_dg * gammaxl);
  const float duz_dzl = static_cast<float>(duz_dxi * xizl + duz_dg * gammazl);
  const float bdux_dxl = static_cast<float>(bdux_dxi * xixl + bdux_dg * gammaxl);
  const float bdux_dzl = static_cast<float>(bdux_dxi * xizl + bdux_dg * gammazl);
  const float bduz_dxl = static_cast<float>(bduz_dxi * xixl + bduz_dg * gammaxl);
  const float bduz_dzl = static_cast<float>(bduz_dxi * xizl + bduz_dg * gammazl);
  const float dsxz = static_cast<float>(0.5 * (static_cast<double>(duz_dxl) + static_cast<double>(dux_dzl)));
  const float bdsxz = static_cast<float>(0.5 * (static_cast<double>(bduz_dxl) + static_cast<double>(bdux_dzl)));
  kap = (dux_dxl + duz_dzl) * (bdux_dxl + bduz_dzl);
  muk = dux_dxl * bdux_dxl + duz_dzl * bduz_dzl + 2.f * dsxz * bdsxz - 1.f / 3.f * kap;
}

// Derivatives along one element line of 5 GLL points (stride st in the
// element's [j][i] order, first local index at le[0]): out[m] = sum_k f_k
// hprime[m][k] with hprime from the kernel parameters (compile-time indices
// after unrolling: constant-bank operands).  Same operation order as a
// point-by-point sum, so the results are the same.
__device__ __forceinline__ void line_derivs(const Params &P, const float2 *fld, const uint16_t *le, int st,
                                            float2 *out) {
  float2 in[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) in[k] = fld[le[st * k]];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    float2 d = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const float h = P.hconst[5 * m + k];
      d.x += in[k].x * h;
      d.y += in[k].y * h;
    }
    out[st * m] = d;
  }
}

// Weighted transpose along one line, in place: out[m] = sum_k t_k hprimewgll[k][m].
__device__ __forceinline__ void line_weighted(const Params &P, float2 *buf, int st) {
  float2 in[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) in[k] = buf[st * k];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    float2 d = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const float w = P.hconst[25 + 5 * k + m];
      d.x += in[k].x * w;
      d.y += in[k].y * w;
    }
    buf[st * m] = d;
  }
}

// PML: the tiles of a CPML layer (isotropic, no attenuation, no kernels):
// mid-step displacement u + dt^2/4 a of the tile's points, the layer's strain
// and displacement memory variables, the modified non-symmetric stress and
// the extra acceleration terms (pml_compute_memory_variables.f90:230-540,
// pml_compute_accel_contribution.f90:187-333, compute_forces_viscoelastic.F90:600-675, 785-797).
// Tiles [tile0, tile0 + gridDim.x) are advanced.
// Resident threads per SM the variants ask for: 1536 for the plain ones (6
// CTAs of 256, at most 40 registers; with the geometry read from global memory
// the tile's shared memory allows it, and the extra warps hide the loads'
// latency), 1024 for the attenuating ones (Newmark: no spill; LDDRK: a
// 32-byte spill, still 3 % faster than 80 registers) and the Newmark gradient
// ones (at most 64 registers; with attenuation a 16-byte spill, still 4 %
// faster: more warps keep the memory variables' and frames' loads in flight),
// 768 for the
// other anisotropic, attenuating, kernel and CPML ones (at most 80 registers;
// left unbounded the compiler takes over 130 and one CTA fits an SM).
template <int NT, bool ANISO, bool ATTEN, bool KERN, bool PML, bool LDDRK>
constexpr int tile_min_blocks() {
  return ((ATTEN && !ANISO && !KERN) || (KERN && !LDDRK)) && !PML ? 1024 / NT
                                                       : (ANISO || ATTEN || KERN || PML) ? 768 / NT : 1536 / NT;
}
template <int NT, bool ANISO, bool ATTEN, bool LDDRK, bool KERN, bool PML = false>
__global__ void __launch_bounds__(NT, tile_min_blocks<NT, ANISO, ATTEN, KERN, PML, LDDRK>())
    k_elastic_tile(const Params P, int record_prev, int stage, int tile0) {
  extern __shared__ __align__(16) unsigned char smem[];
  // the shared-point kernel after it is not released early: its CTAs would sit
  // on the SMs through this kernel's last wave
  wait_previous_kernel();
  const TileInfo &ti = P.tiles[tile0 + blockIdx.x];
  const int tid = threadIdx.x;
  const int n_int = ti.n_int;
  const int n_sh = ti.n_sh;
  const int nl = n_int + n_sh;
  const int nq = ti.nelem * 25;
  const int ebase = ti.elem_base * 25;
  const int int_begin = ti.int_begin;
  const TileSmem L = tile_smem_layout(P.max_q, P.max_local, KERN, PML);
  float2 *s_uold = reinterpret_cast<float2 *>(smem + L.uold);
  float2 *s_pml = reinterpret_cast<float2 *>(smem + L.pml);
  float2 *s_d1 = reinterpret_cast<float2 *>(smem + L.d1);
  float2 *s_d2 = reinterpret_cast<float2 *>(smem + L.d2);
  float2 *s_bd1 = reinterpret_cast<float2 *>(smem + L.bd1);
  float2 *s_bd2 = reinterpret_cast<float2 *>(smem + L.bd2);
  float2 *s_od1 = reinterpret_cast<float2 *>(smem + L.od1);
  float2 *s_od2 = reinterpret_cast<float2 *>(smem + L.od2);
  float2 *s_b = reinterpret_cast<float2 *>(smem + L.b);
  float2 *s_u = reinterpret_cast<float2 *>(smem + L.u);
  float2 *s_v = reinterpret_cast<float2 *>(smem + L.v);
  float2 *s_acc = reinterpret_cast<float2 *>(smem + L.acc);
  float *s_h = reinterpret_cast<float *>(smem + L.h);
  uint16_t *s_lib = reinterpret_cast<uint16_t *>(smem + L.lib);

  const int step = *P.d_step;
  if (blockIdx.x == 0 && tid == 0) *P.d_step_b = step;
  // receivers of the previous step read the old fields before any write
  if (record_prev && tid < ti.rec_n) record_receiver(P, ti.rec_off + tid, step - 1);
  // a masked member neither reads nor writes its points from here on (uniform over the CTA)
  if (P.tile_member && P.member_status[P.tile_member[tile0 + blockIdx.x]]) return;
  const float2 *kframe = nullptr;
  if (KERN) kframe = P.kframes + static_cast<size_t>(*P.kern_base - step) * P.nglob;

  // 1. every load of the tile is issued at once, straight into shared memory
  {
    const uint4 *glib = reinterpret_cast<const uint4 *>(P.lib + ti.lib_off);
    const int nlib16 = (nq + 7) / 8;
    for (int k = tid; k < nlib16; k += NT) cp_async16(s_lib + 8 * k, glib + k);
    for (int l = tid; l < n_int; l += NT) {
      const int g = int_begin + l;
      cp_async8(s_u + l, P.u + g);
      cp_async8(s_v + l, P.v + g);
      if (!LDDRK) cp_async8(s_acc + l, P.a + g);
      if (KERN) cp_async8(s_b + l, kframe + g);
    }
    for (int k = tid; k < n_sh; k += NT) {
      const int g = P.sh_ids[ti.sh_off + k];
      cp_async8(s_u + n_int + k, P.u + g);
      cp_async8(s_v + n_int + k, P.v + g);
      if (!LDDRK) cp_async8(s_acc + n_int + k, P.a + g);
      if (KERN) cp_async8(s_b + n_int + k, kframe + g);
    }
    if (tid < 60) s_h[tid] = P.hconst[tid];
    cp_async_wait_all();
  }
  __syncthreads();

  // 2. Newmark predictor in place, or a cleared accumulator for an LDDRK stage
  const float dt = P.dt, dto2 = P.dto2, dt2o2 = P.dt2o2;
  for (int l = tid; l < nl; l += NT) {
    if (!LDDRK) {
      float2 u = s_u[l], v = s_v[l];
      const float2 a = s_acc[l];
      // mid-step displacement of the layer's convolutions (update_displacement_Newmark.F90:374-380)
      if (PML)
        s_uold[l] = make_float2(static_cast<float>(static_cast<double>(u.x) + P.h_old * static_cast<double>(a.x)),
                                static_cast<float>(static_cast<double>(u.y) + P.h_old * static_cast<double>(a.y)));
      u.x = newmark_displ(u.x, v.x, a.x, dt, dt2o2);
      u.y = newmark_displ(u.y, v.y, a.y, dt, dt2o2);
      v.x = newmark_veloc(v.x, a.x, dto2);
      v.y = newmark_veloc(v.y, a.y, dto2);
      s_u[l] = u;
      s_v[l] = v;
    }
    s_acc[l] = make_float2(0.f, 0.f);
  }
  __syncthreads();
  // outer edge of a CPML layer: displacement, velocity, mid-step displacement
  // and acceleration zeroed before the forces (pml_boundary_elastic,
  // pml_compute.f90:545-574); the layer excludes Stacey terms, so the order
  // against them does not matter
  if (ti.edge_n > 0) {
    for (int k = tid; k < ti.edge_n; k += NT) {
      const int l = P.edge_local[ti.edge_off + k];
      s_u[l] = make_float2(0.f, 0.f);
      s_v[l] = make_float2(0.f, 0.f);
      if (PML && !LDDRK) s_uold[l] = make_float2(0.f, 0.f);
    }
    __syncthreads();
  }

  // 3. boundary terms, coupling and sources: one thread per receiving point,
  //    in the reference's order at that point (overlaps pass 1, which does not
  //    touch the accumulator)
  for (int gi = tid; gi < ti.grp_n; gi += NT) {
    const int4 g = P.bgroups[ti.grp_off + gi];
    const int l = g.x;
    const int *ix = P.bnd_idx + g.y;
    float2 acc = s_acc[l];
    const float2 v = s_v[l];
    const int nst = g.z & 255, ncp = g.z >> 8;
    // Stacey traction on the predicted velocity (compute_stacey_elastic.f90:160-335)
    for (int k = 0; k < nst; ++k) {
      const int p = ix[k];
      const float4 nw = P.st_nw[p];
      const float2 rr = P.st_rho[p];
      const float vn = nw.x * v.x + nw.y * v.y;
      const float tx = rr.x * vn * nw.x + rr.y * (v.x - vn * nw.x);
      const float tz = rr.x * vn * nw.y + rr.y * (v.y - vn * nw.y);
      acc.x -= tx * nw.z;
      acc.y -= tz * nw.z;
    }
    ix += nst;
    // pressure of the fluid on the solid, -chi_dot_dot of this step
    // (compute_coupling_viscoelastic_ac.f90:80-250); a negative source names
    // the CPML entry ~src, whose pressure k_cpl_pml_solid formed
    for (int k = 0; k < ncp; ++k) {
      const int p = ix[k];
      const float4 nw = P.cpl_nw[p];
      const int ga = P.cpl_src[p];
      float pressure;
      if (ga < 0)
        pressure = P.cpl_pml_p[~ga];
      else if (P.cpl_adjoint)
        pressure = newmark_displ(P.p_ac[ga], P.pd_ac[ga], P.pdd_ac[ga], P.dt, P.dt2o2);
      else
        pressure = -P.pdd_ac[ga];
      acc.x += nw.z * nw.x * pressure;
      acc.y += nw.z * nw.y * pressure;
    }
    ix += ncp;
    // sources (compute_add_sources_viscoelastic.f90:36-101)
    for (int k = 0; k < g.w; ++k) {
      const int p = ix[k];
      const float f = step < P.nstep_stf
                          ? P.stf[(static_cast<size_t>(P.src_id[p]) * P.nstep_stf + step) * P.nstage + stage]
                          : 0.f;
      const float2 sa = P.src_arr[p];
      acc.x += sa.x * f;
      acc.y += sa.y * f;
    }
    s_acc[l] = acc;
  }

  // the first point's geometry and material are requested now, so that their
  // latency passes during the derivative lines (software pipelining of 4b)
  float4 g_next = make_float4(0.f, 0.f, 0.f, 0.f);
  float2 m_next = make_float2(0.f, 0.f);
  if (tid < nq) {
    g_next = __ldg(P.geo + ebase + tid);
    m_next = __ldg(P.mat + ebase + tid);
  }

  // 4a. derivative lines: one thread per element row (xi) or column (gamma)
  //     forms the 5 derivatives along it; the loops are fully unrolled, so
  //     hprime comes straight from the kernel's constant bank, and each point's
  //     field is read twice per element instead of ten times
  const int nlines = 10 * ti.nelem;
  for (int t = tid, el = tid / 10; t < nlines; t += NT, el += NT / 10) {
    // with NT a multiple of 10 every thread keeps one line position r
    const int e = NT % 10 == 0 ? el : t / 10;
    const int r = NT % 10 == 0 ? tid % 10 : t - 10 * e;
    const int a0 = r < 5 ? 5 * r : r - 5;  // first point: (j = r, 0) of a row, (0, i = r - 5) of a column
    const int st = r < 5 ? 1 : 5;          // stride along the line
    const uint16_t *le = s_lib + 25 * e + a0;
    const int o = 25 * e + a0;
    float2 *d = r < 5 ? s_d1 : s_d2;
    line_derivs(P, s_u, le, st, d + o);
    if (KERN) line_derivs(P, s_b, le, st, (r < 5 ? s_bd1 : s_bd2) + o);
    if (PML && !LDDRK) line_derivs(P, s_uold, le, st, (r < 5 ? s_od1 : s_od2) + o);
  }
  __syncthreads();

  // 4b. per GLL point: mapping, stress, memory variables, weak-form terms
  //     (t1 = J (sigma . xi_x), t2 = J (sigma . gamma_x) overwrite the derivatives)
  constexpr bool FIXQ = NT % 25 == 0;  // every thread keeps one GLL position
  const int q0 = tid % 25, j0 = q0 / 5, i0 = q0 - 5 * j0;
  for (int f = tid, ef = tid / 25; f < nq; f += NT, ef += NT / 25) {
    const int e = FIXQ ? ef : f / 25;
    const int q = FIXQ ? q0 : f - 25 * e;
    const int j = FIXQ ? j0 : q / 5;
    const int i = FIXQ ? i0 : q - 5 * j;
    const uint16_t *le = s_lib + 25 * e;
    // geometry and material straight from global memory (coalesced in f): not
    // staging them keeps the tile's shared memory small and more tiles resident;
    // the next point's are requested before this one is computed
    const float4 g4 = g_next;
    const float2 m2 = m_next;
    if (f + NT < nq) {
      g_next = __ldg(P.geo + ebase + f + NT);
      m_next = __ldg(P.mat + ebase + f + NT);
    }
    const float2 d1 = s_d1[f], d2 = s_d2[f];
    const float dux_dxi = d1.x, duz_dxi = d1.y, dux_dg = d2.x, duz_dg = d2.y;
    if (KERN) {
      // kernels of this adjoint step: adjoint displacement u' against the forward frame
      const float2 b1 = s_bd1[f], b2 = s_bd2[f];
      float kap, muk;
      kernel_point(dux_dxi, duz_dxi, dux_dg, duz_dg, b1.x, b1.y, b2.x, b2.y, g4, kap, muk);
      float2 km = P.kmu_kl[ebase + f];
      km.x = km.x + kap;
      km.y = km.y + muk;
      P.kmu_kl[ebase + f] = km;
    }
    const float xixl = g4.x, xizl = g4.y, gammaxl = g4.z, gammazl = g4.w;
    const float jacobianl = 1.f / (xixl * gammazl - gammaxl * xizl);
    const float dux_dxl = dux_dxi * xixl + dux_dg * gammaxl;
    const float dux_dzl = dux_dxi * xizl + dux_dg * gammazl;
    const float duz_dxl = duz_dxi * xixl + duz_dg * gammaxl;
    const float duz_dzl = duz_dxi * xizl + duz_dg * gammazl;
    const float mul = m2.y;
    const float lambdal = m2.x;
    const float lambdaplus2mu = lambdal + 2.f * mul;
    if (PML) {
      const int ps = ebase + f - 25 * P.pml_slot0;
      const PmlSet &c = P.pml_sets[P.pml_set_idx[ps]];
      // strains of the mid-step displacement
      float o_dux_dxl = 0.f, o_dux_dzl = 0.f, o_duz_dxl = 0.f, o_duz_dzl = 0.f;
      if (!LDDRK) {
        const float2 od1 = s_od1[f], od2 = s_od2[f];
        const float ox_xi = od1.x, oz_xi = od1.y, ox_g = od2.x, oz_g = od2.y;
        o_dux_dxl = ox_xi * xixl + ox_g * gammaxl;
        o_dux_dzl = ox_xi * xizl + ox_g * gammazl;
        o_duz_dxl = oz_xi * xixl + oz_g * gammaxl;
        o_duz_dzl = oz_xi * xizl + oz_g * gammazl;
      }
      const PmlConv &cax = c.cax, &caz = c.caz, &cbx = c.cbx, &cbz = c.cbz;
      const PmlLik &zx = c.zx, &xz = c.xz;  // poles (alpha_z, beta_x) and (alpha_x, beta_z)
      float4 r0 = P.pml_rm[3 * ps], r1 = P.pml_rm[3 * ps + 1], rd = P.pml_rm[3 * ps + 2];
      float4 l0 = make_float4(0.f, 0.f, 0.f, 0.f), l1 = l0, ld = l0;
      if (LDDRK) {
        l0 = P.pml_rm_l[3 * ps];
        l1 = P.pml_rm_l[3 * ps + 1];
        ld = P.pml_rm_l[3 * ps + 2];
      }
      const float al = P.alpha[stage], be = P.beta[stage];
      pml_update<LDDRK>(r0.x, l0.x, caz, c.az, dux_dxl, o_dux_dxl, al, be, dt);
      pml_update<LDDRK>(r0.y, l0.y, cbx, c.bx, dux_dxl, o_dux_dxl, al, be, dt);
      pml_update<LDDRK>(r0.z, l0.z, caz, c.az, duz_dxl, o_duz_dxl, al, be, dt);
      pml_update<LDDRK>(r0.w, l0.w, cbx, c.bx, duz_dxl, o_duz_dxl, al, be, dt);
      pml_update<LDDRK>(r1.x, l1.x, cax, c.ax, dux_dzl, o_dux_dzl, al, be, dt);
      pml_update<LDDRK>(r1.y, l1.y, cbz, c.bz, dux_dzl, o_dux_dzl, al, be, dt);
      pml_update<LDDRK>(r1.z, l1.z, cax, c.ax, duz_dzl, o_duz_dzl, al, be, dt);
      pml_update<LDDRK>(r1.w, l1.w, cbz, c.bz, duz_dzl, o_duz_dzl, al, be, dt);
      // the layer's acceleration terms at this point (pml_compute_accel_contribution.f90:187-333)
      const PmlL &Lc = c.l;  // poles alpha_x, alpha_z
      const int lq = le[q];
      const float2 uq = s_u[lq], vq = s_v[lq];
      const float2 uo = LDDRK ? make_float2(0.f, 0.f) : s_uold[lq];
      pml_update<LDDRK>(rd.x, ld.x, cax, c.ax, uq.x, uo.x, al, be, dt);
      pml_update<LDDRK>(rd.y, ld.y, cax, c.ax, uq.y, uo.y, al, be, dt);
      pml_update<LDDRK>(rd.z, ld.z, caz, c.az, uq.x, uo.x, al, be, dt);
      pml_update<LDDRK>(rd.w, ld.w, caz, c.az, uq.y, uo.y, al, be, dt);
      const double wwf = static_cast<double>(s_h[50 + i] * s_h[55 + j] * P.pml_rhoj[ps]);
      s_pml[f] = make_float2(
          static_cast<float>(wwf * (Lc.A1 * vq.x + Lc.A2 * uq.x + Lc.A3 * rd.x + Lc.A4 * rd.z)),
          static_cast<float>(wwf * (Lc.A1 * vq.y + Lc.A2 * uq.y + Lc.A3 * rd.y + Lc.A4 * rd.w)));
      P.pml_rm[3 * ps] = r0;
      P.pml_rm[3 * ps + 1] = r1;
      P.pml_rm[3 * ps + 2] = rd;
      if (LDDRK) {
        P.pml_rm_l[3 * ps] = l0;
        P.pml_rm_l[3 * ps + 1] = l1;
        P.pml_rm_l[3 * ps + 2] = ld;
      }
      float sxx, szz, szx, sxz;
      const int vi = (ATTEN && !LDDRK) ? P.pml_vset_idx[ps] : -1;
      if (ATTEN && !LDDRK && vi >= 0) {
        // attenuating layer element (pml_compute_memory_variables.f90:686-892): per
        // SLS the strains convolved with 1/tau_sigma, their Zener and phi-weighted
        // sums; then the modified bulk (k) and shear (m) strains and the stress with
        // the unrelaxed moduli (compute_forces_viscoelastic.F90:545-555)
        const PmlVisco &V = P.pml_vsets[vi];
        float2 *vm = P.pml_vm + static_cast<size_t>(ps) * 9;
        float ks_xx = 0.f, ks_zz = 0.f, ms_xx = 0.f, ms_zz = 0.f, ms_xz = 0.f, ms_zx = 0.f;
        float pk_xx = 0.f, pk_zz = 0.f, pm_xx = 0.f, pm_zz = 0.f, pm_xz = 0.f, pm_zx = 0.f;
        float unused = 0.f;
#pragma unroll
        for (int sl = 0; sl < PML_NSLS; ++sl) {
          float2 a = vm[3 * sl], b = vm[3 * sl + 1], c = vm[3 * sl + 2];
          pml_update<false>(a.x, unused, V.ck[sl], 0.0, dux_dxl, o_dux_dxl, 0.f, 0.f, 0.f);
          pml_update<false>(a.y, unused, V.ck[sl], 0.0, duz_dzl, o_duz_dzl, 0.f, 0.f, 0.f);
          pml_update<false>(b.x, unused, V.cm[sl], 0.0, dux_dxl, o_dux_dxl, 0.f, 0.f, 0.f);
          pml_update<false>(b.y, unused, V.cm[sl], 0.0, duz_dzl, o_duz_dzl, 0.f, 0.f, 0.f);
          pml_update<false>(c.x, unused, V.cm[sl], 0.0, dux_dzl, o_dux_dzl, 0.f, 0.f, 0.f);
          pml_update<false>(c.y, unused, V.cm[sl], 0.0, duz_dxl, o_duz_dxl, 0.f, 0.f, 0.f);
          vm[3 * sl] = a;
          vm[3 * sl + 1] = b;
          vm[3 * sl + 2] = c;
          ks_xx = static_cast<float>(ks_xx + V.k31[sl] * a.x);
          ks_zz = static_cast<float>(ks_zz + V.k13[sl] * a.y);
          ms_xx = static_cast<float>(ms_xx + V.m31[sl] * b.x);
          ms_zz = static_cast<float>(ms_zz + V.m13[sl] * b.y);
          ms_xz = static_cast<float>(ms_xz + V.m13[sl] * c.x);
          ms_zx = static_cast<float>(ms_zx + V.m31[sl] * c.y);
          pk_xx = static_cast<float>(pk_xx + V.phik[sl] * a.x);
          pk_zz = static_cast<float>(pk_zz + V.phik[sl] * a.y);
          pm_xx = static_cast<float>(pm_xx + V.phim[sl] * b.x);
          pm_zz = static_cast<float>(pm_zz + V.phim[sl] * b.y);
          pm_xz = static_cast<float>(pm_xz + V.phim[sl] * c.x);
          pm_zx = static_cast<float>(pm_zx + V.phim[sl] * c.y);
        }
        const float kp_xx = static_cast<float>(V.A01 * dux_dxl + ks_xx + V.k2 * r0.x + V.k3 * r0.y);
        const float kp_zz = static_cast<float>(V.A10 * duz_dzl + ks_zz + V.k4 * r1.z + V.k5 * r1.w);
        const float mp_xx = static_cast<float>(V.A01 * dux_dxl + ms_xx + V.m2 * r0.x + V.m3 * r0.y);
        const float mp_zz = static_cast<float>(V.A10 * duz_dzl + ms_zz + V.m4 * r1.z + V.m5 * r1.w);
        const float mp_xz = static_cast<float>(V.A10 * dux_dzl + ms_xz + V.m4 * r1.x + V.m5 * r1.y);
        const float mp_zx = static_cast<float>(V.A01 * duz_dxl + ms_zx + V.m2 * r0.z + V.m3 * r0.w);
        const float lpm = lambdal + mul;
        sxx = (lpm * kp_xx + mul * mp_xx) + (lpm * (duz_dzl + pk_zz) - mul * (duz_dzl + pm_zz));
        sxz = mul * mp_zx + mul * (dux_dzl + pm_xz);
        szx = mul * (duz_dxl + pm_zx) + mul * mp_xz;
        szz = (lpm * (dux_dxl + pk_xx) - mul * (dux_dxl + pm_xx)) + (lpm * kp_zz + mul * mp_zz);
      } else {
        // modified strains on the diagonal pairs: the stress is not symmetric
        const float m_dux_dxl = static_cast<float>(zx.A0 * dux_dxl + zx.A1 * r0.x + zx.A2 * r0.y);
        const float m_duz_dxl = static_cast<float>(zx.A0 * duz_dxl + zx.A1 * r0.z + zx.A2 * r0.w);
        const float m_dux_dzl = static_cast<float>(xz.A0 * dux_dzl + xz.A1 * r1.x + xz.A2 * r1.y);
        const float m_duz_dzl = static_cast<float>(xz.A0 * duz_dzl + xz.A1 * r1.z + xz.A2 * r1.w);
        sxx = lambdaplus2mu * m_dux_dxl + lambdal * duz_dzl;
        szz = lambdaplus2mu * m_duz_dzl + lambdal * dux_dxl;
        szx = mul * (duz_dxl + m_dux_dzl);
        sxz = mul * (dux_dzl + m_duz_dxl);
      }
      s_d1[f] = make_float2(jacobianl * (sxx * xixl + szx * xizl), jacobianl * (sxz * xixl + szz * xizl));
      s_d2[f] = make_float2(jacobianl * (sxx * gammaxl + szx * gammazl), jacobianl * (sxz * gammaxl + szz * gammazl));
      continue;
    }
    float sxx, szz, sxz;
    int ai = -1;
    if (ANISO) ai = P.aniso_idx[ti.elem_base + e];
    if (ANISO && ai >= 0) {
      const size_t ap = static_cast<size_t>(ai) * 25 + q;
      const float4 ca = P.c4[ap];
      const float2 cb = P.c2[ap];
      const double c11 = ca.x, c13 = ca.y, c15 = ca.z, c33 = ca.w, c35 = cb.x, c55 = cb.y;
      const double sh = static_cast<double>(duz_dxl) + static_cast<double>(dux_dzl);
      sxx = static_cast<float>(c11 * dux_dxl + c13 * duz_dzl + c15 * sh);
      szz = static_cast<float>(c13 * dux_dxl + c33 * duz_dzl + c35 * sh);
      sxz = static_cast<float>(c15 * dux_dxl + c35 * duz_dzl + c55 * sh);
    } else {
      sxx = lambdaplus2mu * dux_dxl + lambdal * duz_dzl;
      szz = lambdaplus2mu * duz_dzl + lambdal * dux_dxl;
      sxz = mul * (duz_dxl + dux_dzl);
    }
    if (ATTEN) {
      float e1s, e11s, e13s;
      attenuation_point<LDDRK>(P, static_cast<size_t>(ebase + f) * 3, dux_dxl, dux_dzl, duz_dxl, duz_dzl, stage, e1s,
                               e11s, e13s);
      const float lambdalplusmul = lambdal + mul;
      sxx = sxx + lambdalplusmul * e1s + 2.f * mul * e11s;
      sxz = sxz + mul * e13s;
      szz = szz + lambdalplusmul * e1s - 2.f * mul * e11s;
    }
    s_d1[f] = make_float2(jacobianl * (sxx * xixl + sxz * xizl), jacobianl * (sxz * xixl + szz * xizl));
    s_d2[f] = make_float2(jacobianl * (sxx * gammaxl + sxz * gammazl), jacobianl * (sxz * gammaxl + szz * gammazl));
  }
  __syncthreads();


  // 4c. weighted transpose lines: rows contract t1 with hprimewgll, columns t2,
  //     in place
  for (int t = tid, el = tid / 10; t < nlines; t += NT, el += NT / 10) {
    // with NT a multiple of 10 every thread keeps one line position r
    const int e = NT % 10 == 0 ? el : t / 10;
    const int r = NT % 10 == 0 ? tid % 10 : t - 10 * e;
    const int a0 = r < 5 ? 5 * r : r - 5;
    const int st = r < 5 ? 1 : 5;
    line_weighted(P, (r < 5 ? s_d1 : s_d2) + 25 * e + a0, st);
  }
  __syncthreads();

  // step-6 operands of the thread's first point, requested before the assembly
  float2 rm_next = make_float2(0.f, 0.f);
  int sp_next = 0;
  if (tid < n_int)
    rm_next = P.rmass[int_begin + tid];
  else if (tid < nl)
    sp_next = P.slot_pos[ti.sh_off + tid - n_int];

  // 5. assembly into the accumulator, one colour at a time (elements of a
  //    colour share no point): a -= wz * row term + wx * column term
  int cb = 0;
  for (int c = 0; c < ti.ncol; ++c) {
    const int ce = ti.col_end[c] * 25;
    for (int f = cb + tid, ef = (cb + tid) / 25; f < ce; f += NT, ef += NT / 25) {  // cb: a multiple of 25
      const int e = FIXQ ? ef : f / 25;
      const int q = FIXQ ? q0 : f - 25 * e;
      const int j = FIXQ ? j0 : q / 5;
      const int i = FIXQ ? i0 : q - 5 * j;
      const float2 rt = s_d1[f], ct = s_d2[f];
      const float wz = s_h[55 + j], wx = s_h[50 + i];
      const int l = s_lib[f];
      float2 acc = s_acc[l];
      acc.x -= wz * rt.x + wx * ct.x;
      acc.y -= wz * rt.y + wx * ct.y;
      if (PML) {
        // the layer's terms after the element's weak-form terms (compute_forces_viscoelastic.F90:785-797)
        const float2 pm = s_pml[f];
        acc.x -= pm.x;
        acc.y -= pm.y;
      }
      s_acc[l] = acc;
    }
    cb = ce;
    __syncthreads();
  }

  // 6. mass matrix, corrector or LDDRK update, write-back
  bool bad = false;
  for (int l = tid; l < nl; l += NT) {
    const float2 acc = s_acc[l];
    const float2 rm = rm_next;
    const int sp = sp_next;
    if (l + NT < n_int)
      rm_next = P.rmass[int_begin + l + NT];
    else if (l + NT < nl)
      sp_next = P.slot_pos[ti.sh_off + l + NT - n_int];
    if (l < n_int) {
      const int g = int_begin + l;
      const float2 a = make_float2(acc.x * rm.x, acc.y * rm.y);
      float2 v = s_v[l];
      float2 u = s_u[l];
      if (!LDDRK) {
        v.x = v.x + dto2 * a.x;
        v.y = v.y + dto2 * a.y;
      } else {
        const float al = P.alpha[stage], be = P.beta[stage];
        float2 vl = P.vL[g], ul = P.uL[g];
        vl.x = al * vl.x + dt * a.x;
        vl.y = al * vl.y + dt * a.y;
        ul.x = al * ul.x + dt * v.x;
        ul.y = al * ul.y + dt * v.y;
        v.x = v.x + be * vl.x;
        v.y = v.y + be * vl.y;
        u.x = u.x + be * ul.x;
        u.y = u.y + be * ul.y;
        P.vL[g] = vl;
        P.uL[g] = ul;
      }
      P.u[g] = u;
      P.v[g] = v;
      P.a[g] = a;
      if (P.frames) {
        const int fi = step - *P.frame_base;
        if (fi >= 0 && fi < P.nframes) {
          P.frames[static_cast<size_t>(fi) * P.nglob + g] = u;
          if (P.aframes) P.aframes[static_cast<size_t>(fi) * P.nglob + g] = a;
        }
      }
      if (KERN) {
        const float2 b = s_b[l];
        P.rho_kl_glob[g] = P.rho_kl_glob[g] + (a.x * b.x + a.y * b.y);
        if (P.hess_glob) {
          // compute_kernels_Hessian: |b_accel|^2 and accel . b_accel at the point
          const float2 ba = P.kaframes[static_cast<size_t>(*P.kern_base - step) * P.nglob + g];
          float2 h = P.hess_glob[g];
          h.x = h.x + (ba.x * ba.x + ba.y * ba.y);
          h.y = h.y + (a.x * ba.x + a.y * ba.y);
          P.hess_glob[g] = h;
        }
      }
      bad |= !(fabsf(u.x) < 1e25f && fabsf(u.y) < 1e25f);
    } else {
      P.partial[sp] = acc;
    }
  }
  if (bad) {
    if (P.tile_member)
      P.member_status[P.tile_member[tile0 + blockIdx.x]] = 1;
    else
      *P.d_status = 1;
  }
}

template <bool LDDRK, bool KERN>
__global__ void __launch_bounds__(SHARED_NT) k_elastic_shared(const Params P, int stage, int last_stage) {
  wait_previous_kernel();
  allow_next_kernel();
  const int s = blockIdx.x * SHARED_NT + threadIdx.x;
  const int step = *P.d_step_b;
  if (s < P.nshared && !(P.shared_member && P.member_status[P.shared_member[s]])) {
    const int g = P.shared_begin + s;
    float2 u = P.u[g], v = P.v[g];
    if (!LDDRK) {
      const float2 a0 = P.a[g];
      u.x = newmark_displ(u.x, v.x, a0.x, P.dt, P.dt2o2);
      u.y = newmark_displ(u.y, v.y, a0.y, P.dt, P.dt2o2);
      v.x = newmark_veloc(v.x, a0.x, P.dto2);
      v.y = newmark_veloc(v.y, a0.y, P.dto2);
    }
    if (P.sh_edge && P.sh_edge[s]) {  // outer edge of a CPML layer
      u = make_float2(0.f, 0.f);
      v = make_float2(0.f, 0.f);
    }
    float2 acc = make_float2(0.f, 0.f);
    for (int k = P.shp_off[s]; k < P.shp_off[s + 1]; ++k) {
      const float2 p = P.partial[k];
      acc.x += p.x;
      acc.y += p.y;
    }
    const float2 rm = P.rmass[g];
    const float2 a = make_float2(acc.x * rm.x, acc.y * rm.y);
    if (!LDDRK) {
      v.x = v.x + P.dto2 * a.x;
      v.y = v.y + P.dto2 * a.y;
    } else {
      const float al = P.alpha[stage], be = P.beta[stage];
      float2 vl = P.vL[g], ul = P.uL[g];
      vl.x = al * vl.x + P.dt * a.x;
      vl.y = al * vl.y + P.dt * a.y;
      ul.x = al * ul.x + P.dt * v.x;
      ul.y = al * ul.y + P.dt * v.y;
      v.x = v.x + be * vl.x;
      v.y = v.y + be * vl.y;
      u.x = u.x + be * ul.x;
      u.y = u.y + be * ul.y;
      P.vL[g] = vl;
      P.uL[g] = ul;
    }
    P.u[g] = u;
    P.v[g] = v;
    P.a[g] = a;
    if (P.frames) {
      const int fi = step - *P.frame_base;
      if (fi >= 0 && fi < P.nframes) {
        P.frames[static_cast<size_t>(fi) * P.nglob + g] = u;
        if (P.aframes) P.aframes[static_cast<size_t>(fi) * P.nglob + g] = a;
      }
    }
    if (KERN) {
      const float2 b = P.kframes[static_cast<size_t>(*P.kern_base - step) * P.nglob + g];
      P.rho_kl_glob[g] = P.rho_kl_glob[g] + (a.x * b.x + a.y * b.y);
      if (P.hess_glob) {
        const float2 ba = P.kaframes[static_cast<size_t>(*P.kern_base - step) * P.nglob + g];
        float2 h = P.hess_glob[g];
        h.x = h.x + (ba.x * ba.x + ba.y * ba.y);
        h.y = h.y + (a.x * ba.x + a.y * ba.y);
        P.hess_glob[g] = h;
      }
    }
    if (!(fabsf(u.x) < 1e25f && fabsf(u.y) < 1e25f)) {
      if (P.shared_member)
        P.member_status[P.shared_member[s]] = 1;
      else
        *P.d_status = 1;
    }
  }
  if (last_stage && blockIdx.x == 0 && threadIdx.x == 0) *P.d_step = step + 1;
}

// records the step before *d_step for every receiver
static __global__ void k_receivers(const Params P) {
  wait_previous_kernel();
  allow_next_kernel();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < P.nrec) record_receiver(P, r, *P.d_step - 1);
}

static __global__ void k_permute_in(const float2 *src, const int *dev2glob, float2 *dst, int n) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) dst[d] = src[dev2glob[d]];
}

static __global__ void k_permute_out(const float2 *src, const int *dev2glob, float2 *dst, int n) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) dst[dev2glob[d]] = src[d];
}

static __global__ void k_max_norm(const float2 *u, int n, unsigned int *out) {
  float m = 0.f;
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
    const float2 x = u[d];
    const float nn = sqrtf(x.x * x.x + x.y * x.y);
    m = (nn == nn) ? fmaxf(m, nn) : __int_as_float(0x7f800000);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

}  // namespace sf2d
