// Tile-staged fused Newmark step for the isotropic elastic SEM (NGLL = 5).
//
// One CTA advances one tile of elements by one time step:
//   1. predictor u' = u + dt v + dt^2/2 a, v' = v + dt/2 a for every point
//      the tile touches (update_displacement_Newmark.F90:408-454), staged in
//      shared memory;
//   2. Stacey traction on the predicted velocity and the force sources
//      (compute_stacey_elastic.f90:160-335, compute_add_sources_viscoelastic.f90)
//      by one thread in reference order;
//   3. per GLL point: gradient through hprime, Jacobian mapping, isotropic
//      stress (lambda and mu as compute_forces_viscoelastic.F90:286-294 forms
//      them), weak-form terms
//      (compute_forces_viscoelastic.F90:184-675);
//   4. weighted transpose contraction with hprimewgll (:760-782);
//   5. assembly into the shared-memory accumulator colour by colour
//      (no two elements of a colour share a point, so no atomics);
//   6. interior points: a *= rmass_inverse, v = v' + dt/2 a
//      (update_displacement_Newmark.F90:564-589) and write-back; shared
//      points: the tile's partial sum is written to its slot.
// A second kernel finishes shared points, adding the partial sums in tile
// order.  Results are bit-identical from run to run.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "sf2d_b200.h"
#include "sf2d_tiler.h"

namespace sf2d {

struct Params {
  float2 *u, *v, *a;
  const float2 *rmass;
  const TileInfo *tiles;
  const uint16_t *lib;
  const float4 *geo;   // xix, xiz, gammax, gammaz per element GLL point (tile slot order)
  const float2 *mat;   // lambda, mu (lambda = rho*cp*cp - 2*mu in FP32, as the CPU solver forms it)
  const int *sh_ids;
  float2 *partial;
  const int *shp_off, *shp_slots;
  const int *st_local;
  const float4 *st_nw;    // nx, nz, weight, 0
  const float2 *st_rho;   // rho*vp, rho*vs
  const int *src_local, *src_id;
  const float2 *src_arr;
  const float *stf;
  const int *rec_id, *rec_dev;
  const double *rec_h;    // 10 per receiver: hxir[5], hgammar[5]
  double *seis;           // [irec][it][2]
  int *d_step, *d_status;
  int nstep_stf, nstep_seis, seismotype, nrec;
  double cosrot, sinrot;
  float dt, dto2, dt2o2;
  int shared_begin, nshared;
  int max_q, max_local;
  float hconst[60];  // hprime[25], hprimewgll[25], wxgll[5], wzgll[5]
};

constexpr int BS = 256;

__device__ __forceinline__ void record_receiver(const Params &P, int r, int step) {
  if (step < 0 || step >= P.nstep_seis) return;
  const float2 *field = P.seismotype == 2 ? P.v : (P.seismotype == 3 ? P.a : P.u);
  const int *dev = P.rec_dev + 25 * r;
  const double *h = P.rec_h + 10 * r;
  double vx = 0.0, vz = 0.0;
  for (int j = 0; j < 5; ++j)
    for (int i = 0; i < 5; ++i) {
      const float2 f = field[dev[j * 5 + i]];
      const double hl = h[i] * h[5 + j];
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

// Shared-memory layout of one tile (sizes from the largest tile); every region
// starts on a 16-byte boundary, as 16-byte cp.async destinations require:
//   geo  float4[max_q]  xix, xiz, gammax, gammaz; overwritten by the weak-form terms
//   mat  float2[max_q]  lambda, mu
//   u, v, acc float2[max_local]  (old u, v, a -> predicted u, v and the accumulator)
//   h    float[64]      hprime, hprimewgll, wxgll, wzgll
//   lib  uint16[max_q rounded up to 8]
struct TileSmem {
  size_t geo, mat, u, v, acc, h, lib, total;
};
__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~static_cast<size_t>(15); }
__host__ __device__ inline TileSmem tile_smem_layout(int max_q, int max_local) {
  TileSmem L;
  size_t o = 0;
  L.geo = o;
  o = align16(o + static_cast<size_t>(max_q) * sizeof(float4));
  L.mat = o;
  o = align16(o + static_cast<size_t>(max_q) * sizeof(float2));
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
  L.total = o;
  return L;
}

template <int NT>
__global__ void __launch_bounds__(NT) k_elastic_tile(const Params P, int record_prev) {
  extern __shared__ __align__(16) unsigned char smem[];
  const TileInfo &ti = P.tiles[blockIdx.x];
  const int tid = threadIdx.x;
  const int n_int = ti.n_int;
  const int n_sh = ti.n_sh;
  const int nl = n_int + n_sh;
  const int nq = ti.nelem * 25;
  const int ebase = ti.elem_base * 25;
  const int int_begin = ti.int_begin;
  const TileSmem L = tile_smem_layout(P.max_q, P.max_local);
  float4 *s_geo = reinterpret_cast<float4 *>(smem + L.geo);
  float2 *s_mat = reinterpret_cast<float2 *>(smem + L.mat);
  float2 *s_u = reinterpret_cast<float2 *>(smem + L.u);
  float2 *s_v = reinterpret_cast<float2 *>(smem + L.v);
  float2 *s_acc = reinterpret_cast<float2 *>(smem + L.acc);
  float *s_h = reinterpret_cast<float *>(smem + L.h);
  uint16_t *s_lib = reinterpret_cast<uint16_t *>(smem + L.lib);

  const int step = *P.d_step;
  // receivers of the previous step read the old fields before any write
  if (record_prev && tid < ti.rec_n) record_receiver(P, ti.rec_off + tid, step - 1);

  // 1. every load of the tile is issued at once, straight into shared memory
  {
    const uint4 *glib = reinterpret_cast<const uint4 *>(P.lib + ti.lib_off);
    const int nlib16 = (nq + 7) / 8;
    for (int k = tid; k < nlib16; k += NT) cp_async16(s_lib + 8 * k, glib + k);
    for (int f = tid; f < nq; f += NT) {
      cp_async16(s_geo + f, P.geo + ebase + f);
      cp_async8(s_mat + f, P.mat + ebase + f);
    }
    for (int l = tid; l < n_int; l += NT) {
      const int g = int_begin + l;
      cp_async8(s_u + l, P.u + g);
      cp_async8(s_v + l, P.v + g);
      cp_async8(s_acc + l, P.a + g);
    }
    for (int k = tid; k < n_sh; k += NT) {
      const int g = P.sh_ids[ti.sh_off + k];
      cp_async8(s_u + n_int + k, P.u + g);
      cp_async8(s_v + n_int + k, P.v + g);
      cp_async8(s_acc + n_int + k, P.a + g);
    }
    if (tid < 60) s_h[tid] = P.hconst[tid];
    cp_async_wait_all();
  }
  __syncthreads();

  // 2. Newmark predictor in place
  const float dt = P.dt, dto2 = P.dto2, dt2o2 = P.dt2o2;
  for (int l = tid; l < nl; l += NT) {
    float2 u = s_u[l], v = s_v[l];
    const float2 a = s_acc[l];
    u.x = u.x + dt * v.x + dt2o2 * a.x;
    u.y = u.y + dt * v.y + dt2o2 * a.y;
    v.x = v.x + dto2 * a.x;
    v.y = v.y + dto2 * a.y;
    s_u[l] = u;
    s_v[l] = v;
    s_acc[l] = make_float2(0.f, 0.f);
  }
  __syncthreads();

  // 3. boundary terms and sources in reference order, one thread (overlaps pass 1)
  if (tid == 0) {
    for (int p = ti.st_off; p < ti.st_off + ti.st_n; ++p) {
      const int l = P.st_local[p];
      const float4 nw = P.st_nw[p];
      const float2 rr = P.st_rho[p];
      const float2 v = s_v[l];
      const float vn = nw.x * v.x + nw.y * v.y;
      const float tx = rr.x * vn * nw.x + rr.y * (v.x - vn * nw.x);
      const float tz = rr.x * vn * nw.y + rr.y * (v.y - vn * nw.y);
      float2 acc = s_acc[l];
      acc.x -= tx * nw.z;
      acc.y -= tz * nw.z;
      s_acc[l] = acc;
    }
    for (int p = ti.src_off; p < ti.src_off + ti.src_n; ++p) {
      const int l = P.src_local[p];
      const float f = step < P.nstep_stf ? P.stf[static_cast<size_t>(P.src_id[p]) * P.nstep_stf + step] : 0.f;
      const float2 sa = P.src_arr[p];
      float2 acc = s_acc[l];
      acc.x += sa.x * f;
      acc.y += sa.y * f;
      s_acc[l] = acc;
    }
  }

  // 4. element pass 1: gradient, stress, weak-form terms (written over the geometry)
  for (int f = tid; f < nq; f += NT) {
    const int e = f / 25;
    const int q = f - 25 * e;
    const int j = q / 5;
    const int i = q - 5 * j;
    const uint16_t *le = s_lib + 25 * e;
    float dux_dxi = 0.f, duz_dxi = 0.f, dux_dg = 0.f, duz_dg = 0.f;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const float2 r = s_u[le[5 * j + k]];
      const float hx = s_h[5 * i + k];
      dux_dxi += r.x * hx;
      duz_dxi += r.y * hx;
      const float2 c = s_u[le[5 * k + i]];
      const float hz = s_h[5 * j + k];
      dux_dg += c.x * hz;
      duz_dg += c.y * hz;
    }
    const float4 g4 = s_geo[f];
    const float2 m2 = s_mat[f];
    const float xixl = g4.x, xizl = g4.y, gammaxl = g4.z, gammazl = g4.w;
    const float jacobianl = 1.f / (xixl * gammazl - gammaxl * xizl);
    const float dux_dxl = dux_dxi * xixl + dux_dg * gammaxl;
    const float dux_dzl = dux_dxi * xizl + dux_dg * gammazl;
    const float duz_dxl = duz_dxi * xixl + duz_dg * gammaxl;
    const float duz_dzl = duz_dxi * xizl + duz_dg * gammazl;
    const float mul = m2.y;
    const float lambdal = m2.x;
    const float lambdaplus2mu = lambdal + 2.f * mul;
    const float sxx = lambdaplus2mu * dux_dxl + lambdal * duz_dzl;
    const float szz = lambdaplus2mu * duz_dzl + lambdal * dux_dxl;
    const float sxz = mul * (duz_dxl + dux_dzl);
    s_geo[f] = make_float4(jacobianl * (sxx * xixl + sxz * xizl), jacobianl * (sxz * xixl + szz * xizl),
                           jacobianl * (sxx * gammaxl + sxz * gammazl), jacobianl * (sxz * gammaxl + szz * gammazl));
  }
  __syncthreads();

  // 5. weighted transpose contraction assembled straight into the accumulator,
  //    one colour at a time (elements of a colour share no point)
  int cb = 0;
  for (int c = 0; c < ti.ncol; ++c) {
    const int ce = ti.col_end[c] * 25;
    for (int f = cb + tid; f < ce; f += NT) {
      const int e = f / 25;
      const int q = f - 25 * e;
      const int j = q / 5;
      const int i = q - 5 * j;
      const float4 *te = s_geo + 25 * e;
      float tx1 = 0.f, tz1 = 0.f, tx2 = 0.f, tz2 = 0.f;
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const float4 r = te[5 * j + k];
        const float w1 = s_h[25 + 5 * k + i];
        tx1 += r.x * w1;
        tz1 += r.y * w1;
        const float4 cc = te[5 * k + i];
        const float w2 = s_h[25 + 5 * k + j];
        tx2 += cc.z * w2;
        tz2 += cc.w * w2;
      }
      const float wz = s_h[55 + j], wx = s_h[50 + i];
      const int l = s_lib[f];
      float2 acc = s_acc[l];
      acc.x -= wz * tx1 + wx * tx2;
      acc.y -= wz * tz1 + wx * tz2;
      s_acc[l] = acc;
    }
    cb = ce;
    __syncthreads();
  }

  // 6. mass matrix, corrector, write-back
  bool bad = false;
  for (int l = tid; l < nl; l += NT) {
    const float2 acc = s_acc[l];
    if (l < n_int) {
      const int g = int_begin + l;
      const float2 rm = P.rmass[g];
      const float2 a = make_float2(acc.x * rm.x, acc.y * rm.y);
      float2 v = s_v[l];
      v.x = v.x + dto2 * a.x;
      v.y = v.y + dto2 * a.y;
      const float2 u = s_u[l];
      P.u[g] = u;
      P.v[g] = v;
      P.a[g] = a;
      bad |= !(fabsf(u.x) < 1e25f && fabsf(u.y) < 1e25f);
    } else {
      P.partial[ti.sh_off + l - n_int] = acc;
    }
  }
  if (bad) *P.d_status = 1;
}

__global__ void __launch_bounds__(BS) k_elastic_shared(const Params P) {
  const int s = blockIdx.x * BS + threadIdx.x;
  if (s < P.nshared) {
    const int g = P.shared_begin + s;
    float2 u = P.u[g], v = P.v[g];
    const float2 a0 = P.a[g];
    u.x = u.x + P.dt * v.x + P.dt2o2 * a0.x;
    u.y = u.y + P.dt * v.y + P.dt2o2 * a0.y;
    v.x = v.x + P.dto2 * a0.x;
    v.y = v.y + P.dto2 * a0.y;
    float2 acc = make_float2(0.f, 0.f);
    for (int k = P.shp_off[s]; k < P.shp_off[s + 1]; ++k) {
      const float2 p = P.partial[P.shp_slots[k]];
      acc.x += p.x;
      acc.y += p.y;
    }
    const float2 rm = P.rmass[g];
    const float2 a = make_float2(acc.x * rm.x, acc.y * rm.y);
    v.x = v.x + P.dto2 * a.x;
    v.y = v.y + P.dto2 * a.y;
    P.u[g] = u;
    P.v[g] = v;
    P.a[g] = a;
    if (!(fabsf(u.x) < 1e25f && fabsf(u.y) < 1e25f)) *P.d_status = 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *P.d_step = *P.d_step + 1;
}

// records the step before *d_step for every receiver
__global__ void k_receivers(const Params P) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < P.nrec) record_receiver(P, r, *P.d_step - 1);
}

__global__ void k_permute_in(const float2 *src, const int *dev2glob, float2 *dst, int n) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) dst[d] = src[dev2glob[d]];
}

__global__ void k_permute_out(const float2 *src, const int *dev2glob, float2 *dst, int n) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) dst[dev2glob[d]] = src[d];
}

__global__ void k_max_norm(const float2 *u, int n, unsigned int *out) {
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

// ---------------------------------------------------------------------------
// host runtime
// ---------------------------------------------------------------------------
namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define SF2D_CUDA(call)                                                                       \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(e_ == cudaErrorMemoryAllocation ? SF2D_ERR_OOM : SF2D_ERR_CUDA,             \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                        \
  } while (0)

}  // namespace

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
  void launch_tile(bool record_prev) {
    const int rp = record_prev ? 1 : 0;
    switch (nt) {
      case 128: sf2d::k_elastic_tile<128><<<T.ntiles, 128, smem, stream>>>(P, rp); break;
      case 512: sf2d::k_elastic_tile<512><<<T.ntiles, 512, smem, stream>>>(P, rp); break;
      default: sf2d::k_elastic_tile<256><<<T.ntiles, 256, smem, stream>>>(P, rp); break;
    }
  }
  int launch_step(bool record_prev) {
    launch_tile(record_prev);
    const int nb = std::max(1, (P.nshared + sf2d::BS - 1) / sf2d::BS);
    sf2d::k_elastic_shared<<<nb, sf2d::BS, 0, stream>>>(P);
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

extern "C" const char *sf2d_last_error(void) { return g_err.c_str(); }

extern "C" int sf2d_elastic_create(const sf2d_elastic_desc *d, sf2d_solver **out) {
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

  auto *S = new sf2d_solver();
  std::unique_ptr<sf2d_solver> guard(S);
  const int te = d->tile_elems > 0 ? d->tile_elems : 64;
  std::string err = build_tiling(d->nspec, d->nglob, d->ibool, d->centroid_xz, te, S->T);
  if (!err.empty()) return fail(SF2D_ERR_INVALID, "tiling: " + err);
  const Tiling &T = S->T;
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

  SF2D_CUDA(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
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
  UP(shp_slots, int, T.shp_slots);
  UP(st_local, int, st_local);
  UP(st_nw, float4, st_nw);
  UP(st_rho, float2, st_rho);
  UP(src_local, int, src_local);
  UP(src_id, int, src_id);
  UP(src_arr, float2, src_arr);
  UP(rec_id, int, rec_id);
  UP(rec_dev, int, rec_dev);
  UP(rec_h, double, rec_h);
#undef UP
  float2 *partial;
  if ((rc = S->alloc(&partial, T.sh_ids.size()))) return rc;
  P.partial = partial;
  std::vector<float> stf(static_cast<size_t>(d->nsrc) * d->nstep);
  if (d->nsrc) std::memcpy(stf.data(), d->stf, stf.size() * sizeof(float));
  float *d_stf;
  if ((rc = S->upload(&d_stf, stf.data(), stf.size()))) return rc;
  P.stf = d_stf;
  double *seis;
  if ((rc = S->alloc(&seis, static_cast<size_t>(d->nrec) * d->nstep * 2))) return rc;
  P.seis = seis;
  if (d->nrec && d->nstep) SF2D_CUDA(cudaMemset(seis, 0, sizeof(double) * d->nrec * d->nstep * 2));
  int *ctr;
  if ((rc = S->alloc(&ctr, 2))) return rc;
  SF2D_CUDA(cudaMemset(ctr, 0, 2 * sizeof(int)));
  P.d_step = ctr;
  P.d_status = ctr + 1;
  if ((rc = S->upload(&S->d_dev2glob, T.dev2glob.data(), T.dev2glob.size()))) return rc;
  if ((rc = S->alloc(&S->d_stage, d->nglob))) return rc;
  if ((rc = S->alloc(&S->d_norm, 1))) return rc;
  P.nstep_stf = d->nstep;
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
  S->smem = tile_smem_layout(P.max_q, P.max_local).total;
  if (S->smem > 220 * 1024) return fail(SF2D_ERR_INVALID, "tile too large for shared memory");
  S->nt = d->threads_per_block > 0 ? d->threads_per_block : 256;
  if (S->nt != 128 && S->nt != 256 && S->nt != 512)
    return fail(SF2D_ERR_INVALID, "threads_per_block must be 128, 256 or 512");
  if (d->nrec > 0) {
    for (const TileInfo &t : tiles)
      if (t.rec_n > S->nt) return fail(SF2D_ERR_INVALID, "more receivers in one tile than threads per CTA");
  }
  SF2D_CUDA(cudaFuncSetAttribute(k_elastic_tile<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(S->smem)));
  SF2D_CUDA(cudaFuncSetAttribute(k_elastic_tile<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(S->smem)));
  SF2D_CUDA(cudaFuncSetAttribute(k_elastic_tile<512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(S->smem)));
  S->nglob = d->nglob;
  S->nrec = d->nrec;
  S->nstep_total = d->nstep;
  SF2D_CUDA(cudaStreamSynchronize(S->stream));
  *out = guard.release();
  return SF2D_OK;
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

extern "C" int sf2d_enqueue(sf2d_solver *S, int nstep) {
  if (!S || nstep < 0) return fail(SF2D_ERR_INVALID, "bad arguments");
  const int K = S->chunk;
  int done = 0;
  if (nstep >= K) {
    if (!S->graph || S->graph_steps != K) {
      if (S->graph) cudaGraphExecDestroy(S->graph);
      S->graph = nullptr;
      cudaGraph_t g;
      SF2D_CUDA(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
      S->launch_chunk(K);
      SF2D_CUDA(cudaStreamEndCapture(S->stream, &g));
      cudaError_t e = cudaGraphInstantiate(&S->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(SF2D_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      S->graph_steps = K;
    }
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
      return fail(SF2D_ERR_CUDA, "timeout waiting for the time loop");
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  int status = 0;
  SF2D_CUDA(cudaMemcpy(&status, S->P.d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (status) return fail(SF2D_ERR_UNSTABLE, "wavefield blew up (NaN or |u| > 1e25)");
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
  std::vector<cudaEvent_t> ev(3 * nstep);
  for (auto &e : ev) SF2D_CUDA(cudaEventCreate(&e));
  for (int k = 0; k < nstep; ++k) {
    SF2D_CUDA(cudaEventRecord(ev[3 * k], S->stream));
    S->launch_tile(k > 0);
    SF2D_CUDA(cudaEventRecord(ev[3 * k + 1], S->stream));
    const int nb = std::max(1, (S->P.nshared + sf2d::BS - 1) / sf2d::BS);
    sf2d::k_elastic_shared<<<nb, sf2d::BS, 0, S->stream>>>(S->P);
    SF2D_CUDA(cudaEventRecord(ev[3 * k + 2], S->stream));
  }
  S->launch_receivers();
  SF2D_CUDA(cudaGetLastError());
  SF2D_CUDA(cudaStreamSynchronize(S->stream));
  double a = 0, b = 0;
  for (int k = 0; k < nstep; ++k) {
    float x = 0, y = 0;
    cudaEventElapsedTime(&x, ev[3 * k], ev[3 * k + 1]);
    cudaEventElapsedTime(&y, ev[3 * k + 1], ev[3 * k + 2]);
    a += x;
    b += y;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  S->steps_done += nstep;
  ms[0] = static_cast<float>(a / nstep);
  ms[1] = static_cast<float>(b / nstep);
  ms[2] = static_cast<float>((a + b) / nstep);
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
  info[7] = 0;
  return SF2D_OK;
}

extern "C" int sf2d_destroy(sf2d_solver *S) {
  if (!S) return SF2D_OK;
  cudaStreamSynchronize(S->stream);
  delete S;
  return SF2D_OK;
}
