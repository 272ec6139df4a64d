// CPU oracle for the SPECFEM2D time-marching hot path -- TEST INFRASTRUCTURE.
//
// A restatement of the reference's CPU routines, used only as the checker of
// the CUDA path and as the timed CPU baseline.  `real` is float for the
// CUSTOM_REAL=4 build and double for the CUSTOM_REAL=8 build.
//
// Summation order follows the serial reference: within a step, Stacey and
// source terms are added first (iphase 1 of
// src/specfem2D/compute_forces_viscoelastic_calling_routine.F90:58-100, all
// elements are "inner" with one process), then element contributions in
// ascending element order.  Element work is spread over host threads into
// a per-element buffer and assembled serially, so results do not depend on
// the thread count.
#include "sf2d_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <thread>
#include <vector>

namespace {

constexpr int NGLL = 5;
constexpr int NGLL2 = 25;

int default_threads() {
  const char *env = std::getenv("SF2D_ORACLE_THREADS");
  if (env && std::atoi(env) > 0) return std::atoi(env);
  const unsigned n = std::thread::hardware_concurrency();
  return n ? static_cast<int>(n) : 1;
}

// Static block partition of [0, n) over `nt` threads.
template <typename F>
void parallel_for(int n, int nt, F &&f) {
  nt = std::max(1, std::min(nt, n));
  if (nt == 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(nt);
  for (int t = 0; t < nt; ++t) {
    const int b = static_cast<int>(static_cast<long long>(n) * t / nt);
    const int e = static_cast<int>(static_cast<long long>(n) * (t + 1) / nt);
    pool.emplace_back([&f, b, e] { f(b, e); });
  }
  for (auto &th : pool) th.join();
}

template <typename real>
struct Db {
  int nspec, nglob;
  const int *ibool;
  std::vector<real> xix, xiz, gammax, gammaz, jacobian, rho, kappa, mu, rho_vp, rmass;
  real hprime[NGLL][NGLL], hprimewgll[NGLL][NGLL], wxgll[NGLL], wzgll[NGLL];
  std::vector<real> st_nx, st_nz, st_w, st_rvp, st_rvs, srcarr;
  std::vector<real> c11, c13, c15, c33, c35, c55;
  const int *aniso;
  real deltat, deltatover2, deltatsquareover2;
};

template <typename real>
std::vector<real> cvt(const double *p, size_t n) {
  std::vector<real> v(n);
  if (p)
    for (size_t k = 0; k < n; ++k) v[k] = static_cast<real>(p[k]);
  return v;
}

template <typename real>
void load(const sf2d_oracle_db *d, Db<real> &o) {
  const size_t nl = static_cast<size_t>(d->nspec) * NGLL2;
  o.nspec = d->nspec;
  o.nglob = d->nglob;
  o.ibool = d->ibool;
  o.xix = cvt<real>(d->xix, nl);
  o.xiz = cvt<real>(d->xiz, nl);
  o.gammax = cvt<real>(d->gammax, nl);
  o.gammaz = cvt<real>(d->gammaz, nl);
  o.jacobian = cvt<real>(d->jacobian, nl);
  o.rho = cvt<real>(d->rhostore, nl);
  o.kappa = cvt<real>(d->kappastore, nl);
  o.mu = cvt<real>(d->mustore, nl);
  o.rho_vp = cvt<real>(d->rho_vpstore, nl);
  o.rmass = cvt<real>(d->rmass_inverse, static_cast<size_t>(d->nglob) * 2);
  for (int a = 0; a < NGLL; ++a) {
    o.wxgll[a] = static_cast<real>(d->wxgll[a]);
    o.wzgll[a] = static_cast<real>(d->wzgll[a]);
    for (int b = 0; b < NGLL; ++b) {
      o.hprime[a][b] = static_cast<real>(d->hprime[a * NGLL + b]);
      o.hprimewgll[a][b] = static_cast<real>(d->hprimewgll[a * NGLL + b]);
    }
  }
  o.st_nx = cvt<real>(d->st_nx, d->nstacey);
  o.st_nz = cvt<real>(d->st_nz, d->nstacey);
  o.st_w = cvt<real>(d->st_w, d->nstacey);
  o.st_rvp = cvt<real>(d->st_rvp, d->nstacey);
  o.st_rvs = cvt<real>(d->st_rvs, d->nstacey);
  o.srcarr = cvt<real>(d->sourcearrays, static_cast<size_t>(d->nsrc) * NGLL2 * 2);
  o.aniso = d->ispec_is_anisotropic;
  if (d->ispec_is_anisotropic) {
    o.c11 = cvt<real>(d->c11, nl);
    o.c13 = cvt<real>(d->c13, nl);
    o.c15 = cvt<real>(d->c15, nl);
    o.c33 = cvt<real>(d->c33, nl);
    o.c35 = cvt<real>(d->c35, nl);
    o.c55 = cvt<real>(d->c55, nl);
  }
  o.deltat = static_cast<real>(d->deltat);
  o.deltatover2 = static_cast<real>(d->deltatover2);
  o.deltatsquareover2 = static_cast<real>(d->deltatsquareover2);
}

// Element internal force -K u for one element (compute_forces_viscoelastic.F90:
// 184-197 gather, :810-883 mxm_4comp_singleA, :220-234 mapping, :286-357
// isotropic P-SV stress with lambda = rho*cp^2 - 2 mu, :372-445 anisotropic,
// :669-675 weak-form terms, :760-782 weighted transpose contraction).
// Writes the 25x2 contributions (to be subtracted) into `out`.
template <typename real>
void element_force(const Db<real> &o, int ispec, const real *displ, real *out) {
  const size_t off = static_cast<size_t>(ispec) * NGLL2;
  real ux[NGLL][NGLL], uz[NGLL][NGLL];  // [j][i]
  for (int j = 0; j < NGLL; ++j)
    for (int i = 0; i < NGLL; ++i) {
      const int g = o.ibool[off + j * NGLL + i];
      ux[j][i] = displ[2 * g];
      uz[j][i] = displ[2 * g + 1];
    }
  real t1x[NGLL][NGLL], t1z[NGLL][NGLL], t2x[NGLL][NGLL], t2z[NGLL][NGLL];
  const bool is_aniso = o.aniso && o.aniso[ispec];
  for (int j = 0; j < NGLL; ++j)
    for (int i = 0; i < NGLL; ++i) {
      // x1 = dux_dxi(i,j) = sum_k A(1,k,j) * hprime(i,k)
      const real dux_dxi = ux[j][0] * o.hprime[i][0] + ux[j][1] * o.hprime[i][1] +
                           ux[j][2] * o.hprime[i][2] + ux[j][3] * o.hprime[i][3] +
                           ux[j][4] * o.hprime[i][4];
      const real duz_dxi = uz[j][0] * o.hprime[i][0] + uz[j][1] * o.hprime[i][1] +
                           uz[j][2] * o.hprime[i][2] + uz[j][3] * o.hprime[i][3] +
                           uz[j][4] * o.hprime[i][4];
      const real dux_dgamma = ux[0][i] * o.hprime[j][0] + ux[1][i] * o.hprime[j][1] +
                              ux[2][i] * o.hprime[j][2] + ux[3][i] * o.hprime[j][3] +
                              ux[4][i] * o.hprime[j][4];
      const real duz_dgamma = uz[0][i] * o.hprime[j][0] + uz[1][i] * o.hprime[j][1] +
                              uz[2][i] * o.hprime[j][2] + uz[3][i] * o.hprime[j][3] +
                              uz[4][i] * o.hprime[j][4];
      const size_t p = off + j * NGLL + i;
      const real xixl = o.xix[p], xizl = o.xiz[p], gammaxl = o.gammax[p], gammazl = o.gammaz[p];
      const real jacobianl = o.jacobian[p];
      const real dux_dxl = dux_dxi * xixl + dux_dgamma * gammaxl;
      const real dux_dzl = dux_dxi * xizl + dux_dgamma * gammazl;
      const real duz_dxl = duz_dxi * xixl + duz_dgamma * gammaxl;
      const real duz_dzl = duz_dxi * xizl + duz_dgamma * gammazl;
      real sigma_xx, sigma_zz, sigma_xz;
      if (!is_aniso) {
        const real mul = o.mu[p];
        const real rhol = o.rho[p];
        const real cpl = o.rho_vp[p] / rhol;
        const real lambdal = rhol * cpl * cpl - real(2) * mul;
        const real lambdaplus2mu = lambdal + real(2) * mul;
        sigma_xx = lambdaplus2mu * dux_dxl + lambdal * duz_dzl;
        sigma_zz = lambdaplus2mu * duz_dzl + lambdal * dux_dxl;
        sigma_xz = mul * (duz_dxl + dux_dzl);
      } else {
        // c_ij are read as double in the reference (compute_forces_viscoelastic.F90:112)
        const double c11 = o.c11[p], c13 = o.c13[p], c15 = o.c15[p];
        const double c33 = o.c33[p], c35 = o.c35[p], c55 = o.c55[p];
        sigma_xx = static_cast<real>(c11 * dux_dxl + c13 * duz_dzl + c15 * (duz_dxl + dux_dzl));
        sigma_zz = static_cast<real>(c13 * dux_dxl + c33 * duz_dzl + c35 * (duz_dxl + dux_dzl));
        sigma_xz = static_cast<real>(c15 * dux_dxl + c35 * duz_dzl + c55 * (duz_dxl + dux_dzl));
      }
      const real sigma_zx = sigma_xz;
      t1x[j][i] = jacobianl * (sigma_xx * xixl + sigma_zx * xizl);
      t1z[j][i] = jacobianl * (sigma_xz * xixl + sigma_zz * xizl);
      t2x[j][i] = jacobianl * (sigma_xx * gammaxl + sigma_zx * gammazl);
      t2z[j][i] = jacobianl * (sigma_xz * gammaxl + sigma_zz * gammazl);
    }
  for (int j = 0; j < NGLL; ++j)
    for (int i = 0; i < NGLL; ++i) {
      real tx1 = 0, tx2 = 0, tz1 = 0, tz2 = 0;
      for (int k = 0; k < NGLL; ++k) {
        tx1 = tx1 + t1x[j][k] * o.hprimewgll[k][i];
        tx2 = tx2 + t2x[k][i] * o.hprimewgll[k][j];
        tz1 = tz1 + t1z[j][k] * o.hprimewgll[k][i];
        tz2 = tz2 + t2z[k][i] * o.hprimewgll[k][j];
      }
      out[2 * (j * NGLL + i)] = o.wzgll[j] * tx1 + o.wxgll[i] * tx2;
      out[2 * (j * NGLL + i) + 1] = o.wzgll[j] * tz1 + o.wxgll[i] * tz2;
    }
}

template <typename real>
int run_newmark(const sf2d_oracle_db *d, int it0, int nstep, real *displ, real *veloc, real *accel,
                double *seis, int nthreads) {
  Db<real> o;
  load(d, o);
  const int nglob = d->nglob;
  const int nspec = d->nspec;
  std::vector<real> contrib(static_cast<size_t>(nspec) * NGLL2 * 2);
  const int nt = nthreads > 0 ? nthreads : default_threads();
  for (int s = 0; s < nstep; ++s) {
    const int it = it0 + s;
    // predictor (update_displacement_Newmark.F90:408-454)
    for (int g = 0; g < 2 * nglob; ++g) {
      displ[g] = displ[g] + o.deltat * veloc[g] + o.deltatsquareover2 * accel[g];
      veloc[g] = veloc[g] + o.deltatover2 * accel[g];
      accel[g] = 0;
    }
    // iphase 1: Stacey (compute_stacey_elastic.f90:160-335) then force sources
    // (compute_add_sources_viscoelastic.f90:36-101)
    for (int p = 0; p < d->nstacey; ++p) {
      const int g = d->st_iglob[p];
      const real vx = veloc[2 * g], vz = veloc[2 * g + 1];
      const real nx = o.st_nx[p], nz = o.st_nz[p];
      const real vn = nx * vx + nz * vz;
      const real tx = o.st_rvp[p] * vn * nx + o.st_rvs[p] * (vx - vn * nx);
      const real tz = o.st_rvp[p] * vn * nz + o.st_rvs[p] * (vz - vn * nz);
      accel[2 * g] = accel[2 * g] - tx * o.st_w[p];
      accel[2 * g + 1] = accel[2 * g + 1] - tz * o.st_w[p];
    }
    for (int isrc = 0; isrc < d->nsrc; ++isrc) {
      const real stf = static_cast<real>(d->stf[(static_cast<size_t>(isrc) * d->nstep_total + it) * d->nstage]);
      const int e = d->src_ispec[isrc];
      for (int j = 0; j < NGLL; ++j)
        for (int i = 0; i < NGLL; ++i) {
          const int g = d->ibool[static_cast<size_t>(e) * NGLL2 + j * NGLL + i];
          const size_t q = (static_cast<size_t>(isrc) * NGLL2 + j * NGLL + i) * 2;
          accel[2 * g] = accel[2 * g] + o.srcarr[q] * stf;
          accel[2 * g + 1] = accel[2 * g + 1] + o.srcarr[q + 1] * stf;
        }
    }
    // iphase 2: all elements
    parallel_for(nspec, nspec > 256 ? nt : 1, [&](int b, int e1) {
      for (int e = b; e < e1; ++e) element_force(o, e, displ, &contrib[static_cast<size_t>(e) * NGLL2 * 2]);
    });
    for (int e = 0; e < nspec; ++e) {
      const real *c = &contrib[static_cast<size_t>(e) * NGLL2 * 2];
      const int *ib = &d->ibool[static_cast<size_t>(e) * NGLL2];
      for (int q = 0; q < NGLL2; ++q) {
        const int g = ib[q];
        accel[2 * g] = accel[2 * g] - c[2 * q];
        accel[2 * g + 1] = accel[2 * g + 1] - c[2 * q + 1];
      }
    }
    // mass matrix and corrector (compute_forces_viscoelastic_calling_routine.F90:181,
    // update_displacement_Newmark.F90:564-589)
    for (int g = 0; g < 2 * nglob; ++g) {
      accel[g] = accel[g] * o.rmass[g];
      veloc[g] = veloc[g] + o.deltatover2 * accel[g];
    }
    // receivers (write_seismograms.F90:150-190, compute_interpolated_dva.f90:34-97)
    if (seis) {
      const real *field = d->seismotype == 2 ? veloc : (d->seismotype == 3 ? accel : displ);
      for (int r = 0; r < d->nrec; ++r) {
        const int e = d->rec_ispec[r];
        double vx = 0.0, vz = 0.0;
        for (int j = 0; j < NGLL; ++j)
          for (int i = 0; i < NGLL; ++i) {
            const int g = d->ibool[static_cast<size_t>(e) * NGLL2 + j * NGLL + i];
            const double h = d->hxir[r * NGLL + i] * d->hgammar[r * NGLL + j];
            vx = vx + static_cast<double>(field[2 * g]) * h;
            vz = vz + static_cast<double>(field[2 * g + 1]) * h;
          }
        double *out = &seis[(static_cast<size_t>(r) * nstep + s) * 2];
        out[0] = d->cosrot * vx + d->sinrot * vz;
        out[1] = -d->sinrot * vx + d->cosrot * vz;
      }
    }
  }
  return 0;
}

}  // namespace

extern "C" int sf2d_oracle_newmark_elastic(const sf2d_oracle_db *db, int precision, int it0, int nstep,
                                           void *displ, void *veloc, void *accel, double *seis,
                                           int nthreads) {
  if (!db || !displ || !veloc || !accel || nstep < 0 || it0 < 0) return -1;
  if (it0 + nstep > db->nstep_total && db->nsrc > 0) return -2;
  if (precision == 4)
    return run_newmark<float>(db, it0, nstep, static_cast<float *>(displ), static_cast<float *>(veloc),
                              static_cast<float *>(accel), seis, nthreads);
  if (precision == 8)
    return run_newmark<double>(db, it0, nstep, static_cast<double *>(displ), static_cast<double *>(veloc),
                               static_cast<double *>(accel), seis, nthreads);
  return -3;
}

extern "C" int sf2d_oracle_max_threads(void) { return default_threads(); }
