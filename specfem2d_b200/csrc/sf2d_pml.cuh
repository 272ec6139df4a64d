// CPML (convolutional perfectly matched layer) coefficients and memory-variable
// updates, shared by the solid and fluid tile kernels and by the host code
// that prepares the coupling entries.  Everything is formed in double, as the
// reference does (pml_compute.f90 declares these quantities double precision),
// from the per-point damping profiles K, d, alpha of prepare_pml.f90 /
// pml_init.F90 and beta = alpha + d / K.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

namespace sf2d {

constexpr int CPML_X_ONLY = 1, CPML_Z_ONLY = 2, CPML_XZ = 3;

// Recursive-convolution weights of one pole bb over one step DT
// (compute_coef_convolution, pml_compute.f90:34-86):
// c0 = exp(-bb DT), c1 = (1 - exp(-bb DT / 2)) / bb, c2 = c1 exp(-bb DT / 2).
struct PmlConv {
  double c0, c1, c2;
};
__host__ __device__ inline PmlConv pml_conv(double bb, double DT) {
  const double t = exp(-0.5 * bb * DT);
  PmlConv c;
  c.c0 = t * t;
  if (fabs(bb) > 1e-5) {
    c.c1 = (1.0 - t) / bb;
    c.c2 = c.c1 * t;
  } else {
    c.c1 = 0.5 * DT;
    c.c2 = c.c1;
  }
  return c;
}

// Strain coefficients A0, A1, A2 of lik_parameter_computation
// (pml_compute.f90:90-169).  Called as (x, z) for index_ik 13, whose poles
// are (alpha_x, beta_z), and as (z, x) with ik13 = false for index_ik 31,
// whose poles are (alpha_z, beta_x); the 31 form exchanges the roles of the
// X-only and Z-only regions.
struct PmlLik {
  double A0, A1, A2;
};
__host__ __device__ inline PmlLik pml_lik(double kx, double bx, double ax, double kz, double bz, double az, int region,
                                          bool ik13) {
  const int xo = ik13 ? CPML_X_ONLY : CPML_Z_ONLY;
  const int zo = ik13 ? CPML_Z_ONLY : CPML_X_ONLY;
  PmlLik L{0.0, 0.0, 0.0};
  if (region == CPML_XZ) {
    L.A0 = kx / kz;
    const double gx = (ax * bz + ax * ax + 2.0 * bx * az - 2.0 * ax * (bx + az)) / (bz - ax);
    const double gz = (ax * bz + bz * bz + 2.0 * bx * az - 2.0 * bz * (bx + az)) / (ax - bz);
    L.A1 = L.A0 / 2.0 * (gx - ax);
    L.A2 = L.A0 / 2.0 * (gz - bz);
  } else if (region == xo) {
    L.A0 = kx;
    L.A1 = -(L.A0 * (ax - bx));
  } else if (region == zo) {
    L.A0 = 1.0 / kz;
    L.A2 = -(L.A0 * (bz - az));
  }
  return L;
}

// Field coefficients A0..A4 of l_parameter_computation (pml_compute.f90:284-359);
// poles (alpha_x, alpha_z).
struct PmlL {
  double A0, A1, A2, A3, A4;
};
__host__ __device__ inline PmlL pml_l(double kx, double bx, double ax, double kz, double bz, double az, int region) {
  PmlL L{0.0, 0.0, 0.0, 0.0, 0.0};
  if (region == CPML_XZ) {
    L.A0 = kx * kz;
    const double gx = (ax * az + ax * ax + 2.0 * bx * bz - 2.0 * ax * (bx + bz)) / (az - ax);
    const double gz = (ax * az + az * az + 2.0 * bx * bz - 2.0 * az * (bx + bz)) / (ax - az);
    L.A1 = L.A0 / 2.0 * (gx - ax + gz - az);
    L.A2 = L.A0 / 2.0 * (ax * ax - gx * ax + az * az - gz * az);
    L.A3 = L.A0 / 2.0 * (ax * ax) * (gx - ax);
    L.A4 = L.A0 / 2.0 * (az * az) * (gz - az);
  } else if (region == CPML_X_ONLY) {
    L.A0 = kx;
    L.A1 = L.A0 * (bx - ax);
    L.A2 = -(L.A0 * ax * (bx - ax));
    L.A3 = L.A0 * (ax * ax) * (bx - ax);
  } else if (region == CPML_Z_ONLY) {
    L.A0 = kz;
    L.A1 = L.A0 * (bz - az);
    L.A2 = -(L.A0 * az * (bz - az));
    L.A4 = L.A0 * (az * az) * (bz - az);
  }
  return L;
}

// One memory variable r of pole bb driven by f: Newmark recursive convolution
// r = c0 r + c1 f + c2 f_old with f_old the field at the step's start plus
// dt^2/4 times its second derivative (pml_compute_memory_variables.f90:176-188
// for the fluid, :392-420 for the solid), or the LDDRK stage
// r_L = alpha r_L + dt (f - bb r), r += beta r_L (:189-212).  The products
// with the double coefficients are double.
template <bool LDDRK>
__device__ __forceinline__ void pml_update(float &r, float &rl, const PmlConv &c, double bb, float f, float fold,
                                           float alpha, float beta, float dt) {
  if (!LDDRK) {
    r = static_cast<float>(c.c0 * static_cast<double>(r) + c.c1 * static_cast<double>(f) +
                           c.c2 * static_cast<double>(fold));
  } else {
    rl = static_cast<float>(static_cast<double>(alpha * rl) +
                            static_cast<double>(dt) * (-bb * static_cast<double>(r) + static_cast<double>(f)));
    r = r + beta * rl;
  }
}

// Every coefficient one GLL point of a layer element needs, formed once on
// the host from its region and (K, alpha, beta) in x and z: the strain
// coefficients of the 31 form (zx, poles alpha_z, beta_x) and of the 13 form
// (xz, poles alpha_x, beta_z), the field coefficients (poles alpha_x,
// alpha_z) and the convolution weights of the four poles.  Points with equal
// damping data share one set, so a layer along a straight edge needs a few
// hundred sets and each point carries only the index of its set.
struct alignas(16) PmlSet {
  PmlLik zx, xz;
  PmlL l;
  PmlConv cax, caz, cbx, cbz;
  double ax, az, bx, bz;  // the poles (LDDRK stages)
};
inline PmlSet pml_set(double kx, double kz, double ax, double az, double bx, double bz, int region, double DT) {
  PmlSet s;
  s.zx = pml_lik(kz, bz, az, kx, bx, ax, region, false);
  s.xz = pml_lik(kx, bx, ax, kz, bz, az, region, true);
  s.l = pml_l(kx, bx, ax, kz, bz, az, region);
  s.cax = pml_conv(ax, DT);
  s.caz = pml_conv(az, DT);
  s.cbx = pml_conv(bx, DT);
  s.cbz = pml_conv(bz, DT);
  s.ax = ax;
  s.az = az;
  s.bx = bx;
  s.bz = bz;
  return s;
}

// The coefficient sets of the layer elements in slots [slot0, slot0 + nslots)
// (slot -> element through elem_order), deduplicated on the exact bits of
// (region, K_x, K_z, d_x, d_z, alpha_x, alpha_z); idx gets one set index per
// GLL point in slot order.  Desc carries the per-point arrays pml_K_x ...
// pml_alpha_z (double, [ispec][j][i]) and pml_region per element.
template <typename Desc>
void pml_build_sets(const Desc *d, const std::vector<int> &elem_order, int slot0, int nslots, double DT,
                    std::vector<PmlSet> &sets, std::vector<int> &idx) {
  std::map<std::array<uint64_t, 7>, int> seen;
  auto bits = [](double x) {
    uint64_t b;
    std::memcpy(&b, &x, sizeof(b));
    return b;
  };
  sets.clear();
  idx.clear();
  for (int s = slot0; s < slot0 + nslots; ++s) {
    const int e = elem_order[s];
    const int region = d->pml_region[e];
    for (int q = 0; q < 25; ++q) {
      const size_t p = static_cast<size_t>(e) * 25 + q;
      const double kx = d->pml_K_x[p], kz = d->pml_K_z[p], dx = d->pml_d_x[p], dz = d->pml_d_z[p];
      const double ax = d->pml_alpha_x[p], az = d->pml_alpha_z[p];
      const std::array<uint64_t, 7> key{static_cast<uint64_t>(region), bits(kx), bits(kz), bits(dx), bits(dz),
                                        bits(ax), bits(az)};
      auto it = seen.find(key);
      if (it == seen.end()) {
        // beta = alpha + d / K (pml_compute_memory_variables.f90:164-165)
        sets.push_back(pml_set(kx, kz, ax, az, ax + dx / kx, az + dz / kz, region, DT));
        it = seen.emplace(key, static_cast<int>(sets.size()) - 1).first;
      }
      idx.push_back(it->second);
    }
  }
}

// CPML in an attenuating solid (Newmark; pml_compute_memory_variables.f90:546-894).
// lik_parameter_computation_viscoelastic (pml_compute.f90:173-280), with the
// two-pole split of decompose_rational_fraction_PML (:578-610) in the XZ
// region: A0, A1, A2 and the Zener term Az of one strain component for one
// relaxation time 1/tau_sigma and strain relaxation time tau_epsilon.
struct PmlViscoLik {
  double A0, A1, A2, Az;
};
inline PmlViscoLik pml_visco_lik(double kx, double bx, double ax, double kz, double bz, double az, int region,
                                 bool ik13, double itau, double teps) {
  const int xo = ik13 ? CPML_X_ONLY : CPML_Z_ONLY;
  const int zo = ik13 ? CPML_Z_ONLY : CPML_X_ONLY;
  const auto gamma = [&](double b, double a) {
    return (b * (itau - a * teps * itau) + a * a * (teps * itau - 1.0)) / (itau - a);
  };
  const auto eta = [&](double b, double a) { return itau * (b - a) / (itau - a); };
  PmlViscoLik L{0.0, 0.0, 0.0, 0.0};
  if (region == CPML_XZ) {
    L.A0 = kx / kz;
    const double a1 = ax, a2 = bz;  // poles of the two fractions, split into (a_k, b_k)
    const double b1 = (a1 * a2 + a1 * a1 + 2.0 * bx * az - 2.0 * a1 * (bx + az)) / (a2 - a1);
    const double b2 = (a1 * a2 + a2 * a2 + 2.0 * bx * az - 2.0 * a2 * (bx + az)) / (a1 - a2);
    L.A1 = L.A0 / 2.0 * (gamma(b1, a1) - a1);
    L.A2 = L.A0 / 2.0 * (gamma(b2, a2) - a2);
    L.Az = L.A0 * (teps * itau - 1.0) * ((eta(b1, a1) + eta(b2, a2)) / 2.0 - itau);
  } else if (region == xo) {
    L.A0 = kx;
    L.A1 = L.A0 * (gamma(bx, ax) - ax);
    L.Az = L.A0 * (teps * itau - 1.0) * (eta(bx, ax) - itau);
  } else if (region == zo) {
    L.A0 = 1.0 / kz;
    L.A2 = L.A0 * (gamma(az, bz) - bz);
    L.Az = L.A0 * (teps * itau - 1.0) * (eta(az, bz) - itau);
  }
  return L;
}

constexpr int PML_NSLS = 3;

// Per-point coefficients of the viscoelastic layer update: for each SLS the
// convolution weights of 1/tau_sigma for the bulk (k) and shear (m) parts,
// the Zener terms divided by Mu = N_SLS Mu_nu (for the 31 and 13 strain
// components) and phi; then A0 of both forms and the SLS sums of A1, A2
// divided by Mu that weight the layer's strain memory variables.
struct alignas(16) PmlVisco {
  PmlConv ck[PML_NSLS], cm[PML_NSLS];
  double k31[PML_NSLS], k13[PML_NSLS], m31[PML_NSLS], m13[PML_NSLS];  // Az / Mu
  double phik[PML_NSLS], phim[PML_NSLS];
  double A01, A10;
  double k2, k3, k4, k5, m2, m3, m4, m5;  // sum over SLS of A1 (31), A2 (31), A1 (13), A2 (13), over Mu
};
inline PmlVisco pml_visco_set(double kx, double kz, double ax, double az, double bx, double bz, int region, double DT,
                              const double *itau1, const double *itau2, const double *teps1, const double *teps2,
                              const double *phi1, const double *phi2, double mu1, double mu2) {
  PmlVisco v{};
  const double Mk = mu1 * PML_NSLS, Mm = mu2 * PML_NSLS;
  double s2k = 0, s2m = 0, s3k = 0, s3m = 0, s4k = 0, s4m = 0, s5k = 0, s5m = 0;
  for (int s = 0; s < PML_NSLS; ++s) {
    const PmlViscoLik k31 = pml_visco_lik(kz, bz, az, kx, bx, ax, region, false, itau1[s], teps1[s]);
    const PmlViscoLik m31 = pml_visco_lik(kz, bz, az, kx, bx, ax, region, false, itau2[s], teps2[s]);
    const PmlViscoLik k13 = pml_visco_lik(kx, bx, ax, kz, bz, az, region, true, itau1[s], teps1[s]);
    const PmlViscoLik m13 = pml_visco_lik(kx, bx, ax, kz, bz, az, region, true, itau2[s], teps2[s]);
    v.A01 = m31.A0;
    v.A10 = m13.A0;
    v.ck[s] = pml_conv(itau1[s], DT);
    v.cm[s] = pml_conv(itau2[s], DT);
    v.k31[s] = k31.Az / Mk;
    v.k13[s] = k13.Az / Mk;
    v.m31[s] = m31.Az / Mm;
    v.m13[s] = m13.Az / Mm;
    v.phik[s] = phi1[s];
    v.phim[s] = phi2[s];
    s2k += k31.A1;
    s2m += m31.A1;
    s3k += k31.A2;
    s3m += m31.A2;
    s4k += k13.A1;
    s4m += m13.A1;
    s5k += k13.A2;
    s5m += m13.A2;
  }
  v.k2 = s2k / Mk;
  v.k3 = s3k / Mk;
  v.k4 = s4k / Mk;
  v.k5 = s5k / Mk;
  v.m2 = s2m / Mm;
  v.m3 = s3m / Mm;
  v.m4 = s4m / Mm;
  v.m5 = s5m / Mm;
  return v;
}

// Viscoelastic coefficient sets of the layer elements in slots [slot0,
// slot0 + nslots) whose pml_visco flag is set, deduplicated on the bits of the
// damping data and the Zener parameters; idx gets one entry per GLL point in
// slot order, -1 for points of elastic layer elements.  Desc carries
// pml_visco per element and att_itau1/2, att_phi1/2, att_teps1/2
// (float, [ispec][j][i][sls]) and att_mu1/2 (float, [ispec][j][i]).
template <typename Desc>
void pml_build_visco_sets(const Desc *d, const std::vector<int> &elem_order, int slot0, int nslots, double DT,
                          std::vector<PmlVisco> &sets, std::vector<int> &idx) {
  std::map<std::vector<uint64_t>, int> seen;
  auto bits = [](double x) {
    uint64_t b;
    std::memcpy(&b, &x, sizeof(b));
    return b;
  };
  sets.clear();
  idx.clear();
  for (int s = slot0; s < slot0 + nslots; ++s) {
    const int e = elem_order[s];
    const int region = d->pml_region[e];
    for (int q = 0; q < 25; ++q) {
      if (!d->pml_visco || !d->pml_visco[e]) {
        idx.push_back(-1);
        continue;
      }
      const size_t p = static_cast<size_t>(e) * 25 + q;
      const double kx = d->pml_K_x[p], kz = d->pml_K_z[p], dx = d->pml_d_x[p], dz = d->pml_d_z[p];
      const double ax = d->pml_alpha_x[p], az = d->pml_alpha_z[p];
      double it1[PML_NSLS], it2[PML_NSLS], te1[PML_NSLS], te2[PML_NSLS], ph1[PML_NSLS], ph2[PML_NSLS];
      std::vector<uint64_t> key{static_cast<uint64_t>(region), bits(kx), bits(kz), bits(dx), bits(dz), bits(ax),
                                bits(az), bits(d->att_mu1[p]), bits(d->att_mu2[p])};
      for (int l = 0; l < PML_NSLS; ++l) {
        const size_t a = p * PML_NSLS + l;
        it1[l] = d->att_itau1[a];
        it2[l] = d->att_itau2[a];
        te1[l] = d->att_teps1[a];
        te2[l] = d->att_teps2[a];
        ph1[l] = d->att_phi1[a];
        ph2[l] = d->att_phi2[a];
        for (double x : {it1[l], it2[l], te1[l], te2[l], ph1[l], ph2[l]}) key.push_back(bits(x));
      }
      auto it = seen.find(key);
      if (it == seen.end()) {
        sets.push_back(pml_visco_set(kx, kz, ax, az, ax + dx / kx, az + dz / kz, region, DT, it1, it2, te1, te2, ph1,
                                     ph2, d->att_mu1[p], d->att_mu2[p]));
        it = seen.emplace(key, static_cast<int>(sets.size()) - 1).first;
      }
      idx.push_back(it->second);
    }
  }
}

}  // namespace sf2d
