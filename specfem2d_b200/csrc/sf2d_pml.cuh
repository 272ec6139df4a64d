// CPML (convolutional perfectly matched layer) coefficients and memory-variable
// updates, shared by the solid and fluid tile kernels and by the host code
// that prepares the coupling entries.  Everything is formed in double, as the
// reference does (pml_compute.f90 declares these quantities double precision),
// from the per-point damping profiles K, d, alpha of prepare_pml.f90 /
// pml_init.F90 and beta = alpha + d / K.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

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

// Per-point damping data as the tile kernels read it: (K_x, K_z),
// (alpha_x, alpha_z), (beta_x, beta_z).
struct PmlPoint {
  double kx, kz, ax, az, bx, bz;
};
__device__ __forceinline__ PmlPoint pml_point(const double2 *coef, int ps) {
  const double2 k = coef[3 * ps], a = coef[3 * ps + 1], b = coef[3 * ps + 2];
  return PmlPoint{k.x, k.y, a.x, a.y, b.x, b.y};
}

}  // namespace sf2d
