// CPU oracle for the SPECFEM2D time-marching hot path -- TEST INFRASTRUCTURE.
//
// A restatement of the reference's CPU routines, used only as the checker of
// the CUDA path and as the timed CPU baseline.  `real` is float for the
// CUSTOM_REAL=4 build and double for the CUSTOM_REAL=8 build; expressions
// that the reference evaluates in double inside a CUSTOM_REAL=4 build are
// evaluated in double here too.
//
// Summation order follows the serial reference: within a step (or LDDRK
// stage), Stacey and source terms are added first (iphase 1 of
// src/specfem2D/compute_forces_viscoelastic_calling_routine.F90:58-100, all
// elements are "inner" with one process), then element contributions in
// ascending element order.  Element work is spread over host threads into
// a per-element buffer; assembly gathers, per global point, the contributions
// of its elements in ascending element order (the serial loop's order at every
// point), so results do not depend on the thread count.
#include "sf2d_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <new>
#include <pthread.h>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr int NGLL = 5;
constexpr int NGLL2 = 25;
constexpr int NSLS = 3;

int default_threads() {
  const char *env = std::getenv("SF2D_ORACLE_THREADS");
  if (env && std::atoi(env) > 0) return std::atoi(env);
  const unsigned n = std::thread::hardware_concurrency();
  return n ? static_cast<int>(n) : 1;
}

// Persistent worker threads.  run(n, nt, f) splits [0, n) into nt static
// blocks, runs block 0 on the calling thread and the others on the workers,
// and returns when every block is done.  Workers spin briefly on a generation
// counter before sleeping, so one call costs microseconds, not a thread
// start per block.  Callers are serialised: a second State waits its turn.
class Pool {
 public:
  static Pool &get() {
    static Pool p;
    return p;
  }
  template <typename F>
  void run(int n, int nt, F &&f) {
    nt = std::max(1, std::min(nt, n));
    if (nt == 1) {
      f(0, n);
      return;
    }
    std::lock_guard<std::mutex> call(call_m_);
    while (static_cast<int>(workers_.size()) < nt - 1) {
      // a new worker starts from the current generation, so it takes the
      // job published below even if it first runs after the publication
      const int k = static_cast<int>(workers_.size()) + 1;
      const unsigned g0 = gen_.load(std::memory_order_acquire);
      workers_.emplace_back([this, k, g0] { worker(k, g0); });
    }
    job_ = [&f, n, nt](int k) {
      const int b = static_cast<int>(static_cast<long long>(n) * k / nt);
      const int e = static_cast<int>(static_cast<long long>(n) * (k + 1) / nt);
      if (b < e) f(b, e);
    };
    nblocks_ = nt;
    pending_.store(static_cast<int>(workers_.size()), std::memory_order_relaxed);
    {
      std::lock_guard<std::mutex> lk(m_);
      gen_.fetch_add(1, std::memory_order_release);
    }
    cv_.notify_all();
    job_(0);
    while (pending_.load(std::memory_order_acquire) != 0) relax();
  }
  Pool() {
    // a forked child has none of the parent's workers: it starts with none
    pthread_atfork(nullptr, nullptr, [] { Pool::get().forget_workers(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_.store(true, std::memory_order_release);
      gen_.fetch_add(1, std::memory_order_release);
    }
    cv_.notify_all();
    for (auto &t : workers_) t.join();
  }

 private:
  // In a child of fork(): the workers' std::thread objects name threads of the
  // parent; they are abandoned (never joined or destroyed) and the locks made
  // anew, so the child's first parallel call starts its own workers.
  void forget_workers() {
    new (&workers_) std::vector<std::thread>();
    new (&call_m_) std::mutex();
    new (&m_) std::mutex();
    new (&cv_) std::condition_variable();
    pending_.store(0, std::memory_order_relaxed);
    nblocks_ = 0;
  }
  static void relax() {
#if defined(__x86_64__)
    __builtin_ia32_pause();
#endif
  }
  void worker(int k, unsigned seen) {
    for (;;) {
      for (int spin = 0; spin < 20000 && gen_.load(std::memory_order_acquire) == seen; ++spin) relax();
      if (gen_.load(std::memory_order_acquire) == seen) {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return gen_.load(std::memory_order_acquire) != seen; });
      }
      seen = gen_.load(std::memory_order_acquire);
      if (stop_.load(std::memory_order_acquire)) return;
      if (k < nblocks_) job_(k);
      pending_.fetch_sub(1, std::memory_order_release);
    }
  }
  std::vector<std::thread> workers_;
  std::mutex call_m_, m_;
  std::condition_variable cv_;
  std::atomic<unsigned> gen_{0};
  std::atomic<int> pending_{0};
  std::atomic<bool> stop_{false};
  std::function<void(int)> job_;
  int nblocks_ = 0;
};

template <typename F>
void parallel_for(int n, int nt, F &&f) {
  Pool::get().run(n, nt, std::forward<F>(f));
}

// Point loops go parallel from this many global points on (smaller meshes
// finish a loop in microseconds).
constexpr int POINT_PARALLEL_MIN = 16384;

template <typename real>
std::vector<real> cvt(const double *p, size_t n) {
  std::vector<real> v(p ? n : 0);
  if (p)
    for (size_t k = 0; k < n; ++k) v[k] = static_cast<real>(p[k]);
  return v;
}

constexpr int CPML_X_ONLY = 1, CPML_Z_ONLY = 2, CPML_XZ = 3;

// compute_coef_convolution (pml_compute.f90:34-86)
void coef_convolution(double bb, double DT, double &c0, double &c1, double &c2) {
  const double temp = std::exp(-0.5 * bb * DT);
  c0 = temp * temp;
  if (std::fabs(bb) > 1e-5) {
    c1 = (1.0 - temp) / bb;
    c2 = c1 * temp;
  } else {
    c1 = 0.5 * DT;
    c2 = c1;
  }
}

struct PmlCoef {
  double A0, A1, A2, A3, A4, bb1, bb2, c0_1, c1_1, c2_1, c0_2, c1_2, c2_2;
};

// lik_parameter_computation (pml_compute.f90:90-169): coefficients of the
// memory variables of one strain component; index_ik 13 or 31 swaps the roles
// of the X-only and Z-only regions.
PmlCoef lik_parameters(double DT, double kx, double bx, double ax, double kz, double bz, double az, int region,
                       int index_ik) {
  const int xo = index_ik == 13 ? CPML_X_ONLY : CPML_Z_ONLY;
  const int zo = index_ik == 13 ? CPML_Z_ONLY : CPML_X_ONLY;
  PmlCoef L{};
  if (region == CPML_XZ) {
    L.A0 = kx / kz;
    const double gx = (ax * bz + ax * ax + 2.0 * bx * az - 2.0 * ax * (bx + az)) / (bz - ax);
    const double gz = (ax * bz + bz * bz + 2.0 * bx * az - 2.0 * bz * (bx + az)) / (ax - bz);
    L.A1 = L.A0 / 2.0 * (gx - ax);
    L.A2 = L.A0 / 2.0 * (gz - bz);
  } else if (region == xo) {
    L.A0 = kx;
    L.A1 = -(L.A0 * (ax - bx));
    L.A2 = 0.0;
  } else if (region == zo) {
    L.A0 = 1.0 / kz;
    L.A1 = 0.0;
    L.A2 = -(L.A0 * (bz - az));
  }
  L.bb1 = ax;
  coef_convolution(L.bb1, DT, L.c0_1, L.c1_1, L.c2_1);
  L.bb2 = bz;
  coef_convolution(L.bb2, DT, L.c0_2, L.c1_2, L.c2_2);
  return L;
}

// l_parameter_computation (pml_compute.f90:284-359): coefficients of the
// acceleration contribution and of the field memory variables.
PmlCoef l_parameters(double DT, double kx, double bx, double ax, double kz, double bz, double az, int region) {
  PmlCoef L{};
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
    L.A4 = 0.0;
  } else if (region == CPML_Z_ONLY) {
    L.A0 = kz;
    L.A1 = L.A0 * (bz - az);
    L.A2 = -(L.A0 * az * (bz - az));
    L.A3 = 0.0;
    L.A4 = L.A0 * (az * az) * (bz - az);
  }
  L.bb1 = ax;
  coef_convolution(L.bb1, DT, L.c0_1, L.c1_1, L.c2_1);
  L.bb2 = az;
  coef_convolution(L.bb2, DT, L.c0_2, L.c1_2, L.c2_2);
  return L;
}

// lik_parameter_computation_viscoelastic (pml_compute.f90:173-280) with the
// two-pole split of decompose_rational_fraction_PML (pml_compute.f90:578-610):
// A0, A1, A2 and the Zener term of one strain component and one relaxation
// time; index_ik 13 or 31 swaps the X-only and Z-only regions.
struct ViscoLik {
  double A0, A1, A2, Az;
};
ViscoLik lik_viscoelastic(double kx, double bx, double ax, double kz, double bz, double az, int region,
                          int index_ik, double itau, double teps) {
  const int xo = index_ik == 13 ? CPML_X_ONLY : CPML_Z_ONLY;
  const int zo = index_ik == 13 ? CPML_Z_ONLY : CPML_X_ONLY;
  const auto gamma = [&](double b, double a) {
    return (b * (itau - a * teps * itau) + a * a * (teps * itau - 1.0)) / (itau - a);
  };
  const auto eta = [&](double b, double a) { return itau * (b - a) / (itau - a); };
  ViscoLik L{};
  if (region == CPML_XZ) {
    L.A0 = kx / kz;
    const double a1 = ax, a2 = bz;
    const double b1 = (a1 * a2 + a1 * a1 + 2.0 * bx * az - 2.0 * a1 * (bx + az)) / (a2 - a1);
    const double b2 = (a1 * a2 + a2 * a2 + 2.0 * bx * az - 2.0 * a2 * (bx + az)) / (a1 - a2);
    L.A1 = L.A0 / 2.0 * (gamma(b1, a1) - a1);
    L.A2 = L.A0 / 2.0 * (gamma(b2, a2) - a2);
    L.Az = L.A0 * (teps * itau - 1.0) * ((eta(b1, a1) + eta(b2, a2)) / 2.0 - itau);
  } else if (region == xo) {
    L.A0 = kx;
    L.A1 = L.A0 * (gamma(bx, ax) - ax);
    L.A2 = 0.0;
    L.Az = L.A0 * (teps * itau - 1.0) * (eta(bx, ax) - itau);
  } else if (region == zo) {
    L.A0 = 1.0 / kz;
    L.A1 = 0.0;
    L.A2 = L.A0 * (gamma(az, bz) - bz);
    L.Az = L.A0 * (teps * itau - 1.0) * (eta(az, bz) - itau);
  }
  return L;
}

struct StateBase {
  virtual ~StateBase() = default;
  virtual int run(int nstep, double *seis, int nthreads) = 0;
  virtual int get(int which, void *out) = 0;
  virtual int set(int which, const void *in) = 0;
  virtual int accumulate(const void *b) = 0;
  virtual int accumulate_hessian(const void *b_accel) = 0;
  virtual int accumulate_acoustic(const void *b_pot) = 0;
  virtual void set_step(int it) = 0;
};

template <typename real>
struct State : StateBase {
  const sf2d_oracle_db d;  // shallow copy of the descriptor (pointers stay with the caller)
  int nspec, nglob;
  std::vector<real> xix, xiz, gammax, gammaz, jacobian, rho, mu, rho_vp, rmass;
  real hprime[NGLL][NGLL], hprimewgll[NGLL][NGLL], wxgll[NGLL], wzgll[NGLL];
  std::vector<real> st_nx, st_nz, st_w, st_rvp, st_rvs, srcarr;
  std::vector<real> c11, c13, c15, c33, c35, c55;
  std::vector<real> a1, b1, a2, b2, phi1, phi2;  // Newmark A/B, LDDRK phi (CUSTOM_REAL)
  std::vector<double> itau1, itau2;             // LDDRK 1/tau_sigma (read as double)
  real deltat, deltatover2, deltatsquareover2;
  real alpha[6], beta[6];
  bool atten;
  // state
  std::vector<real> displ, veloc, accel, displ_l, veloc_l;
  std::vector<real> e1, e11, e13, e1_l, e11_l, e13_l;      // nspec*25*3
  std::vector<real> att_old;                                // nspec*25*3: dux_dxl, duz_dzl, dux_dzl+duz_dxl
  std::vector<real> rho_kl, kappa_kl, mu_kl;                // nspec*25
  std::vector<real> rho_ac_kl, kappa_ac_kl;                 // nspec*25 (fluid elements)
  std::vector<real> hess1, hess2;                           // nspec*25 (approximate Hessian)
  std::vector<real> adj;                                    // nrec*nstep*2
  std::vector<real> contrib;
  // acoustic domain
  bool acoustic = false;
  std::vector<real> kappa, rmass_ac, st_ac_w, st_ac_rvp;
  std::vector<real> cpl_ac_nx, cpl_ac_nz, cpl_ac_w, cpl_el_nx, cpl_el_nz, cpl_el_w;
  std::vector<real> pot, pot_d, pot_dd, pot_l, pot_d_l;     // nglob
  std::vector<real> contrib_ac;                             // nspec*25
  // CPML
  bool pml = false;
  std::vector<real> rm_el, rm_el_l;       // nspec*25*8: dux_dx, dux_dx', duz_dx, duz_dx' (zx), dux_dz.., duz_dz.. (xz)
  std::vector<real> rm_displ, rm_displ_l; // nspec*25*4: (bb1, x), (bb1, z), (bb2, x), (bb2, z)
  std::vector<real> rm_ac, rm_ac_l;       // nspec*25*4: dchi_dx (2, zx), dchi_dz (2, xz)
  std::vector<real> rm_pot, rm_pot_l;     // nspec*25*2
  std::vector<real> rm_fsb, rm_fsb_l;     // 2 per fluid-side coupling entry
  std::vector<real> rm_sfb, rm_sfb_l;     // 1 per solid-side coupling entry
  std::vector<real> displ_old, pot_old;
  // CPML in attenuating solids: memory variables (nspec*25*3*6) and the Zener
  // parameters, all read as double as the reference declares them
  std::vector<real> rm_visco;
  std::vector<double> teps1, teps2, vitau1, vitau2, vphi1, vphi2, mu_nu1, mu_nu2;
  std::vector<real> contrib_pml, contrib_ac_pml;
  // per global point, the (element * 25 + GLL point) entries of its solid and
  // of its fluid elements in ascending element order (gather assembly)
  std::vector<int> gat_el_off, gat_el, gat_ac_off, gat_ac;
  int it = 0;  // steps done

  bool is_acoustic(int e) const { return acoustic && d.ispec_is_acoustic[e] != 0; }
  int pml_region(int e) const { return pml ? d.pml_region[e] : 0; }
  void pml_params(size_t p, double &kx, double &bx, double &ax, double &kz, double &bz, double &az) const {
    kx = d.pml_K_x[p];
    kz = d.pml_K_z[p];
    ax = d.pml_alpha_x[p];
    az = d.pml_alpha_z[p];
    bx = ax + d.pml_d_x[p] / kx;
    bz = az + d.pml_d_z[p] / kz;
  }
  // Newmark memory-variable update r = c0 r + c1 f + c2 f_old, or the LDDRK
  // stage r_L = alpha r_L + dt (-bb r + f), r += beta r_L; coefficients in double
  void rm_update(real &r, real &rl, double c0, double c1, double c2, double bb, real f, real fold, int stage) {
    if (d.time_scheme == 1) {
      r = static_cast<real>(c0 * static_cast<double>(r) + c1 * static_cast<double>(f) + c2 * static_cast<double>(fold));
    } else {
      rl = static_cast<real>(static_cast<double>(alpha[stage] * rl) +
                             static_cast<double>(deltat) * (-bb * static_cast<double>(r) + static_cast<double>(f)));
      r = r + beta[stage] * rl;
    }
  }

  explicit State(const sf2d_oracle_db *p) : d(*p) {
    nspec = d.nspec;
    nglob = d.nglob;
    const size_t nl = static_cast<size_t>(nspec) * NGLL2;
    xix = cvt<real>(d.xix, nl);
    xiz = cvt<real>(d.xiz, nl);
    gammax = cvt<real>(d.gammax, nl);
    gammaz = cvt<real>(d.gammaz, nl);
    jacobian = cvt<real>(d.jacobian, nl);
    rho = cvt<real>(d.rhostore, nl);
    mu = cvt<real>(d.mustore, nl);
    rho_vp = cvt<real>(d.rho_vpstore, nl);
    rmass = cvt<real>(d.rmass_inverse, static_cast<size_t>(nglob) * 2);
    for (int a = 0; a < NGLL; ++a) {
      wxgll[a] = static_cast<real>(d.wxgll[a]);
      wzgll[a] = static_cast<real>(d.wzgll[a]);
      for (int b = 0; b < NGLL; ++b) {
        hprime[a][b] = static_cast<real>(d.hprime[a * NGLL + b]);
        hprimewgll[a][b] = static_cast<real>(d.hprimewgll[a * NGLL + b]);
      }
    }
    st_nx = cvt<real>(d.st_nx, d.nstacey);
    st_nz = cvt<real>(d.st_nz, d.nstacey);
    st_w = cvt<real>(d.st_w, d.nstacey);
    st_rvp = cvt<real>(d.st_rvp, d.nstacey);
    st_rvs = cvt<real>(d.st_rvs, d.nstacey);
    srcarr = cvt<real>(d.sourcearrays, static_cast<size_t>(d.nsrc) * NGLL2 * 2);
    if (d.ispec_is_anisotropic) {
      c11 = cvt<real>(d.c11, nl);
      c13 = cvt<real>(d.c13, nl);
      c15 = cvt<real>(d.c15, nl);
      c33 = cvt<real>(d.c33, nl);
      c35 = cvt<real>(d.c35, nl);
      c55 = cvt<real>(d.c55, nl);
    }
    deltat = static_cast<real>(d.deltat);
    deltatover2 = static_cast<real>(d.deltatover2);
    deltatsquareover2 = static_cast<real>(d.deltatsquareover2);
    for (int s = 0; s < 6; ++s) {
      alpha[s] = d.alpha_lddrk ? static_cast<real>(d.alpha_lddrk[s]) : real(0);
      beta[s] = d.beta_lddrk ? static_cast<real>(d.beta_lddrk[s]) : real(0);
    }
    atten = d.time_scheme == 1 ? (d.att_a1 != nullptr) : (d.att_itau1 != nullptr);
    if (atten) {
      const size_t na = nl * NSLS;
      if (d.time_scheme == 1) {
        a1 = cvt<real>(d.att_a1, na);
        b1 = cvt<real>(d.att_b1, na);
        a2 = cvt<real>(d.att_a2, na);
        b2 = cvt<real>(d.att_b2, na);
      } else {
        phi1 = cvt<real>(d.att_phi1, na);
        phi2 = cvt<real>(d.att_phi2, na);
        itau1.assign(d.att_itau1, d.att_itau1 + na);
        itau2.assign(d.att_itau2, d.att_itau2 + na);
      }
      e1.assign(na, 0);
      e11.assign(na, 0);
      e13.assign(na, 0);
      if (d.time_scheme != 1) {
        e1_l.assign(na, 0);
        e11_l.assign(na, 0);
        e13_l.assign(na, 0);
      }
      att_old.assign(nl * 3, 0);
    }
    const size_t ng = static_cast<size_t>(nglob) * 2;
    displ.assign(ng, 0);
    veloc.assign(ng, 0);
    accel.assign(ng, 0);
    if (d.time_scheme != 1) {
      displ_l.assign(ng, 0);
      veloc_l.assign(ng, 0);
    }
    contrib.assign(nl * 2, 0);
    rho_kl.assign(nl, 0);
    kappa_kl.assign(nl, 0);
    mu_kl.assign(nl, 0);
    hess1.assign(nl, 0);
    hess2.assign(nl, 0);
    rho_ac_kl.assign(nl, 0);
    kappa_ac_kl.assign(nl, 0);
    if (d.adj_src) adj = cvt<real>(d.adj_src, static_cast<size_t>(d.nrec) * d.nstep_total * 2);
    acoustic = d.ispec_is_acoustic != nullptr;
    if (acoustic) {
      kappa = cvt<real>(d.kappastore, nl);
      rmass_ac = cvt<real>(d.rmass_inverse_acoustic, nglob);
      st_ac_w = cvt<real>(d.st_ac_w, d.nstacey_ac);
      st_ac_rvp = cvt<real>(d.st_ac_rvp, d.nstacey_ac);
      cpl_ac_nx = cvt<real>(d.cpl_ac_nx, d.ncpl_ac);
      cpl_ac_nz = cvt<real>(d.cpl_ac_nz, d.ncpl_ac);
      cpl_ac_w = cvt<real>(d.cpl_ac_w, d.ncpl_ac);
      cpl_el_nx = cvt<real>(d.cpl_el_nx, d.ncpl_el);
      cpl_el_nz = cvt<real>(d.cpl_el_nz, d.ncpl_el);
      cpl_el_w = cvt<real>(d.cpl_el_w, d.ncpl_el);
      pot.assign(nglob, 0);
      pot_d.assign(nglob, 0);
      pot_dd.assign(nglob, 0);
      if (d.time_scheme != 1) {
        pot_l.assign(nglob, 0);
        pot_d_l.assign(nglob, 0);
      }
      contrib_ac.assign(nl, 0);
    }
    pml = d.pml_region != nullptr;
    if (pml) {
      rm_el.assign(nl * 8, 0);
      rm_displ.assign(nl * 4, 0);
      displ_old.assign(static_cast<size_t>(nglob) * 2, 0);
      contrib_pml.assign(nl * 2, 0);
      if (d.time_scheme != 1) {
        rm_el_l.assign(nl * 8, 0);
        rm_displ_l.assign(nl * 4, 0);
      }
      if (d.pml_visco) {
        // kaPML_rmemory_dux_dxl, _duz_dzl, muPML_rmemory_dux_dxl, _duz_dzl, _dux_dzl, _duz_dxl per SLS
        rm_visco.assign(nl * NSLS * 6, 0);
        const size_t na = nl * NSLS;
        teps1.assign(d.att_teps1, d.att_teps1 + na);
        teps2.assign(d.att_teps2, d.att_teps2 + na);
        vitau1.assign(d.att_itau1, d.att_itau1 + na);
        vitau2.assign(d.att_itau2, d.att_itau2 + na);
        vphi1.assign(d.att_phi1, d.att_phi1 + na);
        vphi2.assign(d.att_phi2, d.att_phi2 + na);
        mu_nu1.assign(d.att_mu1, d.att_mu1 + nl);
        mu_nu2.assign(d.att_mu2, d.att_mu2 + nl);
      }
      if (acoustic) {
        rm_ac.assign(nl * 4, 0);
        rm_pot.assign(nl * 2, 0);
        pot_old.assign(nglob, 0);
        contrib_ac_pml.assign(nl, 0);
        rm_fsb.assign(static_cast<size_t>(d.ncpl_ac) * 2, 0);
        rm_sfb.assign(d.ncpl_el, 0);
        if (d.time_scheme != 1) {
          rm_ac_l.assign(nl * 4, 0);
          rm_pot_l.assign(nl * 2, 0);
          rm_fsb_l.assign(static_cast<size_t>(d.ncpl_ac) * 2, 0);
          rm_sfb_l.assign(d.ncpl_el, 0);
        }
      }
    }
    build_gather(false, gat_el_off, gat_el);
    if (acoustic) build_gather(true, gat_ac_off, gat_ac);
  }

  void build_gather(bool fluid, std::vector<int> &off, std::vector<int> &idx) const {
    off.assign(static_cast<size_t>(nglob) + 1, 0);
    for (int e = 0; e < nspec; ++e)
      if (is_acoustic(e) == fluid)
        for (int q = 0; q < NGLL2; ++q) ++off[d.ibool[static_cast<size_t>(e) * NGLL2 + q] + 1];
    for (int g = 0; g < nglob; ++g) off[g + 1] += off[g];
    idx.assign(off[nglob], 0);
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int e = 0; e < nspec; ++e)
      if (is_acoustic(e) == fluid)
        for (int q = 0; q < NGLL2; ++q) {
          const int g = d.ibool[static_cast<size_t>(e) * NGLL2 + q];
          idx[fill[g]++] = e * NGLL2 + q;
        }
  }

  // Runs f(b, e) over blocks of [0, nglob) on the pool when the mesh is large.
  template <typename F>
  void points_for(int nt, F &&f) const {
    parallel_for(nglob, nglob >= POINT_PARALLEL_MIN ? nt : 1, std::forward<F>(f));
  }

  // Zeroes the outer PML edge points (pml_boundary_elastic/_acoustic, pml_compute.f90:502-574)
  void pml_boundary_elastic() {
    for (int k = 0; k < (pml ? d.npml_bnd_el : 0); ++k) {
      const int g = d.pml_bnd_el[k];
      for (int c = 0; c < 2; ++c) {
        displ_old[2 * g + c] = 0;
        displ[2 * g + c] = 0;
        veloc[2 * g + c] = 0;
        accel[2 * g + c] = 0;
      }
    }
  }
  void pml_boundary_acoustic() {
    for (int k = 0; k < (pml ? d.npml_bnd_ac : 0); ++k) {
      const int g = d.pml_bnd_ac[k];
      pot_old[g] = 0;
      pot[g] = 0;
      pot_d[g] = 0;
      pot_dd[g] = 0;
    }
  }

  // Acoustic element force for one element (compute_forces_viscoacoustic.f90:
  // 105-125 gather, :420-470 mxm_2comp_singleA, :142-152 mapping, :226-238
  // fac = J / rho weak-form terms, :306-322 weighted transpose contraction).
  // Writes the 25 sums to be subtracted from chi_dot_dot.
  void acoustic_element_force(int ispec, int stage_, real *out, real *pml_out) {
    const size_t off = static_cast<size_t>(ispec) * NGLL2;
    real pe[NGLL][NGLL];  // [j][i]
    for (int j = 0; j < NGLL; ++j)
      for (int i = 0; i < NGLL; ++i) pe[j][i] = pot[d.ibool[off + j * NGLL + i]];
    real t1[NGLL][NGLL], t2[NGLL][NGLL];
    for (int j = 0; j < NGLL; ++j)
      for (int i = 0; i < NGLL; ++i) {
        const real dxi = pe[j][0] * hprime[i][0] + pe[j][1] * hprime[i][1] + pe[j][2] * hprime[i][2] +
                         pe[j][3] * hprime[i][3] + pe[j][4] * hprime[i][4];
        const real dgam = pe[0][i] * hprime[j][0] + pe[1][i] * hprime[j][1] + pe[2][i] * hprime[j][2] +
                          pe[3][i] * hprime[j][3] + pe[4][i] * hprime[j][4];
        const size_t p = off + j * NGLL + i;
        const real xixl = xix[p], xizl = xiz[p], gammaxl = gammax[p], gammazl = gammaz[p];
        real dxl = dxi * xixl + dgam * gammaxl;
        real dzl = dxi * xizl + dgam * gammazl;
        const int region = pml_region(ispec);
        if (region > 0) {
          // pml_compute_memory_variables_acoustic (pml_compute_memory_variables.f90:42-224)
          real dxi_o = 0, dgam_o = 0;
          if (d.time_scheme == 1)
            for (int k = 0; k < NGLL; ++k) {
              dxi_o = dxi_o + pot_old[d.ibool[off + j * NGLL + k]] * hprime[i][k];
              dgam_o = dgam_o + pot_old[d.ibool[off + k * NGLL + i]] * hprime[j][k];
            }
          const real dxl_o = dxi_o * xixl + dgam_o * gammaxl, dzl_o = dxi_o * xizl + dgam_o * gammazl;
          double kx, bx, ax, kz, bz, az;
          pml_params(p, kx, bx, ax, kz, bz, az);
          const PmlCoef zx = lik_parameters(d.DT, kz, bz, az, kx, bx, ax, region, 31);
          const PmlCoef xz = lik_parameters(d.DT, kx, bx, ax, kz, bz, az, region, 13);
          real *r = &rm_ac[p * 4];
          real dummy[4] = {0, 0, 0, 0};
          real *rl = d.time_scheme == 1 ? dummy : &rm_ac_l[p * 4];
          rm_update(r[0], rl[0], zx.c0_1, zx.c1_1, zx.c2_1, zx.bb1, dxl, dxl_o, stage_);
          rm_update(r[1], rl[1], zx.c0_2, zx.c1_2, zx.c2_2, zx.bb2, dxl, dxl_o, stage_);
          rm_update(r[2], rl[2], xz.c0_1, xz.c1_1, xz.c2_1, xz.bb1, dzl, dzl_o, stage_);
          rm_update(r[3], rl[3], xz.c0_2, xz.c1_2, xz.c2_2, xz.bb2, dzl, dzl_o, stage_);
          const real pdx = dxl, pdz = dzl;
          dxl = static_cast<real>(zx.A0 * pdx + zx.A1 * r[0] + zx.A2 * r[1]);
          dzl = static_cast<real>(xz.A0 * pdz + xz.A1 * r[2] + xz.A2 * r[3]);
          // pml_compute_accel_contribution_acoustic (pml_compute_accel_contribution.f90:42-180)
          const int g = d.ibool[p];
          const real fac2 = jacobian[p] / kappa[p];
          const PmlCoef L = l_parameters(d.DT, kx, bx, ax, kz, bz, az, region);
          real *rp = &rm_pot[p * 2];
          real dummy2[2] = {0, 0};
          real *rpl = d.time_scheme == 1 ? dummy2 : &rm_pot_l[p * 2];
          const real po = d.time_scheme == 1 ? pot_old[g] : real(0);
          rm_update(rp[0], rpl[0], L.c0_1, L.c1_1, L.c2_1, L.bb1, pot[g], po, stage_);
          rm_update(rp[1], rpl[1], L.c0_2, L.c1_2, L.c2_2, L.bb2, pot[g], po, stage_);
          const real wwf = wxgll[i] * wzgll[j] * fac2;
          pml_out[j * NGLL + i] = static_cast<real>(static_cast<double>(wwf) *
                                                    (L.A1 * pot_d[g] + L.A2 * pot[g] + L.A3 * rp[0] + L.A4 * rp[1]));
        }
        const real fac = jacobian[p] / rho[p];
        t1[j][i] = fac * (xixl * dxl + xizl * dzl);
        t2[j][i] = fac * (gammaxl * dxl + gammazl * dzl);
      }
    for (int j = 0; j < NGLL; ++j)
      for (int i = 0; i < NGLL; ++i) {
        real s1 = 0, s2 = 0;
        for (int k = 0; k < NGLL; ++k) {
          s1 = s1 + t1[j][k] * hprimewgll[k][i];
          s2 = s2 + t2[k][i] * hprimewgll[k][j];
        }
        out[j * NGLL + i] = wzgll[j] * s1 + wxgll[i] * s2;
      }
  }

  void enforce_free_surface() {
    for (int k = 0; k < d.nfree_ac; ++k) {
      const int g = d.free_ac_iglob[k];
      pot[g] = 0;
      pot_d[g] = 0;
      pot_dd[g] = 0;
    }
  }

  // chi_dd = Stacey(chi_d) + coupling(u) + sources - K chi, in the order of
  // compute_forces_viscoacoustic_calling_routine.F90:40-233 with one process
  // (phase 1 holds no element: boundary terms first, then all elements).
  void acoustic_forces(int stage, int nt) {
    pml_boundary_acoustic();
    for (int p = 0; p < d.nstacey_ac; ++p) {
      const int g = d.st_ac_iglob[p];
      pot_dd[g] = pot_dd[g] - pot_d[g] * st_ac_w[p] / st_ac_rvp[p];
    }
    for (int p = 0; p < d.ncpl_ac; ++p) {
      const int g = d.cpl_ac_iglob[p];
      // the adjoint field takes minus the solid's acceleration of this step
      // (compute_coupling_acoustic_el.f90:89-95, SIMULATION_TYPE 3)
      real ux = d.adj_src ? -accel[2 * g] : displ[2 * g];
      real uz = d.adj_src ? -accel[2 * g + 1] : displ[2 * g + 1];
      if (pml && d.pml_region[d.cpl_ac_elpt[p] / NGLL2] > 0) {
        // solid element in a PML layer (compute_coupling_acoustic_el.f90:78-140)
        const size_t q = d.cpl_ac_elpt[p];
        const int region = d.pml_region[q / NGLL2];
        double kx, bx, ax, kz, bz, az;
        pml_params(q, kx, bx, ax, kz, bz, az);
        const PmlCoef L = region == CPML_X_ONLY ? lik_parameters(d.DT, kx, bx, ax, kz, bz, az, region, 13)
                                                : lik_parameters(d.DT, kz, bz, az, kx, bx, ax, region, 31);
        real *rf = &rm_fsb[p * 2];
        real dummy[2] = {0, 0};
        real *rfl = d.time_scheme == 1 ? dummy : &rm_fsb_l[p * 2];
        const real ox = d.time_scheme == 1 ? displ_old[2 * g] : real(0);
        const real oz = d.time_scheme == 1 ? displ_old[2 * g + 1] : real(0);
        rm_update(rf[0], rfl[0], L.c0_1, L.c1_1, L.c2_1, L.bb1, ux, ox, stage);
        rm_update(rf[1], rfl[1], L.c0_1, L.c1_1, L.c2_1, L.bb1, uz, oz, stage);
        ux = static_cast<real>(L.A0 * displ[2 * g] + L.A1 * rf[0]);
        uz = static_cast<real>(L.A0 * displ[2 * g + 1] + L.A1 * rf[1]);
      }
      const real displ_n = ux * cpl_ac_nx[p] + uz * cpl_ac_nz[p];
      pot_dd[g] = pot_dd[g] + cpl_ac_w[p] * displ_n;
    }
    if (d.adj_src) {
      // adjoint sources of receivers in fluid elements, time-reversed
      // (compute_add_sources_acoustic.f90:247-290): (xir * gammar) * s, in CUSTOM_REAL
      const int it_tmp = d.nstep_total - 1 - it;
      for (int r = 0; r < d.nrec && it_tmp >= 0; ++r) {
        const int e = d.rec_ispec[r];
        if (!is_acoustic(e)) continue;
        const real a = adj[(static_cast<size_t>(r) * d.nstep_total + it_tmp) * 2];
        for (int j = 0; j < NGLL; ++j)
          for (int i = 0; i < NGLL; ++i) {
            const int g = d.ibool[static_cast<size_t>(e) * NGLL2 + j * NGLL + i];
            const real h = static_cast<real>(d.hxir[r * NGLL + i]) * static_cast<real>(d.hgammar[r * NGLL + j]);
            pot_dd[g] = pot_dd[g] + h * a;
          }
      }
    }
    for (int isrc = 0; isrc < d.nsrc && !d.adj_src; ++isrc) {
      const int e = d.src_ispec[isrc];
      if (!is_acoustic(e)) continue;
      real stf = 0;
      if (it < d.nstep_total)
        stf = static_cast<real>(d.stf[(static_cast<size_t>(isrc) * d.nstep_total + it) * d.nstage + stage]);
      // compute_add_sources_acoustic.f90:63-70
      for (int j = 0; j < NGLL; ++j)
        for (int i = 0; i < NGLL; ++i) {
          const size_t p = static_cast<size_t>(e) * NGLL2 + j * NGLL + i;
          const int g = d.ibool[p];
          const real sa = srcarr[(static_cast<size_t>(isrc) * NGLL2 + j * NGLL + i) * 2];
          pot_dd[g] = pot_dd[g] + sa * stf / kappa[p];
        }
    }
    parallel_for(nspec, nspec > 256 ? nt : 1, [&](int b, int e1_) {
      for (int e = b; e < e1_; ++e)
        if (is_acoustic(e))
          acoustic_element_force(e, stage, &contrib_ac[static_cast<size_t>(e) * NGLL2],
                                 pml ? &contrib_ac_pml[static_cast<size_t>(e) * NGLL2] : nullptr);
    });
    // each point takes its elements' contributions in ascending element order,
    // an element's layer term right after its weak-form term
    points_for(nt, [&](int b, int e1_) {
      for (int g = b; g < e1_; ++g)
        for (int k = gat_ac_off[g]; k < gat_ac_off[g + 1]; ++k) {
          const int eq = gat_ac[k];
          pot_dd[g] = pot_dd[g] - contrib_ac[eq];
          if (pml_region(eq / NGLL2) > 0) pot_dd[g] = pot_dd[g] - contrib_ac_pml[eq];
        }
    });
    pml_boundary_acoustic();
  }

  // Memory-variable update at one GLL point; returns the three sums.
  // compute_attenuation_viscoelastic.f90:36-236 (Newmark branch :109-146,
  // LDDRK branch :147-163); stage is 0-based.
  void attenuation(size_t p, real dux_dxl, real dux_dzl, real duz_dxl, real duz_dzl, int stage, real &e1s,
                   real &e11s, real &e13s) {
    const real theta_n = dux_dxl + duz_dzl;
    real *E1 = &e1[p * NSLS], *E11 = &e11[p * NSLS], *E13 = &e13[p * NSLS];
    if (d.time_scheme == 1) {
      real *old = &att_old[p * 3];
      const real theta_n1 = old[0] + old[1];
      for (int s = 0; s < NSLS; ++s) {
        const size_t q = p * NSLS + s;
        real a = a1[q];
        E1[s] = a * a * E1[s] + b1[q] * (theta_n + a * theta_n1);
        a = a2[q];
        E11[s] = a * a * E11[s] + b2[q] * (dux_dxl - theta_n / real(2) + a * (old[0] - theta_n1 / real(2)));
        E13[s] = a * a * E13[s] + b2[q] * (dux_dzl + duz_dxl + a * old[2]);
      }
    } else {
      const real al = alpha[stage], be = beta[stage];
      for (int s = 0; s < NSLS; ++s) {
        const size_t q = p * NSLS + s;
        const real phinu1 = phi1[q], phinu2 = phi2[q];
        const double tauinvnu1 = itau1[q], tauinvnu2 = itau2[q];
        // tauinvnu is double in the reference: the products with it are double
        e1_l[q] = static_cast<real>(static_cast<double>(al * e1_l[q]) +
                                    static_cast<double>(deltat) *
                                        (static_cast<double>(theta_n * phinu1) - static_cast<double>(E1[s]) * tauinvnu1));
        E1[s] = E1[s] + be * e1_l[q];
        e11_l[q] = static_cast<real>(static_cast<double>(al * e11_l[q] + deltat * ((dux_dxl - theta_n / real(2)) * phinu2)) -
                                     static_cast<double>(deltat) * (static_cast<double>(E11[s]) * tauinvnu2));
        E11[s] = E11[s] + be * e11_l[q];
        e13_l[q] = static_cast<real>(static_cast<double>(al * e13_l[q] + deltat * ((dux_dzl + duz_dxl) * phinu2)) -
                                     static_cast<double>(deltat) * (static_cast<double>(E13[s]) * tauinvnu2));
        E13[s] = E13[s] + be * e13_l[q];
      }
    }
    e1s = E1[0] + E1[1] + E1[2];
    e11s = E11[0] + E11[1] + E11[2];
    e13s = E13[0] + E13[1] + E13[2];
    if (d.time_scheme == 1) {
      real *old = &att_old[p * 3];
      old[0] = dux_dxl;
      old[1] = duz_dzl;
      old[2] = dux_dzl + duz_dxl;
    }
  }

  // Element internal force -K u for one element (compute_forces_viscoelastic.F90:
  // 184-197 gather, :810-883 mxm_4comp_singleA, :220-234 mapping, :286-357
  // isotropic P-SV stress with lambda = rho*cp^2 - 2 mu, :372-445 anisotropic,
  // :481-503 attenuation, :669-675 weak-form terms, :760-782 weighted transpose
  // contraction).  Writes the 25x2 contributions (to be subtracted) into `out`.
  void element_force(int ispec, int stage, real *out, real *pml_out) {
    const size_t off = static_cast<size_t>(ispec) * NGLL2;
    real ux[NGLL][NGLL], uz[NGLL][NGLL];  // [j][i]
    for (int j = 0; j < NGLL; ++j)
      for (int i = 0; i < NGLL; ++i) {
        const int g = d.ibool[off + j * NGLL + i];
        ux[j][i] = displ[2 * g];
        uz[j][i] = displ[2 * g + 1];
      }
    real t1x[NGLL][NGLL], t1z[NGLL][NGLL], t2x[NGLL][NGLL], t2z[NGLL][NGLL];
    const bool is_aniso = d.ispec_is_anisotropic && d.ispec_is_anisotropic[ispec];
    for (int j = 0; j < NGLL; ++j)
      for (int i = 0; i < NGLL; ++i) {
        const real dux_dxi = ux[j][0] * hprime[i][0] + ux[j][1] * hprime[i][1] + ux[j][2] * hprime[i][2] +
                             ux[j][3] * hprime[i][3] + ux[j][4] * hprime[i][4];
        const real duz_dxi = uz[j][0] * hprime[i][0] + uz[j][1] * hprime[i][1] + uz[j][2] * hprime[i][2] +
                             uz[j][3] * hprime[i][3] + uz[j][4] * hprime[i][4];
        const real dux_dgamma = ux[0][i] * hprime[j][0] + ux[1][i] * hprime[j][1] + ux[2][i] * hprime[j][2] +
                                ux[3][i] * hprime[j][3] + ux[4][i] * hprime[j][4];
        const real duz_dgamma = uz[0][i] * hprime[j][0] + uz[1][i] * hprime[j][1] + uz[2][i] * hprime[j][2] +
                                uz[3][i] * hprime[j][3] + uz[4][i] * hprime[j][4];
        const size_t p = off + j * NGLL + i;
        const real xixl = xix[p], xizl = xiz[p], gammaxl = gammax[p], gammazl = gammaz[p];
        const real jacobianl = jacobian[p];
        real dux_dxl = dux_dxi * xixl + dux_dgamma * gammaxl;
        real dux_dzl = dux_dxi * xizl + dux_dgamma * gammazl;
        real duz_dxl = duz_dxi * xixl + duz_dgamma * gammaxl;
        real duz_dzl = duz_dxi * xizl + duz_dgamma * gammazl;
        // unmodified strains, kept for the PML stress (compute_forces_viscoelastic.F90:600-610)
        const real p_dux_dxl = dux_dxl, p_dux_dzl = dux_dzl, p_duz_dxl = duz_dxl, p_duz_dzl = duz_dzl;
        const int region = pml_region(ispec);
        const bool visco = region > 0 && d.pml_visco && d.pml_visco[ispec];
        // modified strains of a viscoelastic layer element (kappa and mu parts)
        real vk_pml_xx = 0, vk_pml_zz = 0, vm_pml_xx = 0, vm_pml_zz = 0, vm_pml_xz = 0, vm_pml_zx = 0;
        real vk_xx = 0, vk_zz = 0, vm_xx = 0, vm_zz = 0, vm_xz = 0, vm_zx = 0;
        if (region > 0) {
          // pml_compute_memory_variables_elastic (pml_compute_memory_variables.f90:230-540)
          real dxi_ox = 0, dxi_oz = 0, dg_ox = 0, dg_oz = 0;
          if (d.time_scheme == 1)
            for (int k = 0; k < NGLL; ++k) {
              const int gr = d.ibool[off + j * NGLL + k], gc = d.ibool[off + k * NGLL + i];
              dxi_ox = dxi_ox + displ_old[2 * gr] * hprime[i][k];
              dxi_oz = dxi_oz + displ_old[2 * gr + 1] * hprime[i][k];
              dg_ox = dg_ox + displ_old[2 * gc] * hprime[j][k];
              dg_oz = dg_oz + displ_old[2 * gc + 1] * hprime[j][k];
            }
          const real o_dux_dxl = dxi_ox * xixl + dg_ox * gammaxl, o_dux_dzl = dxi_ox * xizl + dg_ox * gammazl;
          const real o_duz_dxl = dxi_oz * xixl + dg_oz * gammaxl, o_duz_dzl = dxi_oz * xizl + dg_oz * gammazl;
          double kx, bx, ax, kz, bz, az;
          pml_params(p, kx, bx, ax, kz, bz, az);
          const PmlCoef zx = lik_parameters(d.DT, kz, bz, az, kx, bx, ax, region, 31);
          const PmlCoef xz = lik_parameters(d.DT, kx, bx, ax, kz, bz, az, region, 13);
          real *r = &rm_el[p * 8];
          real dummy[8] = {0, 0, 0, 0, 0, 0, 0, 0};
          real *rl = d.time_scheme == 1 ? dummy : &rm_el_l[p * 8];
          rm_update(r[0], rl[0], zx.c0_1, zx.c1_1, zx.c2_1, zx.bb1, p_dux_dxl, o_dux_dxl, stage);
          rm_update(r[1], rl[1], zx.c0_2, zx.c1_2, zx.c2_2, zx.bb2, p_dux_dxl, o_dux_dxl, stage);
          rm_update(r[2], rl[2], zx.c0_1, zx.c1_1, zx.c2_1, zx.bb1, p_duz_dxl, o_duz_dxl, stage);
          rm_update(r[3], rl[3], zx.c0_2, zx.c1_2, zx.c2_2, zx.bb2, p_duz_dxl, o_duz_dxl, stage);
          rm_update(r[4], rl[4], xz.c0_1, xz.c1_1, xz.c2_1, xz.bb1, p_dux_dzl, o_dux_dzl, stage);
          rm_update(r[5], rl[5], xz.c0_2, xz.c1_2, xz.c2_2, xz.bb2, p_dux_dzl, o_dux_dzl, stage);
          rm_update(r[6], rl[6], xz.c0_1, xz.c1_1, xz.c2_1, xz.bb1, p_duz_dzl, o_duz_dzl, stage);
          rm_update(r[7], rl[7], xz.c0_2, xz.c1_2, xz.c2_2, xz.bb2, p_duz_dzl, o_duz_dzl, stage);
          if (visco) {
            // pml_compute_memory_variables_viscoelastic (pml_compute_memory_variables.f90:686-892):
            // per SLS, convolutions of the strains with 1/tau_sigma, their Zener and
            // phi-weighted sums, then the modified strains of the kappa and mu parts
            double A01 = 0, A10 = 0, A2k = 0, A2m = 0, A3k = 0, A3m = 0, A4k = 0, A4m = 0, A5k = 0, A5m = 0;
            double Mk = 0, Mm = 0;
            real ks_xx = 0, ks_zz = 0, ms_xx = 0, ms_zz = 0, ms_xz = 0, ms_zx = 0;
            real pk_xx = 0, pk_zz = 0, pm_xx = 0, pm_zz = 0, pm_xz = 0, pm_zx = 0;
            for (int sl = 0; sl < NSLS; ++sl) {
              const size_t q = p * NSLS + sl;
              const double tik = vitau1[q], tim = vitau2[q], tek = teps1[q], tem = teps2[q];
              Mk = mu_nu1[p] * static_cast<double>(NSLS);
              Mm = mu_nu2[p] * static_cast<double>(NSLS);
              const double Ak = vphi1[q], Am = vphi2[q];
              const ViscoLik k31 = lik_viscoelastic(kz, bz, az, kx, bx, ax, region, 31, tik, tek);
              const ViscoLik m31 = lik_viscoelastic(kz, bz, az, kx, bx, ax, region, 31, tim, tem);
              const ViscoLik k13 = lik_viscoelastic(kx, bx, ax, kz, bz, az, region, 13, tik, tek);
              const ViscoLik m13 = lik_viscoelastic(kx, bx, ax, kz, bz, az, region, 13, tim, tem);
              A01 = m31.A0;
              A10 = m13.A0;
              double ck0, ck1, ck2, cm0, cm1, cm2;
              coef_convolution(tik, d.DT, ck0, ck1, ck2);
              coef_convolution(tim, d.DT, cm0, cm1, cm2);
              real *v = &rm_visco[q * 6];
              v[0] = static_cast<real>(ck0 * v[0] + ck1 * p_dux_dxl + ck2 * o_dux_dxl);
              v[1] = static_cast<real>(ck0 * v[1] + ck1 * p_duz_dzl + ck2 * o_duz_dzl);
              v[2] = static_cast<real>(cm0 * v[2] + cm1 * p_dux_dxl + cm2 * o_dux_dxl);
              v[3] = static_cast<real>(cm0 * v[3] + cm1 * p_duz_dzl + cm2 * o_duz_dzl);
              v[4] = static_cast<real>(cm0 * v[4] + cm1 * p_dux_dzl + cm2 * o_dux_dzl);
              v[5] = static_cast<real>(cm0 * v[5] + cm1 * p_duz_dxl + cm2 * o_duz_dxl);
              A2k = A2k + k31.A1;
              A2m = A2m + m31.A1;
              A3k = A3k + k31.A2;
              A3m = A3m + m31.A2;
              A4k = A4k + k13.A1;
              A4m = A4m + m13.A1;
              A5k = A5k + k13.A2;
              A5m = A5m + m13.A2;
              ks_xx = static_cast<real>(ks_xx + k31.Az * v[0] / Mk);
              ks_zz = static_cast<real>(ks_zz + k13.Az * v[1] / Mk);
              ms_xx = static_cast<real>(ms_xx + m31.Az * v[2] / Mm);
              ms_zz = static_cast<real>(ms_zz + m13.Az * v[3] / Mm);
              ms_xz = static_cast<real>(ms_xz + m13.Az * v[4] / Mm);
              ms_zx = static_cast<real>(ms_zx + m31.Az * v[5] / Mm);
              pk_xx = static_cast<real>(pk_xx + Ak * v[0]);
              pk_zz = static_cast<real>(pk_zz + Ak * v[1]);
              pm_xx = static_cast<real>(pm_xx + Am * v[2]);
              pm_zz = static_cast<real>(pm_zz + Am * v[3]);
              pm_xz = static_cast<real>(pm_xz + Am * v[4]);
              pm_zx = static_cast<real>(pm_zx + Am * v[5]);
            }
            vk_pml_xx = static_cast<real>(A01 * p_dux_dxl + ks_xx + A2k * r[0] / Mk + A3k * r[1] / Mk);
            vk_pml_zz = static_cast<real>(A10 * p_duz_dzl + ks_zz + A4k * r[6] / Mk + A5k * r[7] / Mk);
            vm_pml_xx = static_cast<real>(A01 * p_dux_dxl + ms_xx + A2m * r[0] / Mm + A3m * r[1] / Mm);
            vm_pml_zz = static_cast<real>(A10 * p_duz_dzl + ms_zz + A4m * r[6] / Mm + A5m * r[7] / Mm);
            vm_pml_xz = static_cast<real>(A10 * p_dux_dzl + ms_xz + A4m * r[4] / Mm + A5m * r[5] / Mm);
            vm_pml_zx = static_cast<real>(A01 * p_duz_dxl + ms_zx + A2m * r[2] / Mm + A3m * r[3] / Mm);
            vk_xx = p_dux_dxl + pk_xx;
            vk_zz = p_duz_dzl + pk_zz;
            vm_xx = p_dux_dxl + pm_xx;
            vm_zz = p_duz_dzl + pm_zz;
            vm_xz = p_dux_dzl + pm_xz;
            vm_zx = p_duz_dxl + pm_zx;
          } else {
            dux_dxl = static_cast<real>(zx.A0 * p_dux_dxl + zx.A1 * r[0] + zx.A2 * r[1]);
            duz_dxl = static_cast<real>(zx.A0 * p_duz_dxl + zx.A1 * r[2] + zx.A2 * r[3]);
            dux_dzl = static_cast<real>(xz.A0 * p_dux_dzl + xz.A1 * r[4] + xz.A2 * r[5]);
            duz_dzl = static_cast<real>(xz.A0 * p_duz_dzl + xz.A1 * r[6] + xz.A2 * r[7]);
          }
          // pml_compute_accel_contribution_elastic (pml_compute_accel_contribution.f90:187-333)
          const int g = d.ibool[p];
          const real fac = rho[p] * jacobianl;
          const PmlCoef L = l_parameters(d.DT, kx, bx, ax, kz, bz, az, region);
          real *rd = &rm_displ[p * 4];
          real dummy2[4] = {0, 0, 0, 0};
          real *rdl = d.time_scheme == 1 ? dummy2 : &rm_displ_l[p * 4];
          const real ox = d.time_scheme == 1 ? displ_old[2 * g] : real(0);
          const real oz = d.time_scheme == 1 ? displ_old[2 * g + 1] : real(0);
          rm_update(rd[0], rdl[0], L.c0_1, L.c1_1, L.c2_1, L.bb1, ux[j][i], ox, stage);
          rm_update(rd[1], rdl[1], L.c0_1, L.c1_1, L.c2_1, L.bb1, uz[j][i], oz, stage);
          rm_update(rd[2], rdl[2], L.c0_2, L.c1_2, L.c2_2, L.bb2, ux[j][i], ox, stage);
          rm_update(rd[3], rdl[3], L.c0_2, L.c1_2, L.c2_2, L.bb2, uz[j][i], oz, stage);
          const double wwf = static_cast<double>(wxgll[i] * wzgll[j] * fac);
          pml_out[2 * (j * NGLL + i)] = static_cast<real>(
              wwf * (L.A1 * veloc[2 * g] + L.A2 * ux[j][i] + L.A3 * rd[0] + L.A4 * rd[2]));
          pml_out[2 * (j * NGLL + i) + 1] = static_cast<real>(
              wwf * (L.A1 * veloc[2 * g + 1] + L.A2 * uz[j][i] + L.A3 * rd[1] + L.A4 * rd[3]));
        }
        const real mul = mu[p];
        const real rhol = rho[p];
        const real cpl = rho_vp[p] / rhol;
        const real lambdal = rhol * cpl * cpl - real(2) * mul;
        const real lambdaplus2mu = lambdal + real(2) * mul;
        const real lambdalplusmul = lambdal + mul;
        real sigma_xx, sigma_zz, sigma_xz, sigma_zx;
        if (visco) {
          // viscoelastic layer stress with the unrelaxed moduli (compute_forces_viscoelastic.F90:545-555)
          sigma_xx = (lambdalplusmul * vk_pml_xx + mul * vm_pml_xx) + (lambdalplusmul * vk_zz - mul * vm_zz);
          sigma_xz = (mul * vm_pml_zx + mul * vm_xz);
          sigma_zx = (mul * vm_zx + mul * vm_pml_xz);
          sigma_zz = (lambdalplusmul * vk_xx - mul * vm_xx) + (lambdalplusmul * vk_pml_zz + mul * vm_pml_zz);
        } else if (region > 0) {
          // PML stress: modified strains on the diagonal pairs, not symmetric
          sigma_xx = lambdaplus2mu * dux_dxl + lambdal * p_duz_dzl;
          sigma_zz = lambdaplus2mu * duz_dzl + lambdal * p_dux_dxl;
          sigma_zx = mul * (p_duz_dxl + dux_dzl);
          sigma_xz = mul * (p_dux_dzl + duz_dxl);
        } else if (!is_aniso) {
          sigma_xx = lambdaplus2mu * dux_dxl + lambdal * duz_dzl;
          sigma_zz = lambdaplus2mu * duz_dzl + lambdal * dux_dxl;
          sigma_xz = mul * (duz_dxl + dux_dzl);
          sigma_zx = sigma_xz;
        } else {
          // c_ij are read as double in the reference (compute_forces_viscoelastic.F90:112)
          const double C11 = c11[p], C13 = c13[p], C15 = c15[p], C33 = c33[p], C35 = c35[p], C55 = c55[p];
          sigma_xx = static_cast<real>(C11 * dux_dxl + C13 * duz_dzl + C15 * (duz_dxl + dux_dzl));
          sigma_zz = static_cast<real>(C13 * dux_dxl + C33 * duz_dzl + C35 * (duz_dxl + dux_dzl));
          sigma_xz = static_cast<real>(C15 * dux_dxl + C35 * duz_dzl + C55 * (duz_dxl + dux_dzl));
          sigma_zx = sigma_xz;
        }
        // layer elements keep no attenuation memory variables
        // (compute_attenuation_viscoelastic.f90:85)
        if (atten && region == 0) {
          real e1s, e11s, e13s;
          attenuation(p, dux_dxl, dux_dzl, duz_dxl, duz_dzl, stage, e1s, e11s, e13s);
          sigma_xx = sigma_xx + lambdalplusmul * e1s + real(2) * mul * e11s;
          sigma_xz = sigma_xz + mul * e13s;
          sigma_zz = sigma_zz + lambdalplusmul * e1s - real(2) * mul * e11s;
          sigma_zx = sigma_xz;
        }
        t1x[j][i] = jacobianl * (sigma_xx * xixl + sigma_zx * xizl);
        t1z[j][i] = jacobianl * (sigma_xz * xixl + sigma_zz * xizl);
        t2x[j][i] = jacobianl * (sigma_xx * gammaxl + sigma_zx * gammazl);
        t2z[j][i] = jacobianl * (sigma_xz * gammaxl + sigma_zz * gammazl);
      }
    for (int j = 0; j < NGLL; ++j)
      for (int i = 0; i < NGLL; ++i) {
        real tx1 = 0, tx2 = 0, tz1 = 0, tz2 = 0;
        for (int k = 0; k < NGLL; ++k) {
          tx1 = tx1 + t1x[j][k] * hprimewgll[k][i];
          tx2 = tx2 + t2x[k][i] * hprimewgll[k][j];
          tz1 = tz1 + t1z[j][k] * hprimewgll[k][i];
          tz2 = tz2 + t2z[k][i] * hprimewgll[k][j];
        }
        out[2 * (j * NGLL + i)] = wzgll[j] * tx1 + wxgll[i] * tx2;
        out[2 * (j * NGLL + i) + 1] = wzgll[j] * tz1 + wxgll[i] * tz2;
      }
  }

  // accel = Stacey(veloc) + sources(stf[it, stage]) - K displ, in reference order
  void forces(int stage, int nt) {
    for (int p = 0; p < d.nstacey; ++p) {
      const int g = d.st_iglob[p];
      const real vx = veloc[2 * g], vz = veloc[2 * g + 1];
      const real nx = st_nx[p], nz = st_nz[p];
      const real vn = nx * vx + nz * vz;
      const real tx = st_rvp[p] * vn * nx + st_rvs[p] * (vx - vn * nx);
      const real tz = st_rvp[p] * vn * nz + st_rvs[p] * (vz - vn * nz);
      accel[2 * g] = accel[2 * g] - tx * st_w[p];
      accel[2 * g + 1] = accel[2 * g + 1] - tz * st_w[p];
    }
    pml_boundary_elastic();
    // fluid pressure on the solid (compute_coupling_viscoelastic_ac.f90:80-250)
    for (int p = 0; p < (acoustic ? d.ncpl_el : 0); ++p) {
      const int g = d.cpl_el_iglob[p];
      // the adjoint field takes the fluid's potential of this step
      // (compute_coupling_viscoelastic_ac.f90:89-93, SIMULATION_TYPE 3)
      real pressure = d.adj_src ? pot[g] : -pot_dd[g];
      if (pml && d.pml_region[d.cpl_el_acpt[p] / NGLL2] > 0) {
        // fluid element in a PML layer (:100-150)
        const size_t q = d.cpl_el_acpt[p];
        double kx, bx, ax, kz, bz, az;
        pml_params(q, kx, bx, ax, kz, bz, az);
        const PmlCoef L = l_parameters(d.DT, kx, bx, ax, kz, bz, az, d.pml_region[q / NGLL2]);
        real dummy = 0;
        real &rl = d.time_scheme == 1 ? dummy : rm_sfb_l[p];
        rm_update(rm_sfb[p], rl, L.c0_1, L.c1_1, L.c2_1, L.bb1, pot[g], d.time_scheme == 1 ? pot_old[g] : real(0),
                  stage);
        pressure = static_cast<real>(-(L.A0 * pot_dd[g] + L.A1 * pot_d[g] + L.A2 * pot[g] + L.A3 * rm_sfb[p]));
      }
      accel[2 * g] = accel[2 * g] + cpl_el_w[p] * cpl_el_nx[p] * pressure;
      accel[2 * g + 1] = accel[2 * g + 1] + cpl_el_w[p] * cpl_el_nz[p] * pressure;
    }
    if (d.adj_src) {
      // adjoint sources at the receivers, time-reversed (compute_add_sources_viscoelastic.f90:351-405)
      const int it_tmp = d.nstep_total - 1 - it;
      for (int r = 0; r < d.nrec && it_tmp >= 0; ++r) {
        const int e = d.rec_ispec[r];
        if (is_acoustic(e)) continue;
        const real ax = adj[(static_cast<size_t>(r) * d.nstep_total + it_tmp) * 2];
        const real az = adj[(static_cast<size_t>(r) * d.nstep_total + it_tmp) * 2 + 1];
        for (int j = 0; j < NGLL; ++j)
          for (int i = 0; i < NGLL; ++i) {
            const int g = d.ibool[static_cast<size_t>(e) * NGLL2 + j * NGLL + i];
            const real h = static_cast<real>(d.hxir[r * NGLL + i]) * static_cast<real>(d.hgammar[r * NGLL + j]);
            accel[2 * g] = accel[2 * g] + h * ax;
            accel[2 * g + 1] = accel[2 * g + 1] + h * az;
          }
      }
    }
    for (int isrc = 0; isrc < d.nsrc && !d.adj_src; ++isrc) {
      real stf = 0;
      if (it < d.nstep_total)
        stf = static_cast<real>(d.stf[(static_cast<size_t>(isrc) * d.nstep_total + it) * d.nstage + stage]);
      const int e = d.src_ispec[isrc];
      if (is_acoustic(e)) continue;
      for (int j = 0; j < NGLL; ++j)
        for (int i = 0; i < NGLL; ++i) {
          const int g = d.ibool[static_cast<size_t>(e) * NGLL2 + j * NGLL + i];
          const size_t q = (static_cast<size_t>(isrc) * NGLL2 + j * NGLL + i) * 2;
          accel[2 * g] = accel[2 * g] + srcarr[q] * stf;
          accel[2 * g + 1] = accel[2 * g + 1] + srcarr[q + 1] * stf;
        }
    }
    parallel_for(nspec, nspec > 256 ? nt : 1, [&](int b, int e1_) {
      for (int e = b; e < e1_; ++e)
        if (!is_acoustic(e))
          element_force(e, stage, &contrib[static_cast<size_t>(e) * NGLL2 * 2],
                        pml ? &contrib_pml[static_cast<size_t>(e) * NGLL2 * 2] : nullptr);
    });
    // gather in ascending element order per point; the element's PML
    // contribution right after its weak-form terms (compute_forces_viscoelastic.F90:785-797)
    points_for(nt, [&](int b, int e1_) {
      for (int g = b; g < e1_; ++g)
        for (int k = gat_el_off[g]; k < gat_el_off[g + 1]; ++k) {
          const int eq = gat_el[k];
          accel[2 * g] = accel[2 * g] - contrib[2 * eq];
          accel[2 * g + 1] = accel[2 * g + 1] - contrib[2 * eq + 1];
          if (pml_region(eq / NGLL2) > 0) {
            accel[2 * g] = accel[2 * g] - contrib_pml[2 * eq];
            accel[2 * g + 1] = accel[2 * g + 1] - contrib_pml[2 * eq + 1];
          }
        }
    });
  }

  // Receiver in an acoustic element (write_seismograms.F90:75-150):
  // seismotype 1-3 interpolate grad(chi)/rho of chi, chi_dot or chi_dot_dot
  // formed in double (compute_vector_field.f90:143-207) and stored in
  // CUSTOM_REAL; seismotype 4 interpolates the pressure -chi_dot_dot (or -chi
  // with USE_TRICK_FOR_BETTER_PRESSURE, compute_pressure.f90:542-572),
  // seismotype 6 the potential chi itself (write_seismograms.F90:149-170).
  void record_acoustic(int r, double *out) {
    const int e = d.rec_ispec[r];
    const size_t off = static_cast<size_t>(e) * NGLL2;
    double vx = 0.0, vz = 0.0;
    if (d.seismotype == 6) {
      for (int j = 0; j < NGLL; ++j)
        for (int i = 0; i < NGLL; ++i) {
          const double h = static_cast<double>(static_cast<real>(d.hxir[r * NGLL + i]) *
                                               static_cast<real>(d.hgammar[r * NGLL + j]));
          vx = vx + static_cast<double>(pot[d.ibool[off + j * NGLL + i]]) * h;
        }
      out[0] = vx;
      out[1] = 0.0;
      return;
    }
    if (d.seismotype == 4) {
      const std::vector<real> &f = d.use_trick ? pot : pot_dd;
      for (int j = 0; j < NGLL; ++j)
        for (int i = 0; i < NGLL; ++i) {
          const double h = static_cast<double>(static_cast<real>(d.hxir[r * NGLL + i]) *
                                               static_cast<real>(d.hgammar[r * NGLL + j]));
          const real pr = -f[d.ibool[off + j * NGLL + i]];
          vx = vx + static_cast<double>(pr) * h;
        }
      out[0] = vx;
      out[1] = 0.0;
      return;
    }
    const std::vector<real> &f = d.seismotype == 2 ? pot_d : (d.seismotype == 3 ? pot_dd : pot);
    for (int j = 0; j < NGLL; ++j)
      for (int i = 0; i < NGLL; ++i) {
        double t1 = 0.0, t2 = 0.0;
        for (int k = 0; k < NGLL; ++k) {
          t1 = t1 + static_cast<double>(f[d.ibool[off + j * NGLL + k]]) * static_cast<double>(hprime[i][k]);
          t2 = t2 + static_cast<double>(f[d.ibool[off + k * NGLL + i]]) * static_cast<double>(hprime[j][k]);
        }
        const size_t p = off + j * NGLL + i;
        const double dchi_dx = t1 * static_cast<double>(xix[p]) + t2 * static_cast<double>(gammax[p]);
        const double dchi_dz = t1 * static_cast<double>(xiz[p]) + t2 * static_cast<double>(gammaz[p]);
        const real fx = static_cast<real>(dchi_dx / static_cast<double>(rho[p]));
        const real fz = static_cast<real>(dchi_dz / static_cast<double>(rho[p]));
        const double h = static_cast<double>(static_cast<real>(d.hxir[r * NGLL + i]) *
                                             static_cast<real>(d.hgammar[r * NGLL + j]));
        vx = vx + static_cast<double>(fx) * h;
        vz = vz + static_cast<double>(fz) * h;
      }
    out[0] = d.cosrot * vx + d.sinrot * vz;
    out[1] = -d.sinrot * vx + d.cosrot * vz;
  }

  void record(double *seis, int nstep, int s) {
    if (!seis) return;
    const std::vector<real> &field = d.seismotype == 2 ? veloc : (d.seismotype == 3 ? accel : displ);
    for (int r = 0; r < d.nrec; ++r) {
      const int e = d.rec_ispec[r];
      if (is_acoustic(e)) {
        record_acoustic(r, &seis[(static_cast<size_t>(r) * nstep + s) * 2]);
        continue;
      }
      if (d.seismotype == 6) {
        // a potential receiver in a solid records nothing
        seis[(static_cast<size_t>(r) * nstep + s) * 2] = 0.0;
        seis[(static_cast<size_t>(r) * nstep + s) * 2 + 1] = 0.0;
        continue;
      }
      double vx = 0.0, vz = 0.0;
      for (int j = 0; j < NGLL; ++j)
        for (int i = 0; i < NGLL; ++i) {
          const int g = d.ibool[static_cast<size_t>(e) * NGLL2 + j * NGLL + i];
          // xir_store_loc and gammar_store_loc are CUSTOM_REAL: their product is formed in that precision
          const double h = static_cast<double>(static_cast<real>(d.hxir[r * NGLL + i]) *
                                               static_cast<real>(d.hgammar[r * NGLL + j]));
          vx = vx + static_cast<double>(field[2 * g]) * h;
          vz = vz + static_cast<double>(field[2 * g + 1]) * h;
        }
      double *out = &seis[(static_cast<size_t>(r) * nstep + s) * 2];
      out[0] = d.cosrot * vx + d.sinrot * vz;
      out[1] = -d.sinrot * vx + d.cosrot * vz;
    }
  }

  int run(int nstep, double *seis, int nthreads) override {
    const int nt = nthreads > 0 ? nthreads : default_threads();
    for (int s = 0; s < nstep; ++s, ++it) {
      if (d.time_scheme == 1) {
        if (pml) {
          // mid-step fields of the CPML convolutions (update_displacement_Newmark.F90:374-380, 429-433)
          const double h = static_cast<double>(deltatsquareover2) / 2.0;
          points_for(nt, [&](int b, int e) {
            for (size_t g = 2 * static_cast<size_t>(b); g < 2 * static_cast<size_t>(e); ++g)
              displ_old[g] = static_cast<real>(static_cast<double>(displ[g]) + h * static_cast<double>(accel[g]));
            if (acoustic)
              for (int g = b; g < e; ++g)
                pot_old[g] = static_cast<real>(static_cast<double>(pot[g]) + h * static_cast<double>(pot_dd[g]));
          });
        }
        // predictor (update_displacement_Newmark.F90:408-454)
        points_for(nt, [&](int b, int e) {
          for (size_t g = 2 * static_cast<size_t>(b); g < 2 * static_cast<size_t>(e); ++g) {
            displ[g] = displ[g] + deltat * veloc[g] + deltatsquareover2 * accel[g];
            veloc[g] = veloc[g] + deltatover2 * accel[g];
            accel[g] = 0;
          }
        });
        if (acoustic) {
          // acoustic predictor (update_displacement_Newmark.F90:353-402)
          points_for(nt, [&](int b, int e) {
            for (int g = b; g < e; ++g) {
              pot[g] = pot[g] + deltat * pot_d[g] + deltatsquareover2 * pot_dd[g];
              pot_d[g] = pot_d[g] + deltatover2 * pot_dd[g];
              pot_dd[g] = 0;
            }
          });
        }
        auto fluid_step = [&]() {
          enforce_free_surface();
          acoustic_forces(0, nt);
          points_for(nt, [&](int b, int e) {
            for (int g = b; g < e; ++g) {
              pot_dd[g] = pot_dd[g] * rmass_ac[g];
              pot_d[g] = pot_d[g] + deltatover2 * pot_dd[g];  // update_veloc_acoustic_Newmark
            }
          });
          enforce_free_surface();
        };
        auto solid_step = [&]() {
          forces(0, nt);
          // mass matrix and corrector (compute_forces_viscoelastic_calling_routine.F90:181,
          // update_displacement_Newmark.F90:564-589)
          points_for(nt, [&](int b, int e) {
            for (size_t g = 2 * static_cast<size_t>(b); g < 2 * static_cast<size_t>(e); ++g) {
              accel[g] = accel[g] * rmass[g];
              veloc[g] = veloc[g] + deltatover2 * accel[g];
            }
          });
        };
        // the whole fluid step before the solid one (iterate_time.F90:270-290); an
        // adjoint run switches the order (iterate_time.F90:300-327)
        if (acoustic && !d.adj_src) fluid_step();
        solid_step();
        if (acoustic && d.adj_src) fluid_step();
      } else {
        for (int stage = 0; stage < 6; ++stage) {
          // iterate_time.F90:167-181 clears accel, then forces and the LDDRK update
          // (update_displacement_LDDRK.F90:55-79)
          std::fill(accel.begin(), accel.end(), real(0));
          const real al = alpha[stage], be = beta[stage];
          if (acoustic) {
            std::fill(pot_dd.begin(), pot_dd.end(), real(0));
            enforce_free_surface();
            acoustic_forces(stage, nt);
            // update_veloc_acoustic_LDDRK (update_displacement_LDDRK.F90:88-115)
            points_for(nt, [&](int b, int e) {
              for (int g = b; g < e; ++g) {
                pot_dd[g] = pot_dd[g] * rmass_ac[g];
                pot_d_l[g] = al * pot_d_l[g] + deltat * pot_dd[g];
                pot_l[g] = al * pot_l[g] + deltat * pot_d[g];
                pot_d[g] = pot_d[g] + be * pot_d_l[g];
                pot[g] = pot[g] + be * pot_l[g];
              }
            });
            enforce_free_surface();
          }
          forces(stage, nt);
          points_for(nt, [&](int b, int e) {
            for (size_t g = 2 * static_cast<size_t>(b); g < 2 * static_cast<size_t>(e); ++g) {
              accel[g] = accel[g] * rmass[g];
              veloc_l[g] = al * veloc_l[g] + deltat * accel[g];
              displ_l[g] = al * displ_l[g] + deltat * veloc[g];
              veloc[g] = veloc[g] + be * veloc_l[g];
              displ[g] = displ[g] + be * displ_l[g];
            }
          });
        }
      }
      // receivers (write_seismograms.F90:150-190, compute_interpolated_dva.f90:34-97)
      record(seis, nstep, s);
    }
    return 0;
  }

  // compute_kernels.f90:75-292 (P-SV): strains of both fields with the mapping
  // derivatives read as double, kernel integrands accumulated in CUSTOM_REAL
  // (elements in parallel: each writes only its own points)
  void accumulate_kernels(const real *b) {
    parallel_for(nspec, nspec > 256 ? default_threads() : 1, [&](int eb, int ee) {
    for (int e = eb; e < ee; ++e) {
      if (is_acoustic(e)) continue;  // compute_kernels_el runs over solid elements
      const size_t off = static_cast<size_t>(e) * NGLL2;
      for (int j = 0; j < NGLL; ++j)
        for (int i = 0; i < NGLL; ++i) {
          real dux_dxi = 0, duz_dxi = 0, dux_dg = 0, duz_dg = 0;
          real bdux_dxi = 0, bduz_dxi = 0, bdux_dg = 0, bduz_dg = 0;
          for (int k = 0; k < NGLL; ++k) {
            const int gr = d.ibool[off + j * NGLL + k], gc = d.ibool[off + k * NGLL + i];
            dux_dxi = dux_dxi + displ[2 * gr] * hprime[i][k];
            duz_dxi = duz_dxi + displ[2 * gr + 1] * hprime[i][k];
            dux_dg = dux_dg + displ[2 * gc] * hprime[j][k];
            duz_dg = duz_dg + displ[2 * gc + 1] * hprime[j][k];
            bdux_dxi = bdux_dxi + b[2 * gr] * hprime[i][k];
            bduz_dxi = bduz_dxi + b[2 * gr + 1] * hprime[i][k];
            bdux_dg = bdux_dg + b[2 * gc] * hprime[j][k];
            bduz_dg = bduz_dg + b[2 * gc + 1] * hprime[j][k];
          }
          const size_t p = off + j * NGLL + i;
          const double xixl = xix[p], xizl = xiz[p], gammaxl = gammax[p], gammazl = gammaz[p];
          const real dux_dxl = static_cast<real>(dux_dxi * xixl + dux_dg * gammaxl);
          const real dux_dzl = static_cast<real>(dux_dxi * xizl + dux_dg * gammazl);
          const real duz_dxl = static_cast<real>(duz_dxi * xixl + duz_dg * gammaxl);
          const real duz_dzl = static_cast<real>(duz_dxi * xizl + duz_dg * gammazl);
          const real bdux_dxl = static_cast<real>(bdux_dxi * xixl + bdux_dg * gammaxl);
          const real bdux_dzl = static_cast<real>(bdux_dxi * xizl + bdux_dg * gammazl);
          const real bduz_dxl = static_cast<real>(bduz_dxi * xixl + bduz_dg * gammaxl);
          const real bduz_dzl = static_cast<real>(bduz_dxi * xizl + bduz_dg * gammazl);
          const real dsxx = dux_dxl, dszz = duz_dzl;
          const real dsxz = static_cast<real>(0.5 * (static_cast<double>(duz_dxl) + static_cast<double>(dux_dzl)));
          const real bdsxx = bdux_dxl, bdszz = bduz_dzl;
          const real bdsxz = static_cast<real>(0.5 * (static_cast<double>(bduz_dxl) + static_cast<double>(bdux_dzl)));
          const real kappa_k = (dsxx + dszz) * (bdsxx + bdszz);
          const real mu_k = dsxx * bdsxx + dszz * bdszz + real(2) * dsxz * bdsxz - real(1) / real(3) * kappa_k;
          const int g = d.ibool[p];
          const real rho_k = accel[2 * g] * b[2 * g] + accel[2 * g + 1] * b[2 * g + 1];
          rho_kl[p] = rho_kl[p] + rho_k;
          mu_kl[p] = mu_kl[p] + mu_k;
          kappa_kl[p] = kappa_kl[p] + kappa_k;
        }
    }
    });
  }
  // compute_kernels_Hessian (compute_kernels.f90:749-800), elastic part:
  // per-point temporaries in CUSTOM_REAL, added times deltat at every element point
  int accumulate_hessian(const void *bp) override {
    if (!bp) return -1;
    const real *ba = static_cast<const real *>(bp);
    std::vector<real> t1(nglob), t2(nglob);
    for (int g = 0; g < nglob; ++g) {
      t1[g] = ba[2 * g] * ba[2 * g] + ba[2 * g + 1] * ba[2 * g + 1];
      t2[g] = accel[2 * g] * ba[2 * g] + accel[2 * g + 1] * ba[2 * g + 1];
    }
    for (int e = 0; e < nspec; ++e) {
      if (is_acoustic(e)) continue;
      for (int q = 0; q < NGLL2; ++q) {
        const size_t p = static_cast<size_t>(e) * NGLL2 + q;
        const int g = d.ibool[p];
        hess1[p] = hess1[p] + t1[g] * deltat;
        hess2[p] = hess2[p] + t2[g] * deltat;
      }
    }
    return 0;
  }
  // compute_kernels_ac (compute_kernels.f90:293-449), fluid elements: gradients
  // of the adjoint and forward potentials summed in CUSTOM_REAL, mapped with the
  // derivatives read as double and stored in CUSTOM_REAL;
  //   rho_ac_kl += 1/rho (grad chi_adj . grad chi) deltat,
  //   kappa_ac_kl += 1/kappa chi_adj_dot_dot chi deltat
  int accumulate_acoustic(const void *bp) override {
    if (!bp || !acoustic) return -1;
    const real *b = static_cast<const real *>(bp);
    parallel_for(nspec, nspec > 256 ? default_threads() : 1, [&](int eb, int ee) {
    for (int e = eb; e < ee; ++e) {
      if (!is_acoustic(e)) continue;
      const size_t off = static_cast<size_t>(e) * NGLL2;
      for (int j = 0; j < NGLL; ++j)
        for (int i = 0; i < NGLL; ++i) {
          real t1 = 0, t2 = 0, bt1 = 0, bt2 = 0;
          for (int k = 0; k < NGLL; ++k) {
            const int gr = d.ibool[off + j * NGLL + k], gc = d.ibool[off + k * NGLL + i];
            t1 = t1 + pot[gr] * hprime[i][k];
            bt1 = bt1 + b[gr] * hprime[i][k];
            t2 = t2 + pot[gc] * hprime[j][k];
            bt2 = bt2 + b[gc] * hprime[j][k];
          }
          const size_t p = off + j * NGLL + i;
          const double xixl = xix[p], xizl = xiz[p], gammaxl = gammax[p], gammazl = gammaz[p];
          const real ax = static_cast<real>(t1 * xixl + t2 * gammaxl);
          const real az = static_cast<real>(t1 * xizl + t2 * gammazl);
          const real bx = static_cast<real>(bt1 * xixl + bt2 * gammaxl);
          const real bz = static_cast<real>(bt1 * xizl + bt2 * gammazl);
          const int g = d.ibool[p];
          const real dotp = ax * bx + az * bz;
          rho_ac_kl[p] = rho_ac_kl[p] + real(1) / rho[p] * dotp * deltat;
          kappa_ac_kl[p] = kappa_ac_kl[p] + real(1) / kappa[p] * pot_dd[g] * b[g] * deltat;
        }
    }
    });
    return 0;
  }
  void set_step(int step) override { it = step; }
  int accumulate(const void *b) override {
    if (!b) return -1;
    accumulate_kernels(static_cast<const real *>(b));
    return 0;
  }

  std::vector<real> *field(int which) {
    switch (which) {
      case SF2D_OR_DISPL: return &displ;
      case SF2D_OR_VELOC: return &veloc;
      case SF2D_OR_ACCEL: return &accel;
      case SF2D_OR_DISPL_LDDRK: return &displ_l;
      case SF2D_OR_VELOC_LDDRK: return &veloc_l;
      case SF2D_OR_E1: return &e1;
      case SF2D_OR_E11: return &e11;
      case SF2D_OR_E13: return &e13;
      case SF2D_OR_ATT_OLD: return &att_old;
      case SF2D_OR_RHO_KL: return &rho_kl;
      case SF2D_OR_KAPPA_KL: return &kappa_kl;
      case SF2D_OR_MU_KL: return &mu_kl;
      case SF2D_OR_HESS1: return &hess1;
      case SF2D_OR_HESS2: return &hess2;
      case SF2D_OR_RHO_AC_KL: return &rho_ac_kl;
      case SF2D_OR_KAPPA_AC_KL: return &kappa_ac_kl;
      case SF2D_OR_POT: return &pot;
      case SF2D_OR_POT_DOT: return &pot_d;
      case SF2D_OR_POT_DOT_DOT: return &pot_dd;
      case SF2D_OR_POT_LDDRK: return &pot_l;
      case SF2D_OR_POT_DOT_LDDRK: return &pot_d_l;
      default: return nullptr;
    }
  }
  int get(int which, void *out) override {
    auto *f = field(which);
    if (!f || !out) return -1;
    std::memcpy(out, f->data(), f->size() * sizeof(real));
    return 0;
  }
  int set(int which, const void *in) override {
    auto *f = field(which);
    if (!f || !in) return -1;
    std::memcpy(f->data(), in, f->size() * sizeof(real));
    return 0;
  }
};

}  // namespace

extern "C" void *sf2d_oracle_create(const sf2d_oracle_db *db, int precision) {
  if (!db || db->nspec <= 0 || db->nglob <= 0 || !db->ibool) return nullptr;
  if (db->time_scheme != 1 && db->time_scheme != 2) return nullptr;
  if (db->time_scheme == 2 && (!db->alpha_lddrk || !db->beta_lddrk)) return nullptr;
  if (db->ispec_is_acoustic && (!db->kappastore || !db->rmass_inverse_acoustic)) return nullptr;
  // adjoint runs with fluid elements are restated for Newmark
  if (db->ispec_is_acoustic && db->adj_src && db->time_scheme != 1) return nullptr;
  if (db->pml_region) {
    // CPML is restated for isotropic elements of a forward run
    if (!db->pml_K_x || !db->pml_K_z || !db->pml_d_x || !db->pml_d_z || !db->pml_alpha_x || !db->pml_alpha_z ||
        db->adj_src || db->DT <= 0.0)
      return nullptr;
    // CPML in attenuating solids: Newmark only, as the reference
    // (pml_compute_memory_variables.f90:736-741)
    if (db->pml_visco && (db->time_scheme != 1 || !db->att_itau1 || !db->att_itau2 || !db->att_phi1 ||
                          !db->att_phi2 || !db->att_teps1 || !db->att_teps2 || !db->att_mu1 || !db->att_mu2))
      return nullptr;
    for (int e = 0; e < db->nspec; ++e) {
      if (db->pml_region[e] <= 0) continue;
      if (db->ispec_is_anisotropic && db->ispec_is_anisotropic[e]) return nullptr;
    }
    if (db->ispec_is_acoustic && (!db->cpl_ac_elpt || !db->cpl_el_acpt)) return nullptr;
  }
  if (db->seismotype < 1 || db->seismotype > 6 || db->seismotype == 5) return nullptr;
  if (db->seismotype == 4 && db->nrec > 0) {
    // pressure is recorded in acoustic elements only
    if (!db->ispec_is_acoustic) return nullptr;
    for (int r = 0; r < db->nrec; ++r)
      if (!db->ispec_is_acoustic[db->rec_ispec[r]]) return nullptr;
  }
  if (precision == 4) return static_cast<StateBase *>(new State<float>(db));
  if (precision == 8) return static_cast<StateBase *>(new State<double>(db));
  return nullptr;
}

extern "C" int sf2d_oracle_run(void *h, int nstep, double *seis, int nthreads) {
  if (!h || nstep < 0) return -1;
  return static_cast<StateBase *>(h)->run(nstep, seis, nthreads);
}

extern "C" int sf2d_oracle_get(void *h, int which, void *out) {
  return h ? static_cast<StateBase *>(h)->get(which, out) : -1;
}

extern "C" int sf2d_oracle_set(void *h, int which, const void *in) {
  return h ? static_cast<StateBase *>(h)->set(which, in) : -1;
}

extern "C" int sf2d_oracle_accumulate_kernels(void *h, const void *b_displ) {
  return h ? static_cast<StateBase *>(h)->accumulate(b_displ) : -1;
}

// smooth_sem.F90:63-467, the CPU branch: for every global point (done once,
// by the first element holding it, as imask does), over every element ispec2
// in order: exp_val = exp(-sigma_h2_inv dist_h - sigma_v2_inv dist_v) (CUSTOM_REAL),
// times jacobian * wgll_sq, summed over the 25 points with i fastest (Fortran's
// sum) and added to tk and bk; finally tk / bk at every element point.  Target
// elements run in parallel: a point belongs to exactly one of them.
extern "C" int sf2d_oracle_smooth(int nspec, int nglob, const int *ibool, const float *x, const float *z,
                                  const float *jacobian, const float *wgll_sq, int nfields, const float *fields,
                                  float sigma_h, float sigma_v, float *out) {
  if (nspec < 1 || nglob < 1 || !ibool || !x || !z || !jacobian || !wgll_sq || nfields < 1 || !fields || !out)
    return -1;
  const float sigma_h2_inv = 1.0f / (2.0f * (sigma_h * sigma_h));
  const float sigma_v2_inv = 1.0f / (2.0f * (sigma_v * sigma_v));
  const size_t n = static_cast<size_t>(nspec) * NGLL2;
  std::vector<int> first(nglob, -1);
  for (int e = 0; e < nspec; ++e)
    for (int q = 0; q < NGLL2; ++q) {
      const int g = ibool[static_cast<size_t>(e) * NGLL2 + q];
      if (first[g] < 0) first[g] = e;
    }
  std::vector<float> tk(static_cast<size_t>(nglob) * nfields, 0.f), bk(nglob, 0.f);
  parallel_for(nspec, default_threads(), [&](int b, int e1) {
    float exp_val[NGLL2];
    for (int ispec = b; ispec < e1; ++ispec)
      for (int ispec2 = 0; ispec2 < nspec; ++ispec2) {
        const size_t o2 = static_cast<size_t>(ispec2) * NGLL2;
        for (int j = 0; j < NGLL; ++j)
          for (int i = 0; i < NGLL; ++i) {
            const size_t p = static_cast<size_t>(ispec) * NGLL2 + j * NGLL + i;
            const int g = ibool[p];
            if (first[g] != ispec) continue;
            const float x0 = x[p], z0 = z[p];
            for (int q = 0; q < NGLL2; ++q) {
              const float dh = (x0 - x[o2 + q]) * (x0 - x[o2 + q]);
              const float dv = (z0 - z[o2 + q]) * (z0 - z[o2 + q]);
              exp_val[q] = std::exp(-sigma_h2_inv * dh - sigma_v2_inv * dv);
              exp_val[q] = exp_val[q] * (jacobian[o2 + q] * wgll_sq[q]);
            }
            for (int k = 0; k < nfields; ++k) {
              float sum = 0.f;
              for (int q = 0; q < NGLL2; ++q) sum = sum + exp_val[q] * fields[static_cast<size_t>(k) * n + o2 + q];
              tk[static_cast<size_t>(g) * nfields + k] = tk[static_cast<size_t>(g) * nfields + k] + sum;
            }
            float sum = 0.f;
            for (int q = 0; q < NGLL2; ++q) sum = sum + exp_val[q];
            bk[g] = bk[g] + sum;
          }
      }
  });
  for (size_t p = 0; p < n; ++p) {
    const int g = ibool[p];
    for (int k = 0; k < nfields; ++k) out[static_cast<size_t>(k) * n + p] = tk[static_cast<size_t>(g) * nfields + k] / bk[g];
  }
  return 0;
}

extern "C" int sf2d_oracle_accumulate_kernels_acoustic(void *h, const void *b_pot) {
  return h ? static_cast<StateBase *>(h)->accumulate_acoustic(b_pot) : -1;
}

extern "C" int sf2d_oracle_accumulate_hessian(void *h, const void *b_accel) {
  return h ? static_cast<StateBase *>(h)->accumulate_hessian(b_accel) : -1;
}

extern "C" int sf2d_oracle_set_step(void *h, int it) {
  if (!h || it < 0) return -1;
  static_cast<StateBase *>(h)->set_step(it);
  return 0;
}

extern "C" void sf2d_oracle_destroy(void *h) { delete static_cast<StateBase *>(h); }

extern "C" int sf2d_oracle_max_threads(void) { return default_threads(); }
