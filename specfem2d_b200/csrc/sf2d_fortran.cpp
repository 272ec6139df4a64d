// The reference's Fortran-to-GPU entry points (include/sf2d_fortran.h) over
// this library's fused solvers.  The SPECFEM2D Fortran host (prepare_gpu.f90,
// compute_gpu_acoustic.f90, compute_gpu_elastic.f90,
// update_displacement_Newmark.F90, write_seismograms.F90, check_stability.F90)
// calls them with its own arrays; they gather what sf2d_elastic_create (a
// solid mesh) or sf2d_coupled_create (a mesh with fluid elements: solid and
// fluid sub-meshes with their own point numberings) needs, build the solver
// when the time step is first known (the first update_displacement_*_cuda)
// and advance one fused step per kernel_3_a_cuda (kernel_3_acoustic_cuda on a
// fluid-only mesh).  Errors print and exit, as the reference's exit_on_error
// (src/gpu/helper_functions.cu) does.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sf2d_b200.h"
#include "sf2d_coupled.h"
#include "sf2d_fortran.h"

namespace {

constexpr int NGLL = 5, NGLL2 = 25;

[[noreturn]] void stop(const char *routine, const std::string &msg) {
  std::fprintf(stderr, "Error in %s: %s\n", routine, msg.c_str());
  std::fflush(stderr);
  std::exit(EXIT_FAILURE);
}

void check(const char *routine, int rc) {
  if (rc != SF2D_OK) stop(routine, sf2d_last_error());
}

enum Why { PML, KERNEL_RUN, MPI, DEBUG, OTHER };

[[noreturn]] void unsupported(const char *routine, Why why) {
  static const char *const text[] = {
      "CPML layers run through sf2d_elastic_create / sf2d_coupled_create with the descriptors' pml_* members "
      "(include/sf2d_b200.h, include/sf2d_coupled.h)",
      "kernel runs replay the forward field from checkpoints instead of reconstructing it backwards: "
      "SIMULATION_TYPE = 3 of solid meshes runs through this interface, the rest through sf2d_fwi_create / "
      "sf2d_coupled_fwi_create (include/sf2d_b200.h, include/sf2d_coupled.h)",
      "this library runs one mesh per process: there is no MPI halo exchange",
      "debug helper not provided by libsf2d_b200",
      "not provided by libsf2d_b200"};
  stop(routine, text[why]);
}

// Everything one Mesh_pointer holds: the host copies the descriptor points
// into, the solver once built, and the step bookkeeping.
struct FortranMesh {
  sf2d_elastic_desc d{};
  int nspec = 0, nglob = 0, nstep = 0, nlength = 0, nrec = 0, nsrc = 0;
  bool stacey = false, save_forward = false, have_rmass = false, have_stacey = false;
  std::vector<int> ibool, src_ispec, rec_ispec, st_iglob, aniso_flag;
  std::vector<float> xix, xiz, gammax, gammaz, lambda, mu, hprime, hprimewgll, wxgll, srcarr, stf, rmass;
  std::vector<float> st_nx, st_nz, st_w, st_rvp, st_rvs;
  std::vector<float> c11, c13, c15, c33, c35, c55, a1, b1, a2, b2;
  std::vector<double> hxir, hgammar, centroid;
  sf2d_solver *S = nullptr;
  float dt = 0.f, dtover2 = 0.f, dtsq2 = 0.f;
  int steps = 0;  // steps advanced (the Fortran `it` of the last finished step)
  int stage = 0;  // 0 between steps, 1 after update_displacement_cuda, 2 after the outer forces phase
  std::vector<float> staged_u, staged_v, staged_a;  // fields given before the solver exists
  std::vector<int> sample_step;                     // step of each sample in the host's trace buffer
  // fluid elements (prepare_fields_acoustic_device): the run goes through the coupled solver
  bool fluid = false, have_fluid = false;
  int nspec_acoustic = 0;
  std::vector<unsigned char> is_ac;                 // per element: mustore zero (ispec_is_acoustic)
  std::vector<float> rmass_ac, rho, kappa;          // nglob; nspec*25; nspec*25
  std::vector<int> free_iglob;                      // points of the free-surface faces
  std::vector<int> cpl_iglob;                       // one entry per coupling-face point
  std::vector<float> cpl_nx, cpl_nz, cpl_w;
  std::vector<int> st_ac_iglob;                     // fluid absorbing points
  std::vector<float> st_ac_w, st_ac_rvp;
  sf2d_coupled *C = nullptr;
  std::vector<float> staged_p, staged_pd, staged_pdd;
  // step bookkeeping of a coupled mesh: 0 between steps, 1 fluid predicted,
  // 2 solid predicted, 3 fluid forces, 4 fluid step done, 5 solid forces
  int ac_phase = 0;
  // kernel run (SIMULATION_TYPE = 3, solid meshes): the checkpointed gradient
  // (forward replay and adjoint sweep) runs in full when the first step
  // starts; the calls of each step then follow it and hand out its results
  int sim_type = 1;
  bool adj_prepared = false;
  int nspec_side[4] = {0, 0, 0, 0};  // absorbing faces bottom, left, right, top
  sf2d_fwi *F = nullptr;
  std::vector<float> adj_src;        // [irec][it][comp], forward time order
  std::vector<double> adj_seis;      // adjoint traces [irec][it][comp]
  std::vector<float> rho_sum, kappa_sum, mu_sum;
  int kernel_calls = 0;              // compute_kernels_elastic_cuda calls
  int srcs_added = 0;                // step of the last compute_add_sources_*_s3_cuda
  // with fluid elements: the coupled gradient run; C then points at its adjoint
  // run (owned by CF) for the field and norm queries
  sf2d_coupled_fwi *CF = nullptr;
  bool kr_open = false;              // a time step of the kernel run is open
  bool ac_adj_prepared = false;
  int ac_kernel_calls = 0;           // compute_kernels_acoustic_cuda calls
  std::vector<int> s_elems, f_elems;  // whole-mesh element of each solid / fluid sub-mesh element
  std::vector<float> rho_ac_kl, kappa_ac_kl;  // whole-mesh element order, zero in solid elements
  // CPML layer of a fluid-only mesh (prepare_pml_device): region per element,
  // K, d, alpha per element point, the layer's outer-edge points
  bool pml = false, have_pml = false;
  std::vector<int> pml_region, pml_edge;
  std::vector<double> pml_K_x, pml_K_z, pml_d_x, pml_d_z, pml_alpha_x, pml_alpha_z;
  double pml_dt = 0.0;
  // USE_TRICK_FOR_BETTER_PRESSURE reaches the library only with the first
  // compute_seismograms_cuda, after the first step; the initial fields are kept
  // until then so that a pressure run can be rebuilt with it and step 1 repeated
  int use_trick = 0;
  bool trick_checked = false;
  std::vector<float> init_fields[6];
};

FortranMesh *mesh_of(const char *routine, const long *p) {
  if (!p || *p == 0) stop(routine, "Mesh_pointer was not prepared by prepare_constants_device");
  return reinterpret_cast<FortranMesh *>(*p);
}

// Column-major (n1, n2) -> row-major [i1][i2]: the transpose of the memory order.
template <typename T, typename U>
std::vector<T> transpose(const U *a, int n1, int n2) {
  std::vector<T> out(static_cast<size_t>(n1) * n2);
  for (int i2 = 0; i2 < n2; ++i2)
    for (int i1 = 0; i1 < n1; ++i1) out[static_cast<size_t>(i1) * n2 + i2] = static_cast<T>(a[static_cast<size_t>(i2) * n1 + i1]);
  return out;
}

// Element centres for the tiler's Morton order.  The reference hands the GPU
// no coordinates, so they are rebuilt from the mapping derivatives: x_xi =
// gammaz J, z_xi = -gammax J, x_gamma = -xiz J, z_gamma = xix J with J =
// 1/(xix gammaz - xiz gammax), integrated along GLL lines through the
// Lagrange interpolant of the derivative (exact for the 4- and 9-node
// mappings), and elements placed next to their already placed neighbours
// through shared points.  Only tile shapes depend on them.
void rebuild_centroids(FortranMesh &m) {
  const double s37 = std::sqrt(3.0 / 7.0);
  const double xi[NGLL] = {-1.0, -s37, 0.0, s37, 1.0};
  // W[i][k] = integral from -1 to xi_i of the k-th Lagrange polynomial
  double W[NGLL][NGLL];
  for (int k = 0; k < NGLL; ++k) {
    // coefficients of l_k by expanding the product, lowest degree first
    double c[NGLL] = {1.0, 0, 0, 0, 0};
    double den = 1.0;
    int deg = 0;
    for (int q = 0; q < NGLL; ++q) {
      if (q == k) continue;
      for (int p = deg + 1; p > 0; --p) c[p] = c[p - 1] - xi[q] * c[p];
      c[0] = -xi[q] * c[0];
      ++deg;
      den *= xi[k] - xi[q];
    }
    for (int i = 0; i < NGLL; ++i) {
      double a = 0.0, b = 0.0;
      for (int p = 0; p < NGLL; ++p) {
        a += c[p] / (p + 1) * std::pow(xi[i], p + 1);
        b += c[p] / (p + 1) * std::pow(-1.0, p + 1);
      }
      W[i][k] = (a - b) / den;
    }
  }
  const int ne = m.nspec;
  std::vector<double> lx(static_cast<size_t>(ne) * NGLL2), lz(lx.size());
  for (int e = 0; e < ne; ++e) {
    double xx[NGLL2], zx[NGLL2], xg[NGLL2], zg[NGLL2];
    for (int q = 0; q < NGLL2; ++q) {
      const size_t p = static_cast<size_t>(e) * NGLL2 + q;
      const double det = static_cast<double>(m.xix[p]) * m.gammaz[p] - static_cast<double>(m.xiz[p]) * m.gammax[p];
      const double J = det != 0.0 ? 1.0 / det : 0.0;
      xx[q] = m.gammaz[p] * J;
      zx[q] = -m.gammax[p] * J;
      xg[q] = -m.xiz[p] * J;
      zg[q] = m.xix[p] * J;
    }
    // along gamma on the first column, then along xi on every row
    double cx[NGLL], cz[NGLL];
    for (int j = 0; j < NGLL; ++j) {
      cx[j] = cz[j] = 0.0;
      for (int k = 0; k < NGLL; ++k) {
        cx[j] += W[j][k] * xg[k * NGLL];
        cz[j] += W[j][k] * zg[k * NGLL];
      }
    }
    for (int j = 0; j < NGLL; ++j)
      for (int i = 0; i < NGLL; ++i) {
        double x = cx[j], z = cz[j];
        for (int k = 0; k < NGLL; ++k) {
          x += W[i][k] * xx[j * NGLL + k];
          z += W[i][k] * zx[j * NGLL + k];
        }
        lx[static_cast<size_t>(e) * NGLL2 + j * NGLL + i] = x;
        lz[static_cast<size_t>(e) * NGLL2 + j * NGLL + i] = z;
      }
  }
  // place elements breadth first through shared points
  std::vector<std::vector<int>> elems_of(m.nglob);
  for (int e = 0; e < ne; ++e)
    for (int q = 0; q < NGLL2; ++q) elems_of[m.ibool[static_cast<size_t>(e) * NGLL2 + q]].push_back(e);
  std::vector<double> gx(m.nglob, 0.0), gz(m.nglob, 0.0);
  std::vector<char> known(m.nglob, 0), placed(ne, 0);
  std::vector<int> queue;
  double shift = 0.0;
  for (int seed = 0; seed < ne; ++seed) {
    if (placed[seed]) continue;
    // a new connected part: put it to the right of the previous ones
    queue.assign(1, seed);
    placed[seed] = 1;
    for (size_t h = 0; h < queue.size(); ++h) {
      const int e = queue[h];
      const size_t o = static_cast<size_t>(e) * NGLL2;
      double ox = shift, oz = 0.0;
      for (int q = 0; q < NGLL2; ++q) {
        const int g = m.ibool[o + q];
        if (known[g]) {
          ox = gx[g] - lx[o + q];
          oz = gz[g] - lz[o + q];
          break;
        }
      }
      double cxs = 0.0, czs = 0.0;
      for (int q = 0; q < NGLL2; ++q) {
        const int g = m.ibool[o + q];
        if (!known[g]) {
          gx[g] = lx[o + q] + ox;
          gz[g] = lz[o + q] + oz;
          known[g] = 1;
        }
        cxs += lx[o + q] + ox;
        czs += lz[o + q] + oz;
        for (int nb : elems_of[g])
          if (!placed[nb]) {
            placed[nb] = 1;
            queue.push_back(nb);
          }
      }
      m.centroid[2 * e] = cxs / NGLL2;
      m.centroid[2 * e + 1] = czs / NGLL2;
    }
    double xmax = shift;
    for (int e : queue) xmax = std::max(xmax, m.centroid[2 * e]);
    shift = xmax + 1.0e6;
  }
}

void build_coupled(const char *routine, FortranMesh &m);

void run_kernel_sweep(const char *routine, FortranMesh &m);

void build_solver(const char *routine, FortranMesh &m) {
  if (m.S || m.C || m.F || m.CF) return;
  if (m.fluid) {
    build_coupled(routine, m);
    return;
  }
  if (!m.have_rmass) stop(routine, "prepare_fields_elastic_device has not been called");
  if (m.stacey && !m.have_stacey) stop(routine, "prepare_stacey_device has not been called");
  sf2d_elastic_desc &d = m.d;
  d.nspec = m.nspec;
  d.nglob = m.nglob;
  d.ibool = m.ibool.data();
  d.xix = m.xix.data();
  d.xiz = m.xiz.data();
  d.gammax = m.gammax.data();
  d.gammaz = m.gammaz.data();
  d.lambdastore = m.lambda.data();
  d.mustore = m.mu.data();
  d.rmass_inverse = m.rmass.data();
  d.hprime = m.hprime.data();
  d.hprimewgll = m.hprimewgll.data();
  d.wxgll = d.wzgll = m.wxgll.data();
  d.centroid_xz = m.centroid.data();
  d.nstacey = static_cast<int>(m.st_iglob.size());
  d.st_iglob = m.st_iglob.data();
  d.st_nx = m.st_nx.data();
  d.st_nz = m.st_nz.data();
  d.st_w = m.st_w.data();
  d.st_rho_vp = m.st_rvp.data();
  d.st_rho_vs = m.st_rvs.data();
  d.nsrc = m.nsrc;
  d.src_ispec = m.src_ispec.data();
  d.sourcearrays = m.srcarr.data();
  d.stf = m.stf.data();
  d.nrec = m.nrec;
  d.rec_ispec = m.rec_ispec.data();
  d.hxir = m.hxir.data();
  d.hgammar = m.hgammar.data();
  d.nstep = m.nstep;
  d.deltat = m.dt;
  d.deltatover2 = m.dtover2;
  d.deltatsquareover2 = m.dtsq2;
  d.tile_elems = 32;
  d.threads_per_block = 256;
  d.time_scheme = 1;
  d.nstage = 1;
  if (!m.aniso_flag.empty()) {
    d.ispec_is_anisotropic = m.aniso_flag.data();
    d.c11 = m.c11.data();
    d.c13 = m.c13.data();
    d.c15 = m.c15.data();
    d.c33 = m.c33.data();
    d.c35 = m.c35.data();
    d.c55 = m.c55.data();
  }
  if (!m.a1.empty()) {
    d.att_a1 = m.a1.data();
    d.att_b1 = m.b1.data();
    d.att_a2 = m.a2.data();
    d.att_b2 = m.b2.data();
  }
  if (m.sim_type == 3) {
    run_kernel_sweep(routine, m);
    return;
  }
  check(routine, sf2d_elastic_create(&d, &m.S));
  if (!m.staged_u.empty()) {
    check(routine, sf2d_set_fields(m.S, m.staged_u.data(), m.staged_v.data(), m.staged_a.data()));
    m.staged_u.clear();
    m.staged_v.clear();
    m.staged_a.clear();
  }
}

// A kernel run in full (iterate_time.F90:146-400 with SIMULATION_TYPE = 3):
// the forward field from rest with a checkpoint every min(NSTEP, 200) steps,
// then the adjoint sweep, which injects source_adjoint(:, NSTEP-it+1) at step
// it (compute_gpu_elastic.f90:283-311), replays each forward segment from its
// checkpoint instead of reconstructing it backwards from the last frame and
// the absorbed-boundary records, and sums the kernel integrands at every step
// (compute_kernels_cudakernel, NTSTEP_BETWEEN_COMPUTE_KERNELS = 1).
void run_kernel_sweep(const char *routine, FortranMesh &m) {
  if (!m.adj_prepared) stop(routine, "prepare_fields_elastic_adj_dev has not been called");
  if (m.nrec > 0 && m.adj_src.empty()) stop(routine, "prepare_sim2_or_3_const_device has not been called");
  for (const std::vector<float> *f : {&m.staged_u, &m.staged_v, &m.staged_a})
    for (float x : *f)
      if (x != 0.f) stop(routine, "a kernel run starts from rest: the initial fields must be zero");
  m.staged_u.clear();
  m.staged_v.clear();
  m.staged_a.clear();
  const size_t nl = static_cast<size_t>(m.nspec) * NGLL2;
  // rhostore/kappastore scale the kernels of sf2d_fwi_backward only; the host
  // receives the unscaled sums and scales them itself (save_adjoint_kernels.f90)
  const std::vector<float> ones(nl, 1.f);
  check(routine, sf2d_fwi_create(&m.d, ones.data(), ones.data(), std::min(m.nstep, 200), &m.F));
  int rc = sf2d_fwi_forward(m.F, nullptr);
  if (rc == SF2D_ERR_UNSTABLE) stop(routine, "the forward wavefield of the kernel run became unstable and blew up");
  check(routine, rc);
  const float none = 0.f;
  std::vector<float> rk(nl), kk(nl), mk(nl);
  rc = sf2d_fwi_backward(m.F, m.adj_src.empty() ? &none : m.adj_src.data(), rk.data(), kk.data(), mk.data());
  if (rc == SF2D_ERR_UNSTABLE) stop(routine, "the adjoint wavefield became unstable and blew up");
  check(routine, rc);
  m.adj_seis.assign(static_cast<size_t>(m.nrec) * m.nstep * 2, 0.0);
  if (m.nrec) check(routine, sf2d_fwi_adjoint_seismograms(m.F, m.adj_seis.data()));
  m.rho_sum.resize(nl);
  m.kappa_sum.resize(nl);
  m.mu_sum.resize(nl);
  check(routine, sf2d_fwi_kernel_sums(m.F, m.rho_sum.data(), m.kappa_sum.data(), m.mu_sum.data()));
}

// The elements of one domain with a compact numbering of their points
// (ascending global id), as the coupled solver takes each sub-mesh.
struct SubMesh {
  std::vector<int> elems, pts, gmap, ibool;  // gmap: global point -> local, -1 outside
};

SubMesh submesh(const FortranMesh &m, bool fluid) {
  SubMesh s;
  s.gmap.assign(m.nglob, -1);
  for (int e = 0; e < m.nspec; ++e)
    if ((m.is_ac[e] != 0) == fluid) s.elems.push_back(e);
  std::vector<char> used(m.nglob, 0);
  for (int e : s.elems)
    for (int q = 0; q < NGLL2; ++q) used[m.ibool[static_cast<size_t>(e) * NGLL2 + q]] = 1;
  for (int g = 0; g < m.nglob; ++g)
    if (used[g]) {
      s.gmap[g] = static_cast<int>(s.pts.size());
      s.pts.push_back(g);
    }
  s.ibool.resize(s.elems.size() * NGLL2);
  for (size_t k = 0; k < s.elems.size(); ++k)
    for (int q = 0; q < NGLL2; ++q)
      s.ibool[k * NGLL2 + q] = s.gmap[m.ibool[static_cast<size_t>(s.elems[k]) * NGLL2 + q]];
  return s;
}

template <typename T>
std::vector<T> elem_rows(const std::vector<T> &a, const std::vector<int> &elems, size_t per) {
  std::vector<T> out(elems.size() * per);
  for (size_t k = 0; k < elems.size(); ++k)
    std::copy(a.begin() + static_cast<size_t>(elems[k]) * per, a.begin() + static_cast<size_t>(elems[k] + 1) * per,
              out.begin() + k * per);
  return out;
}

// The coupled solver of a mesh with fluid elements: the solid and fluid
// sub-meshes, the coupling faces of prepare_fields_acoustic_device for both
// directions (the reference's GPU kernels use the fluid element's normals and
// weights for both, compute_coupling_*_kernel.cu), sources and receivers split
// by the domain of their element.
// The kernel run of a mesh with fluid elements (iterate_time.F90:146-400 with
// SIMULATION_TYPE = 3: compute_gpu_elastic.f90 and compute_gpu_acoustic.f90
// with compute_wavefield_1 and _2): the forward field from rest with
// checkpoints, then the adjoint sweep that replays it, at the first step.
// The kernels are summed at every step (NTSTEP_BETWEEN_COMPUTE_KERNELS = 1).
void run_coupled_kernel_sweep(const char *routine, FortranMesh &m, const sf2d_elastic_desc &d,
                              const sf2d_acoustic_desc &a, const sf2d_coupling_desc &c) {
  const bool solid = d.nspec > 0;
  if (!m.ac_adj_prepared || (solid && !m.adj_prepared))
    stop(routine, "prepare_fields_acoustic_adj_dev / prepare_fields_elastic_adj_dev has not been called");
  if (m.nrec > 0 && m.adj_src.empty()) stop(routine, "prepare_sim2_or_3_const_device has not been called");
  for (const std::vector<float> *f : {&m.staged_u, &m.staged_v, &m.staged_a, &m.staged_p, &m.staged_pd,
                                      &m.staged_pdd})
    for (float x : *f)
      if (x != 0.f) stop(routine, "a kernel run starts from rest: the initial fields must be zero");
  for (std::vector<float> *f : {&m.staged_u, &m.staged_v, &m.staged_a, &m.staged_p, &m.staged_pd, &m.staged_pdd})
    f->clear();
  const size_t nls = static_cast<size_t>(d.nspec) * NGLL2, nlf = static_cast<size_t>(a.nspec) * NGLL2;
  // solid rhostore/kappastore scale sf2d_coupled_fwi_backward's kernels only; the
  // host receives the unscaled sums and scales them itself
  const std::vector<float> ones(std::max<size_t>(nls, 1), 1.f);
  check(routine, sf2d_coupled_fwi_create(&d, &a, &c, solid ? ones.data() : nullptr, solid ? ones.data() : nullptr,
                                         std::min(m.nstep, 200), &m.CF));
  int rc = sf2d_coupled_fwi_forward(m.CF, nullptr);
  if (rc == SF2D_ERR_UNSTABLE) stop(routine, "the forward wavefield of the kernel run became unstable and blew up");
  check(routine, rc);
  const float none = 0.f;
  std::vector<float> rk(std::max<size_t>(nls, 1)), kk(rk.size()), mk(rk.size()), rac(std::max<size_t>(nlf, 1)),
      kac(rac.size());
  rc = sf2d_coupled_fwi_backward(m.CF, m.adj_src.empty() ? &none : m.adj_src.data(), solid ? rk.data() : nullptr,
                                 solid ? kk.data() : nullptr, solid ? mk.data() : nullptr, rac.data(), kac.data());
  if (rc == SF2D_ERR_UNSTABLE) stop(routine, "the adjoint wavefield became unstable and blew up");
  check(routine, rc);
  m.adj_seis.assign(static_cast<size_t>(m.nrec) * m.nstep * 2, 0.0);
  if (m.nrec) check(routine, sf2d_coupled_fwi_adjoint_seismograms(m.CF, m.adj_seis.data()));
  // kernels to the whole mesh's element order, zero in the other domain (the
  // reference's kernel arrays span NSPEC_AB)
  const size_t nl = static_cast<size_t>(m.nspec) * NGLL2;
  m.rho_ac_kl.assign(nl, 0.f);
  m.kappa_ac_kl.assign(nl, 0.f);
  for (size_t k = 0; k < m.f_elems.size(); ++k)
    for (int q = 0; q < NGLL2; ++q) {
      m.rho_ac_kl[static_cast<size_t>(m.f_elems[k]) * NGLL2 + q] = rac[k * NGLL2 + q];
      m.kappa_ac_kl[static_cast<size_t>(m.f_elems[k]) * NGLL2 + q] = kac[k * NGLL2 + q];
    }
  m.rho_sum.assign(nl, 0.f);
  m.kappa_sum.assign(nl, 0.f);
  m.mu_sum.assign(nl, 0.f);
  if (solid) {
    check(routine, sf2d_coupled_fwi_kernel_sums(m.CF, rk.data(), kk.data(), mk.data()));
    for (size_t k = 0; k < m.s_elems.size(); ++k)
      for (int q = 0; q < NGLL2; ++q) {
        const size_t p = static_cast<size_t>(m.s_elems[k]) * NGLL2 + q;
        m.rho_sum[p] = rk[k * NGLL2 + q];
        m.kappa_sum[p] = kk[k * NGLL2 + q];
        m.mu_sum[p] = mk[k * NGLL2 + q];
      }
  }
  check(routine, sf2d_coupled_fwi_adjoint_run(m.CF, &m.C));
}

void build_coupled(const char *routine, FortranMesh &m) {
  if (!m.have_fluid) stop(routine, "prepare_fields_acoustic_device has not been called");
  if (m.stacey && !m.have_stacey) stop(routine, "prepare_stacey_device has not been called");
  const SubMesh S = submesh(m, false), F = submesh(m, true);
  const bool solid = !S.elems.empty();
  if (solid && !m.have_rmass) stop(routine, "prepare_fields_elastic_device has not been called");
  // --- solid description (time stepping and GLL arrays only on a fluid-only mesh)
  sf2d_elastic_desc d{};
  d.hprime = m.hprime.data();
  d.hprimewgll = m.hprimewgll.data();
  d.wxgll = d.wzgll = m.wxgll.data();
  d.nstep = m.nstep;
  d.deltat = m.dt;
  d.deltatover2 = m.dtover2;
  d.deltatsquareover2 = m.dtsq2;
  d.tile_elems = 32;
  d.threads_per_block = 256;
  d.time_scheme = 1;
  d.nstage = 1;
  d.seismotype = m.d.seismotype;
  std::vector<float> s_xix, s_xiz, s_gx, s_gz, s_lambda, s_mu, s_rmass, s_srcarr, s_stf, s_st_nx, s_st_nz, s_st_w,
      s_st_rvp, s_st_rvs, s_c[6], s_a[4];
  std::vector<int> s_st_iglob, s_src, s_rec, s_rec_global, s_aniso;
  std::vector<double> s_hxir, s_hgammar, s_cent;
  std::vector<int> s_elem_of(m.nspec, -1), f_elem_of(m.nspec, -1);
  for (size_t k = 0; k < S.elems.size(); ++k) s_elem_of[S.elems[k]] = static_cast<int>(k);
  for (size_t k = 0; k < F.elems.size(); ++k) f_elem_of[F.elems[k]] = static_cast<int>(k);
  if (solid) {
    s_xix = elem_rows(m.xix, S.elems, NGLL2);
    s_xiz = elem_rows(m.xiz, S.elems, NGLL2);
    s_gx = elem_rows(m.gammax, S.elems, NGLL2);
    s_gz = elem_rows(m.gammaz, S.elems, NGLL2);
    s_lambda = elem_rows(m.lambda, S.elems, NGLL2);
    s_mu = elem_rows(m.mu, S.elems, NGLL2);
    s_cent = elem_rows(m.centroid, S.elems, 2);
    s_rmass.resize(2 * S.pts.size());
    for (size_t k = 0; k < S.pts.size(); ++k) {
      s_rmass[2 * k] = m.rmass[2 * static_cast<size_t>(S.pts[k])];
      s_rmass[2 * k + 1] = m.rmass[2 * static_cast<size_t>(S.pts[k]) + 1];
    }
    for (size_t k = 0; k < m.st_iglob.size(); ++k) {
      const int l = S.gmap[m.st_iglob[k]];
      if (l < 0) stop(routine, "a solid absorbing point outside the solid elements");
      s_st_iglob.push_back(l);
      s_st_nx.push_back(m.st_nx[k]);
      s_st_nz.push_back(m.st_nz[k]);
      s_st_w.push_back(m.st_w[k]);
      s_st_rvp.push_back(m.st_rvp[k]);
      s_st_rvs.push_back(m.st_rvs[k]);
    }
    for (int k = 0; k < m.nsrc; ++k) {
      if (m.is_ac[m.src_ispec[k]]) continue;
      s_src.push_back(s_elem_of[m.src_ispec[k]]);
      s_srcarr.insert(s_srcarr.end(), m.srcarr.begin() + static_cast<size_t>(k) * NGLL2 * 2,
                      m.srcarr.begin() + static_cast<size_t>(k + 1) * NGLL2 * 2);
      s_stf.insert(s_stf.end(), m.stf.begin() + static_cast<size_t>(k) * m.nstep,
                   m.stf.begin() + static_cast<size_t>(k + 1) * m.nstep);
    }
    for (int r = 0; r < m.nrec; ++r) {
      if (m.is_ac[m.rec_ispec[r]]) continue;
      s_rec.push_back(s_elem_of[m.rec_ispec[r]]);
      s_rec_global.push_back(r);
      s_hxir.insert(s_hxir.end(), m.hxir.begin() + r * NGLL, m.hxir.begin() + (r + 1) * NGLL);
      s_hgammar.insert(s_hgammar.end(), m.hgammar.begin() + r * NGLL, m.hgammar.begin() + (r + 1) * NGLL);
    }
    d.nspec = static_cast<int>(S.elems.size());
    d.nglob = static_cast<int>(S.pts.size());
    d.ibool = S.ibool.data();
    d.xix = s_xix.data();
    d.xiz = s_xiz.data();
    d.gammax = s_gx.data();
    d.gammaz = s_gz.data();
    d.lambdastore = s_lambda.data();
    d.mustore = s_mu.data();
    d.rmass_inverse = s_rmass.data();
    d.centroid_xz = s_cent.data();
    d.nstacey = static_cast<int>(s_st_iglob.size());
    d.st_iglob = s_st_iglob.data();
    d.st_nx = s_st_nx.data();
    d.st_nz = s_st_nz.data();
    d.st_w = s_st_w.data();
    d.st_rho_vp = s_st_rvp.data();
    d.st_rho_vs = s_st_rvs.data();
    d.nsrc = static_cast<int>(s_src.size());
    d.src_ispec = s_src.data();
    d.sourcearrays = s_srcarr.data();
    d.stf = s_stf.data();
    d.nrec = static_cast<int>(s_rec.size());
    d.rec_ispec = s_rec.data();
    d.hxir = s_hxir.data();
    d.hgammar = s_hgammar.data();
    d.cosrot = m.d.cosrot;
    d.sinrot = m.d.sinrot;
    if (!m.aniso_flag.empty()) {
      s_aniso = elem_rows(m.aniso_flag, S.elems, 1);
      const std::vector<float> *c[6] = {&m.c11, &m.c13, &m.c15, &m.c33, &m.c35, &m.c55};
      for (int k = 0; k < 6; ++k) s_c[k] = elem_rows(*c[k], S.elems, NGLL2);
      d.ispec_is_anisotropic = s_aniso.data();
      d.c11 = s_c[0].data();
      d.c13 = s_c[1].data();
      d.c15 = s_c[2].data();
      d.c33 = s_c[3].data();
      d.c35 = s_c[4].data();
      d.c55 = s_c[5].data();
    }
    if (!m.a1.empty()) {
      const std::vector<float> *a[4] = {&m.a1, &m.b1, &m.a2, &m.b2};
      for (int k = 0; k < 4; ++k) s_a[k] = elem_rows(*a[k], S.elems, NGLL2 * 3);
      d.att_a1 = s_a[0].data();
      d.att_b1 = s_a[1].data();
      d.att_a2 = s_a[2].data();
      d.att_b2 = s_a[3].data();
    }
  }
  // --- fluid description
  sf2d_acoustic_desc a{};
  const std::vector<float> f_xix = elem_rows(m.xix, F.elems, NGLL2), f_xiz = elem_rows(m.xiz, F.elems, NGLL2),
                           f_gx = elem_rows(m.gammax, F.elems, NGLL2), f_gz = elem_rows(m.gammaz, F.elems, NGLL2),
                           f_rho = elem_rows(m.rho, F.elems, NGLL2), f_kappa = elem_rows(m.kappa, F.elems, NGLL2);
  std::vector<float> f_jac(f_xix.size());
  // the reference's GPU kernels form the Jacobian from the inverse mapping in FP32
  // (Kernel_2_acoustic_impl.cu)
  for (size_t p = 0; p < f_jac.size(); ++p) f_jac[p] = 1.f / (f_xix[p] * f_gz[p] - f_gx[p] * f_xiz[p]);
  const std::vector<double> f_cent = elem_rows(m.centroid, F.elems, 2);
  std::vector<float> f_rmass(F.pts.size()), f_st_w, f_st_rvp, f_srcarr, f_stf;
  for (size_t k = 0; k < F.pts.size(); ++k) f_rmass[k] = m.rmass_ac[F.pts[k]];
  std::vector<int> f_free, f_st, f_src, f_rec, f_rec_global;
  std::vector<double> f_hxir, f_hgammar;
  for (int g : m.free_iglob) {
    const int l = F.gmap[g];
    if (l < 0) stop(routine, "a free-surface point outside the fluid elements");
    f_free.push_back(l);
  }
  for (size_t k = 0; k < m.st_ac_iglob.size(); ++k) {
    const int l = F.gmap[m.st_ac_iglob[k]];
    if (l < 0) stop(routine, "a fluid absorbing point outside the fluid elements");
    f_st.push_back(l);
    f_st_w.push_back(m.st_ac_w[k]);
    f_st_rvp.push_back(m.st_ac_rvp[k]);
  }
  for (int k = 0; k < m.nsrc; ++k) {
    if (!m.is_ac[m.src_ispec[k]]) continue;
    f_src.push_back(f_elem_of[m.src_ispec[k]]);
    // sourcearray(1, i, j): the first component drives the potential
    for (int q = 0; q < NGLL2; ++q) f_srcarr.push_back(m.srcarr[(static_cast<size_t>(k) * NGLL2 + q) * 2]);
    f_stf.insert(f_stf.end(), m.stf.begin() + static_cast<size_t>(k) * m.nstep,
                 m.stf.begin() + static_cast<size_t>(k + 1) * m.nstep);
  }
  for (int r = 0; r < m.nrec; ++r) {
    if (!m.is_ac[m.rec_ispec[r]]) continue;
    f_rec.push_back(f_elem_of[m.rec_ispec[r]]);
    f_rec_global.push_back(r);
    f_hxir.insert(f_hxir.end(), m.hxir.begin() + r * NGLL, m.hxir.begin() + (r + 1) * NGLL);
    f_hgammar.insert(f_hgammar.end(), m.hgammar.begin() + r * NGLL, m.hgammar.begin() + (r + 1) * NGLL);
  }
  a.nspec = static_cast<int>(F.elems.size());
  a.nglob = static_cast<int>(F.pts.size());
  a.ibool = F.ibool.data();
  a.xix = f_xix.data();
  a.xiz = f_xiz.data();
  a.gammax = f_gx.data();
  a.gammaz = f_gz.data();
  a.jacobian = f_jac.data();
  a.rhostore = f_rho.data();
  a.kappastore = f_kappa.data();
  a.rmass_inverse = f_rmass.data();
  a.centroid_xz = f_cent.data();
  a.nfree = static_cast<int>(f_free.size());
  a.free_iglob = f_free.data();
  a.nstacey = static_cast<int>(f_st.size());
  a.st_iglob = f_st.data();
  a.st_w = f_st_w.data();
  a.st_rho_vp = f_st_rvp.data();
  a.nsrc = static_cast<int>(f_src.size());
  a.src_ispec = f_src.data();
  a.sourcearrays = f_srcarr.data();
  a.stf = f_stf.data();
  a.nrec = static_cast<int>(f_rec.size());
  a.rec_ispec = f_rec.data();
  a.hxir = f_hxir.data();
  a.hgammar = f_hgammar.data();
  a.rec_global = f_rec_global.data();
  a.tile_elems = 32;
  std::vector<int> f_pml_region, f_pml_edge;
  std::vector<double> f_pml[6];
  if (m.pml) {
    if (!m.have_pml) stop(routine, "prepare_pml_device has not been called");
    f_pml_region = elem_rows(m.pml_region, F.elems, 1);
    const std::vector<double> *src[6] = {&m.pml_K_x, &m.pml_K_z, &m.pml_d_x, &m.pml_d_z, &m.pml_alpha_x,
                                         &m.pml_alpha_z};
    for (int k = 0; k < 6; ++k) f_pml[k] = elem_rows(*src[k], F.elems, NGLL2);
    for (int g : m.pml_edge) {
      const int l = F.gmap[g];
      if (l < 0) stop(routine, "a CPML edge point outside the fluid elements");
      f_pml_edge.push_back(l);
    }
    a.pml_region = f_pml_region.data();
    a.pml_K_x = f_pml[0].data();
    a.pml_K_z = f_pml[1].data();
    a.pml_d_x = f_pml[2].data();
    a.pml_d_z = f_pml[3].data();
    a.pml_alpha_x = f_pml[4].data();
    a.pml_alpha_z = f_pml[5].data();
    a.npml_edge = static_cast<int>(f_pml_edge.size());
    a.pml_edge_iglob = f_pml_edge.data();
    a.pml_dt = m.pml_dt;
  }
  // --- coupling entries, the same faces for both directions
  sf2d_coupling_desc c{};
  std::vector<int> c_f, c_s;
  for (int g : m.cpl_iglob) {
    if (F.gmap[g] < 0 || S.gmap[g] < 0) stop(routine, "a coupling point not shared by a fluid and a solid element");
    c_f.push_back(F.gmap[g]);
    c_s.push_back(S.gmap[g]);
  }
  c.nrec_total = m.nrec;
  c.el_rec_global = s_rec_global.data();
  c.seismotype = m.d.seismotype;
  c.use_trick = m.use_trick;
  c.cosrot = m.d.cosrot;
  c.sinrot = m.d.sinrot;
  c.ncpl_ac = c.ncpl_el = static_cast<int>(c_f.size());
  c.cpl_ac_point = c_f.data();
  c.cpl_ac_el_point = c_s.data();
  c.cpl_ac_nx = c.cpl_el_nx = m.cpl_nx.data();
  c.cpl_ac_nz = c.cpl_el_nz = m.cpl_nz.data();
  c.cpl_ac_w = c.cpl_el_w = m.cpl_w.data();
  c.cpl_el_point = c_s.data();
  c.cpl_el_ac_point = c_f.data();
  m.s_elems = S.elems;
  m.f_elems = F.elems;
  if (m.sim_type == 3) {
    run_coupled_kernel_sweep(routine, m, d, a, c);
    check(routine, sf2d_coupled_set_global_numbering(m.C, m.nglob, solid ? S.pts.data() : nullptr, F.pts.data()));
    return;
  }
  check(routine, sf2d_coupled_create(&d, &a, &c, &m.C));
  check(routine, sf2d_coupled_set_global_numbering(m.C, m.nglob, solid ? S.pts.data() : nullptr, F.pts.data()));
  if (!m.staged_u.empty() || !m.staged_p.empty()) {
    auto ptr = [](std::vector<float> &v) -> const float * { return v.empty() ? nullptr : v.data(); };
    check(routine, sf2d_coupled_set_fields_global(m.C, ptr(m.staged_u), ptr(m.staged_v), ptr(m.staged_a),
                                                  ptr(m.staged_p), ptr(m.staged_pd), ptr(m.staged_pdd)));
  }
  if (m.d.seismotype == 4 && !m.trick_checked) {
    std::vector<float> *st[6] = {&m.staged_u, &m.staged_v, &m.staged_a, &m.staged_p, &m.staged_pd, &m.staged_pdd};
    for (int k = 0; k < 6; ++k) m.init_fields[k] = *st[k];
  }
  m.staged_u.clear();
  m.staged_v.clear();
  m.staged_a.clear();
  m.staged_p.clear();
  m.staged_pd.clear();
  m.staged_pdd.clear();
}

// Whole-mesh fields of a coupled run (points outside a field's domain read zero);
// before the solver exists, the staged copies (or zeros).
void coupled_fields(const char *R, FortranMesh *m, realw *u, realw *v, realw *a, realw *p, realw *pd, realw *pdd) {
  if (m->C) {
    check(R, sf2d_coupled_get_fields_global(m->C, u, v, a, p, pd, pdd));
    return;
  }
  const size_t n2 = 2 * static_cast<size_t>(m->nglob), n1 = m->nglob;
  const std::pair<realw *, std::vector<float> *> f[6] = {{u, &m->staged_u}, {v, &m->staged_v}, {a, &m->staged_a},
                                                           {p, &m->staged_p}, {pd, &m->staged_pd},
                                                           {pdd, &m->staged_pdd}};
  for (int k = 0; k < 6; ++k) {
    if (!f[k].first) continue;
    const size_t n = k < 3 ? n2 : n1;
    if (f[k].second->empty())
      std::memset(f[k].first, 0, n * sizeof(realw));
    else
      std::memcpy(f[k].first, f[k].second->data(), n * sizeof(realw));
  }
}

// Sets some fields of a coupled run, keeping the others.
void coupled_set(const char *R, FortranMesh *m, const realw *u, const realw *v, const realw *a, const realw *p,
                 const realw *pd, const realw *pdd) {
  if (m->CF) stop(R, "the fields of a kernel run cannot be replaced after its first step");
  const size_t n2 = 2 * static_cast<size_t>(m->nglob), n1 = m->nglob;
  std::vector<float> cur[6] = {std::vector<float>(n2), std::vector<float>(n2), std::vector<float>(n2),
                               std::vector<float>(n1), std::vector<float>(n1), std::vector<float>(n1)};
  coupled_fields(R, m, cur[0].data(), cur[1].data(), cur[2].data(), cur[3].data(), cur[4].data(), cur[5].data());
  const realw *in[6] = {u, v, a, p, pd, pdd};
  for (int k = 0; k < 6; ++k)
    if (in[k]) std::memcpy(cur[k].data(), in[k], cur[k].size() * sizeof(float));
  if (m->C) {
    check(R, sf2d_coupled_set_fields_global(m->C, cur[0].data(), cur[1].data(), cur[2].data(), cur[3].data(),
                                            cur[4].data(), cur[5].data()));
    return;
  }
  std::vector<float> *st[6] = {&m->staged_u, &m->staged_v, &m->staged_a, &m->staged_p, &m->staged_pd, &m->staged_pdd};
  for (int k = 0; k < 6; ++k) *st[k] = std::move(cur[k]);
}

// A per-step call of a kernel run on a mesh with fluid elements: the run went
// through in full when the first step started, so only the step must be open.
void kernel_step_call(const char *R, const FortranMesh *m) {
  if (!m->CF || !m->kr_open) stop(R, "called outside a time step of the kernel run");
}

// Ends a time step of a kernel run on a mesh with fluid elements.
void kernel_step_end(const char *R, FortranMesh *m) {
  if (m->srcs_added != m->steps + 1) stop(R, "no compute_add_sources_*_s3_cuda call in this time step");
  ++m->steps;
  m->kr_open = false;
}

void fluid_phase_call(const char *R, FortranMesh *m, const int *compute_wavefield_2) {
  if (compute_wavefield_2 && *compute_wavefield_2) unsupported(R, KERNEL_RUN);
  if (m->ac_phase != 3) stop(R, "called outside the fluid forces of a time step");
}

void need_ac_size(const char *R, const FortranMesh *m, const int *size) {
  if (!m->fluid) stop(R, "the mesh has no fluid element");
  if (!size || *size != m->nglob) stop(R, "size must be NGLOB_AB = " + std::to_string(m->nglob));
}

void need_size(const char *routine, const FortranMesh &m, const int *size) {
  if (!size || *size != 2 * m.nglob) stop(routine, "size must be NDIM*NGLOB_AB = " + std::to_string(2 * m.nglob));
}

void fields_from(const char *R, FortranMesh *m, const int *size, realw *displ, realw *veloc, realw *accel) {
  need_size(R, *m, size);
  if (m->fluid) {
    coupled_fields(R, m, displ, veloc, accel, nullptr, nullptr, nullptr);
    return;
  }
  if (m->S) {
    check(R, sf2d_get_fields(m->S, displ, veloc, accel));
    return;
  }
  if (m->F) {
    check(R, sf2d_fwi_adjoint_fields(m->F, displ, veloc, accel));
    return;
  }
  const size_t n = static_cast<size_t>(*size);
  const bool staged = !m->staged_u.empty();
  for (auto pr : {std::make_pair(displ, &m->staged_u), std::make_pair(veloc, &m->staged_v),
                  std::make_pair(accel, &m->staged_a)})
    if (pr.first) {
      if (staged)
        std::memcpy(pr.first, pr.second->data(), n * sizeof(realw));
      else
        std::memset(pr.first, 0, n * sizeof(realw));
    }
}

}  // namespace

extern "C" {

// ---- device and memory ----

// initialize_cuda_device (src/gpu/initialize_cuda.cu:50): device myrank % count
void initialize_cuda_device_(int *myrank_f, int *ncuda_devices) {
  int n = 0;
  check("initialize_cuda_device", sf2d_initialize_device(myrank_f ? *myrank_f : 0, &n));
  if (ncuda_devices) *ncuda_devices = n;
}

void initialize_cuda_aware_mpi_() {}

void pause_for_debug_() {}

// output_free_device_memory / get_free_device_memory (src/gpu/check_fields_cuda.cu)
void get_free_device_memory_(realw *free_mb, realw *used_mb, realw *total_mb) {
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) stop("get_free_device_memory", "cudaMemGetInfo failed");
  if (free_mb) *free_mb = static_cast<realw>(fr / 1048576.0);
  if (used_mb) *used_mb = static_cast<realw>((tot - fr) / 1048576.0);
  if (total_mb) *total_mb = static_cast<realw>(tot / 1048576.0);
}

void output_free_device_memory_(int *myrank_f) {
  realw fr = 0, used = 0, tot = 0;
  get_free_device_memory_(&fr, &used, &tot);
  std::printf("rank %d: GPU memory usage: used = %f MB, free = %f MB, total = %f MB\n", myrank_f ? *myrank_f : 0,
              used, fr, tot);
  std::fflush(stdout);
}

// ---- set-up and clean-up ----

// prepare_constants_device (src/gpu/prepare_mesh_constants_cuda.cu:83)
void prepare_constants_device_(long *Mesh_pointer, int *h_NGLLX, int *NSPEC_AB, int *NGLOB_AB, realw *h_xix,
                               realw *h_xiz, realw *h_gammax, realw *h_gammaz, realw *h_kappav, realw *h_muv,
                               int *h_ibool, int *num_interfaces_ext_mesh, int *, int *, int *,
                               realw *h_hprime_xx, realw *h_hprimewgll_xx, realw *h_wxgll,
                               int *STACEY_BOUNDARY_CONDITIONS, int *PML_BOUNDARY_CONDITIONS, int *,
                               int *nsources_local_f, realw *h_sourcearrays, realw *h_source_time_function,
                               int *NSTEP, int *h_ispec_selected_source, int *h_ispec_selected_rec_loc,
                               int *nrec_local, realw *h_cosrot, realw *h_sinrot, int *SIMULATION_TYPE, int *P_SV,
                               int *nspec_acoustic, int *, int *ispec_is_acoustic, int *, int *, int *SAVE_FORWARD,
                               realw *h_xir_store, realw *h_gammar_store, int *h_NSIGTYPE, int *h_seismotypeVec,
                               int *nlength_seismogram) {
  const char *R = "prepare_constants_device";
  if (!Mesh_pointer) stop(R, "null Mesh_pointer");
  if (*h_NGLLX != NGLL) stop(R, "NGLLX must be 5");
  if (!*P_SV) stop(R, "SH (membrane) waves are not provided: P_SV only");
  if (*SIMULATION_TYPE != 1 && *SIMULATION_TYPE != 3) unsupported(R, KERNEL_RUN);
  if (*SIMULATION_TYPE == 3 && *nlength_seismogram < 1) stop(R, "nlength_seismogram must be positive");
  if (*PML_BOUNDARY_CONDITIONS) {
    // the reference's GPU path takes CPML layers in fluid-only meshes:
    // compute_forces_viscoelastic_GPU stops them (compute_gpu_elastic.f90:100-101)
    if (*nspec_acoustic != *NSPEC_AB) unsupported(R, PML);
    if (*STACEY_BOUNDARY_CONDITIONS) stop(R, "CPML and Stacey conditions are exclusive");
    if (*SIMULATION_TYPE != 1) stop(R, "kernel runs with CPML layers are not provided");
  }
  if (*num_interfaces_ext_mesh > 0) unsupported(R, MPI);
  if (*h_NSIGTYPE != 1) stop(R, "one seismogram type per run (NSIGTYPE = 1)");
  const int st = h_seismotypeVec[0];
  if (*nspec_acoustic > 0 ? (st < 1 || st > 6 || st == 5) : (st < 1 || st > 3))
    stop(R, "seismotype 1-3 (displacement, velocity, acceleration), with fluid elements also 4 (pressure) "
            "and 6 (potential)");
  auto m = new FortranMesh();
  m->sim_type = *SIMULATION_TYPE;
  m->pml = *PML_BOUNDARY_CONDITIONS != 0;
  if (*SAVE_FORWARD && *SIMULATION_TYPE == 1) {
    // a kernel run through this library replays the forward field from
    // checkpoints and reads neither the last frame nor the absorbed-boundary
    // records; the records this run hands back are zeros
    m->save_forward = true;
    std::fprintf(stderr,
                 "prepare_constants_device: SAVE_FORWARD: the absorbing-boundary records (b_absorb_elastic_*) are "
                 "written as zeros; only a SIMULATION_TYPE = 3 run through this library can follow this run\n");
  }
  const int ns = *NSPEC_AB, ng = *NGLOB_AB;
  const size_t nl = static_cast<size_t>(ns) * NGLL2;
  // ispec_is_acoustic is a Fortran logical array: nonzero is true
  m->is_ac.assign(ns, 0);
  if (*nspec_acoustic > 0) {
    if (!ispec_is_acoustic) stop(R, "missing ispec_is_acoustic");
    for (int e = 0; e < ns; ++e) m->is_ac[e] = ispec_is_acoustic[e] != 0;
    if (std::count(m->is_ac.begin(), m->is_ac.end(), 1) != *nspec_acoustic)
      stop(R, "ispec_is_acoustic disagrees with nspec_acoustic");
    m->fluid = true;
    m->nspec_acoustic = *nspec_acoustic;
  }
  m->nspec = ns;
  m->nglob = ng;
  m->nstep = *NSTEP;
  m->nlength = *nlength_seismogram;
  m->stacey = *STACEY_BOUNDARY_CONDITIONS != 0;
  m->ibool.resize(nl);
  for (size_t p = 0; p < nl; ++p) {
    m->ibool[p] = h_ibool[p] - 1;
    if (m->ibool[p] < 0 || m->ibool[p] >= ng) stop(R, "ibool out of range");
  }
  m->xix.assign(h_xix, h_xix + nl);
  m->xiz.assign(h_xiz, h_xiz + nl);
  m->gammax.assign(h_gammax, h_gammax + nl);
  m->gammaz.assign(h_gammaz, h_gammaz + nl);
  m->mu.assign(h_muv, h_muv + nl);
  // the reference's GPU kernel forms lambda = kappa - mu in CUSTOM_REAL
  // (Kernel_2_viscoelastic_impl.cu:501)
  m->lambda.resize(nl);
  for (size_t p = 0; p < nl; ++p) m->lambda[p] = h_kappav[p] - h_muv[p];
  // hprime_xx(i2, i1) = l'_i1(xi_i2) in Fortran order: the descriptor's [i2][i1]
  m->hprime = transpose<float>(h_hprime_xx, NGLL, NGLL);
  m->hprimewgll = transpose<float>(h_hprimewgll_xx, NGLL, NGLL);
  m->wxgll.assign(h_wxgll, h_wxgll + NGLL);
  // sources: sourcearray_loc(NDIM, NGLLX, NGLLZ, nsrc) is already [isrc][j][i][comp];
  // source_time_function_loc(nsrc, NSTEP) is transposed to [isrc][it]
  m->nsrc = *nsources_local_f;
  m->src_ispec.resize(m->nsrc);
  for (int s = 0; s < m->nsrc; ++s) m->src_ispec[s] = h_ispec_selected_source[s] - 1;
  m->srcarr.assign(h_sourcearrays, h_sourcearrays + static_cast<size_t>(m->nsrc) * NGLL2 * 2);
  m->stf = transpose<float>(h_source_time_function, m->nsrc, m->nstep);
  // receivers: xir_store_loc(nrec, NGLLX) -> [irec][i]; one rotation for all receivers
  m->nrec = *nrec_local;
  m->rec_ispec.resize(m->nrec);
  for (int r = 0; r < m->nrec; ++r) m->rec_ispec[r] = h_ispec_selected_rec_loc[r] - 1;
  m->hxir = transpose<double>(h_xir_store, m->nrec, NGLL);
  m->hgammar = transpose<double>(h_gammar_store, m->nrec, NGLL);
  for (int r = 1; r < m->nrec; ++r)
    if (h_cosrot[r] != h_cosrot[0] || h_sinrot[r] != h_sinrot[0])
      stop(R, "receivers with different rotation angles are not provided");
  m->d.cosrot = m->nrec ? static_cast<double>(h_cosrot[0]) : 1.0;
  m->d.sinrot = m->nrec ? static_cast<double>(h_sinrot[0]) : 0.0;
  m->d.seismotype = h_seismotypeVec[0];
  m->centroid.assign(2 * static_cast<size_t>(ns), 0.0);
  rebuild_centroids(*m);
  *Mesh_pointer = reinterpret_cast<long>(m);
}

// prepare_fields_elastic_device (src/gpu/prepare_mesh_constants_cuda.cu:527)
void prepare_fields_elastic_device_(long *Mesh_pointer, realw *rmassx, realw *rmassz, int *, int *,
                                    int *ispec_is_anisotropic, int *ANISOTROPY, realw *c11store, realw *,
                                    realw *c13store, realw *c15store, realw *, realw *, realw *c33store,
                                    realw *c35store, realw *c55store, int *h_ninterface_elastic, int *,
                                    int *ATTENUATION_VISCOELASTIC, realw *h_A_newmark_mu, realw *h_B_newmark_mu,
                                    realw *h_A_newmark_kappa, realw *h_B_newmark_kappa) {
  const char *R = "prepare_fields_elastic_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->S) stop(R, "called after the time loop started");
  if (*h_ninterface_elastic > 0) unsupported(R, MPI);
  m->rmass.resize(2 * static_cast<size_t>(m->nglob));
  for (int g = 0; g < m->nglob; ++g) {
    m->rmass[2 * g] = rmassx[g];
    m->rmass[2 * g + 1] = rmassz[g];
  }
  m->have_rmass = true;
  const size_t nl = static_cast<size_t>(m->nspec) * NGLL2;
  if (*ANISOTROPY) {
    m->aniso_flag.resize(m->nspec);
    for (int e = 0; e < m->nspec; ++e) m->aniso_flag[e] = ispec_is_anisotropic[e] != 0;
    m->c11.assign(c11store, c11store + nl);
    m->c13.assign(c13store, c13store + nl);
    m->c15.assign(c15store, c15store + nl);
    m->c33.assign(c33store, c33store + nl);
    m->c35.assign(c35store, c35store + nl);
    m->c55.assign(c55store, c55store + nl);
  }
  if (*ATTENUATION_VISCOELASTIC) {
    // A/B_newmark_nu1 (bulk, "kappa") and _nu2 (shear, "mu"), (N_SLS, NGLLX, NGLLZ, nspec)
    const size_t na = nl * 3;
    m->a1.assign(h_A_newmark_kappa, h_A_newmark_kappa + na);
    m->b1.assign(h_B_newmark_kappa, h_B_newmark_kappa + na);
    m->a2.assign(h_A_newmark_mu, h_A_newmark_mu + na);
    m->b2.assign(h_B_newmark_mu, h_B_newmark_mu + na);
  }
}

// prepare_stacey_device (src/gpu/prepare_mesh_constants_cuda.cu:926): faces to
// one entry per absorbing GLL point, in face order; a point whose i or j is
// NGLLX + 1 (a corner a neighbouring face already covers) is left out, as
// compute_stacey_elastic_kernel skips it
void prepare_stacey_device_(long *Mesh_pointer, int *ACOUSTIC_SIMULATION, int *ELASTIC_SIMULATION, realw *rho_vp,
                            realw *rho_vs, int *h_nspec_bottom, int *h_nspec_left, int *h_nspec_right,
                            int *h_nspec_top, int *h_abs_boundary_ispec, int *h_abs_boundary_ij,
                            realw *h_abs_boundary_normal, realw *h_abs_boundary_jacobian1Dw,
                            int *h_num_abs_boundary_faces, int *, int *, int *, int *, int *) {
  const char *R = "prepare_stacey_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->S) stop(R, "called after the time loop started");
  m->st_iglob.clear();
  m->st_nx.clear();
  m->st_nz.clear();
  m->st_w.clear();
  m->st_rvp.clear();
  m->st_rvs.clear();
  m->st_ac_iglob.clear();
  m->st_ac_w.clear();
  m->st_ac_rvp.clear();
  m->nspec_side[0] = *h_nspec_bottom;
  m->nspec_side[1] = *h_nspec_left;
  m->nspec_side[2] = *h_nspec_right;
  m->nspec_side[3] = *h_nspec_top;
  const int nf = *h_num_abs_boundary_faces;
  for (int f = 0; f < nf; ++f) {
    const int e = h_abs_boundary_ispec[f] - 1;
    if (e < 0 || e >= m->nspec) stop(R, "abs_boundary_ispec out of range");
    const bool fluid_face = m->is_ac[e] != 0;
    if (fluid_face ? !*ACOUSTIC_SIMULATION : !*ELASTIC_SIMULATION) continue;
    for (int k = 0; k < NGLL; ++k) {
      const int i = h_abs_boundary_ij[(f * NGLL + k) * 2] - 1;
      const int j = h_abs_boundary_ij[(f * NGLL + k) * 2 + 1] - 1;
      if (i == NGLL || j == NGLL) continue;
      if (i < 0 || i >= NGLL || j < 0 || j >= NGLL) stop(R, "abs_boundary_ij out of range");
      const size_t p = static_cast<size_t>(e) * NGLL2 + j * NGLL + i;
      if (fluid_face) {
        // compute_stacey_acoustic_kernel: chi_dd -= chi_d w / (rho vp)
        m->st_ac_iglob.push_back(m->ibool[p]);
        m->st_ac_w.push_back(h_abs_boundary_jacobian1Dw[f * NGLL + k]);
        m->st_ac_rvp.push_back(rho_vp[p]);
        continue;
      }
      m->st_iglob.push_back(m->ibool[p]);
      m->st_nx.push_back(h_abs_boundary_normal[(f * NGLL + k) * 2]);
      m->st_nz.push_back(h_abs_boundary_normal[(f * NGLL + k) * 2 + 1]);
      m->st_w.push_back(h_abs_boundary_jacobian1Dw[f * NGLL + k]);
      m->st_rvp.push_back(rho_vp[p]);
      m->st_rvs.push_back(rho_vs[p]);
    }
  }
  m->have_stacey = true;
}

// prepare_cleanup_device (src/gpu/prepare_mesh_constants_cuda.cu:1139)
void prepare_cleanup_device_(long *Mesh_pointer, int *, int *, int *, int *, int *, int *, int *, realw *) {
  FortranMesh *m = mesh_of("prepare_cleanup_device", Mesh_pointer);
  if (m->S) sf2d_destroy(m->S);
  if (m->F) sf2d_fwi_destroy(m->F);
  if (m->CF)
    sf2d_coupled_fwi_destroy(m->CF);  // C is its adjoint run
  else if (m->C)
    sf2d_coupled_destroy(m->C);
  delete m;
  *Mesh_pointer = 0;
}

// ---- one elastic time step ----

// update_displacement_cuda (src/gpu/update_displacement_cuda.cu:52): the first
// call of a step; the first one of the run also builds the solver, since this
// is where the host first passes the time step
void update_displacement_cuda_(long *Mesh_pointer, realw *deltat_F, realw *deltatsqover2_F, realw *deltatover2_F,
                               realw *, realw *, realw *) {
  const char *R = "update_displacement_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->fluid) {
    if (m->sim_type == 3) {
      kernel_step_call(R, m);
      return;
    }
    // coupled mesh: the solid predictor follows the fluid's (update_displacement_Newmark.F90:150-240)
    if (m->ac_phase != 1) stop(R, "update_displacement_ac_cuda must start the step");
    m->ac_phase = 2;
    return;
  }
  if (m->stage != 0) stop(R, "the previous time step did not reach kernel_3_a_cuda");
  if (!m->S && !m->F) {
    m->dt = *deltat_F;
    m->dtsq2 = *deltatsqover2_F;
    m->dtover2 = *deltatover2_F;
    build_solver(R, *m);
  } else if (*deltat_F != m->dt || *deltatsqover2_F != m->dtsq2 || *deltatover2_F != m->dtover2) {
    stop(R, "the time step changed during the run");
  }
  if (m->steps >= m->nstep) stop(R, "more time steps than NSTEP");
  m->stage = 1;
}

// compute_forces_viscoelastic_cuda (src/gpu/compute_forces_viscoelastic_cuda.cu:327):
// outer (iphase 1) then inner (iphase 2) elements; with one process every
// element is inner and the fused step covers both
void compute_forces_viscoelastic_cuda_(long *Mesh_pointer, int *iphase, realw *, int *, int *, int *, int *,
                                       int *, int *compute_wavefield_2) {
  const char *R = "compute_forces_viscoelastic_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (*compute_wavefield_2 && m->sim_type != 3) unsupported(R, KERNEL_RUN);
  if (m->fluid) {
    if (m->sim_type == 3) {
      kernel_step_call(R, m);
      return;
    }
    if (*iphase == 1 && m->ac_phase == 4)
      m->ac_phase = 5;
    else if (!(*iphase == 2 && m->ac_phase == 5))
      stop(R, "called out of the order kernel_3_acoustic_cuda, iphase 1, iphase 2, kernel_3_a_cuda");
    return;
  }
  if (*iphase == 1 && m->stage == 1)
    m->stage = 2;
  else if (!(*iphase == 2 && m->stage == 2))
    stop(R, "called out of the order update_displacement_cuda, iphase 1, iphase 2, kernel_3_a_cuda");
}

// compute_stacey_viscoelastic_cuda (src/gpu/compute_stacey_viscoelastic_cuda.cu:40):
// the absorbing terms are part of the fused step
void compute_stacey_viscoelastic_cuda_(long *Mesh_pointer, int *iphase, realw *b_absorb_left,
                                       realw *b_absorb_right, realw *b_absorb_top, realw *b_absorb_bottom, int *,
                                       int *compute_wavefield_2, int *) {
  const char *R = "compute_stacey_viscoelastic_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (*compute_wavefield_2 && m->sim_type != 3) unsupported(R, KERNEL_RUN);
  if (m->fluid && m->sim_type == 3)
    kernel_step_call(R, m);
  else if (m->fluid ? m->ac_phase != 5 : m->stage != 2)
    stop(R, "called outside a time step");
  if (m->save_forward && *iphase == 1) {
    // SIMULATION_TYPE = 1 with SAVE_FORWARD: the host stores these slices as
    // b_absorb_elastic_*(:,:,:,it); a kernel run here does not read them back
    realw *side[4] = {b_absorb_bottom, b_absorb_left, b_absorb_right, b_absorb_top};
    for (int k = 0; k < 4; ++k)
      if (side[k] && m->nspec_side[k] > 0)
        std::memset(side[k], 0, sizeof(realw) * 2 * NGLL * static_cast<size_t>(m->nspec_side[k]));
  }
}

// compute_add_sources_el_cuda (src/gpu/compute_add_sources_viscoelastic_cuda.cu:46):
// the fused step adds source_time_function(:, it) of the step it advances
void compute_add_sources_el_cuda_(long *Mesh_pointer, int *, int *itf) {
  const char *R = "compute_add_sources_el_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->fluid ? m->ac_phase != 5 : m->stage != 2) stop(R, "called outside a time step");
  if (*itf != m->steps + 1) stop(R, "time step " + std::to_string(*itf) + " out of sequence");
}

// kernel_3_a_cuda (src/gpu/update_displacement_cuda.cu:221): the last call of
// the step; the whole fused step is queued here
void kernel_3_a_cuda_(long *Mesh_pointer, realw *, realw *, int *, int *compute_wavefield_2) {
  const char *R = "kernel_3_a_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (*compute_wavefield_2 && m->sim_type != 3) unsupported(R, KERNEL_RUN);
  if (m->fluid) {
    if (m->sim_type == 3) {
      // the backward field's corrector ends a kernel-run step (compute_gpu_elastic.f90
      // with compute_b_wavefield runs last, iterate_time.F90:330-360)
      kernel_step_call(R, m);
      if (*compute_wavefield_2) kernel_step_end(R, m);
      return;
    }
    // the last call of a coupled step: both domains advance in one fused step
    if (m->ac_phase != 5) stop(R, "called before compute_forces_viscoelastic_cuda");
    check(R, sf2d_coupled_enqueue(m->C, 1));
    ++m->steps;
    m->ac_phase = 0;
    return;
  }
  if (m->stage != 2) stop(R, "called before compute_forces_viscoelastic_cuda");
  if (m->sim_type == 3) {
    // the kernel run advanced every step when its first step started
    if (m->srcs_added != m->steps + 1) stop(R, "compute_add_sources_el_s3_cuda was not called in this step");
    ++m->steps;
    m->stage = 0;
    return;
  }
  check(R, sf2d_enqueue(m->S, 1));
  ++m->steps;
  m->stage = 0;
}

// compute_seismograms_cuda (src/gpu/write_seismograms_cuda.cu:41): sample
// seismo_current of the host's buffer is the state after step `it`; the
// buffer sisux/sisuz(nlength_seismogram, nrec_local) is filled when it is
// full or at the last step
void compute_seismograms_cuda_(long *Mesh_pointer_f, int *i_sigf, double *sisux, double *sisuz,
                               int *seismo_currentf, int *nlength_seismogramf, int *, int *,
                               int *USE_TRICK_FOR_BETTER_PRESSURE, int *, int *itf, int *it_endf) {
  const char *R = "compute_seismograms_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer_f);
  if (*i_sigf != 1) stop(R, "one seismogram type per run");
  if (m->d.seismotype == 4 && m->C) {
    // pressure from chi instead of chi_dot_dot (write_seismograms_cuda.cu:160-175)
    const int trick = USE_TRICK_FOR_BETTER_PRESSURE && *USE_TRICK_FOR_BETTER_PRESSURE ? 1 : 0;
    if (!m->trick_checked) {
      m->trick_checked = true;
      if (trick != m->use_trick) {
        if (m->CF || m->steps != 1) stop(R, "USE_TRICK_FOR_BETTER_PRESSURE must be known before the run starts");
        // rebuild the run with it from the kept initial fields and repeat step 1
        m->use_trick = trick;
        sf2d_coupled_destroy(m->C);
        m->C = nullptr;
        std::vector<float> *st[6] = {&m->staged_u, &m->staged_v, &m->staged_a, &m->staged_p, &m->staged_pd,
                                     &m->staged_pdd};
        for (int k = 0; k < 6; ++k) *st[k] = std::move(m->init_fields[k]);
        build_solver(R, *m);
        check(R, sf2d_coupled_enqueue(m->C, 1));
      }
      for (auto &f : m->init_fields) std::vector<float>().swap(f);
    } else if (trick != m->use_trick) {
      stop(R, "USE_TRICK_FOR_BETTER_PRESSURE changed during the run");
    }
  }
  if (m->nrec == 0) return;
  const int j = *seismo_currentf - 1, nlen = *nlength_seismogramf;
  if (j < 0 || j >= nlen) stop(R, "seismo_current out of range");
  if (*itf != m->steps) stop(R, "called for a step that has not been advanced");
  if (static_cast<int>(m->sample_step.size()) != j) m->sample_step.resize(j);
  m->sample_step.push_back(*itf - 1);
  if (j != nlen - 1 && *itf != *it_endf) return;
  const int s0 = m->sample_step.front(), s1 = m->sample_step.back();
  const int n = s1 - s0 + 1;
  std::vector<double> tr(static_cast<size_t>(m->nrec) * n * 2);
  if (m->F || m->CF)
    for (int r = 0; r < m->nrec; ++r)
      std::memcpy(tr.data() + static_cast<size_t>(r) * n * 2,
                  m->adj_seis.data() + (static_cast<size_t>(r) * m->nstep + s0) * 2, sizeof(double) * n * 2);
  else if (m->C)
    check(R, sf2d_coupled_copy_seismograms(m->C, s0, n, tr.data()));
  else
    check(R, sf2d_copy_seismograms(m->S, s0, n, tr.data()));
  for (int r = 0; r < m->nrec; ++r)
    for (size_t k = 0; k < m->sample_step.size(); ++k) {
      const size_t src = (static_cast<size_t>(r) * n + (m->sample_step[k] - s0)) * 2;
      sisux[k + static_cast<size_t>(nlen) * r] = tr[src];
      sisuz[k + static_cast<size_t>(nlen) * r] = tr[src + 1];
    }
  m->sample_step.clear();
}

// get_norm_elastic_from_device (src/gpu/check_fields_cuda.cu:358)
void get_norm_elastic_from_device_(realw *norm, long *Mesh_pointer, const int *FORWARD_OR_ADJOINT) {
  const char *R = "get_norm_elastic_from_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  const bool backward = FORWARD_OR_ADJOINT && *FORWARD_OR_ADJOINT == 3;
  if (backward && m->sim_type != 3) unsupported(R, KERNEL_RUN);
  // a kernel run went through when its first step started and stopped the run
  // if either field blew up; reported: the adjoint field at its end, and the
  // replayed forward field at its end (time zero: at rest)
  if (m->sim_type == 3 && (backward || (!m->F && !m->CF))) {
    *norm = 0.f;
    return;
  }
  if (m->sim_type == 3 && m->F) {
    std::vector<float> u(2 * static_cast<size_t>(m->nglob));
    check(R, sf2d_fwi_adjoint_fields(m->F, u.data(), nullptr, nullptr));
    float mx = 0.f;
    for (int g = 0; g < m->nglob; ++g) mx = std::max(mx, std::sqrt(u[2 * g] * u[2 * g] + u[2 * g + 1] * u[2 * g + 1]));
    *norm = mx;
    return;
  }
  if (m->fluid) {
    std::vector<float> u(2 * static_cast<size_t>(m->nglob));
    coupled_fields(R, m, u.data(), nullptr, nullptr, nullptr, nullptr, nullptr);
    float mx = 0.f;
    for (int g = 0; g < m->nglob; ++g)
      mx = std::max(mx, std::sqrt(u[2 * g] * u[2 * g] + u[2 * g + 1] * u[2 * g + 1]));
    *norm = mx;
    return;
  }
  if (!m->S) {
    float mx = 0.f;
    for (size_t g = 0; g < m->staged_u.size() / 2; ++g)
      mx = std::max(mx, std::sqrt(m->staged_u[2 * g] * m->staged_u[2 * g] + m->staged_u[2 * g + 1] * m->staged_u[2 * g + 1]));
    *norm = mx;
    return;
  }
  check(R, sf2d_get_norm(m->S, norm));
}

// ---- wavefield transfers (src/gpu/transfer_fields_cuda.cu:53-140) ----

void transfer_fields_el_to_device_(int *size, realw *displ, realw *veloc, realw *accel, long *Mesh_pointer) {
  const char *R = "transfer_fields_el_to_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  need_size(R, *m, size);
  if (m->fluid) {
    coupled_set(R, m, displ, veloc, accel, nullptr, nullptr, nullptr);
    return;
  }
  if (m->S) {
    check(R, sf2d_set_fields(m->S, displ, veloc, accel));
    return;
  }
  if (m->F) stop(R, "the fields of a kernel run cannot be replaced after its first step");
  m->staged_u.assign(displ, displ + *size);
  m->staged_v.assign(veloc, veloc + *size);
  m->staged_a.assign(accel, accel + *size);
}

void transfer_fields_el_from_device_(int *size, realw *displ, realw *veloc, realw *accel, long *Mesh_pointer) {
  fields_from("transfer_fields_el_from_device", mesh_of("transfer_fields_el_from_device", Mesh_pointer), size,
              displ, veloc, accel);
}

void transfer_displ_from_device_(int *size, realw *displ, long *Mesh_pointer) {
  fields_from("transfer_displ_from_device", mesh_of("transfer_displ_from_device", Mesh_pointer), size, displ,
              nullptr, nullptr);
}

void transfer_accel_from_device_(int *size, realw *accel, long *Mesh_pointer) {
  fields_from("transfer_accel_from_device", mesh_of("transfer_accel_from_device", Mesh_pointer), size, nullptr,
              nullptr, accel);
}

void transfer_accel_to_device_(int *size, realw *accel, long *Mesh_pointer) {
  const char *R = "transfer_accel_to_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  need_size(R, *m, size);
  std::vector<realw> u(*size), v(*size);
  fields_from(R, m, size, u.data(), v.data(), nullptr);
  transfer_fields_el_to_device_(size, u.data(), v.data(), accel, Mesh_pointer);
}

// ---- the fluid domain (compute_gpu_acoustic.f90, update_displacement_Newmark.F90) ----

// prepare_fields_acoustic_device (src/gpu/prepare_mesh_constants_cuda.cu:319):
// the fluid mass matrix, rho and kappa, the free-surface faces (every point of
// a face is zeroed) and the fluid-solid faces (one entry per face point)
void prepare_fields_acoustic_device_(long *Mesh_pointer, realw *rmass_acoustic, realw *rhostore, realw *kappastore,
                                     int *, int *, int *num_free_surface_faces, int *free_surface_ispec,
                                     int *free_surface_ijk, int *ELASTIC_SIMULATION, int *num_coupling_ac_el_faces,
                                     int *coupling_ac_el_ispec, int *coupling_ac_el_ijk, realw *coupling_ac_el_normal,
                                     realw *coupling_ac_el_jacobian2Dw, int *h_ninterface_acoustic, int *,
                                     int *ATTENUATION_VISCOACOUSTIC, realw *, realw *, int *NO_BACKWARD_RECONSTRUCTION,
                                     realw *) {
  const char *R = "prepare_fields_acoustic_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->S || m->C) stop(R, "called after the time loop started");
  if (!m->fluid) stop(R, "prepare_constants_device was given no fluid element (nspec_acoustic = 0)");
  if (*h_ninterface_acoustic > 0) unsupported(R, MPI);
  if (*ATTENUATION_VISCOACOUSTIC) stop(R, "viscoacoustic attenuation is not provided");
  if (*NO_BACKWARD_RECONSTRUCTION) unsupported(R, KERNEL_RUN);
  const size_t nl = static_cast<size_t>(m->nspec) * NGLL2;
  m->rmass_ac.assign(rmass_acoustic, rmass_acoustic + m->nglob);
  m->rho.assign(rhostore, rhostore + nl);
  m->kappa.assign(kappastore, kappastore + nl);
  auto point_of = [&](int e, const int *ij, int f, int k, const char *what) {
    if (e < 0 || e >= m->nspec || !m->is_ac[e]) stop(R, std::string(what) + ": not a fluid element");
    const int i = ij[(f * NGLL + k) * 2] - 1, j = ij[(f * NGLL + k) * 2 + 1] - 1;
    if (i < 0 || i >= NGLL || j < 0 || j >= NGLL) stop(R, std::string(what) + ": GLL index out of range");
    return m->ibool[static_cast<size_t>(e) * NGLL2 + j * NGLL + i];
  };
  m->free_iglob.clear();
  for (int f = 0; f < *num_free_surface_faces; ++f)
    for (int k = 0; k < NGLL; ++k)
      m->free_iglob.push_back(point_of(free_surface_ispec[f] - 1, free_surface_ijk, f, k, "free_surface_ispec"));
  m->cpl_iglob.clear();
  m->cpl_nx.clear();
  m->cpl_nz.clear();
  m->cpl_w.clear();
  for (int f = 0; f < (*ELASTIC_SIMULATION ? *num_coupling_ac_el_faces : 0); ++f)
    for (int k = 0; k < NGLL; ++k) {
      m->cpl_iglob.push_back(point_of(coupling_ac_el_ispec[f] - 1, coupling_ac_el_ijk, f, k, "coupling_ac_el_ispec"));
      m->cpl_nx.push_back(coupling_ac_el_normal[(f * NGLL + k) * 2]);
      m->cpl_nz.push_back(coupling_ac_el_normal[(f * NGLL + k) * 2 + 1]);
      m->cpl_w.push_back(coupling_ac_el_jacobian2Dw[f * NGLL + k]);
    }
  m->have_fluid = true;
}

// update_displacement_ac_cuda (src/gpu/update_displacement_cuda.cu:133): the
// first call of a step of a mesh with fluid elements; the first one of the
// run builds the coupled solver
void update_displacement_ac_cuda_(long *Mesh_pointer, realw *deltat_F, realw *deltatsqover2_F, realw *deltatover2_F,
                                  realw *, realw *, realw *, int *, int *UNDO_ATTENUATION_AND_OR_PML) {
  const char *R = "update_displacement_ac_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (!m->fluid) stop(R, "the mesh has no fluid element");
  if (UNDO_ATTENUATION_AND_OR_PML && *UNDO_ATTENUATION_AND_OR_PML) unsupported(R, KERNEL_RUN);
  if (m->sim_type == 3) {
    // the first call of a kernel-run step (update_displacement_Newmark.F90:126-160
    // advances both fields here); the first step runs the whole gradient
    if (m->kr_open) stop(R, "the previous time step did not finish");
    if (!m->CF) {
      m->dt = *deltat_F;
      m->dtsq2 = *deltatsqover2_F;
      m->dtover2 = *deltatover2_F;
      build_solver(R, *m);
    } else if (*deltat_F != m->dt || *deltatsqover2_F != m->dtsq2 || *deltatover2_F != m->dtover2) {
      stop(R, "the time step changed during the run");
    }
    if (m->steps >= m->nstep) stop(R, "more time steps than NSTEP");
    m->kr_open = true;
    return;
  }
  if (m->ac_phase != 0) stop(R, "the previous time step did not finish");
  if (!m->C) {
    m->dt = *deltat_F;
    m->dtsq2 = *deltatsqover2_F;
    m->dtover2 = *deltatover2_F;
    build_solver(R, *m);
  } else if (*deltat_F != m->dt || *deltatsqover2_F != m->dtsq2 || *deltatover2_F != m->dtover2) {
    stop(R, "the time step changed during the run");
  }
  if (m->steps >= m->nstep) stop(R, "more time steps than NSTEP");
  // without solid elements no update_displacement_cuda follows
  m->ac_phase = m->nspec_acoustic == m->nspec ? 2 : 1;
}

// acoustic_enforce_free_surf_cuda (src/gpu/enforce_acoustic_free_surface_cuda.cu:46):
// the zeroing before and after the fluid forces is part of the fused step
void acoustic_enforce_free_surf_cuda_(long *Mesh_pointer, int *, int *compute_wavefield_2) {
  const char *R = "acoustic_enforce_free_surf_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type == 3) {
    // before and after each field's forces, the last time after the step ended
    if (!m->CF) stop(R, "called outside a time step of the kernel run");
    return;
  }
  if (*compute_wavefield_2) unsupported(R, KERNEL_RUN);
  const bool fluid_only = m->nspec_acoustic == m->nspec;
  if (!(m->ac_phase == 2 || m->ac_phase == 4 || (fluid_only && m->ac_phase == 0 && m->steps > 0)))
    stop(R, "called outside a time step");
}

// compute_forces_acoustic_cuda (src/gpu/compute_forces_acoustic_cuda.cu:248):
// outer then inner elements; with one process the fused step covers both
void compute_forces_acoustic_cuda_(long *Mesh_pointer, int *iphase, int *, int *, int *ATTENUATION_VISCOACOUSTIC, int *,
                                   int *compute_wavefield_2) {
  const char *R = "compute_forces_acoustic_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (*ATTENUATION_VISCOACOUSTIC) stop(R, "viscoacoustic attenuation is not provided");
  if (m->sim_type == 3) {
    kernel_step_call(R, m);
    return;
  }
  if (*compute_wavefield_2) unsupported(R, KERNEL_RUN);
  if (*iphase == 1 && m->ac_phase == 2)
    m->ac_phase = 3;
  else if (!(*iphase == 2 && m->ac_phase == 3))
    stop(R, "called out of the order update_displacement_*_cuda, iphase 1, iphase 2, kernel_3_acoustic_cuda");
}

// compute_stacey_acoustic_cuda (src/gpu/compute_stacey_acoustic_cuda.cu:40)
void compute_stacey_acoustic_cuda_(long *Mesh_pointer, int *iphase, realw *b_absorb_left, realw *b_absorb_right,
                                   realw *b_absorb_top, realw *b_absorb_bottom, int *, int *compute_wavefield_2,
                                   int *) {
  const char *R = "compute_stacey_acoustic_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type == 3) {
    kernel_step_call(R, m);
    return;
  }
  fluid_phase_call(R, m, compute_wavefield_2);
  if (m->save_forward && *iphase == 1) {
    // SIMULATION_TYPE = 1 with SAVE_FORWARD: the host stores these slices as
    // b_absorb_acoustic_*(:,:,it); a kernel run here does not read them back
    realw *side[4] = {b_absorb_bottom, b_absorb_left, b_absorb_right, b_absorb_top};
    for (int k = 0; k < 4; ++k)
      if (side[k] && m->nspec_side[k] > 0)
        std::memset(side[k], 0, sizeof(realw) * NGLL * static_cast<size_t>(m->nspec_side[k]));
  }
}

// compute_coupling_ac_el_cuda (src/gpu/compute_coupling_cuda.cu:47): the solid's
// normal displacement on the fluid, part of the fused step
void compute_coupling_ac_el_cuda_(long *Mesh_pointer, int *, int *, int *FORWARD_OR_ADJOINT) {
  const char *R = "compute_coupling_ac_el_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type == 3 && (*FORWARD_OR_ADJOINT == 1 || *FORWARD_OR_ADJOINT == 3)) {
    kernel_step_call(R, m);
    return;
  }
  if (*FORWARD_OR_ADJOINT != 1) unsupported(R, KERNEL_RUN);
  fluid_phase_call(R, m, nullptr);
}

// compute_add_sources_ac_cuda (src/gpu/compute_add_sources_viscoacoustic_cuda.cu:46)
void compute_add_sources_ac_cuda_(long *Mesh_pointer, int *, int *itf) {
  const char *R = "compute_add_sources_ac_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  fluid_phase_call(R, m, nullptr);
  if (*itf != m->steps + 1) stop(R, "time step " + std::to_string(*itf) + " out of sequence");
}

// kernel_3_acoustic_cuda (src/gpu/update_displacement_cuda.cu:322): ends the
// fluid step; on a fluid-only mesh the fused step is queued here
void kernel_3_acoustic_cuda_(long *Mesh_pointer, realw *, realw *, int *, int *compute_wavefield_2) {
  const char *R = "kernel_3_acoustic_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type == 3) {
    // on a fluid-only mesh the call with both fields ends the step
    kernel_step_call(R, m);
    if (m->nspec_acoustic == m->nspec && *compute_wavefield_2) kernel_step_end(R, m);
    return;
  }
  fluid_phase_call(R, m, compute_wavefield_2);
  if (m->nspec_acoustic == m->nspec) {
    check(R, sf2d_coupled_enqueue(m->C, 1));
    ++m->steps;
    m->ac_phase = 0;
    return;
  }
  m->ac_phase = 4;
}

// compute_coupling_el_ac_cuda (src/gpu/compute_coupling_cuda.cu:125): the fluid
// pressure on the solid, part of the fused step
void compute_coupling_el_ac_cuda_(long *Mesh_pointer, int *, int *, int *FORWARD_OR_ADJOINT) {
  const char *R = "compute_coupling_el_ac_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type == 3 && (*FORWARD_OR_ADJOINT == 1 || *FORWARD_OR_ADJOINT == 3)) {
    kernel_step_call(R, m);
    return;
  }
  if (*FORWARD_OR_ADJOINT != 1) unsupported(R, KERNEL_RUN);
  if (m->ac_phase != 5) stop(R, "called outside the solid forces of a time step");
}

// get_norm_acoustic_from_device (src/gpu/check_fields_cuda.cu:240): max |chi|
void get_norm_acoustic_from_device_(realw *norm, long *Mesh_pointer, const int *FORWARD_OR_ADJOINT) {
  const char *R = "get_norm_acoustic_from_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  const bool backward = FORWARD_OR_ADJOINT && *FORWARD_OR_ADJOINT == 3;
  if (backward && m->sim_type != 3) unsupported(R, KERNEL_RUN);
  if (!m->fluid) stop(R, "the mesh has no fluid element");
  // a kernel run: the adjoint field at its end, the replayed field at rest
  if (m->sim_type == 3 && (backward || !m->CF)) {
    *norm = 0.f;
    return;
  }
  std::vector<float> p(m->nglob);
  coupled_fields(R, m, nullptr, nullptr, nullptr, p.data(), nullptr, nullptr);
  float mx = 0.f;
  for (float x : p) mx = std::max(mx, std::fabs(x));
  *norm = mx;
}

// transfer_fields_ac_{to,from}_device, transfer_dot_dot_from_device
// (src/gpu/transfer_fields_cuda.cu:223-300): whole-mesh potentials
void transfer_fields_ac_to_device_(int *size, realw *potential_acoustic, realw *potential_dot_acoustic,
                                   realw *potential_dot_dot_acoustic, long *Mesh_pointer) {
  const char *R = "transfer_fields_ac_to_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  need_ac_size(R, m, size);
  coupled_set(R, m, nullptr, nullptr, nullptr, potential_acoustic, potential_dot_acoustic, potential_dot_dot_acoustic);
}

void transfer_fields_ac_from_device_(int *size, realw *potential_acoustic, realw *potential_dot_acoustic,
                                     realw *potential_dot_dot_acoustic, long *Mesh_pointer) {
  const char *R = "transfer_fields_ac_from_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  need_ac_size(R, m, size);
  coupled_fields(R, m, nullptr, nullptr, nullptr, potential_acoustic, potential_dot_acoustic,
                 potential_dot_dot_acoustic);
}

void transfer_dot_dot_from_device_(int *size, realw *potential_dot_dot_acoustic, long *Mesh_pointer) {
  const char *R = "transfer_dot_dot_from_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  need_ac_size(R, m, size);
  coupled_fields(R, m, nullptr, nullptr, nullptr, nullptr, nullptr, potential_dot_dot_acoustic);
}

// ---- not provided ----
// ---- the kernel run (SIMULATION_TYPE = 3) of a solid mesh ----

// prepare_fields_elastic_adj_dev (src/gpu/prepare_mesh_constants_cuda.cu:711):
// the kernel arrays live in the gradient run this library builds at the first
// step
void prepare_fields_elastic_adj_dev_(long *Mesh_pointer, int *size, int *APPROXIMATE_HESS_KL, int *,
                                     int *NO_BACKWARD_RECONSTRUCTION) {
  const char *R = "prepare_fields_elastic_adj_dev";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3)");
  need_size(R, *m, size);
  // prepare_gpu.f90 stops an approximate Hessian on GPUs as well; the
  // library's own sf2d_fwi_enable_hessian computes it
  if (*APPROXIMATE_HESS_KL) stop(R, "APPROXIMATE_HESS_KL: use sf2d_fwi_enable_hessian (include/sf2d_b200.h)");
  if (*NO_BACKWARD_RECONSTRUCTION)
    stop(R, "NO_BACKWARD_RECONSTRUCTION: the forward field is replayed from device checkpoints, no frames are read");
  m->adj_prepared = true;
}

// prepare_sim2_or_3_const_device (src/gpu/prepare_mesh_constants_cuda.cu:815):
// source_adjoint(nadj_rec_local, NSTEP, NDIM) in Fortran order, to [irec][it][comp]
void prepare_sim2_or_3_const_device_(long *Mesh_pointer, int *nadj_rec_local, realw *h_source_adjoint, int *NSTEP) {
  const char *R = "prepare_sim2_or_3_const_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3)");
  if (m->F || m->CF) stop(R, "called after the time loop started");
  if (*NSTEP != m->nstep) stop(R, "NSTEP disagrees with prepare_constants_device");
  if (*nadj_rec_local != m->nrec) stop(R, "every local receiver must be an adjoint source (nadj_rec_local = nrec_local)");
  const size_t nr = static_cast<size_t>(m->nrec), nt = static_cast<size_t>(m->nstep);
  m->adj_src.resize(nr * nt * 2);
  for (size_t r = 0; r < nr; ++r)
    for (size_t it = 0; it < nt; ++it)
      for (size_t c = 0; c < 2; ++c) m->adj_src[(r * nt + it) * 2 + c] = h_source_adjoint[r + nr * (it + nt * c)];
}

// add_sources_el_sim_type_2_or_3 (src/gpu/compute_add_sources_viscoelastic_cuda.cu:131):
// the adjoint sources of step it are source_adjoint(:, NSTEP-it+1)
void add_sources_el_sim_type_2_or_3_(long *Mesh_pointer, int *, int *itf, int *nadj_rec_local, int *NSTEP) {
  const char *R = "add_sources_el_sim_type_2_or_3";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3) unsupported(R, OTHER);
  if (m->fluid)
    kernel_step_call(R, m);
  else if (m->stage != 2)
    stop(R, "called outside a time step");
  if (*nadj_rec_local != m->nrec || *NSTEP != m->nstep) stop(R, "nadj_rec_local or NSTEP changed");
  if (*itf != m->nstep - m->steps) stop(R, "time step " + std::to_string(*itf) + " out of sequence");
}

// compute_add_sources_el_s3_cuda (src/gpu/compute_add_sources_viscoelastic_cuda.cu:86):
// the forward source of the replayed field
void compute_add_sources_el_s3_cuda_(long *Mesh_pointer, int *, int *itf) {
  const char *R = "compute_add_sources_el_s3_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3)");
  if (m->fluid)
    kernel_step_call(R, m);
  else if (m->stage != 2)
    stop(R, "called outside a time step");
  if (*itf != m->nstep - m->steps) stop(R, "time step " + std::to_string(*itf) + " out of sequence");
  m->srcs_added = m->steps + 1;
}

// compute_kernels_elastic_cuda (src/gpu/compute_kernels_cuda.cu:46): the sums
// are accumulated inside the sweep at every step
void compute_kernels_elastic_cuda_(long *Mesh_pointer, realw *) {
  const char *R = "compute_kernels_elastic_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3 || (!m->F && !m->CF)) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3)");
  if (m->fluid ? m->kr_open : m->stage != 0) stop(R, "called inside a time step");
  if (m->kernel_calls >= m->steps) stop(R, "called twice in one time step");
  ++m->kernel_calls;
}

// transfer_b_fields_to_device (src/gpu/transfer_fields_cuda.cu:85): the last
// frame of the forward run (read_forward_arrays.f90); the replayed field
// starts from rest and needs none
void transfer_b_fields_to_device_(int *size, realw *, realw *, realw *, long *Mesh_pointer) {
  const char *R = "transfer_b_fields_to_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3)");
  need_size(R, *m, size);
}

// transfer_kernels_el_to_host (src/gpu/transfer_fields_cuda.cu:194): rho_kl,
// mu_kl and kappa_kl before save_adjoint_kernels.f90 scales them
void transfer_kernels_el_to_host_(long *Mesh_pointer, realw *h_rho_kl, realw *h_mu_kl, realw *h_kappa_kl,
                                  int *NSPEC_AB) {
  const char *R = "transfer_kernels_el_to_host";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3 || (!m->F && !m->CF)) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3)");
  if (*NSPEC_AB != m->nspec) stop(R, "NSPEC_AB disagrees with prepare_constants_device");
  if (m->steps != m->nstep) stop(R, "called before the last time step");
  if (m->kernel_calls != m->nstep)
    stop(R, "NTSTEP_BETWEEN_COMPUTE_KERNELS must be 1: the sums cover every time step");
  const size_t nl = static_cast<size_t>(m->nspec) * NGLL2;
  std::memcpy(h_rho_kl, m->rho_sum.data(), sizeof(realw) * nl);
  std::memcpy(h_mu_kl, m->mu_sum.data(), sizeof(realw) * nl);
  std::memcpy(h_kappa_kl, m->kappa_sum.data(), sizeof(realw) * nl);
}

// ---- CPML layer of a fluid-only mesh ----

// prepare_pml_device (src/gpu/prepare_mesh_constants_cuda.cu:843): the layer's
// profiles as the reference's GPU kernel forms them
// (Kernel_2_acoustic_impl.cu:497-505): in CPML_X_ONLY and CPML_Z_ONLY elements
// alpha = ALPHA_MAX_PML (1 - abs_normalized) and beta = alpha + 2 d0_max
// abs_normalized^2, in CPML_XZ elements alpha and beta from the stores; the
// library's CPML (the reference's CPU convolution scheme,
// pml_compute_memory_variables.f90) takes them as K = 1, d = beta - alpha
void prepare_pml_device_(long *Mesh_pointer, int *NSPEC_PML, int *NSPEC_PML_X, int *NSPEC_PML_Z, int *NSPEC_PML_XZ,
                         int *h_spec_to_pml, realw *h_abs_normalized, realw *ALPHA_MAX_PML, realw *d0_max,
                         realw *deltat, realw *h_alphax_store, realw *h_alphaz_store, realw *h_betax_store,
                         realw *h_betaz_store, int *PML_nglob_abs_acoustic_f, int *h_PML_abs_points_acoustic) {
  const char *R = "prepare_pml_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (!m->pml) stop(R, "PML_BOUNDARY_CONDITIONS is off in prepare_constants_device");
  if (m->C) stop(R, "called after the time loop started");
  const int nx = *NSPEC_PML_X, nz = *NSPEC_PML_Z, nxz = *NSPEC_PML_XZ, np = *NSPEC_PML;
  if (nx < 0 || nz < 0 || nxz < 0 || nx + nz + nxz != np)
    stop(R, "NSPEC_PML_X + NSPEC_PML_Z + NSPEC_PML_XZ must equal NSPEC_PML");
  const size_t nl = static_cast<size_t>(m->nspec) * NGLL2;
  m->pml_region.assign(m->nspec, 0);
  m->pml_K_x.assign(nl, 1.0);
  m->pml_K_z.assign(nl, 1.0);
  m->pml_d_x.assign(nl, 0.0);
  m->pml_d_z.assign(nl, 0.0);
  m->pml_alpha_x.assign(nl, 0.0);
  m->pml_alpha_z.assign(nl, 0.0);
  const float amax = *ALPHA_MAX_PML, d0 = *d0_max;
  for (int e = 0; e < m->nspec; ++e) {
    const int p = h_spec_to_pml[e];
    if (p == 0) continue;
    if (p < 0 || p > np) stop(R, "spec_to_PML out of range");
    const size_t b = static_cast<size_t>(e) * NGLL2;
    if (p <= nx + nz) {
      // one direction: x in CPML_X_ONLY elements, z in CPML_Z_ONLY ones
      const bool xdir = p <= nx;
      m->pml_region[e] = xdir ? 1 : 2;
      std::vector<double> &d = xdir ? m->pml_d_x : m->pml_d_z, &al = xdir ? m->pml_alpha_x : m->pml_alpha_z;
      for (int q = 0; q < NGLL2; ++q) {
        const float an = h_abs_normalized[static_cast<size_t>(p - 1) * NGLL2 + q];
        const float alpha = amax * (1.f - an);
        const float beta = alpha + 2.f * d0 * an * an;
        al[b + q] = alpha;
        d[b + q] = static_cast<double>(beta) - static_cast<double>(alpha);
      }
    } else {
      m->pml_region[e] = 3;
      const size_t k = static_cast<size_t>(p - nx - nz - 1) * NGLL2;
      for (int q = 0; q < NGLL2; ++q) {
        m->pml_alpha_x[b + q] = h_alphax_store[k + q];
        m->pml_alpha_z[b + q] = h_alphaz_store[k + q];
        m->pml_d_x[b + q] = static_cast<double>(h_betax_store[k + q]) - static_cast<double>(h_alphax_store[k + q]);
        m->pml_d_z[b + q] = static_cast<double>(h_betaz_store[k + q]) - static_cast<double>(h_alphaz_store[k + q]);
      }
    }
  }
  m->pml_edge.clear();
  for (int k = 0; k < *PML_nglob_abs_acoustic_f; ++k) {
    const int g = h_PML_abs_points_acoustic[k] - 1;
    if (g < 0 || g >= m->nglob) stop(R, "PML_abs_points_acoustic out of range");
    m->pml_edge.push_back(g);
  }
  m->pml_dt = *deltat;
  m->have_pml = true;
}

// pml_boundary_acoustic_cuda (src/gpu/pml_compute_cuda.cu:47): the
// zeroing of the layer's outer edge is part of the fused step
void pml_boundary_acoustic_cuda_(long *Mesh_pointer, int *, int *compute_wavefield_2) {
  const char *R = "pml_boundary_acoustic_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (!m->pml) stop(R, "the run has no CPML layer");
  fluid_phase_call(R, m, compute_wavefield_2);
}

// ---- the kernel run of a mesh with fluid elements ----

// prepare_fields_acoustic_adj_dev (src/gpu/prepare_mesh_constants_cuda.cu:442)
void prepare_fields_acoustic_adj_dev_(long *Mesh_pointer, int *APPROXIMATE_HESS_KL, int *ATTENUATION_VISCOACOUSTIC,
                                      int *NO_BACKWARD_RECONSTRUCTION) {
  const char *R = "prepare_fields_acoustic_adj_dev";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3 || !m->fluid) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3) with fluid elements");
  if (*APPROXIMATE_HESS_KL) stop(R, "APPROXIMATE_HESS_KL: the fluid Hessian is not provided");
  if (*ATTENUATION_VISCOACOUSTIC) stop(R, "viscoacoustic attenuation is not provided");
  if (*NO_BACKWARD_RECONSTRUCTION)
    stop(R, "NO_BACKWARD_RECONSTRUCTION: the forward field is replayed from device checkpoints, no frames are read");
  m->ac_adj_prepared = true;
}

// add_sources_ac_sim_2_or_3_cuda (src/gpu/compute_add_sources_viscoacoustic_cuda.cu:208):
// source_adjoint(:, NSTEP-it+1, 1) at the fluid receivers, as it is
void add_sources_ac_sim_2_or_3_cuda_(long *Mesh_pointer, int *, int *itf, int *nadj_rec_local, int *NSTEP) {
  const char *R = "add_sources_ac_sim_2_or_3_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3) unsupported(R, OTHER);
  kernel_step_call(R, m);
  if (*nadj_rec_local != m->nrec || *NSTEP != m->nstep) stop(R, "nadj_rec_local or NSTEP changed");
  if (*itf != m->nstep - m->steps) stop(R, "time step " + std::to_string(*itf) + " out of sequence");
}

// compute_add_sources_ac_s3_cuda (src/gpu/compute_add_sources_viscoacoustic_cuda.cu:91):
// the forward source of the replayed field
void compute_add_sources_ac_s3_cuda_(long *Mesh_pointer, int *, int *itf) {
  const char *R = "compute_add_sources_ac_s3_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3)");
  kernel_step_call(R, m);
  if (*itf != m->nstep - m->steps) stop(R, "time step " + std::to_string(*itf) + " out of sequence");
  m->srcs_added = m->steps + 1;
}

// compute_kernels_acoustic_cuda (src/gpu/compute_kernels_cuda.cu:92): summed in the sweep
void compute_kernels_acoustic_cuda_(long *Mesh_pointer, realw *) {
  const char *R = "compute_kernels_acoustic_cuda";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3 || !m->CF) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3) with fluid elements");
  if (m->kr_open) stop(R, "called inside a time step");
  if (m->ac_kernel_calls >= m->steps) stop(R, "called twice in one time step");
  ++m->ac_kernel_calls;
}

// transfer_b_fields_ac_to_device (src/gpu/transfer_fields_cuda.cu:248): the
// replayed field starts from rest and needs no last frame
void transfer_b_fields_ac_to_device_(int *size, realw *, realw *, realw *, long *Mesh_pointer) {
  const char *R = "transfer_b_fields_ac_to_device";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3)");
  need_ac_size(R, m, size);
}

// transfer_kernels_ac_to_host (src/gpu/transfer_fields_cuda.cu:391): rho_ac_kl
// and kappa_ac_kl with deltat and the material factors already in
// (compute_kernels.f90:426-431), zero in solid elements
void transfer_kernels_ac_to_host_(long *Mesh_pointer, realw *h_rho_ac_kl, realw *h_kappa_ac_kl, int *NSPEC_AB) {
  const char *R = "transfer_kernels_ac_to_host";
  FortranMesh *m = mesh_of(R, Mesh_pointer);
  if (m->sim_type != 3 || !m->CF) stop(R, "called outside a kernel run (SIMULATION_TYPE = 3) with fluid elements");
  if (*NSPEC_AB != m->nspec) stop(R, "NSPEC_AB disagrees with prepare_constants_device");
  if (m->steps != m->nstep) stop(R, "called before the last time step");
  if (m->ac_kernel_calls != m->nstep)
    stop(R, "NTSTEP_BETWEEN_COMPUTE_KERNELS must be 1: the sums cover every time step");
  std::memcpy(h_rho_ac_kl, m->rho_ac_kl.data(), sizeof(realw) * m->rho_ac_kl.size());
  std::memcpy(h_kappa_ac_kl, m->kappa_ac_kl.data(), sizeof(realw) * m->kappa_ac_kl.size());
}

void transfer_boun_pot_from_device_(long*, realw*, const int*) { unsupported("transfer_boun_pot_from_device", MPI); }
void transfer_asmbl_pot_to_device_(long*, realw*, const int*) { unsupported("transfer_asmbl_pot_to_device", MPI); }
void transfer_boun_accel_from_device_(long*, realw*, const int*) { unsupported("transfer_boun_accel_from_device", MPI); }
void transfer_boundary_from_device_a_(long*) { unsupported("transfer_boundary_from_device_a", MPI); }
void prepare_boundary_on_device_(long*) { unsupported("prepare_boundary_on_device", MPI); }
void transfer_boundary_to_device_a_(long*, realw*, const int*) { unsupported("transfer_boundary_to_device_a", MPI); }
void transfer_asmbl_accel_to_device_(long*, realw*, const int*, const int*, const int*, const int*) { unsupported("transfer_asmbl_accel_to_device", MPI); }
void sync_copy_from_device_(long*, int*, realw*) { unsupported("sync_copy_from_device", MPI); }
void get_max_accel_(int*, int*, long*) { unsupported("get_max_accel", DEBUG); }
void check_max_norm_displ_gpu_(int*, realw*, long*, int*) { unsupported("check_max_norm_displ_gpu", DEBUG); }
void check_max_norm_vector_(int*, realw*, int*) { unsupported("check_max_norm_vector", DEBUG); }
void check_max_norm_displ_(int*, realw*, int*) { unsupported("check_max_norm_displ", DEBUG); }
void check_max_norm_b_displ_gpu_(int*, realw*, long*, int*) { unsupported("check_max_norm_b_displ_gpu", DEBUG); }
void check_max_norm_b_accel_gpu_(int*, realw*, long*, int*) { unsupported("check_max_norm_b_accel_gpu", DEBUG); }
void check_max_norm_b_veloc_gpu_(int*, realw*, long*, int*) { unsupported("check_max_norm_b_veloc_gpu", DEBUG); }
void check_max_norm_b_displ_(int*, realw*, int*) { unsupported("check_max_norm_b_displ", DEBUG); }
void check_max_norm_b_accel_(int*, realw*, int*) { unsupported("check_max_norm_b_accel", DEBUG); }
void check_error_vectors_(int*, realw*, realw*) { unsupported("check_error_vectors", DEBUG); }
void compute_add_moving_sources_ac_cuda_(long*, int*, int*, int*, int*, int*) { unsupported("compute_add_moving_sources_ac_cuda", OTHER); }
void compute_kernels_hess_cuda_(long*, int*, int*) { unsupported("compute_kernels_hess_cuda", OTHER); }
void prepare_moving_sources_cuda_(long*, int*, int*, realw*, int*, int*, realw*) { unsupported("prepare_moving_sources_cuda", OTHER); }
void prepare_arrays_gpu_(long*, realw*, realw*, realw*, realw*, realw*, realw*, int*, int*, realw*) { unsupported("prepare_arrays_gpu", OTHER); }
void compute_smooth_(long*, realw*, realw*, realw*, realw*, const int*) { unsupported("compute_smooth", OTHER); }
void get_smooth_(long*, realw*) { unsupported("get_smooth", OTHER); }
void transfer_b_fields_from_device_(int*, realw*, realw*, realw*, long*) { unsupported("transfer_b_fields_from_device", KERNEL_RUN); }
void transfer_b_accel_from_device_(int*, realw*, long*) { unsupported("transfer_b_accel_from_device", KERNEL_RUN); }
void transfer_b_displ_from_device_(int*, realw*, long*) { unsupported("transfer_b_displ_from_device", KERNEL_RUN); }
void transfer_b_fields_ac_from_device_(int*, realw*, realw*, realw*, long*) { unsupported("transfer_b_fields_ac_from_device", KERNEL_RUN); }
void transfer_b_potential_ac_from_device_(int*, realw*, long*) { unsupported("transfer_b_potential_ac_from_device", KERNEL_RUN); }
void transfer_b_potential_ac_to_device_(int*, realw*, long*) { unsupported("transfer_b_potential_ac_to_device", KERNEL_RUN); }
void transfer_b_dot_dot_from_device_(int*, realw*, long*) { unsupported("transfer_b_dot_dot_from_device", KERNEL_RUN); }
void transfer_kernels_hess_el_tohost_(long*, realw*, int*) { unsupported("transfer_kernels_hess_el_tohost", OTHER); }
void transfer_kernels_hess_ac_tohost_(long*, realw*, int*) { unsupported("transfer_kernels_hess_ac_tohost", OTHER); }
void transfer_viscoacoustic_b_var_to_device_(int*, realw*, realw*, long*) { unsupported("transfer_viscoacoustic_b_var_to_device", KERNEL_RUN); }
void transfer_viscoacoustic_var_from_device_(int*, realw*, realw*, long*) { unsupported("transfer_viscoacoustic_var_from_device", KERNEL_RUN); }
void transfer_viscoelastic_b_var_to_device_(int*, realw*, realw*, realw*, realw*, realw*, realw*, long*) { unsupported("transfer_viscoelastic_b_var_to_device", KERNEL_RUN); }
void transfer_viscoelastic_var_from_device_(int*, realw*, realw*, realw*, realw*, realw*, realw*, long*) { unsupported("transfer_viscoelastic_var_from_device", KERNEL_RUN); }
void transfer_async_pot_ac_from_device_(realw*, long*) { unsupported("transfer_async_pot_ac_from_device", MPI); }
void transfer_async_pot_ac_to_device_(realw*, long*) { unsupported("transfer_async_pot_ac_to_device", MPI); }
void transfer_compute_kernel_answers_from_device_(long*, realw*, int*, realw*, int*, realw*, int*) { unsupported("transfer_compute_kernel_answers_from_device", KERNEL_RUN); }
void transfer_compute_kernel_fields_from_device_(long*, realw*, int*, realw*, int*, realw*, realw*, realw*, realw*, realw*, int*, realw*, realw*, realw*, realw*, realw*, int*, realw*, int*, realw*, int*, realw*, int*, realw*, realw*, int*) { unsupported("transfer_compute_kernel_fields_from_device", KERNEL_RUN); }
void kernel_3_b_cuda_(long*, realw*, realw*) { unsupported("kernel_3_b_cuda", KERNEL_RUN); }

}  // extern "C"
