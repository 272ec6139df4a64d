// Gaussian smoothing of sensitivity kernels (the post-gradient step of an
// inversion): the computation of src/tomography/postprocess_sensitivity_kernels/
// smooth_sem.F90:63-467 (CPU) and of src/gpu/kernels/process_smooth.cu:37-116.
//
// Every element GLL point i gets
//   out_k(i) = sum_j G(i,j) J_j w_j f_k(j) / sum_j G(i,j) J_j w_j,
//   G = exp(-(x_i - x_j)^2 / (2 sigma_h^2) - (z_i - z_j)^2 / (2 sigma_v^2)),
// the sums running over every element GLL point j (w_j = wxgll * wzgll of
// its position, J_j its Jacobian).  The reference's CPU program sums over all
// pairs; this kernel sums over the points within `cutoff` standard
// deviations (an ellipse), so the weight left out is below exp(-cutoff^2/2)
// of the nearest one.  Points are counting-sorted into cells of `cutoff`
// standard deviations in scaled coordinates (x / sigma_h, z / sigma_v); one
// thread per target point walks the 3 x 3 cells around it and accumulates in
// double.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "sf2d_b200.h"
#include "sf2d_runtime.h"

namespace {

struct SmoothArgs {
  const float2 *pos;      // sorted source points, scaled coordinates
  const float *wj;        // J * w of each sorted source point
  const float *val;       // nfields values per sorted source point [field][point]
  const int *cell_start;  // ncx * ncz + 1 offsets into the sorted points
  const float2 *tpos;     // target points (element GLL points, original order), scaled
  float *out;             // nfields * ntarget
  int ntarget, nsrc, nfields, ncx, ncz;
  float x0, z0, cell, cut2;
};

__global__ void k_smooth(const SmoothArgs A) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.ntarget) return;
  const float2 p = A.tpos[t];
  // the host's cell formula (an IEEE division), so a target sits in the cell the
  // host sorted it into and the 3 x 3 window covers the cutoff ellipse
  const int cx = min(A.ncx - 1, max(0, static_cast<int>((p.x - A.x0) / A.cell)));
  const int cz = min(A.ncz - 1, max(0, static_cast<int>((p.y - A.z0) / A.cell)));
  double norm = 0.0;
  double acc[SF2D_SMOOTH_MAX_FIELDS] = {};
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = cz + dz;
    if (z < 0 || z >= A.ncz) continue;
    const int c0 = max(cx - 1, 0), c1 = min(cx + 1, A.ncx - 1);
    // cells of one row of the grid are contiguous in the sorted order
    const int b = A.cell_start[z * A.ncx + c0], e = A.cell_start[z * A.ncx + c1 + 1];
    for (int j = b; j < e; ++j) {
      const float2 q = A.pos[j];
      const float ddx = p.x - q.x, ddz = p.y - q.y;
      const float r2 = ddx * ddx + ddz * ddz;
      if (r2 > A.cut2) continue;
      const double w = static_cast<double>(expf(-0.5f * r2)) * static_cast<double>(A.wj[j]);
      norm += w;
      for (int k = 0; k < A.nfields && k < SF2D_SMOOTH_MAX_FIELDS; ++k)
        acc[k] += w * static_cast<double>(A.val[static_cast<size_t>(k) * A.nsrc + j]);
    }
  }
  for (int k = 0; k < A.nfields && k < SF2D_SMOOTH_MAX_FIELDS; ++k)
    A.out[static_cast<size_t>(k) * A.ntarget + t] = static_cast<float>(acc[k] / norm);
}

}  // namespace

extern "C" int sf2d_smooth(int nspec, const float *x, const float *z, const float *jacobian, const float *wgll_sq,
                           int nfields, const float *fields, float sigma_h, float sigma_v, float cutoff, float *out,
                           void *stream_v) {
  if (nspec < 1 || !x || !z || !jacobian || !wgll_sq || !fields || !out)
    return fail(SF2D_ERR_INVALID, "sf2d_smooth: null argument");
  if (nfields < 1 || nfields > SF2D_SMOOTH_MAX_FIELDS)
    return fail(SF2D_ERR_INVALID, "sf2d_smooth: 1 to SF2D_SMOOTH_MAX_FIELDS fields per call");
  if (!(sigma_h > 0.f) || !(sigma_v > 0.f) || !(cutoff > 0.f))
    return fail(SF2D_ERR_INVALID, "sf2d_smooth: sigma_h, sigma_v and cutoff must be positive");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
  const size_t n = static_cast<size_t>(nspec) * 25;
  if (n > static_cast<size_t>(INT32_MAX)) return fail(SF2D_ERR_INVALID, "sf2d_smooth: too many points");
  // scaled coordinates and the cell grid
  std::vector<float2> sp(n);
  float xmin = INFINITY, xmax = -INFINITY, zmin = INFINITY, zmax = -INFINITY;
  for (size_t p = 0; p < n; ++p) {
    sp[p] = make_float2(x[p] / sigma_h, z[p] / sigma_v);
    xmin = std::min(xmin, sp[p].x);
    xmax = std::max(xmax, sp[p].x);
    zmin = std::min(zmin, sp[p].y);
    zmax = std::max(zmax, sp[p].y);
  }
  const float cell = cutoff;
  const long long ncx = std::max(1LL, static_cast<long long>((xmax - xmin) / cell) + 1);
  const long long ncz = std::max(1LL, static_cast<long long>((zmax - zmin) / cell) + 1);
  if (ncx * ncz > (1LL << 28)) return fail(SF2D_ERR_INVALID, "sf2d_smooth: sigma too small for the mesh extent");
  std::vector<int> cell_of(n), start(static_cast<size_t>(ncx * ncz) + 1, 0);
  for (size_t p = 0; p < n; ++p) {
    const int cx = std::min<long long>(ncx - 1, static_cast<long long>((sp[p].x - xmin) / cell));
    const int cz = std::min<long long>(ncz - 1, static_cast<long long>((sp[p].y - zmin) / cell));
    cell_of[p] = cz * static_cast<int>(ncx) + cx;
    ++start[cell_of[p] + 1];
  }
  for (size_t c = 0; c + 1 < start.size(); ++c) start[c + 1] += start[c];
  std::vector<int> fill(start.begin(), start.end() - 1);
  std::vector<float2> spos(n);
  std::vector<float> swj(n), sval(n * nfields);
  for (size_t p = 0; p < n; ++p) {
    const int k = fill[cell_of[p]]++;
    spos[k] = sp[p];
    swj[k] = jacobian[p] * wgll_sq[p % 25];
    for (int f = 0; f < nfields; ++f) sval[static_cast<size_t>(f) * n + k] = fields[static_cast<size_t>(f) * n + p];
  }
  // device buffers, one allocation
  const size_t bytes = n * sizeof(float2) * 2 + n * sizeof(float) * (1 + 2 * nfields) + start.size() * sizeof(int);
  char *buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, bytes);
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? SF2D_ERR_OOM : SF2D_ERR_CUDA, "sf2d_smooth: cudaMalloc");
  struct Free {
    char *p;
    ~Free() { cudaFree(p); }
  } guard{buf};
  SmoothArgs A{};
  float2 *d_pos = reinterpret_cast<float2 *>(buf);
  float2 *d_tpos = d_pos + n;
  float *d_wj = reinterpret_cast<float *>(d_tpos + n);
  float *d_val = d_wj + n;
  float *d_out = d_val + n * nfields;
  int *d_start = reinterpret_cast<int *>(d_out + n * nfields);
  SF2D_CUDA(cudaMemcpyAsync(d_pos, spos.data(), n * sizeof(float2), cudaMemcpyHostToDevice, stream));
  SF2D_CUDA(cudaMemcpyAsync(d_tpos, sp.data(), n * sizeof(float2), cudaMemcpyHostToDevice, stream));
  SF2D_CUDA(cudaMemcpyAsync(d_wj, swj.data(), n * sizeof(float), cudaMemcpyHostToDevice, stream));
  SF2D_CUDA(cudaMemcpyAsync(d_val, sval.data(), n * nfields * sizeof(float), cudaMemcpyHostToDevice, stream));
  SF2D_CUDA(cudaMemcpyAsync(d_start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
  A.pos = d_pos;
  A.wj = d_wj;
  A.val = d_val;
  A.cell_start = d_start;
  A.tpos = d_tpos;
  A.out = d_out;
  A.ntarget = static_cast<int>(n);
  A.nsrc = static_cast<int>(n);
  A.nfields = nfields;
  A.ncx = static_cast<int>(ncx);
  A.ncz = static_cast<int>(ncz);
  A.x0 = xmin;
  A.z0 = zmin;
  A.cell = cell;
  A.cut2 = cutoff * cutoff;
  k_smooth<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(A);
  SF2D_CUDA(cudaGetLastError());
  SF2D_CUDA(cudaMemcpyAsync(out, d_out, n * nfields * sizeof(float), cudaMemcpyDeviceToHost, stream));
  SF2D_CUDA(cudaStreamSynchronize(stream));
  return SF2D_OK;
}
