// Per-member maximum displacement norm that allocates no device memory.
//
// The stability check of the time loop (check_stability.F90, through
// get_norm_elastic_from_device in src/gpu/check_fields_cuda.cu:358) reduces
// |u| over all points every few hundred steps.  The reference allocates and
// frees its per-block maxima on every call; sf2d_get_norm keeps a one-word
// buffer in the solver instead.  Neither suits a caller that owns its device
// memory itself:
//
//  * a host code that plans all of its device memory before the time loop
//    (the reference's Fortran side, or a framework whose pooling allocator
//    already holds the GPU's free memory) cannot have a library make device
//    allocations of its own in the middle of the run: a cudaMalloc there can
//    fail for want of memory the pool holds, and cudaFree waits for the
//    whole device, stalling the time steps queued behind the check;
//  * a batch of independent simulations packed into one field (one member
//    per shot or model) needs the maximum per member, so that the member
//    that went unstable can be named, and the batch may be held by a caller
//    that never created a solver here.
//
// sf2d_member_norms_noalloc serves both: it reads a caller-owned device
// field and keeps its intermediates in a static device array of fixed size
// (SF2D_NOALLOC_MAX_MEMBERS members), so it allocates nothing.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "sf2d_b200.h"

namespace sf2d {
int fail(int code, const std::string &msg);
}  // namespace sf2d

namespace {

constexpr int kMaxMembers = SF2D_NOALLOC_MAX_MEMBERS;
constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 8;  // 8 CTAs of 256 threads per SM

// Scratch words: the per-member maxima (float bits as 32-bit words, two per
// 64-bit word) followed by the member offsets copied from the host.
constexpr int kMaxWords = kMaxMembers / 2;
constexpr int kScratchWords = kMaxWords + kMaxMembers + 1;
static_assert(kMaxMembers % 2 == 0, "maxima must fill whole 64-bit words");

// The only device memory this file uses besides the caller's field
// (49,160 bytes).  Every call on a device shares it: overlapping calls on
// one device race on it.
static __device__ __align__(256) unsigned long long g_norm_scratch[kScratchWords];

typedef CUresult (*AddressRangeFn)(CUdeviceptr *base, size_t *size, CUdeviceptr ptr);

std::mutex g_setup_mutex;
unsigned long long *g_scratch[kMaxDevices] = {};
AddressRangeFn g_address_range = nullptr;

#define NA_CUDA(call)                                                                               \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess) return sf2d::fail(SF2D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Looks up, once per device with that device current, the address of the
// scratch array in that device's copy of this module, and the driver's
// allocation-range query used to check the caller's field.
int scratch_of_current_device(unsigned long long **scratch) {
  using sf2d::fail;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SF2D_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return fail(SF2D_ERR_INVALID, "device ordinal " + std::to_string(dev) + " beyond the " +
                                      std::to_string(kMaxDevices) + " devices this entry point supports");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_norm_scratch);
    if (e != cudaSuccess)
      return fail(SF2D_ERR_CUDA, std::string("cudaGetSymbolAddress of the norm scratch: ") + cudaGetErrorString(e));
    if (!g_address_range) {
      void *fn = nullptr;
      cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
      e = cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &fn, 12000, cudaEnableDefault, &q);
      if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
        return fail(SF2D_ERR_CUDA, "driver entry point cuMemGetAddressRange not found");
      g_address_range = reinterpret_cast<AddressRangeFn>(fn);
    }
    g_scratch[dev] = static_cast<unsigned long long *>(p);
  }
  *scratch = g_scratch[dev];
  return SF2D_OK;
}

// Block b covers the points [offsets[0] + b*chunk, +chunk) of the members'
// union; each thread walks its strided share of them in increasing order and
// moves to the next member when a point crosses that member's end offset.
// The norm is sqrtf(ux*ux + uz*uz) and a NaN counts as +inf, as in
// sf2d_get_norm, so that a blown-up member still stands out.
__global__ void __launch_bounds__(kThreads)
k_member_max_norm(const float2 *__restrict__ u, const long long *__restrict__ offsets, int nmembers,
                  long long chunk, unsigned int *__restrict__ maxbits) {
  const long long first = offsets[0];
  const long long last = offsets[nmembers];
  const long long begin = first + static_cast<long long>(blockIdx.x) * chunk;
  const long long end = begin + chunk < last ? begin + chunk : last;
  if (begin >= end) return;  // whole block: no warp below is split by it

  // the member holding `begin`: the largest m < nmembers with offsets[m] <= begin
  int lo = 0, hi = nmembers - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (offsets[mid] <= begin) lo = mid;
    else hi = mid - 1;
  }
  int m = lo;
  long long next = offsets[m + 1];  // > begin, and m + 1 <= nmembers
  float mx = 0.f;
  for (long long d = begin + threadIdx.x; d < end; d += blockDim.x) {
    while (d >= next) {  // d < last = offsets[nmembers], so m + 1 stays <= nmembers
      if (mx > 0.f) atomicMax(&maxbits[m], __float_as_uint(mx));
      mx = 0.f;
      ++m;
      next = offsets[m + 1];
    }
    const float2 x = u[d];
    const float nn = sqrtf(x.x * x.x + x.y * x.y);
    mx = (nn == nn) ? fmaxf(mx, nn) : __int_as_float(0x7f800000);
  }
  // Non-negative floats order like their bit patterns, +inf above all finite values.
  const unsigned int bits = __float_as_uint(mx);
  const int m0 = __shfl_sync(0xffffffffu, m, 0);
  if (__all_sync(0xffffffffu, m == m0)) {
    const unsigned int w = __reduce_max_sync(0xffffffffu, bits);
    if ((threadIdx.x & 31) == 0 && w != 0u) atomicMax(&maxbits[m0], w);
  } else if (bits != 0u) {
    atomicMax(&maxbits[m], bits);
  }
}

}  // namespace

extern "C" int sf2d_member_norms_noalloc(const float *d_field, const int64_t *offsets, int nmembers,
                                         float *max_norm, void *stream) {
  using sf2d::fail;
  if (!d_field || !offsets || !max_norm) return fail(SF2D_ERR_INVALID, "null argument");
  if (nmembers < 1 || nmembers > kMaxMembers)
    return fail(SF2D_ERR_INVALID, "nmembers = " + std::to_string(nmembers) + " outside [1, " +
                                      std::to_string(kMaxMembers) + "], the size of the static scratch");
  if (reinterpret_cast<uintptr_t>(d_field) % 8 != 0)
    return fail(SF2D_ERR_INVALID, "field must be 8-byte aligned (ux, uz pairs)");
  if (offsets[0] < 0) return fail(SF2D_ERR_INVALID, "negative member offset");
  for (int m = 0; m < nmembers; ++m)
    if (offsets[m + 1] < offsets[m])
      return fail(SF2D_ERR_INVALID, "member offsets decrease at member " + std::to_string(m));

  unsigned long long *scratch = nullptr;
  if (int rc = scratch_of_current_device(&scratch)) return rc;

  // The points read must lie inside the allocation holding the field.
  const long long npoints = offsets[nmembers] - offsets[0];
  if (npoints > 0) {
    CUdeviceptr base = 0;
    size_t size = 0;
    if (g_address_range(&base, &size, reinterpret_cast<CUdeviceptr>(d_field)) != CUDA_SUCCESS)
      return fail(SF2D_ERR_INVALID, "field pointer is not device memory");
    // the allocation must live on the current device (a peer's memory passes the range query)
    cudaPointerAttributes attr{};
    int dev = -1;
    if (cudaPointerGetAttributes(&attr, d_field) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
        attr.type != cudaMemoryTypeDevice || attr.device != dev) {
      cudaGetLastError();
      return fail(SF2D_ERR_INVALID, "field pointer is not device memory of the current device");
    }
    // bounds in float2 units before any address is formed: offsets (>= 0, increasing) must stay
    // within the entries between d_field and the end of its allocation
    const unsigned long long f = reinterpret_cast<uintptr_t>(d_field);
    const unsigned long long b = static_cast<unsigned long long>(base);
    if (f < b || f >= b + size) return fail(SF2D_ERR_INVALID, "field pointer outside its allocation");
    const unsigned long long room = (b + size - f) / 8;
    if (static_cast<unsigned long long>(offsets[nmembers]) > room)
      return fail(SF2D_ERR_INVALID, "member offsets reach past the field's allocation");
  }

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned int *maxbits = reinterpret_cast<unsigned int *>(scratch);
  long long *d_offsets = reinterpret_cast<long long *>(scratch + kMaxWords);
  // The maxima start at zero on every call; the offsets are overwritten.
  NA_CUDA(cudaMemsetAsync(maxbits, 0, sizeof(unsigned int) * nmembers, s));
  NA_CUDA(cudaMemcpyAsync(d_offsets, offsets, sizeof(long long) * (nmembers + 1), cudaMemcpyHostToDevice, s));
  if (npoints > 0) {
    long long blocks = (npoints + kThreads - 1) / kThreads;
    if (blocks > kMaxBlocks) blocks = kMaxBlocks;
    long long chunk = (npoints + blocks - 1) / blocks;
    chunk = (chunk + kThreads - 1) / kThreads * kThreads;
    blocks = (npoints + chunk - 1) / chunk;
    k_member_max_norm<<<static_cast<unsigned int>(blocks), kThreads, 0, s>>>(
        reinterpret_cast<const float2 *>(d_field), d_offsets, nmembers, chunk, maxbits);
    NA_CUDA(cudaGetLastError());
  }
  // The maxima are float bit patterns: copy them straight into the floats.
  NA_CUDA(cudaMemcpyAsync(max_norm, maxbits, sizeof(unsigned int) * nmembers, cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaStreamSynchronize(s));
  return SF2D_OK;
}
