// Inverse mass matrix without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need
// the inverse mass matrix: a host framework that owns every device
// allocation through its own pool and forbids plugins from calling
// cudaMalloc, or a real-time loop that must not touch the allocator (a
// cudaMalloc can synchronise the device and take milliseconds).  This entry
// point takes the caller's device inputs and output and keeps its only
// scratch -- the FP64 accumulation buffer of the assembled mass and one
// error word -- in fixed, file-scope device arrays that every GPU loading
// this library holds until the process exits.
//
// Set-up: the first call on a device looks up the array's device address
// with cudaGetSymbolAddress (the array's name is only a host-side stand-in in
// host code) and caches it for that device; make that first call before any
// stream capture.  A device reset (cudaDeviceReset) after that first call is
// not supported: the cached address would belong to the torn-down context.
// The scratch is shared by every call on a device and keeps the last call's
// contents: each call clears the part it uses first, and calls that overlap
// on the GPU (different streams, or threads calling concurrently) race on it.
// A point index outside [0, npoints) is never written through: the kernel
// skips it, counts it in the error word, and the call then fills the whole
// output with NaN so that the bad input cannot pass unnoticed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../../include/specfem_b200.h"

namespace {

__device__ __align__(256) double g_mass_scratch[SFB_NOALLOC_MAX_DOFS];
// Out-of-range point indices seen by the current call (cleared by k_clear).
__device__ unsigned int g_bad_index_count;

constexpr int kMaxDevices = 64;
double *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;
thread_local std::string g_noalloc_error;

struct Weights {
  float w[8];
};

__global__ void k_clear(double *scratch, int n) {
  if (blockIdx.x == 0 && threadIdx.x == 0) g_bad_index_count = 0u;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) scratch[i] = 0.0;
}

// Element mass contributions (reference: compute_mass_matrix.tpp:80-113 and
// the Stacey term of stacey.tpp:644-677, velocity replaced by -dt/2),
// accumulated in FP64.
__global__ void k_mass_noalloc(int medium, int ngll, int nelem, const int *iglob, const float *jac,
                               const float *m0, const float *m1, const float *m2, const uint8_t *bnd,
                               const float *bnx, const float *bnz, const float *bw, float dt, Weights W,
                               int npoints, double *scratch) {
  const int nn = ngll * ngll;
  const int nc = (medium == SFB_MEDIUM_ELASTIC_PSV) ? 2 : 1;
  const size_t total = static_cast<size_t>(nelem) * nn;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(t % nn);
    const int iz = k / ngll, ix = k % ngll;
    float base;
    if (medium == SFB_MEDIUM_ELASTIC_PSV) base = m2[t];      // rho
    else if (medium == SFB_MEDIUM_ELASTIC_SH) base = m1[t];  // rho
    else base = 1.0f / m1[t];                               // 1 / kappa
    float mm[2];
    for (int c = 0; c < nc; ++c) mm[c] = base * (W.w[ix] * W.w[iz] * jac[t]);
    if (bnd && (bnd[t] & 1)) {
      const float v = -1.0f * dt * 0.5f;
      const float nx = bnx[t], nz = bnz[t], we = bw[t];
      const float jac1d = sqrtf(nx * nx + nz * nz);
      if (medium == SFB_MEDIUM_ELASTIC_PSV) {
        const float l2m = m0[t] + static_cast<float>(4.0 / 3.0) * m1[t];
        const float rho_vp = sqrtf(l2m / m2[t]) * m2[t];
        const float rho_vs = sqrtf(m2[t] * m1[t]);
        const float vn = v * nx + v * nz;
        const float dn[2] = {nx, nz};
        for (int c = 0; c < 2; ++c) {
          const float fac = ((vn * dn[c] / (jac1d * jac1d)) * (rho_vp - rho_vs)) + v * rho_vs;
          mm[c] += -1.0f * fac * jac1d * we;
        }
      } else if (medium == SFB_MEDIUM_ELASTIC_SH) {
        mm[0] += -1.0f * (we * jac1d) * sqrtf(m1[t] * m0[t]) * v;
      } else {
        mm[0] += -1.0f * (we * jac1d) * sqrtf(m0[t] * (1.0f / m1[t])) * v;
      }
    }
    const int g = iglob[t];
    if (g < 0 || g >= npoints) {  // never write outside the caller's points
      atomicAdd(&g_bad_index_count, 1u);
      continue;
    }
    for (int c = 0; c < nc; ++c) atomicAdd(scratch + static_cast<size_t>(g) * nc + c, static_cast<double>(mm[c]));
  }
}

// A call that met an out-of-range index returns NaN everywhere.
__global__ void k_invert_noalloc(const double *scratch, float *minv, int n) {
  const bool bad = g_bad_index_count != 0u;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    minv[i] = bad ? __int_as_float(0x7fc00000) : static_cast<float>(1.0 / scratch[i]);
}

int fail(int code, const std::string &msg) {
  g_noalloc_error = msg;
  return code;
}

}  // namespace

SFB_API const char *sfb_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

SFB_API int sfb_assemble_inverse_mass_noalloc(int medium, int ngll, int nelem, int npoints, const int *iglob,
                                             const float *jacobian, const float *mat0, const float *mat1,
                                             const float *mat2, const uint8_t *bnd, const float *bnd_nx,
                                             const float *bnd_nz, const float *bnd_w, const double *wgll,
                                             double dt, float *minv, void *stream) {
  if (medium != SFB_MEDIUM_ELASTIC_PSV && medium != SFB_MEDIUM_ELASTIC_SH && medium != SFB_MEDIUM_ACOUSTIC)
    return fail(SFB_E_INVALID, "unsupported medium tag");
  if (ngll < 2 || ngll > 8) return fail(SFB_E_INVALID, "ngll must be in [2, 8]");
  if (nelem < 0 || npoints < 0) return fail(SFB_E_INVALID, "negative size");
  const int nc = (medium == SFB_MEDIUM_ELASTIC_PSV) ? 2 : 1;
  const long long ndof = static_cast<long long>(npoints) * nc;
  if (ndof > SFB_NOALLOC_MAX_DOFS)
    return fail(SFB_E_INVALID, "npoints * components = " + std::to_string(ndof) +
                                   " exceeds the no-allocation scratch of " +
                                   std::to_string(SFB_NOALLOC_MAX_DOFS) + " degrees of freedom");
  if (!iglob || !jacobian || !mat0 || !mat1 || !minv || !wgll)
    return fail(SFB_E_INVALID, "null input or output pointer");
  if (medium == SFB_MEDIUM_ELASTIC_PSV && !mat2) return fail(SFB_E_INVALID, "P-SV needs mat2 (rho)");
  if (bnd && (!bnd_nx || !bnd_nz || !bnd_w)) return fail(SFB_E_INVALID, "boundary arrays incomplete");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SFB_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(SFB_E_INVALID, "device index out of range");
  double *scratch;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_mass_scratch);
      if (e != cudaSuccess) return fail(SFB_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    scratch = g_scratch_ptr[dev];
  }
  if (ndof == 0) return SFB_OK;
  Weights W{};
  for (int i = 0; i < ngll; ++i) W.w[i] = static_cast<float>(wgll[i]);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int block = 256;
  const int gclear = static_cast<int>(std::min<long long>((ndof + block - 1) / block, 4096));
  k_clear<<<gclear, block, 0, s>>>(scratch, static_cast<int>(ndof));
  const long long nloc = static_cast<long long>(nelem) * ngll * ngll;
  const int gmass = static_cast<int>(std::max<long long>(1, std::min<long long>((nloc + block - 1) / block, 4096)));
  k_mass_noalloc<<<gmass, block, 0, s>>>(medium, ngll, nelem, iglob, jacobian, mat0, mat1, mat2, bnd, bnd_nx,
                                         bnd_nz, bnd_w, static_cast<float>(dt), W, npoints, scratch);
  k_invert_noalloc<<<gclear, block, 0, s>>>(scratch, minv, static_cast<int>(ndof));
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SFB_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return SFB_OK;
}
