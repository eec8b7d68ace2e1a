// sm_100a kernels of the SEM time-marching path.  See kernels.cuh for the
// HBM layout.  Reference operation order is kept so that results track the
// reference's FP32 arithmetic:
//   gradient   include/algorithms/gradient.hpp:78-98
//   stress     include/medium/dim2/elastic/isotropic/stress.hpp:14-85,
//              include/medium/dim2/acoustic/isotropic/stress.hpp:15-31
//   F = J T dxi/dx   core/specfem/point/stress.hpp:123-137
//   divergence include/algorithms/divergence.hpp:83-99 (then * -1)
//   Stacey     include/boundary_conditions/stacey/stacey.tpp:41-212
//   free surface include/boundary_conditions/dirichlet/dirichlet.hpp:19-43
#include "kernels.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>

namespace sfb {
namespace dev {

// GLL tables, one bank per NGLL (N = 2..8): a context writes only its own
// NGLL's bank, so contexts of different NGLL in one process never see each
// other's tables (contexts of the same NGLL write identical values).
//   hprime[i*N + j] = l_j'(xi_i); hprime_wgll[ix*N + l] = hprime[l*N + ix] * w[l]
constexpr int kQBanks = 7;
__constant__ real c_hp_bank[kQBanks][64];
__constant__ real c_hpw_bank[kQBanks][64];
__constant__ real c_w_bank[kQBanks][8];
#ifndef SFB_FP64
// the same tables as (v, v) pairs for the packed two-shot arithmetic
__constant__ float2 c_hp2_bank[kQBanks][64];
__constant__ float2 c_hpw2_bank[kQBanks][64];
__constant__ float2 c_w2_bank[kQBanks][8];
#endif
// accessors: the bank of the NGLL `N` in scope at the use
#define C_HP(i) c_hp_bank[(N) - 2][i]
#define C_HPW(i) c_hpw_bank[(N) - 2][i]
#define C_W(i) c_w_bank[(N) - 2][i]
#define C_HP2(i) c_hp2_bank[(N) - 2][i]
#define C_HPW2(i) c_hpw2_bank[(N) - 2][i]
#define C_W2(i) c_w2_bank[(N) - 2][i]

void set_quadrature(int n, const real *hp, const real *w) {
  real hpw[64];
  for (int ix = 0; ix < n; ++ix)
    for (int l = 0; l < n; ++l) hpw[ix * n + l] = hp[l * n + ix] * w[l];
  const size_t b = static_cast<size_t>(n - 2);
  cudaMemcpyToSymbol(c_hp_bank, hp, sizeof(real) * n * n, b * 64 * sizeof(real));
  cudaMemcpyToSymbol(c_hpw_bank, hpw, sizeof(real) * n * n, b * 64 * sizeof(real));
  cudaMemcpyToSymbol(c_w_bank, w, sizeof(real) * n, b * 8 * sizeof(real));
#ifndef SFB_FP64
  float2 hp2[64], hpw2[64], w2[8];
  for (int k = 0; k < n * n; ++k) {
    hp2[k] = make_float2(hp[k], hp[k]);
    hpw2[k] = make_float2(hpw[k], hpw[k]);
  }
  for (int k = 0; k < n; ++k) w2[k] = make_float2(w[k], w[k]);
  cudaMemcpyToSymbol(c_hp2_bank, hp2, sizeof(float2) * n * n, b * 64 * sizeof(float2));
  cudaMemcpyToSymbol(c_hpw2_bank, hpw2, sizeof(float2) * n * n, b * 64 * sizeof(float2));
  cudaMemcpyToSymbol(c_w2_bank, w2, sizeof(float2) * n, b * 8 * sizeof(float2));
#endif
}

namespace {

template <int NC> struct Vec;
template <> struct Vec<1> {
  using T = real;
  __device__ static T zero() { return 0; }
};
template <> struct Vec<2> {
  using T = real2;
  __device__ static T zero() { return T{0, 0}; }
};

__device__ __forceinline__ real comp(real v, int) { return v; }
__device__ __forceinline__ real comp(real2 v, int c) { return c == 0 ? v.x : v.y; }
__device__ __forceinline__ void set_comp(real &v, int, real x) { v = x; }
__device__ __forceinline__ void set_comp(real2 &v, int c, real x) {
  if (c == 0) v.x = x; else v.y = x;
}

// Vector reduction into global memory (RED.E.ADD.F32x2 on sm_90+; FP64:
// one atomic per component).
__device__ __forceinline__ void red_add(real *p, real v) { atomicAdd(p, v); }
#ifdef SFB_FP64
__device__ __forceinline__ void red_add(real2 *p, real2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}
#else
__device__ __forceinline__ void red_add(float2 *p, float2 v) { atomicAdd(p, v); }
#endif

// The reference's constants are type_real (FP32): 4/3 and 1/3 rounded to
// FP32, kept so in the FP64 build, which computes the same discrete problem.
constexpr real kFourThirds = static_cast<real>(static_cast<float>(4.0 / 3.0));
constexpr real kOneThird = static_cast<real>(static_cast<float>(1.0 / 3.0));

// Square root in the working precision.
__device__ __forceinline__ float msqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double msqrt(double x) { return sqrt(x); }
// A point index held in a `real` word of a packed static block: its int bits
// (FP32) or its value (FP64 build).
__device__ __forceinline__ int pack_index(float v) { return __float_as_int(v); }
__device__ __forceinline__ int pack_index(double v) { return static_cast<int>(v); }

// Stacey traction added to `acc` for velocity `vel` (stacey.tpp:41-75 P-SV,
// :125-145 SH, :178-212 acoustic).
template <int MED>
__device__ __forceinline__ void stacey(real m0, real m1, real m2, real nx, real nz,
                                       real we, const real *vel, real *acc) {
  const real jac1d = msqrt(nx * nx + nz * nz);
  if (MED == MED_PSV) {
    const real kappa = m0, mu = m1, rho = m2;
    const real l2m = kappa + kFourThirds * mu;
    const real rho_vp = msqrt(l2m / rho) * rho;
    const real rho_vs = msqrt(rho * mu);
    const real vn = vel[0] * nx + vel[1] * nz;
    const real dn[2] = {nx, nz};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const real fac = ((vn * dn[c] / (jac1d * jac1d)) * (rho_vp - rho_vs)) + vel[c] * rho_vs;
      acc[c] += static_cast<real>(-1) * fac * jac1d * we;
    }
  } else if (MED == MED_SH) {
    const real mu = m0, rho = m1;
    const real rho_vs = msqrt(rho * mu);
    const real fac = we * jac1d;
    acc[0] += static_cast<real>(-1) * fac * rho_vs * vel[0];
  } else {
    const real rho_inv = m0, kappa = m1;
    const real rvi = msqrt(rho_inv * (static_cast<real>(1) / kappa));
    const real fac = we * jac1d;
    acc[0] += static_cast<real>(-1) * fac * rvi * vel[0];
  }
}

// ---------------------------------------------------------------------------
// Bulk async copy (cp.async.bulk, no multicast) and mbarrier helpers.  Every
// mbarrier wait is bounded; on expiry the kernel records kWaitTimeout in
// st.err and the CTA returns.
// ---------------------------------------------------------------------------
constexpr int kWaitTimeout = 1;
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait (by default 2^32 cycles, about 2 s at 2 GHz).  Returns false
// on expiry.
constexpr long long kWaitLimit = 1LL << 32;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long limit = kWaitLimit) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}

// Per-thread asynchronous global -> shared copies (cp.async, no multicast).
// A thread may read back what it copied itself after cp.async.wait_*; other
// threads' copies need a barrier after that wait as well.
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
  static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async size");
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
  else if constexpr (BYTES == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// all but the newest `PENDING` committed groups of this thread have landed
template <int PENDING>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

// Programmatic dependent launch.  The time-step kernels (stiffness, update)
// are launched with the programmatic-serialization attribute, so a launch
// is set up while the previous one in the stream drains and flushes: it
// stages what no launch writes (static block, GLL tables, barriers), then
// griddepcontrol.wait holds it until the previous launch has completed and
// its writes are visible.  Every block of such a kernel waits before its
// first read or write of a field and before any return, so a completed
// launch implies its predecessors completed.  Kernels trigger their
// dependents at exit: measured on B200, an early trigger let the next
// launch's waiting CTAs occupy SM slots and made the single-shot step about
// 10 % slower, while the implicit trigger at exit makes it about 2 % faster
// than plain stream order.  The exception is an overlapped stiffness pair
// (TailWork::overlap), where the second launch works before it waits.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// Dependency wait of a single-shot stiffness launch at its start, and the
// early trigger of the first launch of an overlapped pair (TailWork::overlap).
// The second launch of a pair may start once every CTA of the first has
// passed its own wait, i.e. after the previous step's update has completed
// and its writes are visible; its element loop reads and writes only its own
// medium's fields, which the first launch does not write, so only its tail
// (sources, coupling from the acoustic force) waits for the first launch.
__device__ __forceinline__ void stiffness_dep_start(const TailWork &tw) {
  if (!(tw.overlap & kOverlapSecond)) grid_dep_wait();
  if (tw.overlap & kOverlapFirst) grid_dep_launch_dependents();
}
// The deferred wait of the second launch of a pair, before its tail work
// (and before any return, so a completed launch still implies completed
// predecessors).
__device__ __forceinline__ void stiffness_dep_tail(const TailWork &tw) {
  if (tw.overlap & kOverlapSecond) grid_dep_wait();
}

// Launch with the programmatic-serialization attribute (off when the
// environment sets SFB_PROGRAMMATIC_LAUNCH=0: plain stream order).
bool programmatic_launch() {
  static const bool on = [] {
    const char *e = std::getenv("SFB_PROGRAMMATIC_LAUNCH");
    return !(e && e[0] == '0');
  }();
  return on;
}
template <typename... KArgs, typename... Args>
void launch_step_kernel(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                        const Args &...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = programmatic_launch() ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kern, args...);
}

// Point sources and fluid-solid coupling of one medium, spread over all CTAs
// of a stiffness launch (`cta`, `ncta`); they only add into the force array.
// Fields are point-major, shot-minor: value (g, s) at g * S + s.
template <int MED, int N>
__device__ __forceinline__ void tail_work(const Static &st, const MediumFields &f, int S, int istep,
                                          const TailWork &tw, int cta, int ncta) {
  constexpr int NC = (MED == MED_PSV) ? 2 : 1;
  constexpr int NN = N * N;
  const int gtid = cta * blockDim.x + threadIdx.x;
  const int gstride = ncta * blockDim.x;
  if (tw.src.n > 0 && istep >= 0 && istep < tw.src.nstep) {
    for (int idx = gtid; idx < tw.src.n * NN; idx += gstride) {
      const int i = idx / NN, kk = idx % NN;
      if (tw.src.medium[i] != MED) continue;
      const size_t p = static_cast<size_t>(tw.src.elem[i]) * NN + kk;
      const int gi = st.iglob[p];
      real *A = f.a + (static_cast<size_t>(gi) * S + tw.src.shot[i]) * NC;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const real stf = tw.src.stf[(static_cast<size_t>(i) * tw.src.nstep + istep) * 2 + c];
        const real arr = tw.src.array[(static_cast<size_t>(i) * 2 + c) * NN + kk];
        real val = stf * arr;
        if (MED == MED_AC) val = stf * arr / st.mat1[p];
        atomicAdd(A + c, val);
      }
    }
  }
  if (tw.cp_mode != 0) {
    const int n = tw.cp.n;
    const MediumFields &o = tw.other;
    for (int idx = gtid; idx < n * S; idx += gstride) {
      const int i = idx / S, s = idx % S;
      if (tw.cp_mode == 1) {  // acoustic self += w (n . u_elastic)
        const real2 u = reinterpret_cast<const real2 *>(o.u)[static_cast<size_t>(tw.cp.other[i]) * S + s];
        atomicAdd(f.a + static_cast<size_t>(tw.cp.self[i]) * S + s,
                  tw.cp.factor[i] * (tw.cp.nx[i] * u.x + tw.cp.nz[i] * u.y));
      } else {  // elastic self += w n chi_ddot
        const int oi = tw.cp.other[i];
        const real r = o.a[static_cast<size_t>(oi) * S + s];
        const real chi_dd = tw.other_divided ? r : r * o.minv[oi];
        real *A = f.a + (static_cast<size_t>(tw.cp.self[i]) * S + s) * 2;
        atomicAdd(A, tw.cp.factor[i] * tw.cp.nx[i] * chi_dd);
        atomicAdd(A + 1, tw.cp.factor[i] * tw.cp.nz[i] * chi_dd);
      }
    }
  }
}

#ifndef SFB_FP64
// Row-per-thread stiffness fed by bulk async copies, software-pipelined.
// A CTA owns EPB elements; thread (el, iz) owns row iz of element el (N
// points: the xi-contractions stay in registers, the gamma-contractions read
// columns from shared memory).  CTAs walk element chunks persistently:
//   - the next chunk's packed static block (iglob, geometry, material:
//     8 x N*N words per element, contiguous in HBM) streams into the other
//     shared-memory stage by one cp.async.bulk (no multicast) completing on
//     an mbarrier while this chunk is computed;
//   - before leaving a chunk, the thread already issues the displacement
//     gathers of its row in the next chunk, so their latency overlaps the
//     barrier, the force reductions and the next chunk's set-up.
// After the chunks every CTA takes a slice of the medium's point sources
// and fluid-solid coupling points (TailWork); they only add into the same
// force array.  Every mbarrier wait is bounded (SFB_DEVICE_WAIT_TIMEOUT).
template <int MED, int N, int EPB, int MINB>
__global__ void __launch_bounds__(N * EPB, MINB)
k_stiffness_rp(Static st, MediumFields f, int nshots, StaceyStore ss, const int *istep_dev, TailWork tw,
               FusedUpdate fu) {
  constexpr int NC = (MED == MED_PSV) ? 2 : 1;
  constexpr int NN = N * N;
  constexpr int ELEM_WORDS = kPackFields * NN;
  constexpr int OFF_M0 = 6 * NN, OFF_M1 = 7 * NN;
  constexpr int STAGE_WORDS = EPB * ELEM_WORDS;
  using V = typename Vec<NC>::T;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float *stage = reinterpret_cast<float *>(smem_raw);      // [2][STAGE_WORDS]
  V *s_u = reinterpret_cast<V *>(stage + 2 * STAGE_WORDS);  // [EPB][NN]
  V *s_fg = s_u + EPB * NN;                                 // [EPB][NN] F(., gamma)
  uint64_t *bar = reinterpret_cast<uint64_t *>(s_fg + EPB * NN);

  const int t = threadIdx.x;
  const int el = t / N, iz = t % N;
  const int nchunks = (f.nelem + EPB - 1) / EPB;
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int chunk, int stg) {
    const int first = chunk * EPB;
    const int count = min(EPB, f.nelem - first);
    const uint32_t bytes = static_cast<uint32_t>(count) * ELEM_WORDS * 4u;
    const float *src = st.pack + static_cast<size_t>(f.elem_begin + first) * ELEM_WORDS;
    mbar_arrive_expect_tx(&bar[stg], bytes);
    bulk_load(stage + stg * STAGE_WORDS, src, bytes, &bar[stg]);
  };
  // the first chunk's static block does not depend on the previous launch
  if (t == 0 && blockIdx.x < nchunks) issue(blockIdx.x, 0);
  float hpz[N], hpwz[N];
#pragma unroll
  for (int l = 0; l < N; ++l) {
    hpz[l] = C_HP(iz * N + l);
    hpwz[l] = C_HPW(iz * N + l);
  }
  const float wz = C_W(iz);
  stiffness_dep_start(tw);
  const int istep = (ss.mode != 0 || tw.src.n > 0) ? *istep_dev : 0;
  const V *vbase = reinterpret_cast<const V *>(f.u);
  V *abase = reinterpret_cast<V *>(f.a);
  bool ok = true;

  // prologue: first chunk's displacement gathers
  int g[N];
  V ur[N];
  if (blockIdx.x < nchunks) {
    if (!mbar_wait_bounded(&bar[0], 0)) ok = false;
    const int li = blockIdx.x * EPB + el;
    const float *blk = stage + el * ELEM_WORDS;
#pragma unroll
    for (int ix = 0; ix < N; ++ix) {
      g[ix] = (ok && li < f.nelem) ? __float_as_int(blk[iz * N + ix]) : 0;
      ur[ix] = (ok && li < f.nelem) ? vbase[static_cast<size_t>(g[ix]) * nshots] : Vec<NC>::zero();
    }
  }

  int iter = 0;
  for (int chunk = blockIdx.x; ok && chunk < nchunks; chunk += gridDim.x, ++iter) {
    const int stg = iter & 1;
    const int next = chunk + gridDim.x;
    if (t == 0 && next < nchunks) issue(next, stg ^ 1);
    const float *blk = stage + stg * STAGE_WORDS + el * ELEM_WORDS;
    const int li = chunk * EPB + el;
    const bool valid = li < f.nelem;
    const int e = f.elem_begin + (valid ? li : 0);
    const uint8_t eflag = valid ? st.eflag[e] : 0;
    const int slot = (ss.mode != 0 && valid) ? ss.slot[e] : -1;
    // element-private points of this row (single shot): their velocity is
    // needed after the divergence, so fetch it now
    const bool fused = fu.enabled && nshots == 1 && (eflag & kElemPrivate) && iz >= 1 && iz <= N - 2;
    V vp[N - 2], mp[N - 2];
    if (fused) {
#pragma unroll
      for (int ix = 1; ix <= N - 2; ++ix) {
        vp[ix - 1] = reinterpret_cast<const V *>(fu.v)[g[ix]];
        mp[ix - 1] = reinterpret_cast<const V *>(fu.minv)[g[ix]];
      }
    }
    for (int s = 0; s < nshots; ++s) {
      if (s > 0) {
#pragma unroll
        for (int ix = 0; ix < N; ++ix) ur[ix] = valid ? vbase[static_cast<size_t>(g[ix]) * nshots + s] : Vec<NC>::zero();
      }
#pragma unroll
      for (int ix = 0; ix < N; ++ix) s_u[el * NN + iz * N + ix] = ur[ix];
      __syncthreads();
      // gamma-derivative by columns (this thread takes column j = iz; same
      // sums in the same order as the row form), left where the owner of
      // each row reads it
      V *sfg = s_fg + el * NN;
      {
        V colv[N];
#pragma unroll
        for (int l = 0; l < N; ++l) colv[l] = s_u[el * NN + l * N + iz];
#pragma unroll
        for (int p = 0; p < N; ++p) {
          V d;
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            float sum = 0.f;
#pragma unroll
            for (int l = 0; l < N; ++l) sum += C_HP(p * N + l) * comp(colv[l], c);
            set_comp(d, c, sum);
          }
          sfg[p * N + iz] = d;
        }
      }
      __syncthreads();
      V fx[N];
#pragma unroll
      for (int ix = 0; ix < N; ++ix) {
        const int k = iz * N + ix;
        const float xix = blk[1 * NN + k], xiz = blk[2 * NN + k];
        const float gax = blk[3 * NN + k], gaz = blk[4 * NN + k];
        const float jac = blk[5 * NN + k];
        const float m0 = blk[OFF_M0 + k], m1 = blk[OFF_M1 + k];
        float dxi[NC], dga[NC];
        const V dg = sfg[k];  // read before this thread overwrites point k with F(., gamma)
#pragma unroll
        for (int c = 0; c < NC; ++c) { dxi[c] = 0.f; dga[c] = comp(dg, c); }
#pragma unroll
        for (int l = 0; l < N; ++l) {
#pragma unroll
          for (int c = 0; c < NC; ++c) dxi[c] += C_HP(ix * N + l) * comp(ur[l], c);
        }
        float du[NC][2];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          du[c][0] = xix * dxi[c] + gax * dga[c];
          du[c][1] = xiz * dxi[c] + gaz * dga[c];
        }
        float T[NC][2];
        if constexpr (MED == MED_PSV) {
          const float l2m = m0 + static_cast<float>(4.0 / 3.0) * m1;
          const float lam = l2m - 2.0f * m1;
          T[0][0] = l2m * du[0][0] + lam * du[1][1];
          T[1][1] = l2m * du[1][1] + lam * du[0][0];
          T[0][1] = m1 * (du[0][1] + du[1][0]);
          T[1][0] = T[0][1];
        } else {
          T[0][0] = m0 * du[0][0];
          T[0][1] = m0 * du[0][1];
        }
        V f0, f1;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          set_comp(f0, c, jac * (T[c][0] * xix + T[c][1] * xiz));
          set_comp(f1, c, jac * (T[c][0] * gax + T[c][1] * gaz));
        }
        fx[ix] = f0;
        sfg[k] = f1;
      }
      __syncthreads();
      // gamma-sum of the divergence by columns, left in the displacement
      // tile (free now: the rows are in registers)
      V *st2 = s_u + el * NN;
      {
        V colf[N];
#pragma unroll
        for (int l = 0; l < N; ++l) colf[l] = sfg[l * N + iz];
#pragma unroll
        for (int p = 0; p < N; ++p) {
          V d;
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            float sum = 0.f;
#pragma unroll
            for (int l = 0; l < N; ++l) sum += comp(colf[l], c) * C_HPW(p * N + l);
            set_comp(d, c, sum);
          }
          st2[p * N + iz] = d;
        }
      }
      __syncthreads();
      float accr[N][2];
#pragma unroll
      for (int ix = 0; ix < N; ++ix) {
        float t1[NC], t2[NC];
        const V g2 = st2[iz * N + ix];
#pragma unroll
        for (int c = 0; c < NC; ++c) { t1[c] = 0.f; t2[c] = comp(g2, c); }
#pragma unroll
        for (int l = 0; l < N; ++l) {
#pragma unroll
          for (int c = 0; c < NC; ++c) t1[c] += comp(fx[l], c) * C_HPW(ix * N + l);
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) accr[ix][c] = (wz * t1[c] + C_W(ix) * t2[c]) * -1.0f;
      }
      if (eflag & 3) {
#pragma unroll
        for (int ix = 0; ix < N; ++ix) {
          const size_t p = (static_cast<size_t>(e) * N + iz) * N + ix;
          const uint8_t b = st.bnd[p];
          if (b & 1) {
            const V vv = reinterpret_cast<const V *>(f.v)[static_cast<size_t>(g[ix]) * nshots + s];
            float vel[2];
#pragma unroll
            for (int c = 0; c < NC; ++c) vel[c] = comp(vv, c);
            stacey<MED>(blk[OFF_M0 + iz * N + ix], blk[OFF_M1 + iz * N + ix], st.mat2 ? st.mat2[p] : 0.f,
                        st.bnd_nx[p], st.bnd_nz[p], st.bnd_w[p], vel, accr[ix]);
          }
          if (b & 2) {
#pragma unroll
            for (int c = 0; c < NC; ++c) accr[ix][c] = 0.f;
          }
        }
      }
      if (slot >= 0) {
#pragma unroll
        for (int ix = 0; ix < N; ++ix) {
          const size_t base =
              ((((static_cast<size_t>(s) * ss.nstep + istep) * ss.nstacey + slot) * N + iz) * N + ix) * 2;
          if (ss.mode == 1) {
#pragma unroll
            for (int c = 0; c < NC; ++c) ss.data[base + c] = accr[ix][c];
          } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) accr[ix][c] = ss.data[base + c];
          }
        }
      }
      const bool last_shot = (s + 1 == nshots);
      int gnext[N];
      if (last_shot && next < nchunks) {
        // next chunk: its static block is (or soon will be) in the other
        // stage; take its indices and start its displacement gathers now
        if (!mbar_wait_bounded(&bar[stg ^ 1], ((iter + 1) >> 1) & 1)) {
          ok = false;
        } else {
          const float *nblk = stage + (stg ^ 1) * STAGE_WORDS + el * ELEM_WORDS;
          const bool nvalid = next * EPB + el < f.nelem;
#pragma unroll
          for (int ix = 0; ix < N; ++ix) gnext[ix] = nvalid ? __float_as_int(nblk[iz * N + ix]) : 0;
        }
      }
      if (valid) {
#pragma unroll
        for (int ix = 0; ix < N; ++ix) {
          if (fused && ix >= 1 && ix <= N - 2) {
            // a = force / M, corrector, next predictor in registers
            // (newmark.tpp:44-47, 98-105); the force never reaches memory
            V vel = vp[ix - 1], uu = ur[ix], aa;
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              const float a_c = accr[ix][c] * comp(mp[ix - 1], c);
              set_comp(aa, c, a_c);
              set_comp(vel, c, comp(vel, c) + fu.dt2 * a_c);
            }
            V *Vw = reinterpret_cast<V *>(fu.v);
            if (fu.last) {
              abase[g[ix]] = aa;
              Vw[g[ix]] = vel;
            } else {
#pragma unroll
              for (int c = 0; c < NC; ++c) {
                set_comp(uu, c, comp(uu, c) + (fu.dt * comp(vel, c) + fu.dtsq2 * comp(aa, c)));
                set_comp(vel, c, comp(vel, c) + fu.dt2 * comp(aa, c));
              }
              reinterpret_cast<V *>(f.u)[g[ix]] = uu;
              Vw[g[ix]] = vel;
            }
            continue;
          }
          V out;
#pragma unroll
          for (int c = 0; c < NC; ++c) set_comp(out, c, accr[ix][c]);
          red_add(abase + static_cast<size_t>(g[ix]) * nshots + s, out);
        }
      }
      if (last_shot && next < nchunks && ok) {
        const bool nvalid = next * EPB + el < f.nelem;
#pragma unroll
        for (int ix = 0; ix < N; ++ix) {
          g[ix] = gnext[ix];
          ur[ix] = nvalid ? vbase[static_cast<size_t>(g[ix]) * nshots] : Vec<NC>::zero();
        }
      }
      __syncthreads();
    }
  }
  stiffness_dep_tail(tw);
  if (!ok) {
    if (t == 0) atomicOr(st.err, kWaitTimeout);
    return;
  }

  tail_work<MED, N>(st, f, nshots, istep, tw, blockIdx.x, gridDim.x);
}

template <int MED, int N, int EPB>
size_t rp_smem_bytes() {
  constexpr int NC = (MED == MED_PSV) ? 2 : 1;
  return 2 * EPB * kPackFields * N * N * 4 + 2 * EPB * N * N * NC * 4 + 16;
}

template <int MED, int N, int EPB, int MINB>
void launch_rp(const Static &st, const MediumFields &f, int nshots, const StaceyStore &ss, const int *istep_dev,
               const TailWork &tw, const FusedUpdate &fu, cudaStream_t stream) {
  static int blocks_per_sm = -1, nsm = 0;
  const size_t smem = rp_smem_bytes<MED, N, EPB>();
  if (blocks_per_sm < 0) {
    cudaFuncSetAttribute(k_stiffness_rp<MED, N, EPB, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_stiffness_rp<MED, N, EPB, MINB>, N * EPB,
                                                  smem);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  const int nchunks = (f.nelem + EPB - 1) / EPB;
  const int grid = std::max(1, std::min(nchunks, nsm * blocks_per_sm));
  launch_step_kernel(k_stiffness_rp<MED, N, EPB, MINB>, grid, N * EPB, smem, stream, st, f, nshots, ss,
                     istep_dev, tw, fu);
}

// Single-shot row kernel for a medium of affine elements (same work,
// arithmetic and outputs as k_stiffness_rp with one shot), reading the
// compact block: per chunk of kAffineChunk elements, chunk-major,
//   [0, E*NN) index, [E*NN, 2E*NN) mat0, [2E*NN, 3E*NN) mat1 (element el,
//   point k at el*NN + k), then xix, xiz, gammax, gammaz, jac ([q][el]),
// so a warp's reads of a stage are conflict-free.  Deeper pipeline: three
// static stages (the block of chunk i+2 streams in while chunk i is
// computed), so the indices of chunk i+1 are in shared memory when chunk i
// starts; each thread then gathers its row of chunk i+1's displacement
// straight into shared memory with cp.async, and those loads have the whole
// of chunk i to land.  The displacement has two shared buffers.  Every
// mbarrier wait is bounded and its outcome is made CTA-uniform with
// __syncthreads_and; on expiry the CTA drains its own copies (bounded),
// records kWaitTimeout in st.err and returns.
template <int MED, int N, int MINB>
__global__ void __launch_bounds__(N * kAffineChunk, MINB)
k_stiffness_rpa(Static st, MediumFields f, StaceyStore ss, const int *istep_dev, TailWork tw, FusedUpdate fu) {
  constexpr int NC = (MED == MED_PSV) ? 2 : 1;
  constexpr int NN = N * N;
  constexpr int EPB = kAffineChunk;
  constexpr int OFF_M0 = EPB * NN, OFF_M1 = 2 * EPB * NN, OFF_GEO = 3 * EPB * NN;
  constexpr int STAGES = 3;
  constexpr int STAGE_WORDS = affine_chunk_words(N);
  using V = typename Vec<NC>::T;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float *stage = reinterpret_cast<float *>(smem_raw);            // [STAGES][STAGE_WORDS]
  V *s_u = reinterpret_cast<V *>(stage + STAGES * STAGE_WORDS);  // [2][EPB][NN]
  V *s_fg = s_u + 2 * EPB * NN;                                  // [EPB][NN] F(., gamma)
  uint64_t *bar = reinterpret_cast<uint64_t *>(s_fg + EPB * NN);  // [STAGES]

  const int t = threadIdx.x;
  const int el = t / N, iz = t % N;
  const int nchunks = (f.nelem + EPB - 1) / EPB;
  const int G = gridDim.x;
  if (t == 0) {
    for (int q = 0; q < STAGES; ++q) mbar_init(&bar[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // whole chunks: the compact block is padded to full chunks per medium
  auto issue = [&](int chunk, int stg) {
    const uint32_t bytes = static_cast<uint32_t>(STAGE_WORDS) * 4u;
    const float *src = st.pack_aff + (static_cast<size_t>(st.aff_chunk0[MED]) + chunk) * STAGE_WORDS;
    mbar_arrive_expect_tx(&bar[stg], bytes);
    bulk_load(stage + stg * STAGE_WORDS, src, bytes, &bar[stg]);
  };
  // static blocks of the first two chunks (no launch writes them)
  if (t == 0) {
    if (blockIdx.x < nchunks) issue(blockIdx.x, 0);
    if (blockIdx.x + G < nchunks) issue(blockIdx.x + G, 1);
  }
  int issued = blockIdx.x + G < nchunks ? 1 : (blockIdx.x < nchunks ? 0 : -1);  // last iteration issued
  int waited = -1;  // last iteration whose static block every thread has waited for
  float hpz[N], hpwz[N];
#pragma unroll
  for (int l = 0; l < N; ++l) {
    hpz[l] = C_HP(iz * N + l);
    hpwz[l] = C_HPW(iz * N + l);
  }
  const float wz = C_W(iz);
  stiffness_dep_start(tw);
  const int istep = (ss.mode != 0 || tw.src.n > 0) ? *istep_dev : 0;
  const V *U = reinterpret_cast<const V *>(f.u);
  V *A = reinterpret_cast<V *>(f.a);

  // this thread's row of chunk `chunk` (iteration `it`) into s_u[it & 1]
  auto gather = [&](int it, int chunk) {
    const float *idx = stage + (it % STAGES) * STAGE_WORDS + el * NN + iz * N;
    V *dst = s_u + (it & 1) * EPB * NN + el * NN + iz * N;
    if (chunk * EPB + el < f.nelem) {
#pragma unroll
      for (int ix = 0; ix < N; ++ix) cp_async<sizeof(V)>(dst + ix, U + __float_as_int(idx[ix]));
    } else {
#pragma unroll
      for (int ix = 0; ix < N; ++ix) dst[ix] = Vec<NC>::zero();
    }
  };
  bool ok = true;
  if (blockIdx.x < nchunks) {
    const bool w0 = mbar_wait_bounded(&bar[0], 0);
    if (w0) gather(0, blockIdx.x);
    cp_async_commit();
    ok = __syncthreads_and(w0);
    if (ok) waited = 0;
  }

  for (int it = 0; ok; ++it) {
    const int chunk = blockIdx.x + it * G;
    if (chunk >= nchunks) break;
    const int stg = it % STAGES;
    // the static block of chunk it+2 into the stage chunk it-1 used
    if (chunk + 2 * G < nchunks) {
      if (t == 0) issue(chunk + 2 * G, (it + 2) % STAGES);
      issued = it + 2;
    }
    // chunk it+1: wait for its static block (issued an iteration ago) and
    // start its displacement gathers
    const bool has_next = chunk + G < nchunks;
    bool okw = true;
    if (has_next) {
      okw = mbar_wait_bounded(&bar[(it + 1) % STAGES], ((it + 1) / STAGES) & 1);
      if (okw) gather(it + 1, chunk + G);
    }
    cp_async_commit();
    cp_async_wait_group<1>();  // chunk it's gathers have landed
    ok = __syncthreads_and(okw);
    if (!ok) break;
    if (has_next) waited = it + 1;

    const float *blk = stage + stg * STAGE_WORDS + el * NN;  // this element's index and material words
    const float *geo = stage + stg * STAGE_WORDS + OFF_GEO + el;
    const V *su = s_u + (it & 1) * EPB * NN + el * NN;
    const int li = chunk * EPB + el;
    const bool valid = li < f.nelem;
    const int e = f.elem_begin + (valid ? li : 0);
    const uint8_t eflag = valid ? st.eflag[e] : 0;
    const int slot = (ss.mode != 0 && valid) ? ss.slot[e] : -1;
    int g[N];
#pragma unroll
    for (int ix = 0; ix < N; ++ix) g[ix] = __float_as_int(blk[iz * N + ix]);
    const float xix = geo[0 * EPB], xiz = geo[1 * EPB], gax = geo[2 * EPB], gaz = geo[3 * EPB];
    const float jac = geo[4 * EPB];
    // element-private points of this row: velocity and inverse mass are
    // needed after the divergence, so fetch them now
    const bool fused = fu.enabled && (eflag & kElemPrivate) && iz >= 1 && iz <= N - 2;
    V vp[N - 2], mp[N - 2];
    if (fused) {
#pragma unroll
      for (int ix = 1; ix <= N - 2; ++ix) {
        vp[ix - 1] = reinterpret_cast<const V *>(fu.v)[g[ix]];
        mp[ix - 1] = reinterpret_cast<const V *>(fu.minv)[g[ix]];
      }
    }
    V ur[N];
#pragma unroll
    for (int ix = 0; ix < N; ++ix) ur[ix] = su[iz * N + ix];
    // gamma-derivative by columns: this thread takes column j = iz of its
    // element (5 shared loads instead of 25 for its row) and leaves the
    // derivative of point (p, j) where the owner of row p reads it; same
    // sums in the same order as the row form
    V *sfg = s_fg + el * NN;
    {
      V colv[N];
#pragma unroll
      for (int l = 0; l < N; ++l) colv[l] = su[l * N + iz];
#pragma unroll
      for (int p = 0; p < N; ++p) {
        V d;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          float sum = 0.f;
#pragma unroll
          for (int l = 0; l < N; ++l) sum += C_HP(p * N + l) * comp(colv[l], c);
          set_comp(d, c, sum);
        }
        sfg[p * N + iz] = d;
      }
    }
    __syncthreads();
    V fx[N];
#pragma unroll
    for (int ix = 0; ix < N; ++ix) {
      const int k = iz * N + ix;
      const float m0 = blk[OFF_M0 + k], m1 = blk[OFF_M1 + k];
      float dxi[NC], dga[NC];
      const V dg = sfg[k];  // read before this thread overwrites point k with F(., gamma)
#pragma unroll
      for (int c = 0; c < NC; ++c) { dxi[c] = 0.f; dga[c] = comp(dg, c); }
#pragma unroll
      for (int l = 0; l < N; ++l) {
#pragma unroll
        for (int c = 0; c < NC; ++c) dxi[c] += C_HP(ix * N + l) * comp(ur[l], c);
      }
      float du[NC][2];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        du[c][0] = xix * dxi[c] + gax * dga[c];
        du[c][1] = xiz * dxi[c] + gaz * dga[c];
      }
      float T[NC][2];
      if constexpr (MED == MED_PSV) {
        const float l2m = m0 + static_cast<float>(4.0 / 3.0) * m1;
        const float lam = l2m - 2.0f * m1;
        T[0][0] = l2m * du[0][0] + lam * du[1][1];
        T[1][1] = l2m * du[1][1] + lam * du[0][0];
        T[0][1] = m1 * (du[0][1] + du[1][0]);
        T[1][0] = T[0][1];
      } else {
        T[0][0] = m0 * du[0][0];
        T[0][1] = m0 * du[0][1];
      }
      V f0, f1;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        set_comp(f0, c, jac * (T[c][0] * xix + T[c][1] * xiz));
        set_comp(f1, c, jac * (T[c][0] * gax + T[c][1] * gaz));
      }
      fx[ix] = f0;
      sfg[k] = f1;
    }
    __syncthreads();
    // gamma-sum of the divergence by columns, left in this chunk's
    // displacement buffer (free now: the rows are in registers, the next
    // chunk's gathers go to the other buffer)
    V *st2 = s_u + (it & 1) * EPB * NN + el * NN;
    {
      V colf[N];
#pragma unroll
      for (int l = 0; l < N; ++l) colf[l] = sfg[l * N + iz];
#pragma unroll
      for (int p = 0; p < N; ++p) {
        V d;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          float sum = 0.f;
#pragma unroll
          for (int l = 0; l < N; ++l) sum += comp(colf[l], c) * C_HPW(p * N + l);
          set_comp(d, c, sum);
        }
        st2[p * N + iz] = d;
      }
    }
    __syncthreads();
    float accr[N][2];
#pragma unroll
    for (int ix = 0; ix < N; ++ix) {
      float t1[NC], t2[NC];
      const V g2 = st2[iz * N + ix];
#pragma unroll
      for (int c = 0; c < NC; ++c) { t1[c] = 0.f; t2[c] = comp(g2, c); }
#pragma unroll
      for (int l = 0; l < N; ++l) {
#pragma unroll
        for (int c = 0; c < NC; ++c) t1[c] += comp(fx[l], c) * C_HPW(ix * N + l);
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) accr[ix][c] = (wz * t1[c] + C_W(ix) * t2[c]) * -1.0f;
    }
    if (eflag & 3) {
#pragma unroll
      for (int ix = 0; ix < N; ++ix) {
        const size_t p = (static_cast<size_t>(e) * N + iz) * N + ix;
        const uint8_t b = st.bnd[p];
        if (b & 1) {
          const V vv = reinterpret_cast<const V *>(f.v)[g[ix]];
          float vel[2];
#pragma unroll
          for (int c = 0; c < NC; ++c) vel[c] = comp(vv, c);
          stacey<MED>(blk[OFF_M0 + iz * N + ix], blk[OFF_M1 + iz * N + ix], st.mat2 ? st.mat2[p] : 0.f,
                      st.bnd_nx[p], st.bnd_nz[p], st.bnd_w[p], vel, accr[ix]);
        }
        if (b & 2) {
#pragma unroll
          for (int c = 0; c < NC; ++c) accr[ix][c] = 0.f;
        }
      }
    }
    if (slot >= 0) {
#pragma unroll
      for (int ix = 0; ix < N; ++ix) {
        const size_t base = (((static_cast<size_t>(istep) * ss.nstacey + slot) * N + iz) * N + ix) * 2;
        if (ss.mode == 1) {
#pragma unroll
          for (int c = 0; c < NC; ++c) ss.data[base + c] = accr[ix][c];
        } else {
#pragma unroll
          for (int c = 0; c < NC; ++c) accr[ix][c] = ss.data[base + c];
        }
      }
    }
    if (valid) {
#pragma unroll
      for (int ix = 0; ix < N; ++ix) {
        if (fused && ix >= 1 && ix <= N - 2) {
          // a = force / M, corrector, next predictor in registers
          // (newmark.tpp:44-47, 98-105); the force never reaches memory
          V vel = vp[ix - 1], uu = ur[ix], aa;
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            const float a_c = accr[ix][c] * comp(mp[ix - 1], c);
            set_comp(aa, c, a_c);
            set_comp(vel, c, comp(vel, c) + fu.dt2 * a_c);
          }
          V *Vw = reinterpret_cast<V *>(fu.v);
          if (fu.last) {
            A[g[ix]] = aa;
            Vw[g[ix]] = vel;
          } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              set_comp(uu, c, comp(uu, c) + (fu.dt * comp(vel, c) + fu.dtsq2 * comp(aa, c)));
              set_comp(vel, c, comp(vel, c) + fu.dt2 * comp(aa, c));
            }
            reinterpret_cast<V *>(f.u)[g[ix]] = uu;
            Vw[g[ix]] = vel;
          }
          continue;
        }
        V out;
#pragma unroll
        for (int c = 0; c < NC; ++c) set_comp(out, c, accr[ix][c]);
        red_add(A + g[ix], out);
      }
    }
    __syncthreads();  // stage stg, s_u[it & 1] and s_fg are free again
  }
  stiffness_dep_tail(tw);
  if (!ok) {
    cp_async_wait_all();
    if (t == 0) {
      for (int j = waited + 1; j <= issued; ++j) mbar_wait_bounded(&bar[j % STAGES], (j / STAGES) & 1);
      atomicOr(st.err, kWaitTimeout);
    }
    return;
  }
  tail_work<MED, N>(st, f, 1, istep, tw, blockIdx.x, gridDim.x);
}

template <int MED, int N>
size_t rpa_smem_bytes() {
  constexpr int NC = (MED == MED_PSV) ? 2 : 1;
  return 3 * affine_chunk_words(N) * 4 + 3 * kAffineChunk * N * N * NC * 4 + 3 * 8;
}

template <int MED, int N, int MINB>
void launch_rpa(const Static &st, const MediumFields &f, const StaceyStore &ss, const int *istep_dev,
                const TailWork &tw, const FusedUpdate &fu, cudaStream_t stream) {
  static int blocks_per_sm = -1, nsm = 0;
  const size_t smem = rpa_smem_bytes<MED, N>();
  if (blocks_per_sm < 0) {
    cudaFuncSetAttribute(k_stiffness_rpa<MED, N, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
    cudaFuncSetAttribute(k_stiffness_rpa<MED, N, MINB>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_stiffness_rpa<MED, N, MINB>, N * kAffineChunk,
                                                  smem);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  const int nchunks = (f.nelem + kAffineChunk - 1) / kAffineChunk;
  int grid = std::max(1, std::min(nchunks, nsm * blocks_per_sm));
  if (tw.overlap & kOverlapFirst) {
    // first launch of an overlapped pair: the fewest CTAs that keep the
    // same number of chunks per CTA, so the slots it leaves go to the second
    const int per = (nchunks + grid - 1) / grid;
    grid = std::max(1, (nchunks + per - 1) / per);
  }
  launch_step_kernel(k_stiffness_rpa<MED, N, MINB>, grid, N * kAffineChunk, smem, stream, st, f, ss, istep_dev, tw,
                     fu);
}
#endif  // !SFB_FP64

// Shot-parallel stiffness for S > 1 independent wavefields (batched shots).
// One CTA per element and group of 32 * SPL shots; warp iz owns row iz of the
// element, lane l owns shots s0 = (group * 32 + l) * SPL .. s0 + SPL - 1.  In
// the point-major, shot-minor layout the SPL shots of a lane are adjacent, so
// each gather of u(g, s0..) and each reduction into f(g, s0..) is one 8- or
// 16-byte access and a warp moves 32 * SPL * NC * 4 contiguous bytes.  The
// element's packed static block (iglob, geometry, material) is staged once
// in shared memory and read by warp-uniform broadcasts.  Row contractions
// stay in registers, column contractions read shared memory.
template <int NV> struct VecN;
template <> struct VecN<1> { using T = real; };
template <> struct VecN<2> { using T = real2; };
template <> struct VecN<4> { using T = real4; };
__device__ __forceinline__ real vget(const real &v, int) { return v; }
__device__ __forceinline__ real vget(const real2 &v, int i) { return i == 0 ? v.x : v.y; }
__device__ __forceinline__ real vget(const real4 &v, int i) {
  return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}
__device__ __forceinline__ void vset(real &v, int, real x) { v = x; }
__device__ __forceinline__ void vset(real2 &v, int i, real x) { if (i == 0) v.x = x; else v.y = x; }
__device__ __forceinline__ void vset(real4 &v, int i, real x) {
  if (i == 0) v.x = x; else if (i == 1) v.y = x; else if (i == 2) v.z = x; else v.w = x;
}
__device__ __forceinline__ void vred(real *p, real v) { atomicAdd(p, v); }
#ifdef SFB_FP64
__device__ __forceinline__ void vred(real2 *p, real2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}
__device__ __forceinline__ void vred(real4 *p, real4 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
  atomicAdd(&p->z, v.z);
  atomicAdd(&p->w, v.w);
}
#else
__device__ __forceinline__ void vred(float2 *p, float2 v) { atomicAdd(p, v); }
__device__ __forceinline__ void vred(float4 *p, float4 v) { atomicAdd(p, v); }
#endif

// Dynamic shared memory of k_stiffness_shots: the displacement and the
// gamma fluxes of the element for the CTA's shots, and the static block.
template <int MED, int N, int SPL>
constexpr size_t shots_smem_bytes() {
  return 2 * static_cast<size_t>(N * N * 32) * sizeof(typename VecN<((MED == MED_PSV) ? 2 : 1) * SPL>::T) +
         static_cast<size_t>(kPackFields * N * N) * sizeof(real);
}

template <int MED, int N, int SPL, int MINB>
__global__ void __launch_bounds__(N * 32, MINB)
k_stiffness_shots(Static st, MediumFields f, int S, StaceyStore ss, const int *istep_dev, TailWork tw,
                  FusedUpdate fu) {
  constexpr int NC = (MED == MED_PSV) ? 2 : 1;
  constexpr int NN = N * N;
  constexpr int NV = NC * SPL;
  using W = typename VecN<NV>::T;
  extern __shared__ __align__(16) unsigned char shots_smem[];
  W *s_u = reinterpret_cast<W *>(shots_smem);         // [NN * 32]
  W *s_fg = s_u + NN * 32;                            // [NN * 32]
  real *s_st = reinterpret_cast<real *>(s_fg + NN * 32);  // [kPackFields * NN]
  const int lane = threadIdx.x & 31, iz = threadIdx.x >> 5;
  const int e = f.elem_begin + blockIdx.x;
  const int s0 = (blockIdx.y * 32 + lane) * SPL;
  const bool act = s0 < S;
  for (int i = threadIdx.x; i < kPackFields * NN; i += blockDim.x)
    s_st[i] = st.pack[static_cast<size_t>(e) * kPackFields * NN + i];
  __syncthreads();
  grid_dep_wait();
  const int istep = (ss.mode != 0 || tw.src.n > 0) ? *istep_dev : 0;
  int g[N];
#pragma unroll
  for (int ix = 0; ix < N; ++ix) g[ix] = pack_index(s_st[iz * N + ix]);
  real hpz[N], hpwz[N];
#pragma unroll
  for (int l = 0; l < N; ++l) {
    hpz[l] = C_HP(iz * N + l);
    hpwz[l] = C_HPW(iz * N + l);
  }
  const real wz = C_W(iz);
  // u(g, s) for s = s0 .. s0+SPL-1, components interleaved: (g*S + s0)*NC floats
  const W *U = reinterpret_cast<const W *>(f.u);
  W *A = reinterpret_cast<W *>(f.a);
  const size_t Sv = static_cast<size_t>(S) / SPL;  // vectors per point
  const size_t lofs = static_cast<size_t>(s0) / SPL;
  W ur[N];
#pragma unroll
  for (int ix = 0; ix < N; ++ix) {
    if (act) ur[ix] = U[g[ix] * Sv + lofs];
    else { for (int q = 0; q < NV; ++q) vset(ur[ix], q, 0); }
    s_u[(iz * N + ix) * 32 + lane] = ur[ix];
  }
  __syncthreads();
  W fx[N];
#pragma unroll
  for (int ix = 0; ix < N; ++ix) {
    const int k = iz * N + ix;
    const real xix = s_st[1 * NN + k], xiz = s_st[2 * NN + k];
    const real gax = s_st[3 * NN + k], gaz = s_st[4 * NN + k];
    const real jac = s_st[5 * NN + k], m0 = s_st[6 * NN + k], m1 = s_st[7 * NN + k];
    real dxi[NV], dga[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) { dxi[q] = 0; dga[q] = 0; }
#pragma unroll
    for (int l = 0; l < N; ++l) {
      const W col = s_u[(l * N + ix) * 32 + lane];
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        dxi[q] += C_HP(ix * N + l) * vget(ur[l], q);
        dga[q] += hpz[l] * vget(col, q);
      }
    }
    W f0, f1;
#pragma unroll
    for (int j = 0; j < SPL; ++j) {
      real du[NC][2];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        du[c][0] = xix * dxi[j * NC + c] + gax * dga[j * NC + c];
        du[c][1] = xiz * dxi[j * NC + c] + gaz * dga[j * NC + c];
      }
      real T[NC][2];
      if constexpr (MED == MED_PSV) {
        const real l2m = m0 + kFourThirds * m1;
        const real lam = l2m - static_cast<real>(2) * m1;
        T[0][0] = l2m * du[0][0] + lam * du[1][1];
        T[1][1] = l2m * du[1][1] + lam * du[0][0];
        T[0][1] = m1 * (du[0][1] + du[1][0]);
        T[1][0] = T[0][1];
      } else {
        T[0][0] = m0 * du[0][0];
        T[0][1] = m0 * du[0][1];
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        vset(f0, j * NC + c, jac * (T[c][0] * xix + T[c][1] * xiz));
        vset(f1, j * NC + c, jac * (T[c][0] * gax + T[c][1] * gaz));
      }
    }
    fx[ix] = f0;
    s_fg[k * 32 + lane] = f1;
  }
  __syncthreads();
  const uint8_t eflag = st.eflag[e];
  const int slot = (ss.mode != 0) ? ss.slot[e] : -1;
  const bool fused = fu.enabled && (eflag & kElemPrivate) && iz >= 1 && iz <= N - 2;
#pragma unroll
  for (int ix = 0; ix < N; ++ix) {
    real t1[NV], t2[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) { t1[q] = 0; t2[q] = 0; }
#pragma unroll
    for (int l = 0; l < N; ++l) {
      const W col = s_fg[(l * N + ix) * 32 + lane];
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        t1[q] += vget(fx[l], q) * C_HPW(ix * N + l);
        t2[q] += vget(col, q) * hpwz[l];
      }
    }
    W out;
#pragma unroll
    for (int j = 0; j < SPL; ++j) {
      real acc[2];
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[c] = (wz * t1[j * NC + c] + C_W(ix) * t2[j * NC + c]) * static_cast<real>(-1);
      if (eflag & 3) {
        const size_t p = (static_cast<size_t>(e) * N + iz) * N + ix;
        const uint8_t b = st.bnd[p];
        if ((b & 1) && act) {
          const real *Vp = f.v + (static_cast<size_t>(g[ix]) * S + s0 + j) * NC;
          real vel[2];
#pragma unroll
          for (int c = 0; c < NC; ++c) vel[c] = Vp[c];
          stacey<MED>(s_st[6 * NN + iz * N + ix], s_st[7 * NN + iz * N + ix], st.mat2 ? st.mat2[p] : real(0),
                      st.bnd_nx[p], st.bnd_nz[p], st.bnd_w[p], vel, acc);
        }
        if (b & 2) {
#pragma unroll
          for (int c = 0; c < NC; ++c) acc[c] = 0;
        }
      }
      if (slot >= 0 && act) {
        const size_t base =
            ((((static_cast<size_t>(s0 + j) * ss.nstep + istep) * ss.nstacey + slot) * N + iz) * N + ix) * 2;
        if (ss.mode == 1) {
#pragma unroll
          for (int c = 0; c < NC; ++c) ss.data[base + c] = acc[c];
        } else {
#pragma unroll
          for (int c = 0; c < NC; ++c) acc[c] = ss.data[base + c];
        }
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) vset(out, j * NC + c, acc[c]);
    }
    if (!act) continue;
    const size_t at = g[ix] * Sv + lofs;
    if (fused && ix >= 1 && ix <= N - 2) {
      // element-private point: a = force / M, corrector, next predictor
      // (the update kernel's arithmetic, newmark.tpp:44-47 and 98-105);
      // u comes back from the shared staging, not from registers
      W *Vw = reinterpret_cast<W *>(fu.v);
      W *Uw = reinterpret_cast<W *>(f.u);
      W vel = Vw[at], uu = s_u[(iz * N + ix) * 32 + lane], aa;
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const real a_q = vget(out, q) * fu.minv[g[ix] * NC + (q % NC)];
        vset(aa, q, a_q);
        vset(vel, q, vget(vel, q) + fu.dt2 * a_q);
      }
      if (fu.last) {
        A[at] = aa;
        Vw[at] = vel;
      } else {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
          vset(uu, q, vget(uu, q) + (fu.dt * vget(vel, q) + fu.dtsq2 * vget(aa, q)));
          vset(vel, q, vget(vel, q) + fu.dt2 * vget(aa, q));
        }
        Uw[at] = uu;
        Vw[at] = vel;
      }
    } else {
      vred(A + at, out);
    }
  }
  tail_work<MED, N>(st, f, S, istep, tw, blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y);
}


#ifndef SFB_FP64
// ---------------------------------------------------------------------------
// Batched stiffness, two shots per lane in packed FP32x2 arithmetic.  Same
// work and launch shape as k_stiffness_shots<..., SPL = 2>, but every
// per-point operation is applied to the (shot 0, shot 1) pair of one
// component with one f32x2 instruction: the lane's float4 / float2 of a
// point (memory order s0c0 s0c1 s1c0 s1c1) is held in component-major pair
// order (s0c0 s1c0 s0c1 s1c1), geometry and material are staged in shared
// memory as (v, v) pairs, and the quadrature tables come as pairs from
// constant memory.  Each f32x2 lane rounds as one IEEE fma / mul / add.
//
// FR (P-SV only): the backward stiffness launch of the combined loop also
// gathers the adjoint displacement and assembled adjoint force of the same
// step and adds the step's Frechet kernels, summed over the launch's shots,
// to the FP64 accumulators (see FrechetFuse).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pr(const float4 &w, int c) { return c == 0 ? make_float2(w.x, w.y) : make_float2(w.z, w.w); }
__device__ __forceinline__ float2 pr(const float2 &w, int) { return w; }
__device__ __forceinline__ void setpr(float4 &w, int c, float2 v) {
  if (c == 0) { w.x = v.x; w.y = v.y; } else { w.z = v.x; w.w = v.y; }
}
__device__ __forceinline__ void setpr(float2 &w, int, float2 v) { w = v; }
// memory order <-> pair order (an involution)
__device__ __forceinline__ float4 swz(const float4 &w) { return make_float4(w.x, w.z, w.y, w.w); }
__device__ __forceinline__ float2 swz(const float2 &w) { return w; }
template <typename W> __device__ __forceinline__ W make_zero_w();
template <> __device__ __forceinline__ float4 make_zero_w<float4>() { return make_float4(0.f, 0.f, 0.f, 0.f); }
template <> __device__ __forceinline__ float2 make_zero_w<float2>() { return make_float2(0.f, 0.f); }


template <int MED, int N, int MINB, bool FR = false, bool AFF = false>
__global__ void __launch_bounds__(N * 32, MINB)
k_stiffness_pk(Static st, MediumFields f, int S, StaceyStore ss, const int *istep_dev, TailWork tw,
               FusedUpdate fu, FrechetFuse fr) {
  constexpr int NC = (MED == MED_PSV) ? 2 : 1;
  constexpr int NN = N * N;
  using W = typename VecN<2 * NC>::T;
  __shared__ W s_u[NN * 32];
  __shared__ W s_fg[NN * 32];
  __shared__ float2 s_g[8 * NN];  // xix, xiz, gammax, gammaz, jac, then P-SV (l+2m, l, m) / SH m / acoustic 1/rho
  __shared__ W s_vp[(N - 2) * (N - 2) * 32];  // velocity of the private points (prefetched)
  // FR: adjoint displacement staging, adjoint force (prefetched) and
  // per-lane kernel values [3][NN][32]
  extern __shared__ float4 s_dyn[];
  W *s_ua = reinterpret_cast<W *>(s_dyn);
  W *s_aa = reinterpret_cast<W *>(s_dyn + (FR ? NN * 32 : 0));
  W *s_av = reinterpret_cast<W *>(s_dyn + (FR ? 2 * NN * 32 : 0));  // adjoint v of private points
  float *s_red = reinterpret_cast<float *>(s_dyn + (FR ? 2 * NN * 32 + (N - 2) * (N - 2) * 32 : 0));
  const int lane = threadIdx.x & 31, iz = threadIdx.x >> 5;
  const int e = f.elem_begin + blockIdx.x;
  const int s0 = (blockIdx.y * 32 + lane) * 2;
  const bool act = s0 < S;
  // static words of this element: index and material per point, geometry
  // per point (full block) or five constants (AFF: the compact block of a
  // medium of affine elements, chunk-major)
  const float *bidx, *bm0, *bm1;
  float2 cgeo[5];
  if constexpr (AFF) {
    const int c = blockIdx.x / kAffineChunk, el = blockIdx.x % kAffineChunk;
    const float *base = st.pack_aff + (static_cast<size_t>(st.aff_chunk0[MED]) + c) * affine_chunk_words(N);
    bidx = base + el * NN;
    bm0 = base + kAffineChunk * NN + el * NN;
    bm1 = base + 2 * kAffineChunk * NN + el * NN;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const float v = __ldg(base + 3 * kAffineChunk * NN + q * kAffineChunk + el);
      cgeo[q] = make_float2(v, v);
    }
  } else {
    const float *blk = st.pack + static_cast<size_t>(e) * kPackFields * NN;
    bidx = blk;
    bm0 = blk + 6 * NN;
    bm1 = blk + 7 * NN;
  }
  int g[N];
#pragma unroll
  for (int ix = 0; ix < N; ++ix) g[ix] = __float_as_int(__ldg(bidx + iz * N + ix));
  // geometry and material pairs: static, staged before the dependency wait
  for (int k = threadIdx.x; k < NN; k += blockDim.x) {
    if constexpr (!AFF) {
#pragma unroll
      for (int q = 1; q <= 5; ++q) {
        const float v = __ldg(bidx + q * NN + k);
        s_g[(q - 1) * NN + k] = make_float2(v, v);
      }
    }
    const float m0 = __ldg(bm0 + k), m1 = __ldg(bm1 + k);
    if constexpr (MED == MED_PSV) {
      const float l2m = m0 + static_cast<float>(4.0 / 3.0) * m1;
      const float lam = l2m - 2.0f * m1;
      s_g[5 * NN + k] = make_float2(l2m, l2m);
      s_g[6 * NN + k] = make_float2(lam, lam);
      s_g[7 * NN + k] = make_float2(m1, m1);
    } else {
      s_g[5 * NN + k] = make_float2(m0, m0);  // SH: mu; acoustic: 1/rho
    }
  }
  grid_dep_wait();
  const int istep = (ss.mode != 0 || tw.src.n > 0) ? *istep_dev : 0;
  const W *U = reinterpret_cast<const W *>(f.u);
  W *A = reinterpret_cast<W *>(f.a);
  const size_t Sv = static_cast<size_t>(S) / 2;
  const size_t lofs = static_cast<size_t>(s0) / 2;
  const uint8_t eflag = st.eflag[e];
  const bool fused = fu.enabled && (eflag & kElemPrivate) && iz >= 1 && iz <= N - 2;
  if (fused && act) {
    // velocity of this row's private points, needed after the divergence
#pragma unroll
    for (int ix = 1; ix <= N - 2; ++ix)
      cp_async<sizeof(W)>(&s_vp[((iz - 1) * (N - 2) + ix - 1) * 32 + lane],
                          reinterpret_cast<const W *>(fu.v) + g[ix] * Sv + lofs);
  }
  bool fused_adj = false;
  if constexpr (FR) {
    fused_adj = fr.adjoint_update && (eflag & kElemPrivate) && iz >= 1 && iz <= N - 2;
    if (act) {
#pragma unroll
      for (int ix = 0; ix < N; ++ix)
        cp_async<sizeof(W)>(&s_aa[(iz * N + ix) * 32 + lane], reinterpret_cast<const W *>(fr.aa) + g[ix] * Sv + lofs);
      if (fused_adj) {
#pragma unroll
        for (int ix = 1; ix <= N - 2; ++ix)
          cp_async<sizeof(W)>(&s_av[((iz - 1) * (N - 2) + ix - 1) * 32 + lane],
                              reinterpret_cast<const W *>(fr.av) + g[ix] * Sv + lofs);
      }
    }
  }
  W ur[N];
#pragma unroll
  for (int ix = 0; ix < N; ++ix) {
    if (act) ur[ix] = swz(U[g[ix] * Sv + lofs]);
    else { for (int c = 0; c < NC; ++c) setpr(ur[ix], c, make_float2(0.f, 0.f)); }
    s_u[(iz * N + ix) * 32 + lane] = ur[ix];
  }
  if constexpr (FR) {
    const W *UA = reinterpret_cast<const W *>(fr.au);
#pragma unroll
    for (int ix = 0; ix < N; ++ix) {
      W w;
      if (act) w = swz(UA[g[ix] * Sv + lofs]);
      else { for (int c = 0; c < NC; ++c) setpr(w, c, make_float2(0.f, 0.f)); }
      s_ua[(iz * N + ix) * 32 + lane] = w;
    }
  }
  __syncthreads();
  float2 hpz[N], hpwz[N];
#pragma unroll
  for (int l = 0; l < N; ++l) {
    hpz[l] = C_HP2(iz * N + l);
    hpwz[l] = C_HPW2(iz * N + l);
  }
  W fx[N];
#pragma unroll
  for (int ix = 0; ix < N; ++ix) {
    const int k = iz * N + ix;
    float2 dxi[NC], dga[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) { dxi[c] = make_float2(0.f, 0.f); dga[c] = make_float2(0.f, 0.f); }
#pragma unroll
    for (int l = 0; l < N; ++l) {
      const W col = s_u[(l * N + ix) * 32 + lane];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        dxi[c] = fma2(C_HP2(ix * N + l), pr(ur[l], c), dxi[c]);
        dga[c] = fma2(hpz[l], pr(col, c), dga[c]);
      }
    }
    const float2 xix = AFF ? cgeo[0] : s_g[0 * NN + k], xiz = AFF ? cgeo[1] : s_g[1 * NN + k];
    const float2 gax = AFF ? cgeo[2] : s_g[2 * NN + k], gaz = AFF ? cgeo[3] : s_g[3 * NN + k];
    const float2 jac = AFF ? cgeo[4] : s_g[4 * NN + k];
    float2 du[NC][2];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      du[c][0] = fma2(xix, dxi[c], mul2(gax, dga[c]));
      du[c][1] = fma2(xiz, dxi[c], mul2(gaz, dga[c]));
    }
    float2 T[NC][2];
    if constexpr (MED == MED_PSV) {
      const float2 l2m = s_g[5 * NN + k], lam = s_g[6 * NN + k], mu = s_g[7 * NN + k];
      T[0][0] = fma2(l2m, du[0][0], mul2(lam, du[1][1]));
      T[1][1] = fma2(l2m, du[1][1], mul2(lam, du[0][0]));
      T[0][1] = mul2(mu, add2(du[0][1], du[1][0]));
      T[1][0] = T[0][1];
    } else {
      const float2 m = s_g[5 * NN + k];
      T[0][0] = mul2(m, du[0][0]);
      T[0][1] = mul2(m, du[0][1]);
    }
    W f1;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      setpr(fx[ix], c, mul2(jac, fma2(T[c][0], xix, mul2(T[c][1], xiz))));
      setpr(f1, c, mul2(jac, fma2(T[c][0], gax, mul2(T[c][1], gaz))));
    }
    s_fg[k * 32 + lane] = f1;
    if constexpr (FR && MED == MED_PSV) {
      // adjoint displacement gradient at this point (same operators)
      float2 axi[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)}, aga[2] = {axi[0], axi[1]};
#pragma unroll
      for (int l = 0; l < N; ++l) {
        const W row = s_ua[(iz * N + l) * 32 + lane];
        const W col = s_ua[(l * N + ix) * 32 + lane];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          axi[c] = fma2(C_HP2(ix * N + l), pr(row, c), axi[c]);
          aga[c] = fma2(hpz[l], pr(col, c), aga[c]);
        }
      }
      float2 da[2][2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        da[c][0] = fma2(xix, axi[c], mul2(gax, aga[c]));
        da[c][1] = fma2(xiz, axi[c], mul2(gaz, aga[c]));
      }
      // frechet_derivative.hpp:14-116 per shot, before the material and dt
      // factors (applied once to the sum over shots):
      //   kappa ~ div(s_adj) div(s_bwd); mu ~ eps_adj : eps_bwd - div div / 3;
      //   rho ~ a_adj . u_bwd
      const float2 half = make_float2(0.5f, 0.5f), two = make_float2(2.0f, 2.0f);
      const float2 mthird = make_float2(static_cast<float>(-1.0 / 3.0), static_cast<float>(-1.0 / 3.0));
      const float2 a_xz = mul2(half, add2(da[1][0], da[0][1]));
      const float2 b_xz = mul2(half, add2(du[1][0], du[0][1]));
      const float2 kap = mul2(add2(da[0][0], da[1][1]), add2(du[0][0], du[1][1]));
      float2 mu = fma2(da[0][0], du[0][0], mul2(da[1][1], du[1][1]));
      mu = fma2(two, mul2(a_xz, b_xz), mu);
      mu = fma2(mthird, kap, mu);
      float2 rho = make_float2(0.f, 0.f);
      if (act) {
        if (ix == 0) cp_async_wait_all();
        const W fa = swz(s_aa[k * 32 + lane]);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const float mi = fr.minv[g[ix] * 2 + c];
          rho = fma2(mul2(pr(fa, c), make_float2(mi, mi)), pr(ur[ix], c), rho);
        }
      }
      s_red[(0 * NN + k) * 32 + lane] = act ? rho.x + rho.y : 0.f;
      s_red[(1 * NN + k) * 32 + lane] = act ? mu.x + mu.y : 0.f;
      s_red[(2 * NN + k) * 32 + lane] = act ? kap.x + kap.y : 0.f;
    }
  }
  __syncthreads();
  if constexpr (FR && MED == MED_PSV) {
    // sum over this launch's shots (32 lanes), material and dt factors,
    // FP64 accumulation (compute_material_derivatives.tpp:130-150)
    for (int q = threadIdx.x; q < 3 * NN; q += blockDim.x) {
      const float4 *r4 = reinterpret_cast<const float4 *>(s_red + q * 32);
      float sum = 0.f;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float4 v = r4[(j + q) & 7];  // rotated start: conflict-free quarter warps
        sum += (v.x + v.y) + (v.z + v.w);
      }
      const int which = q / NN, k = q % NN;
      const size_t p = static_cast<size_t>(e) * NN + k;
      const float m0 = __ldg(bm0 + k), m1 = __ldg(bm1 + k);
      float scale;
      if (which == 0) scale = -1.0f * st.mat2[p] * fr.dt;                            // rho
      else if (which == 1) scale = -2.0f * m1 * fr.dt;                               // mu
      else scale = -1.0f * (m0 + static_cast<float>(4.0 / 3.0) * m1 - m1) * fr.dt;  // kappa' = lambda + mu
      fr.kern[p * 3 + which] += static_cast<double>(sum * scale);
    }
  }
  const int slot = (ss.mode != 0) ? ss.slot[e] : -1;
  if (fused) cp_async_wait_all();
  const float2 wz = C_W2(iz);
  const float2 neg = make_float2(-1.0f, -1.0f);
#pragma unroll
  for (int ix = 0; ix < N; ++ix) {
    float2 t1[NC], t2[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) { t1[c] = make_float2(0.f, 0.f); t2[c] = make_float2(0.f, 0.f); }
#pragma unroll
    for (int l = 0; l < N; ++l) {
      const W col = s_fg[(l * N + ix) * 32 + lane];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        t1[c] = fma2(pr(fx[l], c), C_HPW2(ix * N + l), t1[c]);
        t2[c] = fma2(pr(col, c), hpwz[l], t2[c]);
      }
    }
    float2 acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = mul2(fma2(wz, t1[c], mul2(C_W2(ix), t2[c])), neg);
    if ((eflag & 3) || slot >= 0) {
      // boundary elements: Stacey, free surface and the Stacey store, per shot
      const size_t p = (static_cast<size_t>(e) * N + iz) * N + ix;
      const uint8_t b = (eflag & 3) ? st.bnd[p] : 0;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        float a2[2];
#pragma unroll
        for (int c = 0; c < NC; ++c) a2[c] = j == 0 ? acc[c].x : acc[c].y;
        if ((b & 1) && act) {
          const float *Vp = f.v + (static_cast<size_t>(g[ix]) * S + s0 + j) * NC;
          float vel[2];
#pragma unroll
          for (int c = 0; c < NC; ++c) vel[c] = Vp[c];
          stacey<MED>(__ldg(bm0 + iz * N + ix), __ldg(bm1 + iz * N + ix),
                      st.mat2 ? st.mat2[p] : 0.f, st.bnd_nx[p], st.bnd_nz[p], st.bnd_w[p], vel, a2);
        }
        if (b & 2) {
#pragma unroll
          for (int c = 0; c < NC; ++c) a2[c] = 0.f;
        }
        if (slot >= 0 && act) {
          const size_t base =
              ((((static_cast<size_t>(s0 + j) * ss.nstep + istep) * ss.nstacey + slot) * N + iz) * N + ix) * 2;
          if (ss.mode == 1) {
#pragma unroll
            for (int c = 0; c < NC; ++c) ss.data[base + c] = a2[c];
          } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) a2[c] = ss.data[base + c];
          }
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          if (j == 0) acc[c].x = a2[c]; else acc[c].y = a2[c];
        }
      }
    }
    if (!act) continue;
    const size_t at = g[ix] * Sv + lofs;
    if constexpr (FR && MED == MED_PSV) {
      if (fused_adj && ix >= 1 && ix <= N - 2) {
        // the adjoint wavefield's private point: its Frechet contribution
        // was taken above; now a = force / M, corrector, next predictor
        W va = swz(s_av[((iz - 1) * (N - 2) + ix - 1) * 32 + lane]), ua = s_ua[(iz * N + ix) * 32 + lane], aa;
        const W fa = swz(s_aa[(iz * N + ix) * 32 + lane]);
        const float2 adt = make_float2(fr.adt, fr.adt), adt2 = make_float2(fr.adt2, fr.adt2);
        const float2 adtsq2 = make_float2(fr.adtsq2, fr.adtsq2);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const float mi = fr.minv[g[ix] * NC + c];
          const float2 a_c = mul2(pr(fa, c), make_float2(mi, mi));
          setpr(aa, c, a_c);
          setpr(va, c, fma2(adt2, a_c, pr(va, c)));
        }
        if (fr.last) {
          reinterpret_cast<W *>(fr.aa)[at] = swz(aa);
          reinterpret_cast<W *>(fr.av)[at] = swz(va);
        } else {
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            setpr(ua, c, add2(pr(ua, c), fma2(adt, pr(va, c), mul2(adtsq2, pr(aa, c)))));
            setpr(va, c, fma2(adt2, pr(aa, c), pr(va, c)));
          }
          reinterpret_cast<W *>(fr.au)[at] = swz(ua);
          reinterpret_cast<W *>(fr.av)[at] = swz(va);
          reinterpret_cast<W *>(fr.aa)[at] = swz(make_zero_w<W>());
        }
      }
    }
    if (fused && ix >= 1 && ix <= N - 2) {
      // element-private point: a = force / M, corrector, next predictor
      // (the update kernel's arithmetic, newmark.tpp:44-47 and 98-105)
      W *Vw = reinterpret_cast<W *>(fu.v);
      W *Uw = reinterpret_cast<W *>(f.u);
      W vel = swz(s_vp[((iz - 1) * (N - 2) + ix - 1) * 32 + lane]), uu = s_u[(iz * N + ix) * 32 + lane], aa;
      const float2 dt = make_float2(fu.dt, fu.dt), dt2 = make_float2(fu.dt2, fu.dt2);
      const float2 dtsq2 = make_float2(fu.dtsq2, fu.dtsq2);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float mi = fu.minv[g[ix] * NC + c];
        const float2 a_c = mul2(acc[c], make_float2(mi, mi));
        setpr(aa, c, a_c);
        setpr(vel, c, fma2(dt2, a_c, pr(vel, c)));
      }
      if (fu.last) {
        A[at] = swz(aa);
        Vw[at] = swz(vel);
      } else {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          setpr(uu, c, add2(pr(uu, c), fma2(dt, pr(vel, c), mul2(dtsq2, pr(aa, c)))));
          setpr(vel, c, fma2(dt2, pr(aa, c), pr(vel, c)));
        }
        Uw[at] = swz(uu);
        Vw[at] = swz(vel);
      }
    } else {
      W out;
#pragma unroll
      for (int c = 0; c < NC; ++c) setpr(out, c, acc[c]);
      vred(A + at, swz(out));
    }
  }
  tail_work<MED, N>(st, f, S, istep, tw, blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y);
}

#endif  // !SFB_FP64

// Dynamic shared memory above the default 48 KiB needs an opt-in once per
// kernel instantiation.
template <int MED, int N, int SPL, int MINB>
size_t shots_smem_opt_in() {
  constexpr size_t bytes = shots_smem_bytes<MED, N, SPL>();
  if constexpr (bytes > 48 * 1024) {
    static bool done = false;
    if (!done) {
      cudaFuncSetAttribute(k_stiffness_shots<MED, N, SPL, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(bytes));
      done = true;
    }
  }
  return bytes;
}

// variant: kShotsPacked (two shots per lane, f32x2), kShotsPair (two shots
// per lane, scalar), kShotsSingle (one shot per lane); kShotsAuto picks the
// packed kernel when it applies.  Two shots per lane need an even S and
// (for the static shared staging) NGLL <= 5.  The FP64 build has the
// one-shot-per-lane kernel only.
template <int MED, int N, int MINB>
void launch_shots(const Static &st, const MediumFields &f, int S, const StaceyStore &ss, const int *istep_dev,
                  const TailWork &tw, const FusedUpdate &fu, int variant, cudaStream_t stream) {
#ifndef SFB_FP64
  if constexpr (N <= 5) {
    if (S % 2 == 0 && variant != kShotsSingle) {
      dim3 grid(f.nelem, (S / 2 + 31) / 32);
      if (variant == kShotsPair)
        launch_step_kernel(k_stiffness_shots<MED, N, 2, MINB>, grid, N * 32, shots_smem_opt_in<MED, N, 2, MINB>(),
                           stream, st, f, S, ss, istep_dev, tw, fu);
      else if (st.affine[MED] && st.pack_aff)  // compact block: geometry constants in registers
        launch_step_kernel(k_stiffness_pk<MED, N, MINB, false, true>, grid, N * 32, 0, stream, st, f, S, ss, istep_dev,
                           tw, fu, FrechetFuse{});
      else
        launch_step_kernel(k_stiffness_pk<MED, N, MINB, false>, grid, N * 32, 0, stream, st, f, S, ss, istep_dev, tw, fu,
                           FrechetFuse{});
      return;
    }
  }
#else
  (void)variant;
#endif
  dim3 grid(f.nelem, (S + 31) / 32);
  launch_step_kernel(k_stiffness_shots<MED, N, 1, MINB>, grid, N * 32, shots_smem_opt_in<MED, N, 1, MINB>(), stream,
                     st, f, S, ss, istep_dev, tw, fu);
}

#ifndef SFB_FP64
constexpr size_t kFrechetDynSmem = (2 * 25 + 9) * 32 * sizeof(float4) + 3 * 25 * 32 * sizeof(float);
#endif


// ---------------------------------------------------------------------------
// Point sources (compute_source_interaction.tpp:77-95): one block per source.
// ---------------------------------------------------------------------------
__global__ void k_sources(Static st, SourceSet src, MediumFields f, int medium, int N,
                          const int *istep_dev, int nshots) {
  const int i = blockIdx.x;
  const int k = threadIdx.x;
  if (k >= N * N) return;
  if (src.medium[i] != medium) return;
  const int istep = *istep_dev;
  if (istep < 0 || istep >= src.nstep) return;
  const int e = src.elem[i];
  const size_t p = static_cast<size_t>(e) * N * N + k;
  const int gi = st.iglob[p];
  const int s = src.shot[i];
  real *A = f.a + (static_cast<size_t>(gi) * nshots + s) * f.nc;
  for (int c = 0; c < f.nc; ++c) {
    const real stf = src.stf[(static_cast<size_t>(i) * src.nstep + istep) * 2 + c];
    const real arr = src.array[(static_cast<size_t>(i) * 2 + c) * N * N + k];
    real val = stf * arr;
    if (medium == MED_AC) val = stf * arr / st.mat1[p];
    atomicAdd(A + c, val);
  }
}

// ---------------------------------------------------------------------------
// Fluid-solid coupling (coupled_interface.tpp:55-86, compute_coupling.hpp).
// ---------------------------------------------------------------------------
__global__ void k_couple_acoustic(CouplingSet c, MediumFields ac, MediumFields el, int nshots) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= c.n || s >= nshots) return;
  const real2 u = reinterpret_cast<const real2 *>(el.u)[static_cast<size_t>(c.other[i]) * nshots + s];
  atomicAdd(ac.a + static_cast<size_t>(c.self[i]) * nshots + s, c.factor[i] * (c.nx[i] * u.x + c.nz[i] * u.y));
}

__global__ void k_couple_elastic(CouplingSet c, MediumFields el, MediumFields ac, int nshots,
                                 int ac_divided) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= c.n || s >= nshots) return;
  const int o = c.other[i];
  const real r = ac.a[static_cast<size_t>(o) * nshots + s];
  const real chi_dd = ac_divided ? r : r * ac.minv[o];
  real *A = el.a + (static_cast<size_t>(c.self[i]) * nshots + s) * 2;
  atomicAdd(A, c.factor[i] * c.nx[i] * chi_dd);
  atomicAdd(A + 1, c.factor[i] * c.nz[i] * chi_dd);
}

// ---------------------------------------------------------------------------
// Deterministic sources and coupling (see DetTail): the terms of tail_work,
// summed per target point and shot in a fixed order.
// ---------------------------------------------------------------------------
template <int MED, int N>
__global__ void k_tail_det(Static st, MediumFields f, int S, const int *istep_dev, TailWork tw, DetTail dt) {
  constexpr int NC = (MED == MED_PSV) ? 2 : 1;
  constexpr int NN = N * N;
  const int istep = *istep_dev;
  const bool src_on = tw.src.n > 0 && istep >= 0 && istep < tw.src.nstep;
  const size_t total = static_cast<size_t>(dt.ntarget) * S;
  for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(idx / S), s = static_cast<int>(idx % S);
    real acc[2] = {0, 0};
    for (int q = dt.tgt_begin[t]; q < dt.tgt_begin[t + 1]; ++q) {
      const int e = dt.ent[q];
      if (e >= 0) {
        const int i = e / NN, kk = e % NN;
        if (!src_on || tw.src.shot[i] != s) continue;
        const size_t p = static_cast<size_t>(tw.src.elem[i]) * NN + kk;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const real stf = tw.src.stf[(static_cast<size_t>(i) * tw.src.nstep + istep) * 2 + c];
          const real arr = tw.src.array[(static_cast<size_t>(i) * 2 + c) * NN + kk];
          acc[c] += (MED == MED_AC) ? stf * arr / st.mat1[p] : stf * arr;
        }
      } else if (tw.cp_mode == 1) {  // acoustic self += w (n . u_elastic)
        const int i = -e - 1;
        const real2 u = reinterpret_cast<const real2 *>(tw.other.u)[static_cast<size_t>(tw.cp.other[i]) * S + s];
        acc[0] += tw.cp.factor[i] * (tw.cp.nx[i] * u.x + tw.cp.nz[i] * u.y);
      } else if (tw.cp_mode == 2) {  // elastic self += w n chi_ddot
        const int i = -e - 1;
        const int oi = tw.cp.other[i];
        const real r = tw.other.a[static_cast<size_t>(oi) * S + s];
        const real chi_dd = tw.other_divided ? r : r * tw.other.minv[oi];
        acc[0] += tw.cp.factor[i] * tw.cp.nx[i] * chi_dd;
        acc[1] += tw.cp.factor[i] * tw.cp.nz[i] * chi_dd;
      }
    }
    real *A = f.a + (static_cast<size_t>(dt.tgt_g[t]) * S + s) * NC;
#pragma unroll
    for (int c = 0; c < NC; ++c) A[c] += acc[c];
  }
}

// ---------------------------------------------------------------------------
// Receivers (compute_seismogram.tpp:98-135, wavefield.hpp): one block of 64
// threads per (receiver, shot).
// ---------------------------------------------------------------------------
__device__ __forceinline__ real ld_comp(const MediumFields &f, int which, int s, int g, int c,
                                        real dt2, int mode, int S) {
  const size_t idx = (static_cast<size_t>(g) * S + s) * f.nc + c;
  const size_t m = static_cast<size_t>(g) * f.nc + c;
  if (which == 0) return f.u[idx];
  if (mode == 0) return which == 1 ? f.v[idx] : f.a[idx];
  const real a = f.a[idx] * f.minv[m];
  if (which == 2) return a;
  return f.v[idx] + dt2 * a;
}

__global__ void k_receivers(Static st, ReceiverSet rec, MediumFields f_psv, MediumFields f_sh,
                            MediumFields f_ac, int N, real dt2, int mode, const int *istep_dev, int S) {
  __shared__ real s_val[2][64];
  __shared__ real s_red[2][64];
  const int r = blockIdx.x, s = blockIdx.y, k = threadIdx.x;
  const int istep = *istep_dev;
  if (istep < 0 || istep % rec.nsbs != 0) return;
  const int isig = rec.backward_nstep > 0 ? (rec.backward_nstep - 1) / rec.nsbs - istep / rec.nsbs
                                          : istep / rec.nsbs;
  if (isig >= rec.max_sig) return;
  const int e = rec.elem[r];
  const int NN = N * N;
  const int iz = k / N, ix = k % N;
  const size_t p = static_cast<size_t>(e) * NN + k;
  // medium of this receiver's element: decided from the element ranges
  int med;
  const MediumFields *F;
  if (e >= f_psv.elem_begin && e < f_psv.elem_begin + f_psv.nelem) { med = MED_PSV; F = &f_psv; }
  else if (e >= f_sh.elem_begin && e < f_sh.elem_begin + f_sh.nelem) { med = MED_SH; F = &f_sh; }
  else { med = MED_AC; F = &f_ac; }
  const int g = (k < NN) ? st.iglob[p] : 0;
  const real h = (k < NN) ? rec.lagrange[static_cast<size_t>(r) * NN + k] : real(0);
  for (int it = 0; it < rec.ntypes; ++it) {
    const int type = rec.types[it];
    real w0 = 0, w1 = 0;
    const bool need_grad = (med == MED_AC && type != 3) || (med == MED_PSV && type == 3);
    if (need_grad) {
      // field on all points of the element, then gradient at this point
      const int which = (med == MED_AC) ? (type == 3 ? 2 : type) : 0;
      if (k < NN) {
        s_val[0][k] = ld_comp(*F, which, s, g, 0, dt2, mode, S);
        s_val[1][k] = (F->nc > 1) ? ld_comp(*F, which, s, g, 1, dt2, mode, S) : real(0);
      }
      __syncthreads();
      if (k < NN) {
        real dxi[2] = {0, 0}, dga[2] = {0, 0};
        for (int l = 0; l < N; ++l)
          for (int c = 0; c < F->nc; ++c) {
            dxi[c] += C_HP(ix * N + l) * s_val[c][iz * N + l];
            dga[c] += C_HP(iz * N + l) * s_val[c][l * N + ix];
          }
        const real xix = st.xix[p], xiz = st.xiz[p], gax = st.gax[p], gaz = st.gaz[p];
        real du[2][2];
        for (int c = 0; c < F->nc; ++c) {
          du[c][0] = xix * dxi[c] + gax * dga[c];
          du[c][1] = xiz * dxi[c] + gaz * dga[c];
        }
        if (med == MED_AC) {
          const real ri = st.mat0[p];
          w0 = ri * du[0][0];
          w1 = ri * du[0][1];
        } else {
          const real kappa = st.mat0[p], mu = st.mat1[p];
          const real l2m = kappa + kFourThirds * mu;
          const real lam = l2m - static_cast<real>(2) * mu;
          w0 = static_cast<real>(-1) * ((lam + static_cast<real>(2.0 / 3.0) * mu) * (du[0][0] + du[1][1]));
          w1 = 0;
        }
      }
      __syncthreads();
    } else if (k < NN) {
      if (med == MED_AC) {  // pressure = -chi_ddot
        w0 = static_cast<real>(-1) * ld_comp(*F, 2, s, g, 0, dt2, mode, S);
      } else {
        w0 = ld_comp(*F, type, s, g, 0, dt2, mode, S);
        w1 = (F->nc > 1) ? ld_comp(*F, type, s, g, 1, dt2, mode, S) : real(0);
      }
    }
    s_red[0][k] = h * w0;
    s_red[1][k] = h * w1;
    __syncthreads();
    if (k == 0) {
      real a0 = 0, a1 = 0;
      for (int j = 0; j < NN; ++j) {
        a0 += s_red[0][j];
        a1 += s_red[1][j];
      }
      const real sn = rec.sinv[r], cs = rec.cosv[r];
      real *o = rec.seis + ((((static_cast<size_t>(s) * rec.max_sig + isig) * rec.ntypes + it) *
                              rec.n + r) * 2);
      o[0] = cs * a0 - sn * a1;
      o[1] = sn * a0 + cs * a1;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Newmark (newmark.tpp) and the fused update.  Fields of one medium are
// [S][ld] floats with ld = (nglob + nglob%2) * nc, a multiple of 4 for P-SV
// and of 2 otherwise; the float4 / float2 paths below rely on that.
// ---------------------------------------------------------------------------
// Kahan-compensated accumulation s += x with running compensation c
// (Kahan 1965): the low-order bits lost by each FP32 add are carried to the
// next one.  Explicit round-to-nearest adds keep the compiler from
// contracting or reassociating the compensation away.
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ real kahan_add(real s, real &c, real x) {
  const real y = sub_rn(x, c);
  const real t = add_rn(s, y);
  c = sub_rn(sub_rn(t, s), y);
  return t;
}

__global__ void k_predictor(real *u, real *v, real *a, size_t n, real dt, real dt2,
                            real dtsq2, real *cu, real *cv) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const real ai = a[i];
    const real vi = v[i];
    if (cu) {
      real c_u = cu[i], c_v = cv[i];
      u[i] = kahan_add(u[i], c_u, dt * vi + dtsq2 * ai);
      v[i] = kahan_add(vi, c_v, dt2 * ai);
      cu[i] = c_u;
      cv[i] = c_v;
    } else {
      u[i] += dt * vi + dtsq2 * ai;
      v[i] = vi + dt2 * ai;
    }
    a[i] = 0;
  }
}
__global__ void k_corrector(real *v, const real *a, size_t n, real dt2) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    v[i] += dt2 * a[i];
}
__global__ void k_divide(real *a, const real *minv, size_t n, int nshots, int nc) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t c = i % nc, g = (i / nc) / nshots;
    a[i] = a[i] * minv[g * nc + c];
  }
}

__global__ void k_advance(Control *ctrl) { ctrl->istep += 1; }

// Snapshot restore at the start of combined step istep: backward u := u at
// step istep, v := v half a step later, both from the forward run.
__global__ void k_restore(RestoreParams P) {
  const int istep = P.ctrl->istep;
  if (istep <= 0 || istep % P.interval != 0) return;
  const int slot = istep / P.interval - 1;
  if (slot >= P.count) return;
  for (int m = 0; m < P.nm; ++m) {
    const real *su = P.ck_u[m] + slot * P.ck_stride[m];
    const real *sv = P.ck_v[m] + slot * P.ck_stride[m];
    const size_t n4 = P.n[m] / 4;  // slots and fields start aligned to four values
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
      reinterpret_cast<real4 *>(P.u[m])[i] = reinterpret_cast<const real4 *>(su)[i];
      reinterpret_cast<real4 *>(P.v[m])[i] = reinterpret_cast<const real4 *>(sv)[i];
    }
    for (size_t i = n4 * 4 + blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < P.n[m];
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
      P.u[m][i] = su[i];
      P.v[m][i] = sv[i];
    }
  }
}

// ---------------------------------------------------------------------------
// Unified update: for every medium and shot, a = force * minv, v += dt/2 a
// (corrector, newmark.tpp:44-47), seismogram taps on (u, v, a), then unless
// this is the last step the next predictor u += dt v + dt^2/2 a,
// v += dt/2 a, force = 0 (newmark.tpp:98-105).  The step counter is read at
// entry by every CTA and advanced by the last CTA to finish.
// ---------------------------------------------------------------------------
// The tapped nodal value: field (0 u, 1 v, 2 a) * 2 + component, picked
// with selects (no indexed local array).
__device__ __forceinline__ real pick6(int wh, real a0, real a1, real b0, real b1, real c0, real c1) {
  const real lo = (wh & 1) ? a1 : a0, mid = (wh & 1) ? b1 : b0, hi = (wh & 1) ? c1 : c0;
  return wh < 2 ? lo : (wh < 4 ? mid : hi);
}

__device__ __forceinline__ real2 mk2(real x, real y) { return real2{x, y}; }
__device__ __forceinline__ real4 mk4(real x, real y, real z, real w) { return real4{x, y, z, w}; }

__device__ __forceinline__ void apply_taps(const ReceiverTaps &tp, int g, real u0, real u1, real v0, real v1,
                                           real a0, real a1, real *seis_row) {
  if (!((tp.mask[g >> 5] >> (g & 31)) & 1u)) return;
  int lo = 0, hi = tp.nsup - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (tp.sup_g[mid] < g) lo = mid + 1; else hi = mid;
  }
  if (tp.sup_g[lo] != g) return;
  for (int q = tp.sup_begin[lo]; q < tp.sup_begin[lo + 1]; ++q)
    atomicAdd(seis_row + tp.slot[q], tp.w[q] * pick6(tp.which[q], u0, u1, v0, v1, a0, a1));
}

// EXTRA: Kahan terms or snapshot writes present (a separate instantiation
// keeps the plain update free of their registers and branches).
template <bool EXTRA>
__global__ void k_update_all(UpdateParams P) {
  grid_dep_wait();
  const int istep = P.ctrl ? P.ctrl->istep : -1;
  // Sample index: istep / nsbs forward; in the backward run of the combined
  // loop (dir -1) samples are numbered in the order the loop reaches them,
  // from step nstep - 1 down (time_marching.tpp:208-212, the seismogram
  // step counter of the time scheme).
  const int isig_raw = P.dir < 0 ? (P.nstep - 1) / P.nsbs - istep / P.nsbs : istep / P.nsbs;
  const bool record = P.seis != nullptr && istep >= 0 && (istep % P.nsbs) == 0 && isig_raw < P.max_sig;
  const int isig = record ? isig_raw : 0;
  const size_t total = P.begin[P.nm];
  const int S = P.nshots;
  // snapshot slots this step writes (forward run with checkpoints)
  int ck_uslot = -1, ck_vslot = -1;
  if (EXTRA && P.ck_interval > 0 && istep >= 0 && !P.last) {
    if ((istep + 1) % P.ck_interval == 0) ck_uslot = (istep + 1) / P.ck_interval - 1;
    if (istep % P.ck_interval == 0) ck_vslot = istep / P.ck_interval - 1;
    if (ck_uslot >= P.ck_count) ck_uslot = -1;
    if (ck_vslot >= P.ck_count) ck_vslot = -1;
  }
  if constexpr (!EXTRA) {
    // plain update: unit w of a medium is its pairs 2w and 2w + 1, read and
    // written as one float4 per array (a medium with an odd number of pairs
    // ends with a one-pair unit).  A pair is (g, s) with both components
    // (nc = 2) or two consecutive entries of [g][s] (nc = 1); entry e of a
    // unit is component e % 2 of its pair e / 2 (nc = 2) or entry e (nc = 1).
    // first unit of media 1 and 2 (at most three media), in registers
    const size_t ub1 = (P.begin[1] - P.begin[0] + 1) / 2;
    const size_t ub2 = P.nm > 1 ? ub1 + (P.begin[2] - P.begin[1] + 1) / 2 : ub1;
    const size_t units = P.nm > 2 ? ub2 + (P.begin[3] - P.begin[2] + 1) / 2 : ub2;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t w = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; w < units; w += stride) {
      int mi = 0;
      size_t ub = 0;
      if (P.nm > 1 && w >= ub1) { mi = 1; ub = ub1; }
      if (P.nm > 2 && w >= ub2) { mi = 2; ub = ub2; }
      const UpdateMedium &M = P.m[mi];
      const size_t ld2 = P.begin[mi + 1] - P.begin[mi];
      const size_t p0 = 2 * (w - ub);
      const bool two = p0 + 1 < ld2;
      real4 r, vel, uu;
      if (two) {
        r = reinterpret_cast<const real4 *>(M.a)[p0 / 2];
        vel = reinterpret_cast<const real4 *>(M.v)[p0 / 2];
        uu = reinterpret_cast<const real4 *>(M.u)[p0 / 2];
      } else {
        const real2 r2 = reinterpret_cast<const real2 *>(M.a)[p0];
        const real2 v2 = reinterpret_cast<const real2 *>(M.v)[p0];
        const real2 u2 = reinterpret_cast<const real2 *>(M.u)[p0];
        r = mk4(r2.x, r2.y, 0, 0);
        vel = mk4(v2.x, v2.y, 0, 0);
        uu = mk4(u2.x, u2.y, 0, 0);
      }
      real m[4] = {0, 0, 0, 0};
      int g[4] = {0, 0, 0, 0}, sh[4] = {0, 0, 0, 0};
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        if (i == 1 && !two) continue;
        if (M.nc == 2) {
          const uint32_t n = static_cast<uint32_t>(p0 + i);
          const int gi = static_cast<int>(P.sdiv.div(n));
          const real2 mm = reinterpret_cast<const real2 *>(M.minv)[gi];
          g[2 * i] = g[2 * i + 1] = gi;
          sh[2 * i] = sh[2 * i + 1] = static_cast<int>(n - static_cast<uint32_t>(gi) * S);
          m[2 * i] = mm.x;
          m[2 * i + 1] = mm.y;
        } else {
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const uint32_t n = static_cast<uint32_t>(2 * (p0 + i) + j);
            g[2 * i + j] = static_cast<int>(P.sdiv.div(n));
            sh[2 * i + j] = static_cast<int>(n - static_cast<uint32_t>(g[2 * i + j]) * S);
            m[2 * i + j] = M.minv[g[2 * i + j]];
          }
        }
      }
      const real4 acc = mk4(r.x * m[0], r.y * m[1], r.z * m[2], r.w * m[3]);
      vel.x += P.dt2 * acc.x;  // corrector (newmark.tpp:44-47)
      vel.y += P.dt2 * acc.y;
      vel.z += P.dt2 * acc.z;
      vel.w += P.dt2 * acc.w;
      if (record && M.taps.nsup > 0) {
        if (M.nc == 2) {
          apply_taps(M.taps, g[0], uu.x, uu.y, vel.x, vel.y, acc.x, acc.y,
                     P.seis + (static_cast<size_t>(sh[0]) * P.max_sig + isig) * P.slots);
          if (two)
            apply_taps(M.taps, g[2], uu.z, uu.w, vel.z, vel.w, acc.z, acc.w,
                       P.seis + (static_cast<size_t>(sh[2]) * P.max_sig + isig) * P.slots);
        } else {
          const real us[4] = {uu.x, uu.y, uu.z, uu.w}, vs[4] = {vel.x, vel.y, vel.z, vel.w};
          const real as[4] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (e < 2 || two)
              apply_taps(M.taps, g[e], us[e], 0, vs[e], 0, as[e], 0,
                         P.seis + (static_cast<size_t>(sh[e]) * P.max_sig + isig) * P.slots);
        }
      }
      if (!P.last) {
        uu.x += P.dt * vel.x + P.dtsq2 * acc.x;  // next predictor (newmark.tpp:98-105)
        uu.y += P.dt * vel.y + P.dtsq2 * acc.y;
        uu.z += P.dt * vel.z + P.dtsq2 * acc.z;
        uu.w += P.dt * vel.w + P.dtsq2 * acc.w;
        vel.x += P.dt2 * acc.x;
        vel.y += P.dt2 * acc.y;
        vel.z += P.dt2 * acc.z;
        vel.w += P.dt2 * acc.w;
      }
      // last step: a and v stored, u kept; otherwise u, v stored and a = 0
      const real4 a_out = P.last ? acc : mk4(0, 0, 0, 0);
      if (two) {
        if (!P.last) reinterpret_cast<real4 *>(M.u)[p0 / 2] = uu;
        reinterpret_cast<real4 *>(M.v)[p0 / 2] = vel;
        reinterpret_cast<real4 *>(M.a)[p0 / 2] = a_out;
      } else {
        if (!P.last) reinterpret_cast<real2 *>(M.u)[p0] = mk2(uu.x, uu.y);
        reinterpret_cast<real2 *>(M.v)[p0] = mk2(vel.x, vel.y);
        reinterpret_cast<real2 *>(M.a)[p0] = mk2(a_out.x, a_out.y);
      }
    }
  } else
  for (size_t j = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; j < total;
       j += static_cast<size_t>(gridDim.x) * blockDim.x) {
    int mi = 0;
    while (mi + 1 < P.nm && j >= P.begin[mi + 1]) ++mi;
    const UpdateMedium &M = P.m[mi];
    const size_t jj = j - P.begin[mi];
    // pair jj holds (g, s) with both components (nc = 2), or the two
    // consecutive entries 2jj, 2jj + 1 of [g][s] (nc = 1)
    int g0, s0, g1, s1;
    real2 m;
    const size_t at = jj;  // pair index in the field arrays
    if (M.nc == 2) {
      const uint32_t n = static_cast<uint32_t>(jj);
      g0 = g1 = static_cast<int>(P.sdiv.div(n));
      s0 = s1 = static_cast<int>(n - static_cast<uint32_t>(g0) * S);
      m = reinterpret_cast<const real2 *>(M.minv)[g0];
    } else {
      const uint32_t n0 = static_cast<uint32_t>(2 * jj), n1 = n0 + 1;
      g0 = static_cast<int>(P.sdiv.div(n0));
      s0 = static_cast<int>(n0 - static_cast<uint32_t>(g0) * S);
      g1 = static_cast<int>(P.sdiv.div(n1));
      s1 = static_cast<int>(n1 - static_cast<uint32_t>(g1) * S);
      m = mk2(M.minv[g0], M.minv[g1]);
    }
    real2 *U = reinterpret_cast<real2 *>(M.u);
    real2 *Vv = reinterpret_cast<real2 *>(M.v);
    real2 *A = reinterpret_cast<real2 *>(M.a);
    const real2 r = A[at];
    real2 acc, vel = Vv[at];
    acc.x = r.x * m.x;
    acc.y = r.y * m.y;
    real2 cu = mk2(0, 0), cv = cu;
    if (EXTRA && M.cu) {
      cu = reinterpret_cast<const real2 *>(M.cu)[at];
      cv = reinterpret_cast<const real2 *>(M.cv)[at];
      vel.x = kahan_add(vel.x, cv.x, P.dt2 * acc.x);
      vel.y = kahan_add(vel.y, cv.y, P.dt2 * acc.y);
    } else {
      vel.x += P.dt2 * acc.x;  // corrector (newmark.tpp:44-47)
      vel.y += P.dt2 * acc.y;
    }
    real2 uu = U[at];
    if (record && M.taps.nsup > 0) {
      if (M.nc == 2) {
        apply_taps(M.taps, g0, uu.x, uu.y, vel.x, vel.y, acc.x, acc.y,
                   P.seis + (static_cast<size_t>(s0) * P.max_sig + isig) * P.slots);
      } else {
        apply_taps(M.taps, g0, uu.x, 0, vel.x, 0, acc.x, 0,
                   P.seis + (static_cast<size_t>(s0) * P.max_sig + isig) * P.slots);
        apply_taps(M.taps, g1, uu.y, 0, vel.y, 0, acc.y, 0,
                   P.seis + (static_cast<size_t>(s1) * P.max_sig + isig) * P.slots);
      }
    }
    if (P.last) {
      A[at] = acc;
      Vv[at] = vel;
    } else if (EXTRA && M.cu) {
      uu.x = kahan_add(uu.x, cu.x, P.dt * vel.x + P.dtsq2 * acc.x);
      uu.y = kahan_add(uu.y, cu.y, P.dt * vel.y + P.dtsq2 * acc.y);
      vel.x = kahan_add(vel.x, cv.x, P.dt2 * acc.x);
      vel.y = kahan_add(vel.y, cv.y, P.dt2 * acc.y);
      U[at] = uu;
      Vv[at] = vel;
      A[at] = mk2(0, 0);
      reinterpret_cast<real2 *>(M.cu)[at] = cu;
    } else {
      uu.x += P.dt * vel.x + P.dtsq2 * acc.x;  // next predictor (newmark.tpp:98-105)
      uu.y += P.dt * vel.y + P.dtsq2 * acc.y;
      vel.x += P.dt2 * acc.x;
      vel.y += P.dt2 * acc.y;
      U[at] = uu;
      Vv[at] = vel;
      A[at] = mk2(0, 0);
    }
    if constexpr (EXTRA) {
      if (M.cu) reinterpret_cast<real2 *>(M.cv)[at] = cv;
      if (M.ck_u && ck_uslot >= 0) reinterpret_cast<real2 *>(M.ck_u + ck_uslot * M.ck_stride)[at] = uu;
      if (M.ck_u && ck_vslot >= 0) reinterpret_cast<real2 *>(M.ck_v + ck_vslot * M.ck_stride)[at] = vel;
    }
  }
  if (P.ctrl) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned prev = atomicAdd(P.done, 1u);
      if (prev == gridDim.x - 1) {
        P.ctrl->istep = istep + P.dir;
        *P.done = 0u;
        __threadfence();
      }
    }
  }
}


// ---------------------------------------------------------------------------
// Frechet kernels (compute_material_derivatives.tpp:84-153 with
// medium/dim2/elastic/isotropic/frechet_derivative.hpp:14-138 and
// medium/dim2/acoustic/isotropic/frechet_derivative.hpp:12-41).  Thread per
// local point, EPB elements per CTA; gradients of the adjoint and backward
// displacements through shared memory; the per-step FP32 contributions of
// all shots are summed in FP64 registers and added once into the per-point
// FP64 accumulators kern[p][3] = (rho, mu, kappa) elastic, (rho, kappa,
// sum of rho_kl * kappa_kl) acoustic.  The adjoint acceleration is its force times the inverse mass.
// ---------------------------------------------------------------------------
template <int MED, int N, int EPB>
__global__ void __launch_bounds__(EPB * N * N)
k_frechet(Static st, MediumFields A, MediumFields B, int S, real dt, double *kern, int a_is_force) {
  constexpr int NC = (MED == MED_PSV) ? 2 : 1;
  constexpr int NN = N * N;
  __shared__ real s_a[EPB][NC][NN];
  __shared__ real s_b[EPB][NC][NN];
  const int t = threadIdx.x;
  const int el = t / NN, k = t % NN, iz = k / N, ix = k % N;
  const int li = blockIdx.x * EPB + el;
  const bool valid = li < A.nelem;
  const int e = A.elem_begin + (valid ? li : 0);
  const size_t p = static_cast<size_t>(e) * NN + k;
  const int g = valid ? st.iglob[p] : 0;
  const real xix = st.xix[p], xiz = st.xiz[p], gax = st.gax[p], gaz = st.gaz[p];
  const real m0 = st.mat0[p], m1 = st.mat1[p];
  const real m2 = st.mat2 ? st.mat2[p] : real(0);
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
  for (int s = 0; s < S; ++s) {
    const size_t base = (static_cast<size_t>(g) * S + s) * NC;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      s_a[el][c][k] = valid ? A.u[base + c] : real(0);
      s_b[el][c][k] = valid ? B.u[base + c] : real(0);
    }
    __syncthreads();
    real da[NC][2], db[NC][2];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      real axi = 0, aga = 0, bxi = 0, bga = 0;
#pragma unroll
      for (int l = 0; l < N; ++l) {
        axi += C_HP(ix * N + l) * s_a[el][c][iz * N + l];
        aga += C_HP(iz * N + l) * s_a[el][c][l * N + ix];
        bxi += C_HP(ix * N + l) * s_b[el][c][iz * N + l];
        bga += C_HP(iz * N + l) * s_b[el][c][l * N + ix];
      }
      da[c][0] = xix * axi + gax * aga;
      da[c][1] = xiz * axi + gaz * aga;
      db[c][0] = xix * bxi + gax * bga;
      db[c][1] = xiz * bxi + gaz * bga;
    }
    if (valid) {
      if constexpr (MED == MED_PSV) {
        const real l2m = m0 + kFourThirds * m1;
        const real kappa = l2m - m1;
        const real half = static_cast<real>(0.5);
        const real ad_dsxx = da[0][0], ad_dsxz = half * (da[1][0] + da[0][1]), ad_dszz = da[1][1];
        const real b_dsxx = db[0][0], b_dsxz = half * (db[1][0] + db[0][1]), b_dszz = db[1][1];
        real kappa_kl = (ad_dsxx + ad_dszz) * (b_dsxx + b_dszz);
        real mu_kl = (ad_dsxx * b_dsxx + ad_dszz * b_dszz + static_cast<real>(2) * ad_dsxz * b_dsxz -
                      kOneThird * kappa_kl);
        const real ax = a_is_force ? A.a[base] * A.minv[static_cast<size_t>(g) * 2] : A.a[base];
        const real az = a_is_force ? A.a[base + 1] * A.minv[static_cast<size_t>(g) * 2 + 1] : A.a[base + 1];
        real rho_kl = ax * B.u[base] + az * B.u[base + 1];
        kappa_kl = static_cast<real>(-1) * kappa * dt * kappa_kl;
        mu_kl = static_cast<real>(-2) * m1 * dt * mu_kl;
        rho_kl = static_cast<real>(-1) * m2 * dt * rho_kl;
        acc0 += static_cast<double>(rho_kl);
        acc1 += static_cast<double>(mu_kl);
        acc2 += static_cast<double>(kappa_kl);
      } else {
        const real rho_kl = (da[0][0] * db[0][0] + da[0][1] * db[0][1]) * m0 * dt;
        const real chi_dd = a_is_force ? A.a[base] * A.minv[g] : A.a[base];
        const real kappa_kl = chi_dd * B.u[base] * static_cast<real>(1) / m1 * dt;
        acc0 += static_cast<double>(rho_kl);
        acc1 += static_cast<double>(kappa_kl);
        acc2 += static_cast<double>(rho_kl * kappa_kl);  // rhop per step (point/kernels.hpp:189-192)
      }
    }
    __syncthreads();
  }
  if (valid) {
    kern[p * 3 + 0] += acc0;
    kern[p * 3 + 1] += acc1;
    kern[p * 3 + 2] += acc2;
  }
}

// Model derivative of the Stacey traction, which the reference's kernels
// leave out (frechet_derivative.hpp:14-138 has no boundary term).  With the
// kernels' convention dchi/dm = dt sum_steps s_adj . d(force)/dm and the P-SV
// Stacey force -w |n| [(rho vp - rho vs)(v.n^)n^ + rho vs v]
// (stacey.tpp:41-75), per Stacey point of a P-SV element
//   kb[p][0] += -dt w |n| (s_adj.n^)(v.n^)              dchi / d(rho vp)
//   kb[p][1] += -dt w |n| (s_adj.v - (s_adj.n^)(v.n^))  dchi / d(rho vs)
// summed over the shots, with v the backward wavefield's velocity at the end
// of the step: the field value plus vcorr * force * M^-1 when the update
// has not run yet (the implicit dt/2 mass term makes the damping act on the
// corrected velocity).
template <int N>
__global__ void k_stacey_frechet(Static st, MediumFields A, MediumFields B, int S, real dt, real vcorr,
                                 double *kb) {
  constexpr int NN = N * N;
  const size_t total = static_cast<size_t>(A.nelem) * NN;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int e = A.elem_begin + static_cast<int>(t / NN);
    if (!(st.eflag[e] & 1)) continue;
    const size_t p = static_cast<size_t>(e) * NN + t % NN;
    if (!(st.bnd[p] & 1)) continue;
    const int g = st.iglob[p];
    const real nx = st.bnd_nx[p], nz = st.bnd_nz[p], we = st.bnd_w[p];
    const real jac1d = msqrt(nx * nx + nz * nz);
    const real ux = nx / jac1d, uz = nz / jac1d;
    double k0 = 0.0, k1 = 0.0;
    for (int s = 0; s < S; ++s) {
      const size_t base = (static_cast<size_t>(g) * S + s) * 2;
      real vx = B.v[base], vz = B.v[base + 1];
      if (vcorr != real(0)) {
        vx += vcorr * B.a[base] * B.minv[static_cast<size_t>(g) * 2];
        vz += vcorr * B.a[base + 1] * B.minv[static_cast<size_t>(g) * 2 + 1];
      }
      const real ax = A.u[base], az = A.u[base + 1];
      const double an = static_cast<double>(ax) * ux + static_cast<double>(az) * uz;
      const double vn = static_cast<double>(vx) * ux + static_cast<double>(vz) * uz;
      const double av = static_cast<double>(ax) * vx + static_cast<double>(az) * vz;
      k0 += an * vn;
      k1 += av - an * vn;
    }
    const double f = -static_cast<double>(dt) * we * jac1d;
    kb[p * 2 + 0] += f * k0;
    kb[p * 2 + 1] += f * k1;
  }
}

// Mass matrix (compute_mass_matrix.tpp:80-113) accumulated in FP64.
template <int MED>
__global__ void k_mass(Static st, MediumFields f, int N, real dt) {
  constexpr int NC = (MED == MED_PSV) ? 2 : 1;
  const size_t nn = static_cast<size_t>(N) * N;
  const size_t total = static_cast<size_t>(f.nelem) * nn;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int e = f.elem_begin + static_cast<int>(t / nn);
    const int k = static_cast<int>(t % nn);
    const int iz = k / N, ix = k % N;
    const size_t p = static_cast<size_t>(e) * nn + k;
    real base;
    if (MED == MED_PSV) base = st.mat2[p];                    // rho
    else if (MED == MED_SH) base = st.mat1[p];                // rho
    else base = static_cast<real>(1) / st.mat1[p];            // 1 / kappa
    real mm[2];
    for (int c = 0; c < NC; ++c) mm[c] = base * (C_W(ix) * C_W(iz) * st.jac[p]);
    if (st.bnd[p] & 1) {
      const real hv = static_cast<real>(-1) * dt * static_cast<real>(0.5);
      const real vf[2] = {hv, hv};
      stacey<MED>(st.mat0[p], st.mat1[p], st.mat2 ? st.mat2[p] : real(0), st.bnd_nx[p], st.bnd_nz[p],
                  st.bnd_w[p], vf, mm);
    }
    const int g = st.iglob[p];
    for (int c = 0; c < NC; ++c) atomicAdd(f.mass + static_cast<size_t>(g) * NC + c, static_cast<double>(mm[c]));
  }
}

__global__ void k_invert(const double *mass, real *minv, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    minv[i] = static_cast<real>(1.0 / mass[i]);
}

// Error word bit set by k_nonfinite.
constexpr int kNonFinite = 2;

// NaN / Inf watchdog: sets kNonFinite in *err when any of p[0, n) is not
// finite.
template <typename T>
__global__ void k_nonfinite(const T *p, size_t n, int *err) {
  bool bad = false;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    bad = bad || !isfinite(p[i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(err, kNonFinite);
}

// The bounded mbarrier wait of the stiffness kernels, run out on purpose: a
// barrier in shared memory that expects one arrival which never comes, a
// limit of `limit` cycles, then the timeout is recorded in *err exactly as
// the stiffness kernels record it.  Nothing else is waited for or copied.
__global__ void k_wait_probe(long long limit, int *err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait_bounded(&bar, 0, limit)) atomicOr(err, kWaitTimeout);
}

__global__ void k_zero(real *p, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    p[i] = 0;
}

int grid_for(size_t n, int block) {
  size_t g = (n + block - 1) / block;
  const size_t cap = 148 * 32;  // 148 SMs x resident blocks
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return static_cast<int>(g);
}

size_t field_ld(const MediumFields &f) { return static_cast<size_t>(f.nglob + (f.nglob & 1)) * f.nc; }

}  // namespace

void init_kernel_attributes() {
#ifndef SFB_FP64
  cudaFuncSetAttribute(k_stiffness_pk<MED_PSV, 5, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(kFrechetDynSmem));
  cudaFuncSetAttribute(k_stiffness_pk<MED_PSV, 5, 3, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(kFrechetDynSmem));
#endif
}

bool frechet_fusable(int medium, int ngll, int nshots) {
#ifdef SFB_FP64
  (void)medium;
  (void)ngll;
  (void)nshots;
  return false;  // the fused Frechet launch is the packed FP32 kernel
#else
  return medium == MED_PSV && ngll == 5 && nshots > 1 && nshots % 2 == 0;
#endif
}

void launch_stiffness_frechet(int ngll, const Static &st, const MediumFields &f, int S, const StaceyStore &ss,
                              const int *istep_dev, const TailWork &tw, const FrechetFuse &fr,
                              const FusedUpdate &fu, cudaStream_t stream) {
  if (f.nelem == 0 || !frechet_fusable(MED_PSV, ngll, S)) return;
#ifndef SFB_FP64
  dim3 grid(f.nelem, (S / 2 + 31) / 32);
  if (st.affine[MED_PSV] && st.pack_aff)
    launch_step_kernel(k_stiffness_pk<MED_PSV, 5, 3, true, true>, grid, 5 * 32, kFrechetDynSmem, stream, st, f, S, ss,
                       istep_dev, tw, fu, fr);
  else
    launch_step_kernel(k_stiffness_pk<MED_PSV, 5, 3, true>, grid, 5 * 32, kFrechetDynSmem, stream, st, f, S, ss,
                       istep_dev, tw, fu, fr);
#else
  (void)st;
  (void)ss;
  (void)istep_dev;
  (void)tw;
  (void)fr;
  (void)fu;
  (void)stream;
#endif
}

void launch_stiffness(int medium, int ngll, const Static &st, const MediumFields &f, int nshots,
                      const StaceyStore &ss, const int *istep_dev, cudaStream_t stream, const TailWork *tw,
                      const FusedUpdate *fu, int variant) {
  if (f.nelem == 0) return;
  const TailWork none{};
  const TailWork &w = tw ? *tw : none;
  const FusedUpdate nofu{};
  // the in-launch update of private points exists for the P-SV kernels
  const FusedUpdate &u = (fu && medium == MED_PSV) ? *fu : nofu;
#ifdef SFB_FP64
  // FP64 build: the scalar shot-parallel kernel for every shot count
  (void)variant;
  if (ngll == 5) {
    if (medium == MED_PSV) launch_shots<MED_PSV, 5, 1>(st, f, nshots, ss, istep_dev, w, u, kShotsSingle, stream);
    else if (medium == MED_SH) launch_shots<MED_SH, 5, 1>(st, f, nshots, ss, istep_dev, w, nofu, kShotsSingle, stream);
    else launch_shots<MED_AC, 5, 1>(st, f, nshots, ss, istep_dev, w, nofu, kShotsSingle, stream);
  } else if (ngll == 8) {
    if (medium == MED_PSV) launch_shots<MED_PSV, 8, 1>(st, f, nshots, ss, istep_dev, w, u, kShotsSingle, stream);
    else if (medium == MED_SH) launch_shots<MED_SH, 8, 1>(st, f, nshots, ss, istep_dev, w, nofu, kShotsSingle, stream);
    else launch_shots<MED_AC, 8, 1>(st, f, nshots, ss, istep_dev, w, nofu, kShotsSingle, stream);
  }
  return;
#else
  if (nshots > 1) {
    if (ngll == 5) {
      if (medium == MED_PSV) launch_shots<MED_PSV, 5, 4>(st, f, nshots, ss, istep_dev, w, u, variant, stream);
      else if (medium == MED_SH) launch_shots<MED_SH, 5, 4>(st, f, nshots, ss, istep_dev, w, nofu, variant, stream);
      else launch_shots<MED_AC, 5, 4>(st, f, nshots, ss, istep_dev, w, nofu, variant, stream);
    } else if (ngll == 8) {
      if (medium == MED_PSV) launch_shots<MED_PSV, 8, 2>(st, f, nshots, ss, istep_dev, w, u, variant, stream);
      else if (medium == MED_SH) launch_shots<MED_SH, 8, 3>(st, f, nshots, ss, istep_dev, w, nofu, variant, stream);
      else launch_shots<MED_AC, 8, 3>(st, f, nshots, ss, istep_dev, w, nofu, variant, stream);
    }
    return;
  }
  // single shot: the row kernel with 32- or 16-element chunks (NGLL 8: 16),
  // or, where every element of the medium is affine (NGLL 5), the compact
  // block kernel
  if (variant == kRowAffine && ngll == 5 && st.affine[medium] && st.pack_aff) {
    if (medium == MED_PSV) launch_rpa<MED_PSV, 5, 4>(st, f, ss, istep_dev, w, u, stream);
    else if (medium == MED_SH) launch_rpa<MED_SH, 5, 4>(st, f, ss, istep_dev, w, nofu, stream);
    else launch_rpa<MED_AC, 5, 4>(st, f, ss, istep_dev, w, nofu, stream);
  } else if (ngll == 5) {
    if (variant == kRowHalfChunk) {
      if (medium == MED_PSV) launch_rp<MED_PSV, 5, 16, 6>(st, f, nshots, ss, istep_dev, w, u, stream);
      else if (medium == MED_SH) launch_rp<MED_SH, 5, 16, 6>(st, f, nshots, ss, istep_dev, w, nofu, stream);
      else launch_rp<MED_AC, 5, 16, 6>(st, f, nshots, ss, istep_dev, w, nofu, stream);
    } else {
      if (medium == MED_PSV) launch_rp<MED_PSV, 5, 32, 3>(st, f, nshots, ss, istep_dev, w, u, stream);
      else if (medium == MED_SH) launch_rp<MED_SH, 5, 32, 3>(st, f, nshots, ss, istep_dev, w, nofu, stream);
      else launch_rp<MED_AC, 5, 32, 3>(st, f, nshots, ss, istep_dev, w, nofu, stream);
    }
  } else if (ngll == 8) {
    if (medium == MED_PSV) launch_rp<MED_PSV, 8, 16, 2>(st, f, nshots, ss, istep_dev, w, u, stream);
    else if (medium == MED_SH) launch_rp<MED_SH, 8, 16, 2>(st, f, nshots, ss, istep_dev, w, nofu, stream);
    else launch_rp<MED_AC, 8, 16, 2>(st, f, nshots, ss, istep_dev, w, nofu, stream);
  }
#endif
}

void launch_sources(int ngll, const Static &st, const SourceSet &src, MediumFields *fields,
                    int nshots, int medium, const int *istep_dev, int, cudaStream_t stream) {
  if (src.n == 0) return;
  const MediumFields &f = fields[medium];
  if (f.nelem == 0) return;
  k_sources<<<src.n, ngll * ngll <= 32 ? 32 : 64, 0, stream>>>(st, src, f, medium, ngll, istep_dev, nshots);
}

void launch_coupling_acoustic(const CouplingSet &c, const MediumFields &ac, const MediumFields &el,
                              int nshots, cudaStream_t stream) {
  if (c.n == 0) return;
  dim3 grid((c.n + 127) / 128, nshots);
  k_couple_acoustic<<<grid, 128, 0, stream>>>(c, ac, el, nshots);
}

void launch_coupling_elastic(const CouplingSet &c, const MediumFields &el, const MediumFields &ac,
                             int nshots, int ac_divided, cudaStream_t stream) {
  if (c.n == 0) return;
  dim3 grid((c.n + 127) / 128, nshots);
  k_couple_elastic<<<grid, 128, 0, stream>>>(c, el, ac, nshots, ac_divided);
}

void launch_tail_det(int medium, int ngll, const Static &st, const MediumFields &f, int nshots,
                     const int *istep_dev, const TailWork &tw, const DetTail &dt, cudaStream_t stream) {
  if (dt.ntarget == 0) return;
  const int grid = grid_for(static_cast<size_t>(dt.ntarget) * nshots, 128);
  if (ngll == 5) {
    if (medium == MED_PSV) k_tail_det<MED_PSV, 5><<<grid, 128, 0, stream>>>(st, f, nshots, istep_dev, tw, dt);
    else if (medium == MED_SH) k_tail_det<MED_SH, 5><<<grid, 128, 0, stream>>>(st, f, nshots, istep_dev, tw, dt);
    else k_tail_det<MED_AC, 5><<<grid, 128, 0, stream>>>(st, f, nshots, istep_dev, tw, dt);
  } else if (ngll == 8) {
    if (medium == MED_PSV) k_tail_det<MED_PSV, 8><<<grid, 128, 0, stream>>>(st, f, nshots, istep_dev, tw, dt);
    else if (medium == MED_SH) k_tail_det<MED_SH, 8><<<grid, 128, 0, stream>>>(st, f, nshots, istep_dev, tw, dt);
    else k_tail_det<MED_AC, 8><<<grid, 128, 0, stream>>>(st, f, nshots, istep_dev, tw, dt);
  }
}

void launch_receivers(int ngll, const Static &st, const ReceiverSet &rec, const MediumFields *fields,
                      int nshots, real dt2, int mode, const int *istep_dev, cudaStream_t stream) {
  if (rec.n == 0 || rec.ntypes == 0) return;
  dim3 grid(rec.n, nshots);
  k_receivers<<<grid, 64, 0, stream>>>(st, rec, fields[MED_PSV], fields[MED_SH], fields[MED_AC], ngll,
                                       dt2, mode, istep_dev, nshots);
}

void launch_predictor(const MediumFields &f, int nshots, real dt, real dt2, real dtsq2,
                      cudaStream_t stream, real *cu, real *cv) {
  const size_t n = field_ld(f) * nshots;
  if (n == 0) return;
  k_predictor<<<grid_for(n, 256), 256, 0, stream>>>(f.u, f.v, f.a, n, dt, dt2, dtsq2, cu, cv);
}
void launch_corrector(const MediumFields &f, int nshots, real dt2, cudaStream_t stream) {
  const size_t n = field_ld(f) * nshots;
  if (n == 0) return;
  k_corrector<<<grid_for(n, 256), 256, 0, stream>>>(f.v, f.a, n, dt2);
}
void launch_divide(const MediumFields &f, int nshots, cudaStream_t stream) {
  const size_t n = field_ld(f) * nshots;
  if (n == 0) return;
  k_divide<<<grid_for(n, 256), 256, 0, stream>>>(f.a, f.minv, n, nshots, f.nc);
}
void launch_advance_step(Control *ctrl, cudaStream_t stream) { k_advance<<<1, 1, 0, stream>>>(ctrl); }

void launch_restore(const RestoreParams &p, cudaStream_t stream) {
  if (p.nm == 0 || p.interval <= 0 || p.count <= 0) return;
  static int nsm = 0;
  if (nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  k_restore<<<nsm * 4, 256, 0, stream>>>(p);
}

void launch_update_all(const UpdateParams &p, cudaStream_t stream) {
  const size_t total = p.begin[p.nm];
  if (total == 0) {
    if (p.ctrl) k_advance<<<1, 1, 0, stream>>>(p.ctrl);
    return;
  }
  // one wave of resident CTAs (grid-stride): a grid beyond what fits leaves
  // a partial second wave
  static int nsm = 0, per_sm[2] = {0, 0};
  if (nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0], k_update_all<false>, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1], k_update_all<true>, 256, 0);
    for (int &b : per_sm) b = std::max(b, 1);
  }
  bool extra = p.ck_interval > 0;
  for (int m = 0; m < p.nm; ++m) extra = extra || p.m[m].cu != nullptr || p.m[m].ck_u != nullptr;
  const size_t want = (total + 255) / 256;
  const int grid = static_cast<int>(std::min<size_t>(want, static_cast<size_t>(nsm) * per_sm[extra ? 1 : 0]));
  if (extra)
    launch_step_kernel(k_update_all<true>, std::max(grid, 1), 256, 0, stream, p);
  else
    launch_step_kernel(k_update_all<false>, std::max(grid, 1), 256, 0, stream, p);
}


void launch_mass(int medium, int ngll, const Static &st, const MediumFields &f, real dt,
                 cudaStream_t stream) {
  if (f.nelem == 0) return;
  const size_t n = static_cast<size_t>(f.nelem) * ngll * ngll;
  const int grid = grid_for(n, 256);
  if (medium == MED_PSV) k_mass<MED_PSV><<<grid, 256, 0, stream>>>(st, f, ngll, dt);
  else if (medium == MED_SH) k_mass<MED_SH><<<grid, 256, 0, stream>>>(st, f, ngll, dt);
  else k_mass<MED_AC><<<grid, 256, 0, stream>>>(st, f, ngll, dt);
}
void launch_invert_mass(const MediumFields &f, cudaStream_t stream) {
  const size_t n = static_cast<size_t>(f.nglob) * f.nc;
  if (n == 0) return;
  k_invert<<<grid_for(n, 256), 256, 0, stream>>>(f.mass, f.minv, n);
}
void launch_frechet(int medium, int ngll, const Static &st, const MediumFields &adj, const MediumFields &bwd,
                    int nshots, real dt, double *kern, int a_is_force, cudaStream_t stream) {
  if (adj.nelem == 0) return;
  if (ngll == 5) {
    constexpr int EPB = 8;
    const int grid = (adj.nelem + EPB - 1) / EPB;
    if (medium == MED_PSV) k_frechet<MED_PSV, 5, EPB><<<grid, EPB * 25, 0, stream>>>(st, adj, bwd, nshots, dt, kern, a_is_force);
    else if (medium == MED_AC) k_frechet<MED_AC, 5, EPB><<<grid, EPB * 25, 0, stream>>>(st, adj, bwd, nshots, dt, kern, a_is_force);
  } else if (ngll == 8) {
    constexpr int EPB = 4;
    const int grid = (adj.nelem + EPB - 1) / EPB;
    if (medium == MED_PSV) k_frechet<MED_PSV, 8, EPB><<<grid, EPB * 64, 0, stream>>>(st, adj, bwd, nshots, dt, kern, a_is_force);
    else if (medium == MED_AC) k_frechet<MED_AC, 8, EPB><<<grid, EPB * 64, 0, stream>>>(st, adj, bwd, nshots, dt, kern, a_is_force);
  }
}

void launch_stacey_frechet(int ngll, const Static &st, const MediumFields &adj, const MediumFields &bwd, int nshots,
                           real dt, real vcorr, double *kb, cudaStream_t stream) {
  if (adj.nelem == 0) return;
  const size_t n = static_cast<size_t>(adj.nelem) * ngll * ngll;
  if (ngll == 5) k_stacey_frechet<5><<<grid_for(n, 256), 256, 0, stream>>>(st, adj, bwd, nshots, dt, vcorr, kb);
  else if (ngll == 8) k_stacey_frechet<8><<<grid_for(n, 256), 256, 0, stream>>>(st, adj, bwd, nshots, dt, vcorr, kb);
}

void launch_nonfinite_check(const real *p, size_t n, int *err, cudaStream_t stream) {
  if (n == 0) return;
  k_nonfinite<real><<<grid_for(n, 256), 256, 0, stream>>>(p, n, err);
}
#ifndef SFB_FP64
void launch_nonfinite_check(const double *p, size_t n, int *err, cudaStream_t stream) {
  if (n == 0) return;
  k_nonfinite<double><<<grid_for(n, 256), 256, 0, stream>>>(p, n, err);
}
#endif

void launch_wait_probe(long long limit_cycles, int *err, cudaStream_t stream) {
  k_wait_probe<<<1, 32, 0, stream>>>(limit_cycles, err);
}

void launch_zero(real *p, size_t n, cudaStream_t stream) {
  if (n == 0) return;
  k_zero<<<grid_for(n, 256), 256, 0, stream>>>(p, n);
}

}  // namespace dev
}  // namespace sfb
