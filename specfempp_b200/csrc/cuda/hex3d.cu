// 3D elastic path on hexahedral spectral elements (include/specfem_b200_3d.h).
//
// The reference has no 3D solver (src/specfem3d.cpp:49-73); this restates its
// 2D weak form with a third dimension, term by term:
//   gradient    include/algorithms/gradient.hpp:78-98: du_c/dxi(k,j,i) =
//               sum_l hprime(i,l) u_c(k,j,l), likewise along eta (j) and
//               zeta (k); physical derivatives through the inverse Jacobian
//               (axis-aligned hexahedra: d/dx = xix d/dxi, d/dy = etay d/deta,
//               d/dz = gammaz d/dzeta)
//   stress      medium/dim2/elastic/isotropic/stress.hpp:14-50 with
//               lambda + 2 mu = kappa + 4/3 mu, lambda = lambda + 2 mu - 2 mu
//   F = J T dxi/dx  core/specfem/point/stress.hpp:117-139
//   divergence  include/algorithms/divergence.hpp:83-99, negated:
//               r(k,j,i) = -( w_j w_k sum_l F_xi(k,j,l) hpw(i,l)
//                           + w_i w_k sum_l F_eta(k,l,i) hpw(j,l)
//                           + w_i w_j sum_l F_zeta(l,j,i) hpw(k,l) ),
//               hpw(i,l) = hprime(l,i) w_l
//   Stacey      boundary_conditions/stacey/stacey.tpp:41-75 summed over the
//               absorbing element faces through a global point: with
//               axis-aligned normals the traction is -A v, A diagonal
//   mass        compute_mass_matrix.tpp:80-113 plus the Stacey term at
//               velocity -dt/2 (stacey.tpp:644-677): M_c + dt/2 A_c
//   Newmark     timescheme/newmark.tpp (predictor / corrector, -dt backward)
//   sources     moment tensor (src/source/moment_tensor_source.cpp:125-135):
//               array_c = sum_d M_cd d(h_i h_j h_k)/dx_d, Ricker time function
//   Frechet     frechet_derivative.hpp:14-138 with the 3D strain:
//               K_kappa = -kappa dt div(s_adj) div(s), K_mu = -2 mu dt
//               (eps_adj : eps - 1/3 div div), K_rho = -rho dt a_adj . s
//   combined    solver/time_marching.tpp:126-247 (adjoint in reversed time,
//               backward with -dt replaying the forward run's Stacey
//               tractions, kernels every step; the backward wavefield is
//               the forward run's last state at the first reversed step)
//
// Device layout: every wavefield is [g][c][S] (value of global point g,
// component c, shot s at (g * 3 + c) * S + s): the shots of one point and
// component are contiguous, so 16 shots make one 64-byte access.  Per local
// point p = e * 125 + (k * 5 + j) * 5 + i: global index, kappa, mu, rho; per
// element the geometry (xix, etay, gammaz, J).  The stiffness kernel is one
// CTA per element and group of 16 shots: thread (lane = shot, row = (k, j))
// owns the five points of its row along x; the eta and zeta contractions
// read shared memory.
#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/specfem_b200_3d.h"
#include "../host/assembly.hpp"
#include "../host/quadrature.hpp"

namespace {

constexpr int N = 5, NN = 25, NNN = 125;
constexpr int SG = 16;                       // shots per CTA (lanes of a half-warp)
constexpr int TILE = NNN * 3 * SG;           // floats of one element tile in shared memory
constexpr float kFourThirds = static_cast<float>(4.0 / 3.0);
constexpr float kOneThird = static_cast<float>(1.0 / 3.0);

__constant__ float c3_hp[NN];   // hprime[i*5 + l] = l_l'(xi_i)
__constant__ float c3_hpw[NN];  // hprime[l*5 + i] * w[l] at [i*5 + l]
__constant__ float c3_w[N];

struct Dev3 {
  int nspec, S;
  const int *iglob;       // [nspec * 125]
  const float4 *geo;      // [nspec]: xix, etay, gammaz, jacobian
  const float *kappa, *mu, *rho;
  const unsigned char *priv;  // [nspec]: 1 = the element's 27 interior points are private
  // Deterministic mode: a launch covers one colour of elements (elist[elist_off
  // + blockIdx.x]; no two elements of a colour share a point) and one group
  // of 16 shots (sgroup + blockIdx.y), and scatters with plain adds.
  const int *elist;
  int elist_off, sgroup, det;
};

__device__ __forceinline__ int elem_of(const Dev3 &d) { return d.elist ? d.elist[d.elist_off + blockIdx.x] : blockIdx.x; }
__device__ __forceinline__ int group_of(const Dev3 &d) { return d.sgroup + blockIdx.y; }

// Forward steps: the stiffness launch finishes the private points of marked
// elements (a = f M^-1, corrector, and unless `last` the next predictor).
struct PrivArgs {
  float *v;
  const float *minv;
  float dt, dt2, dtsq2;
  int last;
  int enabled;
};

__device__ __forceinline__ size_t fidx(int g, int c, int s, int S) {
  return (static_cast<size_t>(g) * 3 + c) * S + s;
}

// Stiffness of every element, scatter-added into the force accumulator a.
__global__ void __launch_bounds__(SG * NN, 2) k3_stiffness(Dev3 d, const float *__restrict__ u, float *a) {
  extern __shared__ float smem[];
  float *s_u = smem, *s_fy = smem + TILE, *s_fz = smem + 2 * TILE;
  const int lane = threadIdx.x, row = threadIdx.y;  // row = k * 5 + j
  const int k = row / N, j = row % N;
  const int e = elem_of(d);
  const int S = d.S;
  const int s = group_of(d) * SG + lane;
  const bool act = s < S;
  const float4 gg = d.geo[e];
  const float xix = gg.x, etay = gg.y, gaz = gg.z, jac = gg.w;
  const size_t p0 = static_cast<size_t>(e) * NNN + row * N;
  int g[N];
  float ur[N][3];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    g[i] = d.iglob[p0 + i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ur[i][c] = act ? u[fidx(g[i], c, s, S)] : 0.f;
      s_u[((row * N + i) * 3 + c) * SG + lane] = ur[i][c];
    }
  }
  __syncthreads();
  float fx[N][3];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    float dxi[3] = {0.f, 0.f, 0.f}, deta[3] = {0.f, 0.f, 0.f}, dzeta[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int l = 0; l < N; ++l) {
      const float hx = c3_hp[i * N + l], hy = c3_hp[j * N + l], hz = c3_hp[k * N + l];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        dxi[c] += hx * ur[l][c];
        deta[c] += hy * s_u[(((k * N + l) * N + i) * 3 + c) * SG + lane];
        dzeta[c] += hz * s_u[(((l * N + j) * N + i) * 3 + c) * SG + lane];
      }
    }
    const float kap = d.kappa[p0 + i], mu = d.mu[p0 + i];
    const float l2m = kap + kFourThirds * mu;
    const float lam = l2m - 2.0f * mu;
    float du[3][3];  // du[c][x] = d u_c / d x
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      du[c][0] = xix * dxi[c];
      du[c][1] = etay * deta[c];
      du[c][2] = gaz * dzeta[c];
    }
    const float sxx = l2m * du[0][0] + lam * (du[1][1] + du[2][2]);
    const float syy = l2m * du[1][1] + lam * (du[0][0] + du[2][2]);
    const float szz = l2m * du[2][2] + lam * (du[0][0] + du[1][1]);
    const float sxy = mu * (du[0][1] + du[1][0]);
    const float sxz = mu * (du[0][2] + du[2][0]);
    const float syz = mu * (du[1][2] + du[2][1]);
    const float T[3][3] = {{sxx, sxy, sxz}, {sxy, syy, syz}, {sxz, syz, szz}};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      fx[i][c] = jac * (T[c][0] * xix);
      s_fy[((row * N + i) * 3 + c) * SG + lane] = jac * (T[c][1] * etay);
      s_fz[((row * N + i) * 3 + c) * SG + lane] = jac * (T[c][2] * gaz);
    }
  }
  __syncthreads();
  if (!act) return;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    float t1[3] = {0.f, 0.f, 0.f}, t2[3] = {0.f, 0.f, 0.f}, t3[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int l = 0; l < N; ++l) {
      const float hx = c3_hpw[i * N + l], hy = c3_hpw[j * N + l], hz = c3_hpw[k * N + l];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        t1[c] += fx[l][c] * hx;
        t2[c] += s_fy[(((k * N + l) * N + i) * 3 + c) * SG + lane] * hy;
        t3[c] += s_fz[(((l * N + j) * N + i) * 3 + c) * SG + lane] * hz;
      }
    }
    const float wjk = c3_w[j] * c3_w[k], wik = c3_w[i] * c3_w[k], wij = c3_w[i] * c3_w[j];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float r = (wjk * t1[c] + wik * t2[c] + wij * t3[c]) * -1.0f;
      if (d.det) a[fidx(g[i], c, s, S)] += r;
      else atomicAdd(a + fidx(g[i], c, s, S), r);
    }
  }
}

// ---------------------------------------------------------------------------
// Packed variants for an even number of shots: each thread holds two
// adjacent shots of its row and applies every per-point operation to the
// pair with one f32x2 instruction (each lane rounds as one IEEE fma / mul /
// add), loads and stores the pair as one float2 and adds it to the force
// with one vector atomic.  CTA: 8 lanes x 25 rows (16 shots).
// ---------------------------------------------------------------------------
constexpr int PL = SG / 2;  // lanes of a row in the packed kernels

__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 dup(float v) { return make_float2(v, v); }
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.commit_group;\ncp.async.wait_all;\n" ::: "memory"); }

// Shared words of the private-point prefetch: velocity [27][3][16], inverse mass [27][3].
constexpr int PRIV_WORDS = 27 * 3 * SG + 27 * 3;

__device__ __forceinline__ float2 lds2(const float *t, int q, int c, int lane) {
  return *reinterpret_cast<const float2 *>(t + (q * 3 + c) * SG + 2 * lane);
}
__device__ __forceinline__ void sts2(float *t, int q, int c, int lane, float2 v) {
  *reinterpret_cast<float2 *>(t + (q * 3 + c) * SG + 2 * lane) = v;
}

// Frechet accumulation fused into the backward stiffness launch of the
// combined run: the adjoint displacement, the adjoint force of the same
// step (complete: its stiffness, Stacey and sources launches came first)
// and the inverse mass give the adjoint acceleration a = f M^-1 the
// corrector would produce; the backward displacement is the launch's own.
struct FrArgs {
  const float *au, *af, *minv;
  double *kern;
  float dt;
  int atomic;
};

// Kernels of one point for the lane's two shots, summed in FP64 over the
// pair and the 8 lanes of the row; value v = i * 3 + q lands in lane v % 8,
// slot v / 8 of `mine`.
__device__ __forceinline__ void frechet_point(const float2 (&da)[3][3], const float2 (&db)[3][3], float2 rho_dot,
                                              float kap, float muv, float rhov, float dt, bool act, int i, int lane,
                                              unsigned seg, double (&mine)[2]) {
  const float2 zero = make_float2(0.f, 0.f), half = dup(0.5f);
  const float2 diva = add2(add2(da[0][0], da[1][1]), da[2][2]);
  const float2 divb = add2(add2(db[0][0], db[1][1]), db[2][2]);
  float2 ee = zero;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int x = 0; x < 3; ++x)
      ee = fma2(mul2(half, add2(da[c][x], da[x][c])), mul2(half, add2(db[c][x], db[x][c])), ee);
  float2 kappa_kl = mul2(diva, divb);
  float2 mu_kl = fma2(dup(-kOneThird), kappa_kl, ee);
  kappa_kl = mul2(mul2(dup(-1.0f * kap), dup(dt)), kappa_kl);
  mu_kl = mul2(mul2(dup(-2.0f * muv), dup(dt)), mu_kl);
  const float2 rho_kl = mul2(mul2(dup(-1.0f * rhov), dup(dt)), rho_dot);
  double r[3] = {act ? static_cast<double>(rho_kl.x) + static_cast<double>(rho_kl.y) : 0.0,
                 act ? static_cast<double>(mu_kl.x) + static_cast<double>(mu_kl.y) : 0.0,
                 act ? static_cast<double>(kappa_kl.x) + static_cast<double>(kappa_kl.y) : 0.0};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
#pragma unroll
    for (int off = PL / 2; off > 0; off >>= 1) r[q] += __shfl_xor_sync(seg, r[q], off, PL);
    const int v = i * 3 + q;
    if (lane == (v & (PL - 1))) mine[v / PL] = r[q];
  }
}

// The row's 15 kernel values: lanes 0-7 hold values 0-7, lanes 0-6 values 8-14.
__device__ __forceinline__ void frechet_store(double *kern, size_t p0, int lane, const double (&mine)[2], int atomic) {
#pragma unroll
  for (int slot = 0; slot < 2; ++slot) {
    const int v = slot * PL + lane;
    if (v < 3 * N) {
      double *dst = kern + p0 * 3 + v;
      if (atomic) atomicAdd(dst, mine[slot]);
      else *dst += mine[slot];
    }
  }
}

template <int MINB, bool FR>
__global__ void __launch_bounds__(PL * NN, MINB) k3_stiffness_pk(Dev3 d, const float *u, float *a, FrArgs fr,
                                                                 PrivArgs pv) {
  extern __shared__ float smem[];
  float *s_u = smem, *s_fy = smem + TILE, *s_fz = smem + 2 * TILE, *s_a = smem + 3 * TILE;
  float *s_pv = smem + 3 * TILE, *s_pm = s_pv + 27 * 3 * SG;  // private prefetch (not with FR)
  const int lane = threadIdx.x, row = threadIdx.y;
  const int k = row / N, j = row % N;
  const int e = elem_of(d);
  const int S = d.S;
  const int s = group_of(d) * SG + 2 * lane;  // the lane's shots s, s + 1
  const bool act = s < S;
  const float4 gg = d.geo[e];
  const float2 xix = dup(gg.x), etay = dup(gg.y), gaz = dup(gg.z), jac = dup(gg.w);
  const size_t p0 = static_cast<size_t>(e) * NNN + row * N;
  const float2 zero = make_float2(0.f, 0.f);
  const bool private_row = !FR && pv.enabled && d.priv[e] && j >= 1 && j <= N - 2 && k >= 1 && k <= N - 2;
  int g[N];
  float2 ur[N][3];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    g[i] = d.iglob[p0 + i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ur[i][c] = act ? *reinterpret_cast<const float2 *>(u + fidx(g[i], c, s, S)) : zero;
      sts2(s_u, row * N + i, c, lane, ur[i][c]);
      if (FR) sts2(s_a, row * N + i, c, lane, act ? *reinterpret_cast<const float2 *>(fr.au + fidx(g[i], c, s, S)) : zero);
    }
  }
  if (private_row) {
    // the private points' velocity and inverse mass, needed after the
    // divergence: copied to shared memory while the element is computed
#pragma unroll
    for (int i = 1; i <= N - 2; ++i) {
      const int pi = ((k - 1) * 3 + (j - 1)) * 3 + (i - 1);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (act) cp_async8(s_pv + (pi * 3 + c) * SG + 2 * lane, pv.v + fidx(g[i], c, s, S));
        if (lane == 0) cp_async4(s_pm + pi * 3 + c, pv.minv + static_cast<size_t>(g[i]) * 3 + c);
      }
    }
  }
  __syncthreads();
  const unsigned seg = 0xffu << (8 * (threadIdx.y & 3));  // a warp holds four rows of 8 lanes
  double mine[2] = {0.0, 0.0};
  float2 fx[N][3];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    float2 dxi[3] = {zero, zero, zero}, deta[3] = {zero, zero, zero}, dzeta[3] = {zero, zero, zero};
#pragma unroll
    for (int l = 0; l < N; ++l) {
      const float2 hx = dup(c3_hp[i * N + l]), hy = dup(c3_hp[j * N + l]), hz = dup(c3_hp[k * N + l]);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        dxi[c] = fma2(hx, ur[l][c], dxi[c]);
        deta[c] = fma2(hy, lds2(s_u, (k * N + l) * N + i, c, lane), deta[c]);
        dzeta[c] = fma2(hz, lds2(s_u, (l * N + j) * N + i, c, lane), dzeta[c]);
      }
    }
    const float kap = d.kappa[p0 + i], muv = d.mu[p0 + i];
    const float l2ms = kap + kFourThirds * muv;
    const float2 l2m = dup(l2ms), lam = dup(l2ms - 2.0f * muv), mu = dup(muv);
    float2 du[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      du[c][0] = mul2(xix, dxi[c]);
      du[c][1] = mul2(etay, deta[c]);
      du[c][2] = mul2(gaz, dzeta[c]);
    }
    if (FR) {
      // the adjoint gradient at this point (all three directions from the
      // shared tile) and the adjoint acceleration
      float2 da[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float2 axi = zero, aeta = zero, azeta = zero;
#pragma unroll
        for (int l = 0; l < N; ++l) {
          axi = fma2(dup(c3_hp[i * N + l]), lds2(s_a, (k * N + j) * N + l, c, lane), axi);
          aeta = fma2(dup(c3_hp[j * N + l]), lds2(s_a, (k * N + l) * N + i, c, lane), aeta);
          azeta = fma2(dup(c3_hp[k * N + l]), lds2(s_a, (l * N + j) * N + i, c, lane), azeta);
        }
        da[c][0] = mul2(xix, axi);
        da[c][1] = mul2(etay, aeta);
        da[c][2] = mul2(gaz, azeta);
      }
      float2 rho_dot = zero;
      if (act) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float m = fr.minv[static_cast<size_t>(g[i]) * 3 + c];
          const float2 acc = mul2(*reinterpret_cast<const float2 *>(fr.af + fidx(g[i], c, s, S)), dup(m));
          rho_dot = fma2(acc, ur[i][c], rho_dot);
        }
      }
      frechet_point(da, du, rho_dot, kap, muv, d.rho[p0 + i], fr.dt, act, i, lane, seg, mine);
    }
    const float2 sxx = fma2(l2m, du[0][0], mul2(lam, add2(du[1][1], du[2][2])));
    const float2 syy = fma2(l2m, du[1][1], mul2(lam, add2(du[0][0], du[2][2])));
    const float2 szz = fma2(l2m, du[2][2], mul2(lam, add2(du[0][0], du[1][1])));
    const float2 sxy = mul2(mu, add2(du[0][1], du[1][0]));
    const float2 sxz = mul2(mu, add2(du[0][2], du[2][0]));
    const float2 syz = mul2(mu, add2(du[1][2], du[2][1]));
    const float2 T[3][3] = {{sxx, sxy, sxz}, {sxy, syy, syz}, {sxz, syz, szz}};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      fx[i][c] = mul2(jac, mul2(T[c][0], xix));
      sts2(s_fy, row * N + i, c, lane, mul2(jac, mul2(T[c][1], etay)));
      sts2(s_fz, row * N + i, c, lane, mul2(jac, mul2(T[c][2], gaz)));
    }
  }
  if (FR) frechet_store(fr.kern, p0, lane, mine, fr.atomic);
  if (private_row) cp_async_wait_all();
  __syncthreads();
  if (!act) return;
  const float2 neg = dup(-1.0f);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    float2 t1[3] = {zero, zero, zero}, t2[3] = {zero, zero, zero}, t3[3] = {zero, zero, zero};
#pragma unroll
    for (int l = 0; l < N; ++l) {
      const float2 hx = dup(c3_hpw[i * N + l]), hy = dup(c3_hpw[j * N + l]), hz = dup(c3_hpw[k * N + l]);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        t1[c] = fma2(fx[l][c], hx, t1[c]);
        t2[c] = fma2(lds2(s_fy, (k * N + l) * N + i, c, lane), hy, t2[c]);
        t3[c] = fma2(lds2(s_fz, (l * N + j) * N + i, c, lane), hz, t3[c]);
      }
    }
    const float2 wjk = dup(c3_w[j] * c3_w[k]), wik = dup(c3_w[i] * c3_w[k]), wij = dup(c3_w[i] * c3_w[j]);
    float2 r[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) r[c] = mul2(fma2(wjk, t1[c], fma2(wik, t2[c], mul2(wij, t3[c]))), neg);
    if (private_row) {
      if (i >= 1 && i <= N - 2) {
        // a = f M^-1, corrector and next predictor in registers
        // (newmark.tpp:44-47, 98-105); the force never reaches memory
        const int pi = ((k - 1) * 3 + (j - 1)) * 3 + (i - 1);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const size_t at = fidx(g[i], c, s, S);
          const float2 acc = mul2(r[c], dup(s_pm[pi * 3 + c]));
          float2 vel = fma2(dup(pv.dt2), acc, lds2(s_pv, pi, c, lane));
          if (pv.last) {
            *reinterpret_cast<float2 *>(a + at) = acc;
          } else {
            *reinterpret_cast<float2 *>(const_cast<float *>(u) + at) =
                add2(ur[i][c], fma2(dup(pv.dt), vel, mul2(dup(pv.dtsq2), acc)));
            vel = fma2(dup(pv.dt2), acc, vel);
          }
          *reinterpret_cast<float2 *>(pv.v + at) = vel;
        }
        continue;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 *dst = reinterpret_cast<float2 *>(a + fidx(g[i], c, s, S));
      if (d.det) *dst = add2(*dst, r[c]);
      else atomicAdd(dst, r[c]);
    }
  }
}

// Frechet kernels, packed: the lane's two shots are summed in FP64, then
// the 8 lanes of the row by shuffles.
template <int MINB>
__global__ void __launch_bounds__(PL * NN, MINB) k3_frechet_pk(Dev3 d, const float *__restrict__ au,
                                                           const float *__restrict__ aa,
                                                           const float *__restrict__ bu, float dt, double *kern,
                                                           int atomic) {
  extern __shared__ float smem[];
  float *s_a = smem, *s_b = smem + TILE;
  const int lane = threadIdx.x, row = threadIdx.y;
  const int k = row / N, j = row % N;
  const int e = elem_of(d);
  const int S = d.S;
  const int s = group_of(d) * SG + 2 * lane;
  const bool act = s < S;
  const float4 gg = d.geo[e];
  const float2 xix = dup(gg.x), etay = dup(gg.y), gaz = dup(gg.z);
  const size_t p0 = static_cast<size_t>(e) * NNN + row * N;
  const float2 zero = make_float2(0.f, 0.f);
  int g[N];
  float2 ra[N][3], rb[N][3];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    g[i] = d.iglob[p0 + i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ra[i][c] = act ? *reinterpret_cast<const float2 *>(au + fidx(g[i], c, s, S)) : zero;
      rb[i][c] = act ? *reinterpret_cast<const float2 *>(bu + fidx(g[i], c, s, S)) : zero;
      sts2(s_a, row * N + i, c, lane, ra[i][c]);
      sts2(s_b, row * N + i, c, lane, rb[i][c]);
    }
  }
  __syncthreads();
  // a warp holds four rows of 8 lanes
  const unsigned seg = 0xffu << (8 * (threadIdx.y & 3));
  double mine[2] = {0.0, 0.0};
  const float2 half = dup(0.5f);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    float2 da[3][3], db[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 axi = zero, aeta = zero, azeta = zero, bxi = zero, beta = zero, bzeta = zero;
#pragma unroll
      for (int l = 0; l < N; ++l) {
        const float2 hx = dup(c3_hp[i * N + l]), hy = dup(c3_hp[j * N + l]), hz = dup(c3_hp[k * N + l]);
        axi = fma2(hx, ra[l][c], axi);
        bxi = fma2(hx, rb[l][c], bxi);
        aeta = fma2(hy, lds2(s_a, (k * N + l) * N + i, c, lane), aeta);
        beta = fma2(hy, lds2(s_b, (k * N + l) * N + i, c, lane), beta);
        azeta = fma2(hz, lds2(s_a, (l * N + j) * N + i, c, lane), azeta);
        bzeta = fma2(hz, lds2(s_b, (l * N + j) * N + i, c, lane), bzeta);
      }
      da[c][0] = mul2(xix, axi);
      da[c][1] = mul2(etay, aeta);
      da[c][2] = mul2(gaz, azeta);
      db[c][0] = mul2(xix, bxi);
      db[c][1] = mul2(etay, beta);
      db[c][2] = mul2(gaz, bzeta);
    }
    const size_t p = p0 + i;
    const float2 diva = add2(add2(da[0][0], da[1][1]), da[2][2]);
    const float2 divb = add2(add2(db[0][0], db[1][1]), db[2][2]);
    float2 ee = zero;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int x = 0; x < 3; ++x)
        ee = fma2(mul2(half, add2(da[c][x], da[x][c])), mul2(half, add2(db[c][x], db[x][c])), ee);
    float2 kappa_kl = mul2(diva, divb);
    float2 mu_kl = fma2(dup(-kOneThird), kappa_kl, ee);
    float2 rho_kl = zero;
    if (act) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
        rho_kl = fma2(*reinterpret_cast<const float2 *>(aa + fidx(g[i], c, s, S)), rb[i][c], rho_kl);
    }
    kappa_kl = mul2(mul2(dup(-1.0f * d.kappa[p]), dup(dt)), kappa_kl);
    mu_kl = mul2(mul2(dup(-2.0f * d.mu[p]), dup(dt)), mu_kl);
    rho_kl = mul2(mul2(dup(-1.0f * d.rho[p]), dup(dt)), rho_kl);
    double r[3] = {act ? static_cast<double>(rho_kl.x) + static_cast<double>(rho_kl.y) : 0.0,
                   act ? static_cast<double>(mu_kl.x) + static_cast<double>(mu_kl.y) : 0.0,
                   act ? static_cast<double>(kappa_kl.x) + static_cast<double>(kappa_kl.y) : 0.0};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
#pragma unroll
      for (int off = PL / 2; off > 0; off >>= 1) r[q] += __shfl_xor_sync(seg, r[q], off, PL);
      const int v = i * 3 + q;  // value v of the row goes to lane v % 8, slot v / 8
      if (lane == (v & (PL - 1))) mine[v / PL] = r[q];
    }
  }
  // the row's 15 values: lanes 0-7 (values 0-7), lanes 0-6 (values 8-14)
#pragma unroll
  for (int slot = 0; slot < 2; ++slot) {
    const int v = slot * PL + lane;
    if (v < 3 * N) {
      double *dst = kern + p0 * 3 + v;
      if (atomic) atomicAdd(dst, mine[slot]);
      else *dst += mine[slot];
    }
  }
}

// Stacey traction at the boundary points: a += -A v (mode 0), the same and
// kept in `slot` (mode 1), or the kept traction (mode 2).
__global__ void k3_stacey(const int *__restrict__ bpoint, const float *__restrict__ bdiag, const float *__restrict__ v,
                          float *a, float *slot, int nb, int S, int mode) {
  const size_t n = static_cast<size_t>(nb) * 3 * S;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t b = t / (3 * static_cast<size_t>(S));
    const size_t rem = t - b * 3 * S;
    const size_t at = static_cast<size_t>(bpoint[b]) * 3 * S + rem;
    float tr;
    if (mode == 2) {
      tr = slot[t];
    } else {
      tr = -1.0f * bdiag[b * 3 + rem / S] * v[at];
      if (mode == 1) slot[t] = tr;
    }
    a[at] += tr;
  }
}

// Moment-tensor sources: force += stf(istep) * array at the source element.
__global__ void k3_sources(Dev3 d, int nsrc, const int *elem, const int *shot, const float *array, const float *stf,
                           int nstep, float *a, int istep) {
  const int q = threadIdx.x;
  const int i = blockIdx.x;
  if (i >= nsrc || q >= NNN) return;
  const int g = d.iglob[static_cast<size_t>(elem[i]) * NNN + q];
  const float f = stf[static_cast<size_t>(i) * nstep + istep];
#pragma unroll
  for (int c = 0; c < 3; ++c)
    atomicAdd(a + fidx(g, c, shot[i], d.S), f * array[(static_cast<size_t>(i) * 3 + c) * NNN + q]);
}

// Adjoint sources at the receivers (src/source/adjoint_source.cpp): force
// component c += stf[istep][r][c][s] * h(r, point); one CTA per receiver and
// group of 16 shots, thread (lane = shot, row) over five points.
__global__ void __launch_bounds__(SG * NN) k3_adjoint_sources(Dev3 d, int nrec, const int *relem, const float *rlag,
                                                              const float *stf, float *a, int istep) {
  const int lane = threadIdx.x, row = threadIdx.y;
  const int r = blockIdx.x, s = blockIdx.y * SG + lane;
  const int S = d.S;
  if (s >= S) return;
  const size_t at = (static_cast<size_t>(istep) * nrec + r) * 3 * S;
  const float f[3] = {stf[at + s], stf[at + S + s], stf[at + 2 * S + s]};
  const size_t p0 = static_cast<size_t>(relem[r]) * NNN + row * N;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const int g = d.iglob[p0 + i];
    const float h = rlag[static_cast<size_t>(r) * NNN + row * N + i];
#pragma unroll
    for (int c = 0; c < 3; ++c) atomicAdd(a + fidx(g, c, s, S), f[c] * h);
  }
}

// Displacement seismograms seis[isig][r][c][s] = sum_p h(r, p) u_c(p, s).
__global__ void __launch_bounds__(SG * NN) k3_receivers(Dev3 d, int nrec, const int *relem, const float *rlag,
                                                        const float *u, float *seis, int isig) {
  __shared__ float red[NN][3][SG];
  const int lane = threadIdx.x, row = threadIdx.y;
  const int r = blockIdx.x, s = blockIdx.y * SG + lane;
  const int S = d.S;
  const bool act = s < S;
  float acc[3] = {0.f, 0.f, 0.f};
  const size_t p0 = static_cast<size_t>(relem[r]) * NNN + row * N;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const int g = d.iglob[p0 + i];
    const float h = rlag[static_cast<size_t>(r) * NNN + row * N + i];
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] += act ? h * u[fidx(g, c, s, S)] : 0.f;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) red[row][c][lane] = acc[c];
  __syncthreads();
  if (row < 3 && act) {
    float v = 0.f;
    for (int q = 0; q < NN; ++q) v += red[q][row][lane];
    seis[((static_cast<size_t>(isig) * nrec + r) * 3 + row) * S + s] = v;
  }
}

// Newmark pieces over the [g][c][S] arrays (timescheme/newmark.tpp).
// mode 0 predictor: u += dt v + dt^2/2 a, v += dt/2 a, a = 0;
// mode 1: a *= minv, corrector v += dt/2 a;
// mode 2: mode 1 then the next step's predictor (a is not kept).
template <int MODE>
__global__ void k3_newmark(float *u, float *v, float *a, const float *__restrict__ minv, size_t n4, int S4, float dt,
                           float dt2, float dtsq2) {
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < n4;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    float4 ai = reinterpret_cast<float4 *>(a)[t];
    float4 vi = reinterpret_cast<float4 *>(v)[t];
    if (MODE >= 1) {
      const float m = minv[t / S4];
      ai.x *= m; ai.y *= m; ai.z *= m; ai.w *= m;
      vi.x += dt2 * ai.x; vi.y += dt2 * ai.y; vi.z += dt2 * ai.z; vi.w += dt2 * ai.w;
    }
    if (MODE == 1) {
      reinterpret_cast<float4 *>(a)[t] = ai;
      reinterpret_cast<float4 *>(v)[t] = vi;
      continue;
    }
    float4 ui = reinterpret_cast<float4 *>(u)[t];
    ui.x += dt * vi.x + dtsq2 * ai.x; ui.y += dt * vi.y + dtsq2 * ai.y;
    ui.z += dt * vi.z + dtsq2 * ai.z; ui.w += dt * vi.w + dtsq2 * ai.w;
    vi.x += dt2 * ai.x; vi.y += dt2 * ai.y; vi.z += dt2 * ai.z; vi.w += dt2 * ai.w;
    reinterpret_cast<float4 *>(u)[t] = ui;
    reinterpret_cast<float4 *>(v)[t] = vi;
    reinterpret_cast<float4 *>(a)[t] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}
// The same for shot counts that are not a multiple of 4.
__global__ void k3_newmark_scalar(float *u, float *v, float *a, const float *__restrict__ minv, size_t n, int S,
                                  float dt, float dt2, float dtsq2, int mode) {
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    float ai = a[t], vi = v[t];
    if (mode >= 1) {
      ai = ai * minv[t / S];
      vi = vi + dt2 * ai;
    }
    if (mode == 1) {
      a[t] = ai;
      v[t] = vi;
      continue;
    }
    u[t] += dt * vi + dtsq2 * ai;
    v[t] = vi + dt2 * ai;
    a[t] = 0.f;
  }
}

// Mass matrix: rho w_i w_j w_k J per local point, FP64 accumulation.
// `count` elements: all of them, or (deterministic mode) one colour of
// d.elist, whose points no other element of the launch shares (plain adds).
__global__ void k3_mass(Dev3 d, double *mass, int count) {
  const size_t total = static_cast<size_t>(count) * NNN;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int le = static_cast<int>(t / NNN), q = static_cast<int>(t % NNN);
    const int e = d.elist ? d.elist[d.elist_off + le] : le;
    const int k = q / NN, j = (q / N) % N, i = q % N;
    const size_t p = static_cast<size_t>(e) * NNN + q;
    const float m = d.rho[p] * (c3_w[i] * c3_w[j] * c3_w[k] * d.geo[e].w);
    if (d.det) mass[d.iglob[p]] += static_cast<double>(m);
    else atomicAdd(mass + d.iglob[p], static_cast<double>(m));
  }
}

// Point sources one after another (deterministic mode): one CTA, thread q
// = local point.
__global__ void k3_sources_det(Dev3 d, int nsrc, const int *elem, const int *shot, const float *array,
                               const float *stf, int nstep, float *a, int istep) {
  const int q = threadIdx.x;
  for (int i = 0; i < nsrc; ++i) {
    if (q < NNN) {
      const int g = d.iglob[static_cast<size_t>(elem[i]) * NNN + q];
      const float f = stf[static_cast<size_t>(i) * nstep + istep];
#pragma unroll
      for (int c = 0; c < 3; ++c) a[fidx(g, c, shot[i], d.S)] += f * array[(static_cast<size_t>(i) * 3 + c) * NNN + q];
    }
    __syncthreads();
  }
}

// Adjoint sources one receiver after another (deterministic mode): one CTA
// per group of 16 shots, thread (lane, row) over five points.
__global__ void __launch_bounds__(SG * NN) k3_adjoint_sources_det(Dev3 d, int nrec, const int *relem,
                                                                  const float *rlag, const float *stf, float *a,
                                                                  int istep) {
  const int lane = threadIdx.x, row = threadIdx.y;
  const int S = d.S;
  const int s = blockIdx.x * SG + lane;
  for (int r = 0; r < nrec; ++r) {
    if (s < S) {
      const size_t at = (static_cast<size_t>(istep) * nrec + r) * 3 * S;
      const float f[3] = {stf[at + s], stf[at + S + s], stf[at + 2 * S + s]};
      const size_t p0 = static_cast<size_t>(relem[r]) * NNN + row * N;
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const int g = d.iglob[p0 + i];
        const float h = rlag[static_cast<size_t>(r) * NNN + row * N + i];
#pragma unroll
        for (int c = 0; c < 3; ++c) a[fidx(g, c, s, S)] += f[c] * h;
      }
    }
    __syncthreads();
  }
}

// Inverse mass per (point, component) with the Stacey term dt/2 A_c.
__global__ void k3_invert(const double *mass, const int *bindex, const float *bdiag, float dt, float *minv,
                          size_t nglob) {
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < nglob * 3;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t g = t / 3;
    double m = mass[g];
    const int b = bindex[g];
    if (b >= 0) m += static_cast<double>(dt * 0.5f * bdiag[static_cast<size_t>(b) * 3 + t % 3]);
    minv[t] = static_cast<float>(1.0 / m);
  }
}

// Frechet kernels of one step, summed over the CTA's shots in FP64 and
// added to kern[p][3] = (rho, mu, kappa).  `atomic`: several CTAs share an
// element (more than 16 shots).
__global__ void __launch_bounds__(SG * NN, 2) k3_frechet(Dev3 d, const float *__restrict__ au,
                                                        const float *__restrict__ aa, const float *__restrict__ bu,
                                                        float dt, double *kern, int atomic) {
  extern __shared__ float smem[];
  float *s_a = smem, *s_b = smem + TILE;
  const int lane = threadIdx.x, row = threadIdx.y;
  const int k = row / N, j = row % N;
  const int e = elem_of(d);
  const int S = d.S;
  const int s = group_of(d) * SG + lane;
  const bool act = s < S;
  const float4 gg = d.geo[e];
  const float xix = gg.x, etay = gg.y, gaz = gg.z;
  const size_t p0 = static_cast<size_t>(e) * NNN + row * N;
  int g[N];
  float ra[N][3], rb[N][3];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    g[i] = d.iglob[p0 + i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ra[i][c] = act ? au[fidx(g[i], c, s, S)] : 0.f;
      rb[i][c] = act ? bu[fidx(g[i], c, s, S)] : 0.f;
      s_a[((row * N + i) * 3 + c) * SG + lane] = ra[i][c];
      s_b[((row * N + i) * 3 + c) * SG + lane] = rb[i][c];
    }
  }
  __syncthreads();
  // lanes 0-15 of a warp are one row, 16-31 the next
  const unsigned seg = ((threadIdx.y & 1) ? 0xffff0000u : 0x0000ffffu);
  double mine = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    float da[3][3], db[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float axi = 0.f, aeta = 0.f, azeta = 0.f, bxi = 0.f, beta = 0.f, bzeta = 0.f;
#pragma unroll
      for (int l = 0; l < N; ++l) {
        const float hx = c3_hp[i * N + l], hy = c3_hp[j * N + l], hz = c3_hp[k * N + l];
        axi += hx * ra[l][c];
        bxi += hx * rb[l][c];
        aeta += hy * s_a[(((k * N + l) * N + i) * 3 + c) * SG + lane];
        beta += hy * s_b[(((k * N + l) * N + i) * 3 + c) * SG + lane];
        azeta += hz * s_a[(((l * N + j) * N + i) * 3 + c) * SG + lane];
        bzeta += hz * s_b[(((l * N + j) * N + i) * 3 + c) * SG + lane];
      }
      da[c][0] = xix * axi;
      da[c][1] = etay * aeta;
      da[c][2] = gaz * azeta;
      db[c][0] = xix * bxi;
      db[c][1] = etay * beta;
      db[c][2] = gaz * bzeta;
    }
    const size_t p = p0 + i;
    const float diva = da[0][0] + da[1][1] + da[2][2], divb = db[0][0] + db[1][1] + db[2][2];
    float ee = 0.f;  // eps_adj : eps
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int x = 0; x < 3; ++x) ee += (0.5f * (da[c][x] + da[x][c])) * (0.5f * (db[c][x] + db[x][c]));
    float kappa_kl = diva * divb;
    float mu_kl = ee - kOneThird * kappa_kl;
    float rho_kl = 0.f;
    if (act) {
#pragma unroll
      for (int c = 0; c < 3; ++c) rho_kl += aa[fidx(g[i], c, s, S)] * rb[i][c];
    }
    kappa_kl = -1.0f * d.kappa[p] * dt * kappa_kl;
    mu_kl = -2.0f * d.mu[p] * dt * mu_kl;
    rho_kl = -1.0f * d.rho[p] * dt * rho_kl;
    double r[3] = {act ? static_cast<double>(rho_kl) : 0.0, act ? static_cast<double>(mu_kl) : 0.0,
                   act ? static_cast<double>(kappa_kl) : 0.0};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
#pragma unroll
      for (int off = SG / 2; off > 0; off >>= 1) r[q] += __shfl_xor_sync(seg, r[q], off, SG);
      if (lane == i * 3 + q) mine = r[q];
    }
  }
  // lanes 0-14 hold the row's 5 points x 3 kernels: one contiguous write
  if (lane < 3 * N) {
    double *dst = kern + p0 * 3 + lane;
    if (atomic) atomicAdd(dst, mine);
    else *dst += mine;
  }
}

// dst[m] = src[m * S + s]: one shot out of a shot-minor array.
__global__ void k3_gather(const float *src, float *dst, size_t m, int S, int s) {
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < m;
       t += static_cast<size_t>(gridDim.x) * blockDim.x)
    dst[t] = src[t * S + s];
}
// dst[m * S + s] = src[m]
__global__ void k3_scatter(const float *src, float *dst, size_t m, int S, int s) {
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < m;
       t += static_cast<size_t>(gridDim.x) * blockDim.x)
    dst[t * S + s] = src[t];
}

int grid_of(size_t n, int block) {
  const size_t g = (n + block - 1) / block;
  return static_cast<int>(std::max<size_t>(1, std::min<size_t>(g, static_cast<size_t>(148) * 16)));
}

// Device or host memory that could not be had: reported as SFB_E_NOMEM.
struct NoMemError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void ck3(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T> struct Buf {
  T *p = nullptr;
  size_t n = 0;
  size_t *total = nullptr;
  void alloc(size_t count, size_t *tot) {
    release();
    n = count;
    total = tot;
    if (!count) return;
    if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      n = 0;
      throw NoMemError("cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
    }
    // zeroed on the legacy default stream, which the contexts' non-blocking
    // streams do not wait for: finish it before any kernel can read the
    // buffer (reused memory still holds a freed buffer's data)
    ck3(cudaMemset(p, 0, count * sizeof(T)), "cudaMemset");
    ck3(cudaStreamSynchronize(0), "cudaMemset");
    *tot += count * sizeof(T);
  }
  void upload(const std::vector<T> &h, size_t *tot) {
    alloc(h.size(), tot);
    if (!h.empty()) ck3(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
  }
  void release() {
    if (p) {
      cudaFree(p);
      if (total) *total -= n * sizeof(T);
    }
    p = nullptr;
    n = 0;
  }
  ~Buf() { release(); }
};

struct Wave {
  Buf<float> u, v, a;
  void alloc(size_t n, size_t *tot) {
    u.alloc(n, tot);
    v.alloc(n, tot);
    a.alloc(n, tot);
  }
  bool ready() const { return u.p != nullptr; }
};

thread_local std::string g_err3;

}  // namespace

struct sfb3_context {
  std::string err;
  int nx = 0, ny = 0, nz = 0, nspec = 0, nglob = 0, S = 0, nstep = 0, nrec = 0, nsrc = 0, nb = 0;
  int nshared = 0, nprivate = 0;  // point numbering: shared points first, private points last
  std::vector<int> perm;          // lattice index -> device point index
  double x0 = 0, y0 = 0, z0 = 0, dx = 0, dy = 0, dz = 0, dt = 0, t0 = 0;
  bool save = false;
  int step = 0;
  int seg_len = 0, nseg = 1;
  bool ckpt_host = false;
  bool fwd_final = true;       // the forward fields hold the state after `step` steps
  int variant = 0;             // kernel variant (variant_of)
  bool det = false;            // deterministic assembly (colour launches, fixed-order sums)
  int col_off[9] = {0};        // elements of colour c: elist[col_off[c], col_off[c + 1])
  sfb::Quadrature quad{N};
  cudaStream_t stream = nullptr;
  size_t bytes = 0, host_bytes = 0;
  unsigned long long launches = 0;
  // mesh, model, boundary
  Buf<int> iglob, bpoint, bindex;
  Buf<unsigned char> priv;
  Buf<int> elist;
  Buf<float4> geo;
  Buf<float> kappa, mu, rho, bdiag, minv;
  // sources and receivers
  Buf<int> src_elem, src_shot, rec_elem;
  Buf<float> src_array, src_stf, rec_lag, adj_stf;
  // state
  Wave fwd, adj, bwd;
  Buf<float> seis_f, seis_b, store, scratch;
  Buf<double> kern;
  // checkpoints: slot k < nseg - 1 holds the state after (k + 1) * seg_len
  // steps, slot nseg - 1 the final state; each slot u, v, a
  Buf<float> ckpt_dev;
  float *ckpt_host_p = nullptr;
  float *ckpt_pageable = nullptr;
  float *host_ckpt() const { return ckpt_host_p ? ckpt_host_p : ckpt_pageable; }
  size_t field_n() const { return static_cast<size_t>(nglob) * 3 * S; }
  Dev3 dev() const {
    Dev3 d{};
    d.nspec = nspec;
    d.S = S;
    d.iglob = iglob.p;
    d.geo = geo.p;
    d.kappa = kappa.p;
    d.mu = mu.p;
    d.rho = rho.p;
    d.priv = priv.p;
    d.det = det ? 1 : 0;
    return d;
  }
  ~sfb3_context() {
    if (stream) cudaStreamSynchronize(stream);
    if (ckpt_host_p) cudaFreeHost(ckpt_host_p);
    std::free(ckpt_pageable);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

template <typename F> int guarded3(sfb3_context *c, F &&fn) {
  try {
    return fn();
  } catch (const std::invalid_argument &e) {
    (c ? c->err : g_err3) = e.what();
    return SFB_E_INVALID;
  } catch (const NoMemError &e) {
    (c ? c->err : g_err3) = e.what();
    return SFB_E_NOMEM;
  } catch (const std::exception &e) {
    (c ? c->err : g_err3) = e.what();
    return SFB_E_CUDA;
  }
}

// Element containing (x, y, z) and the reference coordinates there.
// Points outside the mesh are rejected rather than extrapolated from the
// nearest element's interpolants.
void locate(const sfb3_context *c, double x, double y, double z, int &e, double r[3]) {
  const double v[3] = {x, y, z}, o[3] = {c->x0, c->y0, c->z0}, h[3] = {c->dx, c->dy, c->dz};
  const int n[3] = {c->nx, c->ny, c->nz};
  int ie[3];
  for (int a = 0; a < 3; ++a) {
    const double tol = 1e-9 * h[a] * n[a];
    if (!(v[a] >= o[a] - tol && v[a] <= o[a] + h[a] * n[a] + tol))
      throw std::invalid_argument("point (" + std::to_string(x) + ", " + std::to_string(y) + ", " +
                                  std::to_string(z) + ") lies outside the mesh");
    ie[a] = static_cast<int>(std::floor((v[a] - o[a]) / h[a]));
    ie[a] = std::min(std::max(ie[a], 0), n[a] - 1);
    r[a] = 2.0 * (v[a] - (o[a] + ie[a] * h[a])) / h[a] - 1.0;
  }
  e = (ie[2] * c->ny + ie[1]) * c->nx + ie[0];
}

// Kernel variant: packed kernels for an even shot count (pairs stay 8-byte
// aligned), the scalar ones otherwise.  Variant 1 forces the scalar
// kernels; 2 (default) and 3 are the packed kernels compiled for two and
// three resident CTAs per SM.
int variant_of(const sfb3_context *c) {
  if (c->S % 2 != 0 || c->variant == 1) return 1;
  return c->variant == 3 ? 3 : 2;
}

// Does the forward stiffness launch finish the private points?  (Packed
// kernels only; otherwise the update kernel walks every point.)
bool private_on(const sfb3_context *c) { return c->nprivate > 0 && variant_of(c) != 1; }

// `pv` null: every point's force is scattered (adjoint and backward runs,
// timing); otherwise the private points of marked elements are finished.
// The element kernels' launches: one over all elements and shot groups, or
// in the deterministic mode one per shot group and element colour (group
// outer, colours 0-7 inner), so that every point's sum is taken in the same
// order on every run.  `launch(d, grid)` issues one launch.
template <typename F> void element_launches(sfb3_context *c, F &&launch) {
  const int groups = (c->S + SG - 1) / SG;
  Dev3 d = c->dev();
  if (!c->det) {
    launch(d, dim3(c->nspec, groups));
    return;
  }
  d.elist = c->elist.p;
  for (int g = 0; g < groups; ++g)
    for (int col = 0; col < 8; ++col) {
      const int n = c->col_off[col + 1] - c->col_off[col];
      if (n == 0) continue;
      d.elist_off = c->col_off[col];
      d.sgroup = g;
      launch(d, dim3(n, 1));
    }
}

void launch_stiffness(sfb3_context *c, const float *u, float *a, const PrivArgs *pv = nullptr) {
  const size_t sm = (3 * TILE + PRIV_WORDS) * sizeof(float);
  const FrArgs none{};
  const PrivArgs off{};
  const PrivArgs &p = (pv && private_on(c)) ? *pv : off;
  const int v = variant_of(c);
  element_launches(c, [&](const Dev3 &d, dim3 grid) {
    switch (v) {
      case 1: k3_stiffness<<<grid, dim3(SG, NN), 3 * TILE * sizeof(float), c->stream>>>(d, u, a); break;
      case 3: k3_stiffness_pk<3, false><<<grid, dim3(PL, NN), sm, c->stream>>>(d, u, a, none, p); break;
      default: k3_stiffness_pk<2, false><<<grid, dim3(PL, NN), sm, c->stream>>>(d, u, a, none, p); break;
    }
    ++c->launches;
  });
}

// The backward stiffness with the step's Frechet kernels (packed variants):
// au / af the adjoint displacement and complete adjoint force of the step.
void launch_stiffness_frechet(sfb3_context *c, const float *u, float *a, const float *au, const float *af) {
  const size_t sm = 4 * TILE * sizeof(float);
  const PrivArgs off{};
  const int v = variant_of(c);
  element_launches(c, [&](const Dev3 &d, dim3 grid) {
    const FrArgs fr{au, af, c->minv.p, c->kern.p, static_cast<float>(c->dt), grid.y > 1 ? 1 : 0};
    if (v == 3) k3_stiffness_pk<3, true><<<grid, dim3(PL, NN), sm, c->stream>>>(d, u, a, fr, off);
    else k3_stiffness_pk<2, true><<<grid, dim3(PL, NN), sm, c->stream>>>(d, u, a, fr, off);
    ++c->launches;
  });
}

void launch_stacey(sfb3_context *c, const float *v, float *a, int mode, int slot) {
  if (c->nb == 0) return;
  const size_t n = static_cast<size_t>(c->nb) * 3 * c->S;
  float *sl = c->store.p ? c->store.p + static_cast<size_t>(slot) * n : nullptr;
  if (mode != 0 && !sl) throw std::logic_error("no Stacey store for this run");
  k3_stacey<<<grid_of(n, 256), 256, 0, c->stream>>>(c->bpoint.p, c->bdiag.p, v, a, sl, c->nb, c->S, mode);
  ++c->launches;
}

// `shared_only`: the update walks the shared points (the prefix of the
// numbering); the forward stiffness launch finished the private ones.
void newmark(sfb3_context *c, Wave &w, double sdt, int mode, bool shared_only = false) {
  const size_t n = static_cast<size_t>(shared_only && private_on(c) ? c->nshared : c->nglob) * 3 * c->S;
  const float dt = static_cast<float>(sdt), dt2 = static_cast<float>(sdt / 2.0),
              dtsq2 = static_cast<float>(c->dt * c->dt / 2.0);
  if (c->S % 4 == 0) {
    const size_t n4 = n / 4;
    const int S4 = c->S / 4;
    const int grid = grid_of(n4, 256);
    if (mode == 0) k3_newmark<0><<<grid, 256, 0, c->stream>>>(w.u.p, w.v.p, w.a.p, c->minv.p, n4, S4, dt, dt2, dtsq2);
    else if (mode == 1) k3_newmark<1><<<grid, 256, 0, c->stream>>>(w.u.p, w.v.p, w.a.p, c->minv.p, n4, S4, dt, dt2, dtsq2);
    else k3_newmark<2><<<grid, 256, 0, c->stream>>>(w.u.p, w.v.p, w.a.p, c->minv.p, n4, S4, dt, dt2, dtsq2);
  } else {
    k3_newmark_scalar<<<grid_of(n, 256), 256, 0, c->stream>>>(w.u.p, w.v.p, w.a.p, c->minv.p, n, c->S, dt, dt2, dtsq2,
                                                              mode);
  }
  ++c->launches;
}

void forward_sources(sfb3_context *c, float *a, int istep) {
  if (c->nsrc == 0) return;
  if (c->det)
    k3_sources_det<<<1, 128, 0, c->stream>>>(c->dev(), c->nsrc, c->src_elem.p, c->src_shot.p, c->src_array.p,
                                              c->src_stf.p, c->nstep, a, istep);
  else
    k3_sources<<<c->nsrc, 128, 0, c->stream>>>(c->dev(), c->nsrc, c->src_elem.p, c->src_shot.p, c->src_array.p,
                                                c->src_stf.p, c->nstep, a, istep);
  ++c->launches;
}

void adjoint_sources(sfb3_context *c, float *a, int istep) {
  if (c->nrec == 0) return;
  if (c->det)
    k3_adjoint_sources_det<<<(c->S + SG - 1) / SG, dim3(SG, NN), 0, c->stream>>>(
        c->dev(), c->nrec, c->rec_elem.p, c->rec_lag.p, c->adj_stf.p, a, istep);
  else
    k3_adjoint_sources<<<dim3(c->nrec, (c->S + SG - 1) / SG), dim3(SG, NN), 0, c->stream>>>(
        c->dev(), c->nrec, c->rec_elem.p, c->rec_lag.p, c->adj_stf.p, a, istep);
  ++c->launches;
}

void receivers(sfb3_context *c, const float *u, float *seis, int isig) {
  if (c->nrec == 0) return;
  k3_receivers<<<dim3(c->nrec, (c->S + SG - 1) / SG), dim3(SG, NN), 0, c->stream>>>(
      c->dev(), c->nrec, c->rec_elem.p, c->rec_lag.p, u, seis, isig);
  ++c->launches;
}

void frechet(sfb3_context *c, const float *au, const float *aa, const float *bu) {
  const size_t sm = 2 * TILE * sizeof(float);
  const float dt = static_cast<float>(c->dt);
  const int v = variant_of(c);
  element_launches(c, [&](const Dev3 &d, dim3 grid) {
    const int atomic = grid.y > 1 ? 1 : 0;
    switch (v) {
      case 1: k3_frechet<<<grid, dim3(SG, NN), sm, c->stream>>>(d, au, aa, bu, dt, c->kern.p, atomic); break;
      case 3: k3_frechet_pk<3><<<grid, dim3(PL, NN), sm, c->stream>>>(d, au, aa, bu, dt, c->kern.p, atomic); break;
      default: k3_frechet_pk<2><<<grid, dim3(PL, NN), sm, c->stream>>>(d, au, aa, bu, dt, c->kern.p, atomic); break;
    }
    ++c->launches;
  });
}

void copy_wave(sfb3_context *c, Wave &dst, const Wave &src) {
  const size_t b = c->field_n() * sizeof(float);
  ck3(cudaMemcpyAsync(dst.u.p, src.u.p, b, cudaMemcpyDeviceToDevice, c->stream), "copy");
  ck3(cudaMemcpyAsync(dst.v.p, src.v.p, b, cudaMemcpyDeviceToDevice, c->stream), "copy");
  ck3(cudaMemcpyAsync(dst.a.p, src.a.p, b, cudaMemcpyDeviceToDevice, c->stream), "copy");
}

void zero_wave(sfb3_context *c, Wave &w) {
  const size_t b = c->field_n() * sizeof(float);
  for (Buf<float> *f : {&w.u, &w.v, &w.a})
    if (f->p) ck3(cudaMemsetAsync(f->p, 0, b, c->stream), "zero");
}

// Checkpoint slot <-> wavefield (three fields, device or pinned host).
void checkpoint(sfb3_context *c, int slot, Wave &w, bool save) {
  const size_t n = c->field_n();
  Buf<float> *f[3] = {&w.u, &w.v, &w.a};
  for (int q = 0; q < 3; ++q) {
    const size_t off = (static_cast<size_t>(slot) * 3 + q) * n;
    float *ck = c->ckpt_host ? c->host_ckpt() + off : c->ckpt_dev.p + off;
    const cudaMemcpyKind kind = c->ckpt_host ? (save ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice)
                                             : cudaMemcpyDeviceToDevice;
    if (save) ck3(cudaMemcpyAsync(ck, f[q]->p, n * sizeof(float), kind, c->stream), "checkpoint");
    else ck3(cudaMemcpyAsync(f[q]->p, ck, n * sizeof(float), kind, c->stream), "checkpoint");
  }
}

// Forward steps [s0, s1) from the state after s0 steps (time_marching.tpp
// forward loop: predictor; sources + stiffness + Stacey; seismograms;
// divide by the mass and corrector, fused with the next step's predictor).
// store_mode 1 keeps the Stacey tractions in slot istep - slot_base.
void march_forward(sfb3_context *c, int s0, int s1, int store_mode, int slot_base, bool record) {
  if (s1 <= s0) return;
  newmark(c, c->fwd, c->dt, 0);
  PrivArgs pv{c->fwd.v.p, c->minv.p, static_cast<float>(c->dt), static_cast<float>(c->dt / 2.0),
              static_cast<float>(c->dt * c->dt / 2.0), 0, 1};
  for (int istep = s0; istep < s1; ++istep) {
    pv.last = istep + 1 == s1 ? 1 : 0;
    forward_sources(c, c->fwd.a.p, istep);
    launch_stiffness(c, c->fwd.u.p, c->fwd.a.p, &pv);
    launch_stacey(c, c->fwd.v.p, c->fwd.a.p, store_mode, istep - slot_base);
    if (record) receivers(c, c->fwd.u.p, c->seis_f.p, istep);
    newmark(c, c->fwd, c->dt, pv.last ? 1 : 2, true);
  }
}

void run_forward_impl(sfb3_context *c, int nstep) {
  const int end = c->step + nstep;
  const int store_mode = (c->save && c->nseg == 1 && c->nb) ? 1 : 0;
  while (c->step < end) {
    int stop = end;
    if (c->nseg > 1) stop = std::min(end, (c->step / c->seg_len + 1) * c->seg_len);
    march_forward(c, c->step, stop, store_mode, 0, true);
    c->step = stop;
    if (c->nseg > 1 && c->step % c->seg_len == 0 && c->step < c->nstep)
      checkpoint(c, c->step / c->seg_len - 1, c->fwd, true);
  }
  if (c->nseg > 1 && c->step == c->nstep && nstep > 0) checkpoint(c, c->nseg - 1, c->fwd, true);
  c->fwd_final = true;
}

// The combined run (time_marching.tpp:126-247), enqueued on the context's stream.
void run_combined_impl(sfb3_context *c) {
  if (!c->save) throw std::invalid_argument("the context keeps no adjoint state (save_boundary_values)");
  if (c->step != c->nstep) throw std::invalid_argument("run the whole forward simulation first");
  zero_wave(c, c->adj);
  ck3(cudaMemsetAsync(c->kern.p, 0, c->kern.n * sizeof(double), c->stream), "zero");
  // the backward wavefield starts from the forward run's last state (the
  // reference overwrites its first reversed step with it)
  if (c->nseg == 1) copy_wave(c, c->bwd, c->fwd);
  else checkpoint(c, c->nseg - 1, c->bwd, false);
  // Per reversed step: adjoint predictor (+dt), adjoint sources,
  // stiffness and Stacey; backward predictor (-dt), forward sources,
  // stiffness, replayed tractions; correctors; the step's kernels; the
  // backward seismogram.  With the packed kernels the kernels are added
  // by the backward stiffness launch (from the adjoint force before its
  // corrector) and each wavefield's corrector is fused with its next
  // step's predictor; the first reversed step keeps the forward run's
  // last state as the backward state (no backward step) and adds its
  // kernels with the separate Frechet launch.
  const bool fused = variant_of(c) != 1;
  newmark(c, c->adj, c->dt, 0);
  int isig = 0;
  for (int seg = c->nseg - 1; seg >= 0; --seg) {
    const int s0 = seg * c->seg_len, s1 = std::min(c->nstep, s0 + c->seg_len);
    if (c->nseg > 1) {
      // recompute this segment's forward steps, keeping the tractions
      if (seg == 0) zero_wave(c, c->fwd);
      else checkpoint(c, seg - 1, c->fwd, false);
      c->fwd_final = false;
      march_forward(c, s0, s1, c->nb ? 1 : 0, s0, false);
    }
    for (int istep = s1 - 1; istep >= s0; --istep) {
      const bool last = istep == 0;
      adjoint_sources(c, c->adj.a.p, istep);
      launch_stiffness(c, c->adj.u.p, c->adj.a.p);
      launch_stacey(c, c->adj.v.p, c->adj.a.p, 0, 0);
      if (istep == c->nstep - 1) {
        newmark(c, c->adj, c->dt, 1);
        frechet(c, c->adj.u.p, c->adj.a.p, c->bwd.u.p);
        receivers(c, c->bwd.u.p, c->seis_b.p, isig++);
        if (!last) {
          newmark(c, c->adj, c->dt, 0);
          newmark(c, c->bwd, -c->dt, 0);
        }
        continue;
      }
      forward_sources(c, c->bwd.a.p, istep);
      if (fused) launch_stiffness_frechet(c, c->bwd.u.p, c->bwd.a.p, c->adj.u.p, c->adj.a.p);
      else launch_stiffness(c, c->bwd.u.p, c->bwd.a.p);
      launch_stacey(c, c->bwd.v.p, c->bwd.a.p, 2, istep - s0);
      if (fused) {
        receivers(c, c->bwd.u.p, c->seis_b.p, isig++);
        newmark(c, c->adj, c->dt, last ? 1 : 2);
        newmark(c, c->bwd, -c->dt, last ? 1 : 2);
      } else {
        newmark(c, c->adj, c->dt, 1);
        newmark(c, c->bwd, -c->dt, 1);
        frechet(c, c->adj.u.p, c->adj.a.p, c->bwd.u.p);
        receivers(c, c->bwd.u.p, c->seis_b.p, isig++);
        if (!last) {
          newmark(c, c->adj, c->dt, 0);
          newmark(c, c->bwd, -c->dt, 0);
        }
      }
    }
  }
  if (c->nseg > 1) {
    checkpoint(c, c->nseg - 1, c->fwd, false);
    c->fwd_final = true;
  }
}

void ensure_scratch(sfb3_context *c) {
  if (!c->adj.ready()) c->adj.alloc(c->field_n(), &c->bytes);
}

}  // namespace

extern "C" {

SFB_API const char *sfb3_last_error(const sfb3_context *ctx) { return ctx ? ctx->err.c_str() : g_err3.c_str(); }

SFB_API int sfb3_create(const sfb3_desc *d, sfb3_context **out) {
  if (!d || !out) return SFB_E_INVALID;
  *out = nullptr;
  return guarded3(nullptr, [&]() {
    if (d->nx < 1 || d->ny < 1 || d->nz < 1) throw std::invalid_argument("the mesh needs an element per axis");
    if (d->nshots < 1 || d->nstep < 1 || !(d->dt > 0)) throw std::invalid_argument("bad nshots, nstep or dt");
    if (!(d->x1 > d->x0 && d->y1 > d->y0 && d->z1 > d->z0)) throw std::invalid_argument("empty domain");
    if (!d->rho || !d->vp || !d->vs) throw std::invalid_argument("no model");
    if (d->nsources < 0 || (d->nsources && !d->sources) || d->nreceivers < 0 || (d->nreceivers && !d->receivers))
      throw std::invalid_argument("bad source or receiver list");
    const long long gx = 4LL * d->nx + 1, gy = 4LL * d->ny + 1, gz = 4LL * d->nz + 1;
    if (gx * gy * gz >= (1LL << 31) || static_cast<long long>(d->nx) * d->ny * d->nz * NNN >= (1LL << 31))
      throw std::invalid_argument("mesh too large");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw std::runtime_error("no CUDA device available");
    std::unique_ptr<sfb3_context> c(new sfb3_context());
    c->nx = d->nx;
    c->ny = d->ny;
    c->nz = d->nz;
    c->nspec = d->nx * d->ny * d->nz;
    c->nglob = static_cast<int>(gx * gy * gz);
    c->x0 = d->x0;
    c->y0 = d->y0;
    c->z0 = d->z0;
    c->dx = (d->x1 - d->x0) / d->nx;
    c->dy = (d->y1 - d->y0) / d->ny;
    c->dz = (d->z1 - d->z0) / d->nz;
    c->dt = d->dt;
    c->nstep = d->nstep;
    c->S = d->nshots;
    c->save = d->save_boundary_values != 0;
    c->nrec = d->nreceivers;
    c->nsrc = d->nsources;
    c->det = d->deterministic != 0;
    ck3(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream");
    ck3(cudaFuncSetAttribute(k3_stiffness, cudaFuncAttributeMaxDynamicSharedMemorySize, 3 * TILE * sizeof(float)),
        "attribute");
    ck3(cudaFuncSetAttribute(k3_frechet, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * TILE * sizeof(float)),
        "attribute");
    for (const void *f : {reinterpret_cast<const void *>(k3_stiffness_pk<2, false>),
                          reinterpret_cast<const void *>(k3_stiffness_pk<3, false>)})
      ck3(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (3 * TILE + PRIV_WORDS) * sizeof(float)),
          "attribute");
    for (const void *f : {reinterpret_cast<const void *>(k3_stiffness_pk<2, true>),
                          reinterpret_cast<const void *>(k3_stiffness_pk<3, true>)})
      ck3(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * TILE * sizeof(float)),
          "attribute");
    for (const void *f : {reinterpret_cast<const void *>(k3_frechet_pk<2>),
                          reinterpret_cast<const void *>(k3_frechet_pk<3>)})
      ck3(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * TILE * sizeof(float)),
          "attribute");
    size_t *tot = &c->bytes;
    const int nspec = c->nspec;
    const size_t nloc = static_cast<size_t>(nspec) * NNN;
    // quadrature tables (FP32, the reference's type_real)
    float hp[NN], hpw[NN], w[N];
    for (int i = 0; i < N; ++i) w[i] = static_cast<float>(c->quad.w[i]);
    for (int i = 0; i < NN; ++i) hp[i] = static_cast<float>(c->quad.hprime[i]);
    for (int i = 0; i < N; ++i)
      for (int l = 0; l < N; ++l) hpw[i * N + l] = hp[l * N + i] * w[l];
    ck3(cudaMemcpyToSymbol(c3_hp, hp, sizeof(hp)), "tables");
    ck3(cudaMemcpyToSymbol(c3_hpw, hpw, sizeof(hpw)), "tables");
    ck3(cudaMemcpyToSymbol(c3_w, w, sizeof(w)), "tables");
    // numbering and model
    std::vector<int> iglob(nloc);
    std::vector<float> kap(nloc), mu(nloc), rho(nloc);
    for (int ez = 0; ez < d->nz; ++ez)
      for (int ey = 0; ey < d->ny; ++ey)
        for (int ex = 0; ex < d->nx; ++ex) {
          const int e = (ez * d->ny + ey) * d->nx + ex;
          for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
              for (int i = 0; i < N; ++i) {
                const size_t p = static_cast<size_t>(e) * NNN + (k * N + j) * N + i;
                iglob[p] = static_cast<int>(((4 * ez + k) * gy + (4 * ey + j)) * gx + (4 * ex + i));
                // properties.hpp: mu = rho vs^2, kappa = rho (vp^2 - 4/3 vs^2)
                const float r = d->rho[p], a = d->vp[p], b = d->vs[p];
                if (!(r > 0) || !(a > 0) || !(b >= 0)) throw std::invalid_argument("non-positive model value");
                rho[p] = r;
                mu[p] = r * b * b;
                kap[p] = r * (a * a - kFourThirds * b * b);
              }
        }
    // Stacey: per global point the diagonal A_c = sum over absorbing element
    // faces through it of w_a w_b |J_face| (rho vs + (rho vp - rho vs) n_c^2)
    std::vector<double> adiag(static_cast<size_t>(c->nglob) * 3, 0.0);
    std::vector<char> onb(c->nglob, 0);
    const double fj[3] = {c->dy * c->dz / 4.0, c->dx * c->dz / 4.0, c->dx * c->dy / 4.0};
    for (int ez = 0; ez < d->nz; ++ez)
      for (int ey = 0; ey < d->ny; ++ey)
        for (int ex = 0; ex < d->nx; ++ex) {
          const int e = (ez * d->ny + ey) * d->nx + ex;
          const bool on[6] = {ex == 0, ex == d->nx - 1, ey == 0, ey == d->ny - 1, ez == 0, ez == d->nz - 1};
          for (int f = 0; f < 6; ++f) {
            if (!on[f] || !((d->absorb >> f) & 1)) continue;
            const int axis = f / 2;
            const int fixed = (f & 1) ? N - 1 : 0;
            for (int b1 = 0; b1 < N; ++b1)
              for (int b0 = 0; b0 < N; ++b0) {
                int k, j, i;
                if (axis == 0) { i = fixed; j = b0; k = b1; }
                else if (axis == 1) { j = fixed; i = b0; k = b1; }
                else { k = fixed; i = b0; j = b1; }
                const size_t p = static_cast<size_t>(e) * NNN + (k * N + j) * N + i;
                const float l2m = kap[p] + kFourThirds * mu[p];
                const float rho_vp = std::sqrt(l2m / rho[p]) * rho[p];
                const float rho_vs = std::sqrt(rho[p] * mu[p]);
                const double wf = c->quad.w[b0] * c->quad.w[b1] * fj[axis];
                const int g = iglob[p];
                onb[g] = 1;
                for (int cc = 0; cc < 3; ++cc)
                  adiag[static_cast<size_t>(g) * 3 + cc] += wf * (cc == axis ? rho_vp : rho_vs);
              }
          }
        }
    std::vector<int> bpoint, bindex(c->nglob, -1);
    std::vector<float> bdiag;
    for (int g = 0; g < c->nglob; ++g)
      if (onb[g]) {
        bindex[g] = static_cast<int>(bpoint.size());
        bpoint.push_back(g);
        for (int cc = 0; cc < 3; ++cc) bdiag.push_back(static_cast<float>(adiag[static_cast<size_t>(g) * 3 + cc]));
      }
    c->nb = static_cast<int>(bpoint.size());
    const float4 g4 = make_float4(static_cast<float>(2.0 / c->dx), static_cast<float>(2.0 / c->dy),
                                  static_cast<float>(2.0 / c->dz),
                                  static_cast<float>(c->dx * c->dy * c->dz / 8.0));
    c->geo.upload(std::vector<float4>(nspec, g4), tot);
    c->kappa.upload(kap, tot);
    c->mu.upload(mu, tot);
    c->rho.upload(rho, tot);
    c->bdiag.upload(bdiag, tot);
    // sources: t0 and time shifts as io/sources.cpp:128-158 sets them
    std::vector<sfb::Source> srcs(d->nsources);
    for (int q = 0; q < d->nsources; ++q) {
      const sfb3_source &s = d->sources[q];
      if (s.shot < 0 || s.shot >= c->S) throw std::invalid_argument("source shot out of range");
      if (!(s.f0 > 0)) throw std::invalid_argument("source frequency must be positive");
      srcs[q].kind = sfb::Source::MOMENT_TENSOR;
      srcs[q].stf = sfb::Source::RICKER;
      srcs[q].f0 = s.f0;
      srcs[q].tshift = s.tshift;
      srcs[q].factor = s.factor;
    }
    c->t0 = d->nsources ? sfb::resolve_t0(srcs, 0.0) : 0.0;
    std::vector<int> selem(d->nsources), sshot(d->nsources);
    std::vector<float> sarr(static_cast<size_t>(d->nsources) * 3 * NNN),
        sstf(static_cast<size_t>(d->nsources) * d->nstep);
    const double inv[3] = {2.0 / c->dx, 2.0 / c->dy, 2.0 / c->dz};
    for (int q = 0; q < d->nsources; ++q) {
      const sfb3_source &s = d->sources[q];
      int e;
      double r[3];
      locate(c.get(), s.x, s.y, s.z, e, r);
      selem[q] = e;
      sshot[q] = s.shot;
      double h[3][N], hd[3][N];
      for (int a = 0; a < 3; ++a) sfb::lagrange_interpolants(c->quad, r[a], h[a], hd[a]);
      const double M[3][3] = {{s.mxx, s.mxy, s.mxz}, {s.mxy, s.myy, s.myz}, {s.mxz, s.myz, s.mzz}};
      for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i) {
            const double dd[3] = {hd[0][i] * inv[0] * h[1][j] * h[2][k], h[0][i] * hd[1][j] * inv[1] * h[2][k],
                                  h[0][i] * h[1][j] * hd[2][k] * inv[2]};
            for (int cc = 0; cc < 3; ++cc)
              sarr[(static_cast<size_t>(q) * 3 + cc) * NNN + (k * N + j) * N + i] =
                  static_cast<float>(M[cc][0] * dd[0] + M[cc][1] * dd[1] + M[cc][2] * dd[2]);
          }
      for (int t = 0; t < d->nstep; ++t)
        sstf[static_cast<size_t>(q) * d->nstep + t] = static_cast<float>(srcs[q].value(c->t0 + t * c->dt));
    }
    c->src_elem.upload(selem, tot);
    c->src_shot.upload(sshot, tot);
    c->src_array.upload(sarr, tot);
    c->src_stf.upload(sstf, tot);
    // receivers
    std::vector<int> relem(c->nrec);
    std::vector<float> rlag(static_cast<size_t>(c->nrec) * NNN);
    for (int r = 0; r < c->nrec; ++r) {
      int e;
      double rr[3];
      locate(c.get(), d->receivers[r * 3], d->receivers[r * 3 + 1], d->receivers[r * 3 + 2], e, rr);
      relem[r] = e;
      double h[3][N], hd[3][N];
      for (int a = 0; a < 3; ++a) sfb::lagrange_interpolants(c->quad, rr[a], h[a], hd[a]);
      for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i)
            rlag[static_cast<size_t>(r) * NNN + (k * N + j) * N + i] = static_cast<float>(h[0][i] * h[1][j] * h[2][k]);
    }
    c->rec_elem.upload(relem, tot);
    c->rec_lag.upload(rlag, tot);
    // Element-private points: the 27 interior points of an element without
    // sources or receivers belong to it alone; they are numbered after all
    // shared points so that the forward update walks a prefix, and the
    // forward stiffness launch finishes them (lattice order kept in each
    // group).
    {
      std::vector<unsigned char> priv(nspec, 1);
      for (int e : selem) priv[e] = 0;
      for (int e : relem) priv[e] = 0;
      std::vector<char> is_private(c->nglob, 0);
      for (int e = 0; e < nspec; ++e) {
        if (!priv[e]) continue;
        for (int k = 1; k < N - 1; ++k)
          for (int j = 1; j < N - 1; ++j)
            for (int i = 1; i < N - 1; ++i) is_private[iglob[static_cast<size_t>(e) * NNN + (k * N + j) * N + i]] = 1;
      }
      c->perm.assign(c->nglob, 0);
      int next = 0;
      for (int g = 0; g < c->nglob; ++g)
        if (!is_private[g]) c->perm[g] = next++;
      c->nshared = next;
      for (int g = 0; g < c->nglob; ++g)
        if (is_private[g]) c->perm[g] = next++;
      c->nprivate = c->nglob - c->nshared;
      for (auto &g : iglob) g = c->perm[g];
      for (auto &g : bpoint) g = c->perm[g];
      std::vector<int> bidx(c->nglob, -1);
      for (int g = 0; g < c->nglob; ++g) bidx[c->perm[g]] = bindex[g];
      c->iglob.upload(iglob, tot);
      // element colours by coordinate parity: hexahedra of one colour share
      // no point (deterministic mode)
      std::vector<int> el;
      el.reserve(nspec);
      c->col_off[0] = 0;
      for (int col = 0; col < 8; ++col) {
        for (int ez = col >> 2 & 1; ez < d->nz; ez += 2)
          for (int ey = col >> 1 & 1; ey < d->ny; ey += 2)
            for (int ex = col & 1; ex < d->nx; ex += 2) el.push_back((ez * d->ny + ey) * d->nx + ex);
        c->col_off[col + 1] = static_cast<int>(el.size());
      }
      c->elist.upload(el, tot);
      c->bpoint.upload(bpoint, tot);
      c->bindex.upload(bidx, tot);
      c->priv.upload(priv, tot);
    }
    // state
    const size_t nf = c->field_n();
    const size_t nseis = std::max<size_t>(1, static_cast<size_t>(c->nstep) * c->nrec * 3 * c->S);
    c->fwd.alloc(nf, tot);
    c->minv.alloc(static_cast<size_t>(c->nglob) * 3, tot);
    c->seis_f.alloc(nseis, tot);
    c->scratch.alloc(std::max<size_t>(static_cast<size_t>(c->nglob) * 3, static_cast<size_t>(c->nstep) * c->nrec * 3),
                     tot);
    // mass
    {
      Buf<double> mass;
      size_t tmp = 0;
      mass.alloc(c->nglob, &tmp);
      if (c->det) {
        // colour by colour: each point's terms added in the same order
        Dev3 dd = c->dev();
        dd.elist = c->elist.p;
        for (int col = 0; col < 8; ++col) {
          const int n = c->col_off[col + 1] - c->col_off[col];
          if (n == 0) continue;
          dd.elist_off = c->col_off[col];
          k3_mass<<<grid_of(static_cast<size_t>(n) * NNN, 256), 256, 0, c->stream>>>(dd, mass.p, n);
          ++c->launches;
        }
      } else {
        k3_mass<<<grid_of(nloc, 256), 256, 0, c->stream>>>(c->dev(), mass.p, nspec);
        ++c->launches;
      }
      k3_invert<<<grid_of(static_cast<size_t>(c->nglob) * 3, 256), 256, 0, c->stream>>>(
          mass.p, c->bindex.p, c->bdiag.p, static_cast<float>(c->dt), c->minv.p, c->nglob);
      ++c->launches;
      ck3(cudaGetLastError(), "mass");
      ck3(cudaStreamSynchronize(c->stream), "mass");
    }
    c->seg_len = c->nstep;
    c->nseg = 1;
    if (c->save) {
      c->adj.alloc(nf, tot);
      c->bwd.alloc(nf, tot);
      c->kern.alloc(nloc * 3, tot);
      c->seis_b.alloc(nseis, tot);
      c->adj_stf.alloc(nseis, tot);
      // Stacey store: the whole run when it fits, else segments with
      // checkpoints (device when they fit beside the store, else host)
      const size_t sps = static_cast<size_t>(c->nb) * 3 * c->S * sizeof(float);
      const size_t ck = 3 * nf * sizeof(float);
      size_t freeb = 0, totalb = 0;
      ck3(cudaMemGetInfo(&freeb, &totalb), "memory info");
      const size_t margin = std::max<size_t>(size_t(2) << 30, totalb / 20);
      const size_t budget = freeb > margin ? freeb - margin : 0;
      int len = c->nstep;
      bool host = d->host_checkpoints != 0;
      if (d->segment_steps > 0) {
        len = std::min(d->segment_steps, c->nstep);
      } else if (sps && static_cast<double>(sps) * c->nstep > static_cast<double>(budget)) {
        len = 0;
        if (!host)
          for (int nseg = 2; nseg <= c->nstep; ++nseg) {
            const int l = (c->nstep + nseg - 1) / nseg;
            if (static_cast<double>(nseg) * ck + static_cast<double>(l) * sps <= static_cast<double>(budget)) {
              len = l;
              break;
            }
          }
        if (len == 0) {
          host = true;
          len = static_cast<int>(std::min<size_t>(c->nstep, budget / sps));
          if (len < 1) throw NoMemError("not enough device memory for one step of Stacey tractions");
        }
      }
      c->seg_len = std::max(1, len);
      c->nseg = (c->nstep + c->seg_len - 1) / c->seg_len;
      if (c->nb) c->store.alloc(static_cast<size_t>(c->seg_len) * (sps / sizeof(float)), tot);
      if (c->nseg > 1) {
        const size_t nck = static_cast<size_t>(c->nseg) * 3 * nf;
        if (!host && static_cast<double>(nck) * sizeof(float) >
                         static_cast<double>(budget) - static_cast<double>(c->store.n) * sizeof(float))
          host = true;
        c->ckpt_host = host;
        if (host) {
          // pinned when the host allows it, else pageable (staged copies);
          // never more than half of the host memory still available
          const double avail = static_cast<double>(sysconf(_SC_AVPHYS_PAGES)) * sysconf(_SC_PAGESIZE);
          if (static_cast<double>(nck) * sizeof(float) > 0.5 * avail)
            throw NoMemError("the checkpoints (" + std::to_string(nck * sizeof(float) >> 20) +
                                     " MiB) need more host memory than is available");
          if (cudaHostAlloc(reinterpret_cast<void **>(&c->ckpt_host_p), nck * sizeof(float), cudaHostAllocDefault) !=
              cudaSuccess) {
            cudaGetLastError();
            c->ckpt_host_p = nullptr;
            c->ckpt_pageable = static_cast<float *>(std::malloc(nck * sizeof(float)));
            if (!c->ckpt_pageable) throw NoMemError("host allocation of the checkpoints failed");
          }
          c->host_bytes = nck * sizeof(float);
        } else {
          c->ckpt_dev.alloc(nck, tot);
        }
      }
    }
    ck3(cudaDeviceSynchronize(), "setup");
    *out = c.release();
    return SFB_OK;
  });
}

SFB_API void sfb3_destroy(sfb3_context *ctx) { delete ctx; }

SFB_API int sfb3_get_info(const sfb3_context *c, sfb3_info *info) {
  if (!c || !info) return SFB_E_INVALID;
  *info = sfb3_info{};
  info->nspec = c->nspec;
  info->nglob = c->nglob;
  info->nshots = c->S;
  info->nstep = c->nstep;
  info->nreceivers = c->nrec;
  info->nboundary_points = c->nb;
  info->segment_steps = c->seg_len;
  info->nsegments = c->nseg;
  info->checkpoints_on_host = c->ckpt_host ? 1 : 0;
  info->dt = c->dt;
  info->t0 = c->t0;
  info->device_bytes = c->bytes;
  info->host_bytes = c->host_bytes;
  info->kernel_launches = c->launches;
  return SFB_OK;
}

SFB_API int sfb3_run_forward(sfb3_context *c, int nstep) {
  if (!c) return SFB_E_INVALID;
  return guarded3(c, [&]() {
    if (nstep < 0 || c->step + nstep > c->nstep) throw std::invalid_argument("the run would pass the configured steps");
    if (!c->fwd_final) throw std::invalid_argument("the forward fields were recomputed: reset first");
    run_forward_impl(c, nstep);
    ck3(cudaGetLastError(), "forward");
    ck3(cudaStreamSynchronize(c->stream), "forward");
    return SFB_OK;
  });
}

SFB_API int sfb3_get_seismograms(sfb3_context *c, int wavefield, int shot, float *host, size_t count) {
  if (!c || !host) return SFB_E_INVALID;
  return guarded3(c, [&]() {
    const size_t per = static_cast<size_t>(c->nstep) * c->nrec * 3;
    if (shot < 0 || shot >= c->S || count < per || (wavefield != 0 && wavefield != 2))
      throw std::invalid_argument("bad wavefield, shot or buffer size");
    const Buf<float> &b = wavefield == 2 ? c->seis_b : c->seis_f;
    if (!b.p) throw std::invalid_argument("no backward seismograms: the context keeps no adjoint state");
    if (per == 0) return SFB_OK;
    k3_gather<<<grid_of(per, 256), 256, 0, c->stream>>>(b.p, c->scratch.p, per, c->S, shot);
    ++c->launches;
    ck3(cudaMemcpyAsync(host, c->scratch.p, per * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "d2h");
    ck3(cudaStreamSynchronize(c->stream), "d2h");
    return SFB_OK;
  });
}

SFB_API int sfb3_get_field(sfb3_context *c, int wavefield, int which, int shot, float *host, size_t count) {
  if (!c || !host) return SFB_E_INVALID;
  return guarded3(c, [&]() {
    const size_t n = static_cast<size_t>(c->nglob);
    if (which < 0 || which > 3 || wavefield < 0 || wavefield > 2 || shot < 0 || shot >= c->S || count < 3 * n)
      throw std::invalid_argument("bad selector or buffer size");
    std::vector<float> tmp(3 * n);
    if (which == 3) {
      ck3(cudaMemcpyAsync(tmp.data(), c->minv.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "d2h");
    } else {
      const Wave &w = wavefield == 0 ? c->fwd : wavefield == 1 ? c->adj : c->bwd;
      if (!w.ready()) throw std::invalid_argument("the context keeps no such wavefield");
      const float *src = which == 0 ? w.u.p : which == 1 ? w.v.p : w.a.p;
      k3_gather<<<grid_of(3 * n, 256), 256, 0, c->stream>>>(src, c->scratch.p, 3 * n, c->S, shot);
      ++c->launches;
      ck3(cudaMemcpyAsync(tmp.data(), c->scratch.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "d2h");
    }
    ck3(cudaStreamSynchronize(c->stream), "d2h");
    for (size_t g = 0; g < n; ++g)  // lattice order
      for (int cc = 0; cc < 3; ++cc) host[cc * n + g] = tmp[static_cast<size_t>(c->perm[g]) * 3 + cc];
    return SFB_OK;
  });
}

SFB_API int sfb3_set_adjoint_sources(sfb3_context *c, int shot, const float *host, size_t count) {
  if (!c || !host) return SFB_E_INVALID;
  return guarded3(c, [&]() {
    const size_t per = static_cast<size_t>(c->nstep) * c->nrec * 3;
    if (shot < 0 || shot >= c->S || count < per) throw std::invalid_argument("bad shot or buffer size");
    if (!c->adj_stf.p) throw std::invalid_argument("the context keeps no adjoint state (save_boundary_values)");
    if (per == 0) return SFB_OK;
    ck3(cudaMemcpyAsync(c->scratch.p, host, per * sizeof(float), cudaMemcpyHostToDevice, c->stream), "h2d");
    k3_scatter<<<grid_of(per, 256), 256, 0, c->stream>>>(c->scratch.p, c->adj_stf.p, per, c->S, shot);
    ++c->launches;
    ck3(cudaStreamSynchronize(c->stream), "h2d");
    return SFB_OK;
  });
}

SFB_API int sfb3_run_combined(sfb3_context *c) {
  if (!c) return SFB_E_INVALID;
  return guarded3(c, [&]() {
    run_combined_impl(c);
    ck3(cudaGetLastError(), "combined");
    ck3(cudaStreamSynchronize(c->stream), "combined");
    return SFB_OK;
  });
}

SFB_API int sfb3_get_kernels(sfb3_context *c, int which, double *host, size_t count) {
  if (!c || !host) return SFB_E_INVALID;
  return guarded3(c, [&]() {
    const size_t nloc = static_cast<size_t>(c->nspec) * NNN;
    if (which < 0 || which > 2 || count < nloc) throw std::invalid_argument("bad selector or buffer size");
    if (!c->kern.p) throw std::invalid_argument("the context keeps no kernels (save_boundary_values)");
    std::vector<double> k(nloc * 3);
    ck3(cudaMemcpyAsync(k.data(), c->kern.p, k.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h");
    ck3(cudaStreamSynchronize(c->stream), "d2h");
    for (size_t p = 0; p < nloc; ++p) host[p] = k[p * 3 + which];
    return SFB_OK;
  });
}

SFB_API int sfb3_reset(sfb3_context *c) {
  if (!c) return SFB_E_INVALID;
  return guarded3(c, [&]() {
    for (Wave *w : {&c->fwd, &c->adj, &c->bwd}) zero_wave(c, *w);
    for (Buf<float> *b : {&c->seis_f, &c->seis_b})
      if (b->p) ck3(cudaMemsetAsync(b->p, 0, b->n * sizeof(float), c->stream), "zero");
    if (c->kern.p) ck3(cudaMemsetAsync(c->kern.p, 0, c->kern.n * sizeof(double), c->stream), "zero");
    ck3(cudaStreamSynchronize(c->stream), "zero");
    c->step = 0;
    c->fwd_final = true;
    return SFB_OK;
  });
}

SFB_API int sfb3_set_variant(sfb3_context *c, int variant) {
  if (!c || variant < 0 || variant > 3) return SFB_E_INVALID;
  c->variant = variant;
  return SFB_OK;
}

SFB_API int sfb3_get_variant(const sfb3_context *c) { return c ? variant_of(c) : SFB_E_INVALID; }

SFB_API int sfb3_time_kernel(sfb3_context *c, int what, int reps, double *mean_ms) {
  if (!c || !mean_ms || reps < 1 || what < 0 || what > 5) return SFB_E_INVALID;
  return guarded3(c, [&]() {
    if (what == 5) {
      // the whole combined run, timed on the context's stream: mean per step
      if (!c->save || c->step != c->nstep) throw std::invalid_argument("run the whole forward simulation first");
      cudaEvent_t e0, e1;
      ck3(cudaEventCreate(&e0), "event");
      ck3(cudaEventCreate(&e1), "event");
      ck3(cudaEventRecord(e0, c->stream), "event");
      run_combined_impl(c);
      ck3(cudaEventRecord(e1, c->stream), "event");
      ck3(cudaEventSynchronize(e1), "event");
      float ms = 0.f;
      ck3(cudaEventElapsedTime(&ms, e0, e1), "event");
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      ck3(cudaGetLastError(), "timing");
      *mean_ms = ms / c->nstep;
      return SFB_OK;
    }
    if (what == 3 && (c->step + reps > c->nstep || !c->fwd_final))
      throw std::invalid_argument("the timed steps would pass the configured steps");
    if ((what == 2 || what == 4) && !c->kern.p)
      throw std::invalid_argument("the context keeps no kernels (save_boundary_values)");
    if (what == 4 && variant_of(c) == 1) throw std::invalid_argument("the fused launch needs the packed kernels");
    if (what != 3) {
      ensure_scratch(c);
      copy_wave(c, c->adj, c->fwd);
    }
    cudaEvent_t e0, e1;
    ck3(cudaEventCreate(&e0), "event");
    ck3(cudaEventCreate(&e1), "event");
    ck3(cudaEventRecord(e0, c->stream), "event");
    if (what == 3) {
      run_forward_impl(c, reps);
    } else {
      for (int r = 0; r < reps; ++r) {
        if (what == 0) launch_stiffness(c, c->adj.u.p, c->adj.a.p);
        else if (what == 1) newmark(c, c->adj, c->dt, 2);
        else if (what == 2) frechet(c, c->adj.u.p, c->adj.a.p, c->fwd.u.p);
        else launch_stiffness_frechet(c, c->adj.u.p, c->adj.a.p, c->fwd.u.p, c->fwd.a.p);
      }
    }
    ck3(cudaEventRecord(e1, c->stream), "event");
    ck3(cudaEventSynchronize(e1), "event");
    float ms = 0.f;
    ck3(cudaEventElapsedTime(&ms, e0, e1), "event");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *mean_ms = ms / reps;
    if (what == 2 || what == 4) ck3(cudaMemsetAsync(c->kern.p, 0, c->kern.n * sizeof(double), c->stream), "zero");
    if (what != 3) zero_wave(c, c->adj);
    ck3(cudaGetLastError(), "timing");
    ck3(cudaStreamSynchronize(c->stream), "timing");
    return SFB_OK;
  });
}

}  // extern "C"
