// ORACLE -- test infrastructure only.  A CPU restatement of the 3D elastic
// time-marching path (include/specfem_b200_3d.h), used by the tests as the
// checker.  It is never linked into, loaded by or called from the product
// library.
//
// It builds its own mesh, numbering, quadrature, Lagrange interpolants,
// source and receiver arrays from the same sfb3_desc, so it shares no setup
// code with the product.  The reference has no 3D solver; the restatement
// follows its 2D weak form with a third dimension:
//   time loop        include/solver/time_marching.tpp:9-124 (forward),
//                    :126-247 (combined)
//   Newmark          include/timescheme/newmark.tpp:11-117, 181-242
//   gradient         include/algorithms/gradient.hpp:36-111
//   divergence       include/algorithms/divergence.hpp:40-103
//   stress           include/medium/dim2/elastic/isotropic/stress.hpp:14-85
//   F = J T d(xi)/dx core/specfem/point/stress.hpp:117-139
//   Stacey           include/boundary_conditions/stacey/stacey.tpp:41-75,
//                    625-677, evaluated per absorbing element face point
//                    with the face's outward normal; the forward run keeps
//                    each face point's traction and the backward run
//                    replays it (the reference keeps element-local
//                    accelerations of its Stacey elements)
//   mass matrix      include/kokkos_kernels/impl/compute_mass_matrix.tpp:80-113
//   sources          src/source/moment_tensor_source.cpp:125-135 (array),
//                    io/sources.cpp:128-158 (t0, time shifts), Ricker
//   seismograms      include/kokkos_kernels/impl/compute_seismogram.tpp:98-135
//   Frechet kernels  include/medium/dim2/elastic/isotropic/frechet_derivative.hpp:14-138
//                    with the 3D strain and deviatoric part
// Templated on the arithmetic type: float restates the FP32 build, double
// gives the FP64 oracle of the same discrete problem.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/specfem_b200_3d.h"

namespace {

constexpr int N = 5, NNN = 125;

// Gauss-Lobatto-Legendre points and weights for 5 points (exact values:
// 0, +-sqrt(3/7), +-1; 32/45, 49/90, 1/10).
struct Gll {
  double x[N], w[N], hp[N][N];  // hp[i][j] = l_j'(x_i)
  Gll() {
    const double a = std::sqrt(3.0 / 7.0);
    const double xs[N] = {-1.0, -a, 0.0, a, 1.0}, ws[N] = {0.1, 49.0 / 90.0, 32.0 / 45.0, 49.0 / 90.0, 0.1};
    for (int i = 0; i < N; ++i) {
      x[i] = xs[i];
      w[i] = ws[i];
    }
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        double h, d;
        lagrange(j, x[i], h, d);
        hp[i][j] = d;
      }
  }
  // l_j(t) and l_j'(t) from the product formula.
  void lagrange(int j, double t, double &h, double &d) const {
    h = 1.0;
    d = 0.0;
    for (int m = 0; m < N; ++m) {
      if (m == j) continue;
      double term = 1.0 / (x[j] - x[m]);
      for (int k = 0; k < N; ++k)
        if (k != j && k != m) term *= (t - x[k]) / (x[j] - x[k]);
      d += term;
      h *= (t - x[m]) / (x[j] - x[m]);
    }
  }
};

template <typename T> struct Sim3 {
  const sfb3_desc &D;
  Gll q;
  int nx, ny, nz, nspec, gx, gy, gz, nglob;
  double dx, dy, dz;
  T xix, etay, gaz, jac;
  T w[N], hp[N][N], hpw[N][N];
  std::vector<int> iglob;
  std::vector<T> kappa, mu, rho;
  std::vector<T> u, v, a, minv;  // [3][nglob]
  std::vector<T> floc;           // [nspec][125][3]
  T dt, dt2, dtsq2;
  int threads = 1;
  bool backward = false;
  // Stacey face entries: (element, face) -> first entry, 25 per face
  std::vector<int> fbase;        // [nspec][6]
  int nentries = 0;
  const double *replay = nullptr;  // [nstep][nentries][3]
  double *keep = nullptr;
  // point sources of the run
  std::vector<int> selem;
  std::vector<std::vector<T>> sarr;    // [3][125]
  std::vector<std::vector<T>> sstf;    // [nstep]
  // receivers
  std::vector<int> relem;
  std::vector<std::vector<T>> rlag;    // [125]
  const double *adj_stf = nullptr;     // [nstep][nrec][3]

  Sim3(const sfb3_desc &d, int shot) : D(d) {
    nx = d.nx;
    ny = d.ny;
    nz = d.nz;
    nspec = nx * ny * nz;
    gx = 4 * nx + 1;
    gy = 4 * ny + 1;
    gz = 4 * nz + 1;
    nglob = gx * gy * gz;
    dx = (d.x1 - d.x0) / nx;
    dy = (d.y1 - d.y0) / ny;
    dz = (d.z1 - d.z0) / nz;
    xix = static_cast<T>(2.0 / dx);
    etay = static_cast<T>(2.0 / dy);
    gaz = static_cast<T>(2.0 / dz);
    jac = static_cast<T>(dx * dy * dz / 8.0);
    for (int i = 0; i < N; ++i) {
      w[i] = static_cast<T>(q.w[i]);
      for (int j = 0; j < N; ++j) hp[i][j] = static_cast<T>(q.hp[i][j]);
    }
    for (int i = 0; i < N; ++i)
      for (int l = 0; l < N; ++l) hpw[i][l] = hp[l][i] * w[l];
    dt = static_cast<T>(d.dt);
    dt2 = static_cast<T>(d.dt / 2.0);
    dtsq2 = static_cast<T>(d.dt * d.dt / 2.0);
    const size_t nloc = static_cast<size_t>(nspec) * NNN;
    iglob.resize(nloc);
    kappa.resize(nloc);
    mu.resize(nloc);
    rho.resize(nloc);
    fbase.assign(static_cast<size_t>(nspec) * 6, -1);
    for (int ez = 0; ez < nz; ++ez)
      for (int ey = 0; ey < ny; ++ey)
        for (int ex = 0; ex < nx; ++ex) {
          const int e = (ez * ny + ey) * nx + ex;
          for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
              for (int i = 0; i < N; ++i) {
                const size_t p = P(e, k, j, i);
                iglob[p] = ((4 * ez + k) * gy + (4 * ey + j)) * gx + (4 * ex + i);
                const T r = static_cast<T>(d.rho[p]), vp = static_cast<T>(d.vp[p]), vs = static_cast<T>(d.vs[p]);
                rho[p] = r;
                mu[p] = r * vs * vs;
                kappa[p] = r * (vp * vp - static_cast<T>(static_cast<float>(4.0 / 3.0)) * vs * vs);
              }
          const bool on[6] = {ex == 0, ex == nx - 1, ey == 0, ey == ny - 1, ez == 0, ez == nz - 1};
          for (int f = 0; f < 6; ++f)
            if (on[f] && ((d.absorb >> f) & 1)) {
              fbase[static_cast<size_t>(e) * 6 + f] = nentries;
              nentries += 25;
            }
        }
    u.assign(static_cast<size_t>(3) * nglob, T(0));
    v = u;
    a = u;
    minv = u;
    floc.assign(nloc * 3, T(0));
    // sources of this shot; t0 and time shifts over all sources
    double min_t0 = 1e300;
    for (int s = 0; s < d.nsources; ++s) min_t0 = std::min(min_t0, -1.2 / d.sources[s].f0 + d.sources[s].tshift);
    for (int s = 0; s < d.nsources; ++s) {
      const sfb3_source &S = d.sources[s];
      if (S.shot != shot) continue;
      int e;
      double r[3];
      locate(S.x, S.y, S.z, e, r);
      double h[3][N], hd[3][N];
      for (int ax = 0; ax < 3; ++ax)
        for (int j = 0; j < N; ++j) q.lagrange(j, r[ax], h[ax][j], hd[ax][j]);
      const double M[3][3] = {{S.mxx, S.mxy, S.mxz}, {S.mxy, S.myy, S.myz}, {S.mxz, S.myz, S.mzz}};
      std::vector<T> arr(3 * NNN);
      for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i) {
            const double g[3] = {hd[0][i] * (2.0 / dx) * h[1][j] * h[2][k], h[0][i] * hd[1][j] * (2.0 / dy) * h[2][k],
                                 h[0][i] * h[1][j] * hd[2][k] * (2.0 / dz)};
            for (int c = 0; c < 3; ++c)
              arr[c * NNN + (k * N + j) * N + i] = static_cast<T>(M[c][0] * g[0] + M[c][1] * g[1] + M[c][2] * g[2]);
          }
      // shifted Ricker: -factor (1 - 2 a t^2) exp(-a t^2), a = (pi f0)^2,
      // t measured from the source's own t0 - min t0
      const double tshift = (-1.2 / S.f0 + S.tshift) - min_t0;
      std::vector<T> stf(d.nstep);
      for (int t = 0; t < d.nstep; ++t) {
        const double tt = (min_t0 + t * d.dt) - tshift;
        const double aa = M_PI * M_PI * S.f0 * S.f0;
        stf[t] = static_cast<T>(-S.factor * (1.0 - 2.0 * aa * tt * tt) * std::exp(-aa * tt * tt));
      }
      selem.push_back(e);
      sarr.push_back(arr);
      sstf.push_back(stf);
    }
    for (int r = 0; r < d.nreceivers; ++r) {
      int e;
      double rr[3];
      locate(d.receivers[3 * r], d.receivers[3 * r + 1], d.receivers[3 * r + 2], e, rr);
      double h[3][N], hd[3][N];
      for (int ax = 0; ax < 3; ++ax)
        for (int j = 0; j < N; ++j) q.lagrange(j, rr[ax], h[ax][j], hd[ax][j]);
      std::vector<T> lag(NNN);
      for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i) lag[(k * N + j) * N + i] = static_cast<T>(h[0][i] * h[1][j] * h[2][k]);
      relem.push_back(e);
      rlag.push_back(lag);
    }
  }

  size_t P(int e, int k, int j, int i) const { return static_cast<size_t>(e) * NNN + (k * N + j) * N + i; }
  size_t F(int c, int g) const { return static_cast<size_t>(c) * nglob + g; }

  void locate(double x, double y, double z, int &e, double r[3]) const {
    const double vv[3] = {x, y, z}, o[3] = {D.x0, D.y0, D.z0}, h[3] = {dx, dy, dz};
    const int n[3] = {nx, ny, nz};
    int ie[3];
    for (int ax = 0; ax < 3; ++ax) {
      ie[ax] = static_cast<int>(std::floor((vv[ax] - o[ax]) / h[ax]));
      ie[ax] = std::min(std::max(ie[ax], 0), n[ax] - 1);
      r[ax] = 2.0 * (vv[ax] - (o[ax] + ie[ax] * h[ax])) / h[ax] - 1.0;
    }
    e = (ie[2] * ny + ie[1]) * nx + ie[0];
  }

  // face f of element e: local point of face slot (b0, b1), outward normal,
  // face Jacobian
  void face_point(int f, int b0, int b1, int &k, int &j, int &i) const {
    const int fixed = (f & 1) ? N - 1 : 0;
    if (f < 2) { i = fixed; j = b0; k = b1; }
    else if (f < 4) { j = fixed; i = b0; k = b1; }
    else { k = fixed; i = b0; j = b1; }
  }
  T face_jac(int f) const {
    if (f < 2) return static_cast<T>(dy * dz / 4.0);
    if (f < 4) return static_cast<T>(dx * dz / 4.0);
    return static_cast<T>(dx * dy / 4.0);
  }
  // stacey.tpp:41-75 with a 3D normal
  void stacey(size_t p, int f, T wgt, const T *vel, T *out) const {
    T n[3] = {T(0), T(0), T(0)};
    n[f / 2] = (f & 1) ? T(1) : T(-1);
    const T l2m = kappa[p] + static_cast<T>(static_cast<float>(4.0 / 3.0)) * mu[p];
    const T rho_vp = std::sqrt(l2m / rho[p]) * rho[p];
    const T rho_vs = std::sqrt(rho[p] * mu[p]);
    const T vn = vel[0] * n[0] + vel[1] * n[1] + vel[2] * n[2];
    for (int c = 0; c < 3; ++c) {
      const T fac = (vn * n[c]) * (rho_vp - rho_vs) + vel[c] * rho_vs;
      out[c] += T(-1) * fac * wgt;
    }
  }

  void init_mass() {
    std::vector<T> mass(static_cast<size_t>(3) * nglob, T(0));
    for (int e = 0; e < nspec; ++e)
      for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i) {
            const size_t p = P(e, k, j, i);
            const T m = rho[p] * (w[i] * w[j] * w[k] * jac);
            for (int c = 0; c < 3; ++c) mass[F(c, iglob[p])] += m;
          }
    for (int e = 0; e < nspec; ++e)
      for (int f = 0; f < 6; ++f) {
        if (fbase[static_cast<size_t>(e) * 6 + f] < 0) continue;
        for (int b1 = 0; b1 < N; ++b1)
          for (int b0 = 0; b0 < N; ++b0) {
            int k, j, i;
            face_point(f, b0, b1, k, j, i);
            const size_t p = P(e, k, j, i);
            const T vf[3] = {T(-1) * dt * T(0.5), T(-1) * dt * T(0.5), T(-1) * dt * T(0.5)};
            T mm[3] = {T(0), T(0), T(0)};
            stacey(p, f, w[b0] * w[b1] * face_jac(f), vf, mm);
            for (int c = 0; c < 3; ++c) mass[F(c, iglob[p])] += mm[c];
          }
      }
    for (size_t t = 0; t < mass.size(); ++t) minv[t] = T(1) / mass[t];
  }

  void predictor(T sgn) {
    const T d = sgn * dt, d2 = sgn * dt2;
    for (size_t t = 0; t < u.size(); ++t) {
      u[t] += d * v[t] + dtsq2 * a[t];
      v[t] += d2 * a[t];
      a[t] = T(0);
    }
  }
  void corrector(T sgn) {
    const T d2 = sgn * dt2;
    for (size_t t = 0; t < u.size(); ++t) {
      a[t] = a[t] * minv[t];
      v[t] += d2 * a[t];
    }
  }

  // Element-local stiffness (+ Stacey faces) into floc, then assembly.
  void stiffness(int istep) {
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int e = 0; e < nspec; ++e) {
      T ue[N][N][N][3], fxi[N][N][N][3], feta[N][N][N][3], fzeta[N][N][N][3];
      for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i)
            for (int c = 0; c < 3; ++c) ue[k][j][i][c] = u[F(c, iglob[P(e, k, j, i)])];
      for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i) {
            T du[3][3];
            for (int c = 0; c < 3; ++c) {
              T d1 = T(0), d2 = T(0), d3 = T(0);
              for (int l = 0; l < N; ++l) {
                d1 += hp[i][l] * ue[k][j][l][c];
                d2 += hp[j][l] * ue[k][l][i][c];
                d3 += hp[k][l] * ue[l][j][i][c];
              }
              du[c][0] = xix * d1;
              du[c][1] = etay * d2;
              du[c][2] = gaz * d3;
            }
            const size_t p = P(e, k, j, i);
            const T l2m = kappa[p] + static_cast<T>(static_cast<float>(4.0 / 3.0)) * mu[p];
            const T lam = l2m - T(2) * mu[p];
            T s[3][3];
            s[0][0] = l2m * du[0][0] + lam * (du[1][1] + du[2][2]);
            s[1][1] = l2m * du[1][1] + lam * (du[0][0] + du[2][2]);
            s[2][2] = l2m * du[2][2] + lam * (du[0][0] + du[1][1]);
            s[0][1] = s[1][0] = mu[p] * (du[0][1] + du[1][0]);
            s[0][2] = s[2][0] = mu[p] * (du[0][2] + du[2][0]);
            s[1][2] = s[2][1] = mu[p] * (du[1][2] + du[2][1]);
            for (int c = 0; c < 3; ++c) {
              fxi[k][j][i][c] = jac * (s[c][0] * xix);
              feta[k][j][i][c] = jac * (s[c][1] * etay);
              fzeta[k][j][i][c] = jac * (s[c][2] * gaz);
            }
          }
      for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i)
            for (int c = 0; c < 3; ++c) {
              T t1 = T(0), t2 = T(0), t3 = T(0);
              for (int l = 0; l < N; ++l) {
                t1 += fxi[k][j][l][c] * hpw[i][l];
                t2 += feta[k][l][i][c] * hpw[j][l];
                t3 += fzeta[l][j][i][c] * hpw[k][l];
              }
              floc[P(e, k, j, i) * 3 + c] =
                  (w[j] * w[k] * t1 + w[i] * w[k] * t2 + w[i] * w[j] * t3) * T(-1);
            }
      for (int f = 0; f < 6; ++f) {
        const int base = fbase[static_cast<size_t>(e) * 6 + f];
        if (base < 0) continue;
        for (int b1 = 0; b1 < N; ++b1)
          for (int b0 = 0; b0 < N; ++b0) {
            int k, j, i;
            face_point(f, b0, b1, k, j, i);
            const size_t p = P(e, k, j, i);
            const size_t entry = static_cast<size_t>(base) + b1 * N + b0;
            const size_t at = (static_cast<size_t>(istep) * nentries + entry) * 3;
            T tr[3] = {T(0), T(0), T(0)};
            if (backward && replay) {
              for (int c = 0; c < 3; ++c) tr[c] = static_cast<T>(replay[at + c]);
            } else {
              const int g = iglob[p];
              const T vel[3] = {v[F(0, g)], v[F(1, g)], v[F(2, g)]};
              stacey(p, f, w[b0] * w[b1] * face_jac(f), vel, tr);
              if (keep)
                for (int c = 0; c < 3; ++c) keep[at + c] = static_cast<double>(tr[c]);
            }
            for (int c = 0; c < 3; ++c) floc[p * 3 + c] += tr[c];
          }
      }
    }
    for (size_t p = 0; p < iglob.size(); ++p)
      for (int c = 0; c < 3; ++c) a[F(c, iglob[p])] += floc[p * 3 + c];
  }

  void sources(int istep) {
    for (size_t s = 0; s < selem.size(); ++s)
      for (int qq = 0; qq < NNN; ++qq)
        for (int c = 0; c < 3; ++c)
          a[F(c, iglob[static_cast<size_t>(selem[s]) * NNN + qq])] += sstf[s][istep] * sarr[s][c * NNN + qq];
  }
  void adjoint_sources(int istep) {
    const int nrec = static_cast<int>(relem.size());
    for (int r = 0; r < nrec; ++r)
      for (int qq = 0; qq < NNN; ++qq)
        for (int c = 0; c < 3; ++c) {
          const T f = static_cast<T>(adj_stf[(static_cast<size_t>(istep) * nrec + r) * 3 + c]);
          a[F(c, iglob[static_cast<size_t>(relem[r]) * NNN + qq])] += f * rlag[r][qq];
        }
  }
  void seismograms(double *out) const {
    for (size_t r = 0; r < relem.size(); ++r)
      for (int c = 0; c < 3; ++c) {
        T acc = T(0);
        for (int qq = 0; qq < NNN; ++qq) acc += rlag[r][qq] * u[F(c, iglob[static_cast<size_t>(relem[r]) * NNN + qq])];
        out[r * 3 + c] = static_cast<double>(acc);
      }
  }

  // frechet_derivative.hpp:14-138 with the 3D strain, added to k[p][3]
  static void frechet(const Sim3 &adj, const Sim3 &bwd, double *k, int threads) {
    const int nspec = adj.nspec;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int e = 0; e < nspec; ++e)
      for (int kk = 0; kk < N; ++kk)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i) {
            const size_t p = adj.P(e, kk, j, i);
            T d[2][3][3];
            for (int wv = 0; wv < 2; ++wv) {
              const Sim3 &S = wv == 0 ? adj : bwd;
              for (int c = 0; c < 3; ++c) {
                T d1 = T(0), d2 = T(0), d3 = T(0);
                for (int l = 0; l < N; ++l) {
                  d1 += adj.hp[i][l] * S.u[S.F(c, S.iglob[adj.P(e, kk, j, l)])];
                  d2 += adj.hp[j][l] * S.u[S.F(c, S.iglob[adj.P(e, kk, l, i)])];
                  d3 += adj.hp[kk][l] * S.u[S.F(c, S.iglob[adj.P(e, l, j, i)])];
                }
                d[wv][c][0] = adj.xix * d1;
                d[wv][c][1] = adj.etay * d2;
                d[wv][c][2] = adj.gaz * d3;
              }
            }
            const T diva = d[0][0][0] + d[0][1][1] + d[0][2][2], divb = d[1][0][0] + d[1][1][1] + d[1][2][2];
            T ee = T(0);
            for (int c = 0; c < 3; ++c)
              for (int x = 0; x < 3; ++x)
                ee += (T(0.5) * (d[0][c][x] + d[0][x][c])) * (T(0.5) * (d[1][c][x] + d[1][x][c]));
            T kappa_kl = diva * divb;
            T mu_kl = ee - static_cast<T>(static_cast<float>(1.0 / 3.0)) * kappa_kl;
            const int g = adj.iglob[p];
            T rho_kl = T(0);
            for (int c = 0; c < 3; ++c) rho_kl += adj.a[adj.F(c, g)] * bwd.u[bwd.F(c, g)];
            kappa_kl = T(-1) * adj.kappa[p] * adj.dt * kappa_kl;
            mu_kl = T(-2) * adj.mu[p] * adj.dt * mu_kl;
            rho_kl = T(-1) * adj.rho[p] * adj.dt * rho_kl;
            k[p * 3 + 0] += static_cast<double>(rho_kl);
            k[p * 3 + 1] += static_cast<double>(mu_kl);
            k[p * 3 + 2] += static_cast<double>(kappa_kl);
          }
  }
};

thread_local std::string g_err3;

template <typename T>
int forward3(const sfb3_desc *d, int shot, int threads, double *seis, double *final_fields, double *store) {
  Sim3<T> s(*d, shot);
  s.threads = threads;
  s.keep = store;
  s.init_mass();
  const int nrec = d->nreceivers;
  for (int istep = 0; istep < d->nstep; ++istep) {
    s.predictor(T(1));
    s.sources(istep);
    s.stiffness(istep);
    if (seis) s.seismograms(seis + static_cast<size_t>(istep) * nrec * 3);
    s.corrector(T(1));
  }
  if (final_fields) {
    const std::vector<T> *f[3] = {&s.u, &s.v, &s.a};
    for (int q = 0; q < 3; ++q)
      for (size_t t = 0; t < f[q]->size(); ++t) final_fields[q * f[q]->size() + t] = static_cast<double>((*f[q])[t]);
  }
  return 0;
}

template <typename T>
int combined3(const sfb3_desc *d, int shot, int threads, const double *adj_stf, const double *final_fields,
              const double *store, double *kernels, double *bseis) {
  Sim3<T> adj(*d, shot), bwd(*d, shot);
  adj.threads = bwd.threads = threads;
  adj.adj_stf = adj_stf;
  bwd.backward = true;
  bwd.replay = store;
  adj.init_mass();
  bwd.init_mass();
  const int nrec = d->nreceivers;
  int isig = 0;
  for (int istep = d->nstep - 1; istep >= 0; --istep) {
    adj.predictor(T(1));
    adj.adjoint_sources(istep);
    adj.stiffness(istep);
    adj.corrector(T(1));
    bwd.predictor(T(-1));
    bwd.sources(istep);
    bwd.stiffness(istep);
    bwd.corrector(T(-1));
    if (istep == d->nstep - 1) {
      std::vector<T> *f[3] = {&bwd.u, &bwd.v, &bwd.a};
      for (int q = 0; q < 3; ++q)
        for (size_t t = 0; t < f[q]->size(); ++t) (*f[q])[t] = static_cast<T>(final_fields[q * f[q]->size() + t]);
    }
    Sim3<T>::frechet(adj, bwd, kernels, threads);
    if (bseis) bwd.seismograms(bseis + static_cast<size_t>(isig) * nrec * 3);
    ++isig;
  }
  return 0;
}

}  // namespace

extern "C" {

const char *oracle3d_last_error() { return g_err3.c_str(); }

// Number of Stacey face entries (25 per absorbing element face).
int oracle3d_nentries(const sfb3_desc *d) {
  int n = 0;
  for (int ez = 0; ez < d->nz; ++ez)
    for (int ey = 0; ey < d->ny; ++ey)
      for (int ex = 0; ex < d->nx; ++ex) {
        const bool on[6] = {ex == 0, ex == d->nx - 1, ey == 0, ey == d->ny - 1, ez == 0, ez == d->nz - 1};
        for (int f = 0; f < 6; ++f)
          if (on[f] && ((d->absorb >> f) & 1)) n += 25;
      }
  return n;
}

// Forward run of one shot: seismograms [nstep][nrec][3], the final u, v, a
// ([3][3][nglob]) and, when `store` is given, the Stacey tractions
// [nstep][nentries][3].
int oracle3d_forward(const sfb3_desc *d, int shot, int precision, int threads, double *seis, double *final_fields,
                     double *store) {
  try {
    return precision == 64 ? forward3<double>(d, shot, threads, seis, final_fields, store)
                           : forward3<float>(d, shot, threads, seis, final_fields, store);
  } catch (const std::exception &e) {
    g_err3 = e.what();
    return -1;
  }
}

// Combined run of one shot: adjoint sources [nstep][nrec][3], the forward
// run's final fields and store; kernels [nspec*125][3] (rho, mu, kappa)
// are added to, backward seismograms [nstep][nrec][3] in loop order.
int oracle3d_combined(const sfb3_desc *d, int shot, int precision, int threads, const double *adj_stf,
                      const double *final_fields, const double *store, double *kernels, double *bseis) {
  try {
    return precision == 64 ? combined3<double>(d, shot, threads, adj_stf, final_fields, store, kernels, bseis)
                           : combined3<float>(d, shot, threads, adj_stf, final_fields, store, kernels, bseis);
  } catch (const std::exception &e) {
    g_err3 = e.what();
    return -1;
  }
}

}  // extern "C"
