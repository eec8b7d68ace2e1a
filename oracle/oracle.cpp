// ORACLE -- test infrastructure only.  A CPU restatement of SPECFEM++'s 2D
// time-marching path, used by the tests, the smoke check and the CPU
// baseline leg of bench.py as the checker.  It is never linked into, loaded
// by or called from the product library.
//
// It consumes the flat problem view the product exports
// (sfb_get_problem_view in include/specfem_b200.h) so that both sides start
// from identical discrete inputs, and restates, in the reference's step
// order and operation order:
//   time loop        include/solver/time_marching.tpp:9-124 (forward),
//                    :126-247 (combined)
//   Newmark          include/timescheme/newmark.tpp:11-117, 181-242
//   update_wavefields include/kokkos_kernels/domain_kernels.hpp:68-126
//   stiffness        include/kokkos_kernels/impl/compute_stiffness_interaction.tpp:140-260
//   gradient         include/algorithms/gradient.hpp:36-111
//   divergence       include/algorithms/divergence.hpp:40-103
//   stress           include/medium/dim2/elastic/isotropic/stress.hpp:14-85,
//                    include/medium/dim2/acoustic/isotropic/stress.hpp:15-31
//   F = J T d(xi)/dx core/specfem/point/stress.hpp:117-139
//   Stacey           include/boundary_conditions/stacey/stacey.tpp:41-250, 625-677
//   free surface     include/boundary_conditions/dirichlet/dirichlet.hpp:19-43
//   mass matrix      include/kokkos_kernels/impl/compute_mass_matrix.tpp:80-113,
//                    invert_mass_matrix.tpp:40-47, divide_mass_matrix.tpp:40-49
//   sources          include/kokkos_kernels/impl/compute_source_interaction.tpp:77-95
//   coupling         include/coupled_interface/coupled_interface.tpp:55-86,
//                    impl/compute_coupling.hpp:22-56
//   seismograms      include/kokkos_kernels/impl/compute_seismogram.tpp:98-135,
//                    include/medium/dim2/*/isotropic/wavefield.hpp,
//                    include/compute/receivers/receivers.hpp:126-141 (rotation)
//   Frechet kernels  include/kokkos_kernels/impl/compute_material_derivatives.tpp:84-153,
//                    include/medium/dim2/elastic/isotropic/frechet_derivative.hpp:14-196,
//                    include/medium/dim2/acoustic/isotropic/frechet_derivative.hpp:12-41
// Templated on the arithmetic type: float restates the reference's FP32
// build, double gives the FP64 oracle of the same discrete problem.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/specfem_b200.h"

namespace {

constexpr int ACOUSTIC = 3, PSV = 0, SH = 1;

template <typename T> struct Field {
  int nglob = 0, nc = 0;
  std::vector<T> u, v, a, minv;  // [nc][nglob]
  void init(int n, int c) {
    nglob = n;
    nc = c;
    u.assign(static_cast<size_t>(n) * c, T(0));
    v = u;
    a = u;
    minv = u;
  }
};

template <typename T> struct Sim {
  const sfb_problem_view &pv;
  int n, nspec, shot;
  T dt, dt2, dtsq2;
  Field<T> f[4];  // by medium tag
  std::vector<T> hp, hpw, w;  // hprime, hprime_wgll(ix,l)=hprime(l,ix)w(l), weights
  std::vector<std::vector<int>> elems;  // per medium
  bool store_stacey = false;
  int istep_store = 0;
  // [nstep][nloc][2] accelerations, FP32 as the reference's store, or in the
  // working precision for the FP64 oracle's exact outputs
  std::vector<float> *stacey_store = nullptr;
  std::vector<double> *stacey_store64 = nullptr;
  const std::vector<float> *stacey_replay = nullptr;
  const std::vector<double> *stacey_replay64 = nullptr;
  bool backward = false;
  int threads = 1;
  // Optional adjoint sources: [nstep][nrec][2] acting through receiver arrays.
  const float *adjoint_stf = nullptr;

  Sim(const sfb_problem_view &v, int s) : pv(v), n(v.ngll), nspec(v.nspec), shot(s) {
    dt = static_cast<T>(v.dt);
    dt2 = static_cast<T>(v.dt / 2.0);
    dtsq2 = static_cast<T>(v.dt * v.dt / 2.0);
    hp.resize(n * n);
    hpw.resize(n * n);
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = static_cast<T>(static_cast<float>(v.wgll[i]));
    for (int i = 0; i < n * n; ++i) hp[i] = static_cast<T>(static_cast<float>(v.hprime[i]));
    // element_quadrature.hprime_wgll(ix, iz) = hprime(iz, ix) * w(iz)
    // (include/compute/compute_mesh.hpp:265-277)
    for (int ix = 0; ix < n; ++ix)
      for (int l = 0; l < n; ++l) hpw[ix * n + l] = hp[l * n + ix] * w[l];
    elems.resize(4);
    for (int e = 0; e < nspec; ++e) elems[v.medium[e]].push_back(e);
    f[ACOUSTIC].init(v.nglob[ACOUSTIC], 1);
    f[PSV].init(v.nglob[PSV], 2);
    f[SH].init(v.nglob[SH], 1);
  }

  size_t P(int e, int iz, int ix) const { return (static_cast<size_t>(e) * n + iz) * n + ix; }

  // The element's boundary tag is stacey: Stacey points and no acoustic
  // free-surface point (enumerations/boundary.hpp:50-105 makes an element
  // with both composite_stacey_dirichlet).  Only these are stored by the
  // forward run and replayed by the backward run
  // (compute_stiffness_interaction.tpp:123-137, 251-255); composite
  // elements are computed in the backward run like any other.
  bool stacey_tagged(int e) const {
    const int nn = n * n;
    bool st = false, fs = false;
    for (int k = 0; k < nn; ++k) {
      st = st || (pv.bnd[static_cast<size_t>(e) * nn + k] & 1);
      fs = fs || (pv.bnd[static_cast<size_t>(e) * nn + k] & 2);
    }
    return st && !fs;
  }

  // ---- Newmark (newmark.tpp:60-117 predictor, :11-56 corrector) ---------
  void predictor(int m, T sgn) {
    Field<T> &F = f[m];
    const T d = sgn * dt, d2 = sgn * dt2, dsq = dtsq2;
    for (size_t i = 0; i < F.u.size(); ++i) {
      F.u[i] += d * F.v[i] + dsq * F.a[i];
      F.v[i] += d2 * F.a[i];
      F.a[i] = T(0);
    }
  }
  void corrector(int m, T sgn) {
    Field<T> &F = f[m];
    const T d2 = sgn * dt2;
    for (size_t i = 0; i < F.u.size(); ++i) F.v[i] += d2 * F.a[i];
  }

  // ---- mass matrix (compute_mass_matrix.tpp, stacey.tpp:644-677) --------
  void stacey_terms(int m, size_t p, const T *vel, T *out) const {
    const T nx = pv.bnd_nx[p], nz = pv.bnd_nz[p], we = pv.bnd_w[p];
    const T jac1d = std::sqrt(nx * nx + nz * nz);
    if (m == PSV) {
      const T kappa = pv.kappa[p], mu = pv.mu[p], rho = pv.rho[p];
      const T l2m = kappa + static_cast<T>(static_cast<float>(4.0 / 3.0)) * mu;
      const T rho_vp = std::sqrt(l2m / rho) * rho;
      const T rho_vs = std::sqrt(rho * mu);
      const T vn = vel[0] * nx + vel[1] * nz;
      const T dn[2] = {nx, nz};
      for (int c = 0; c < 2; ++c) {
        const T fac = ((vn * dn[c] / (jac1d * jac1d)) * (rho_vp - rho_vs)) + vel[c] * rho_vs;
        out[c] += T(-1) * fac * jac1d * we;
      }
    } else if (m == SH) {
      const T rho_vs = std::sqrt(static_cast<T>(pv.rho[p]) * static_cast<T>(pv.mu[p]));
      const T fac = we * jac1d;
      out[0] += T(-1) * fac * rho_vs * vel[0];
    } else {
      const T rvi = std::sqrt(static_cast<T>(pv.rho_inverse[p]) * (T(1) / static_cast<T>(pv.kappa[p])));
      const T fac = we * jac1d;
      out[0] += T(-1) * fac * rvi * vel[0];
    }
  }

  void init_mass() {
    for (int m : {ACOUSTIC, PSV, SH}) {
      Field<T> &F = f[m];
      std::vector<double> mass(F.minv.size(), 0.0);
      std::vector<T> massT(F.minv.size(), T(0));
      for (int e : elems[m])
        for (int iz = 0; iz < n; ++iz)
          for (int ix = 0; ix < n; ++ix) {
            const size_t p = P(e, iz, ix);
            T mm[2];
            const T base = (m == ACOUSTIC) ? T(1) / static_cast<T>(pv.kappa[p]) : static_cast<T>(pv.rho[p]);
            for (int c = 0; c < F.nc; ++c) mm[c] = base * (w[ix] * w[iz] * static_cast<T>(pv.jacobian[p]));
            if (pv.bnd[p] & 1) {
              const T vf[2] = {T(-1) * dt * T(0.5), T(-1) * dt * T(0.5)};
              stacey_terms(m, p, vf, mm);
            }
            const int g = pv.iglob[p];
            for (int c = 0; c < F.nc; ++c) massT[static_cast<size_t>(c) * F.nglob + g] += mm[c];
          }
      for (size_t i = 0; i < massT.size(); ++i) F.minv[i] = T(1) / massT[i];
    }
  }

  // ---- stiffness (compute_stiffness_interaction.tpp:140-260) ------------
  void stiffness(int m, int istep) {
    Field<T> &F = f[m];
    const int nc = F.nc;
    const std::vector<int> &E = elems[m];
    const int nn = n * n;
    if (backward && stacey_replay) {
      // Stacey elements replay the stored element-local acceleration
      // (:123-137); other elements are computed below.
    }
#pragma omp parallel for num_threads(threads) schedule(static)
    for (long ie = 0; ie < static_cast<long>(E.size()); ++ie) {
      const int e = E[ie];
      T u[8 * 8 * 2], Fs[8 * 8 * 2 * 2];
      bool replay = false;
      if (backward && (stacey_replay || stacey_replay64)) replay = stacey_tagged(e);
      if (replay) {
        for (int k = 0; k < nn; ++k) {
          const size_t p = static_cast<size_t>(e) * nn + k;
          const size_t at = (static_cast<size_t>(istep) * pv.nspec * nn + p) * 2;
          const int g = pv.iglob[p];
          for (int c = 0; c < nc; ++c) {
            T val = stacey_replay64 ? static_cast<T>((*stacey_replay64)[at + c])
                                    : static_cast<T>((*stacey_replay)[at + c]);
#pragma omp atomic
            F.a[static_cast<size_t>(c) * F.nglob + g] += val;
          }
        }
        continue;
      }
      for (int k = 0; k < nn; ++k) {
        const int g = pv.iglob[static_cast<size_t>(e) * nn + k];
        for (int c = 0; c < nc; ++c) u[k * nc + c] = F.u[static_cast<size_t>(c) * F.nglob + g];
      }
      // gradient + stress + stress integrand
      for (int iz = 0; iz < n; ++iz)
        for (int ix = 0; ix < n; ++ix) {
          const size_t p = P(e, iz, ix);
          T dxi[2] = {T(0), T(0)}, dga[2] = {T(0), T(0)};
          for (int l = 0; l < n; ++l)
            for (int c = 0; c < nc; ++c) {
              dxi[c] += hp[ix * n + l] * u[(iz * n + l) * nc + c];
              dga[c] += hp[iz * n + l] * u[(l * n + ix) * nc + c];
            }
          const T xix = pv.xix[p], xiz = pv.xiz[p], gax = pv.gammax[p], gaz = pv.gammaz[p];
          const T J = pv.jacobian[p];
          T du[2][2];
          for (int c = 0; c < nc; ++c) {
            du[c][0] = xix * dxi[c] + gax * dga[c];
            du[c][1] = xiz * dxi[c] + gaz * dga[c];
          }
          T Tm[2][2];
          if (m == PSV) {
            const T kappa = pv.kappa[p], mu = pv.mu[p];
            const T l2m = kappa + static_cast<T>(static_cast<float>(4.0 / 3.0)) * mu;
            const T lam = l2m - T(2) * mu;
            const T sxx = l2m * du[0][0] + lam * du[1][1];
            const T szz = l2m * du[1][1] + lam * du[0][0];
            const T sxz = mu * (du[0][1] + du[1][0]);
            Tm[0][0] = sxx;
            Tm[0][1] = sxz;
            Tm[1][0] = sxz;
            Tm[1][1] = szz;
          } else if (m == SH) {
            const T mu = pv.mu[p];
            Tm[0][0] = mu * du[0][0];
            Tm[0][1] = mu * du[0][1];
          } else {
            const T ri = pv.rho_inverse[p];
            Tm[0][0] = ri * du[0][0];
            Tm[0][1] = ri * du[0][1];
          }
          const int k = iz * n + ix;
          for (int c = 0; c < nc; ++c) {
            Fs[(k * nc + c) * 2 + 0] = J * (Tm[c][0] * xix + Tm[c][1] * xiz);
            Fs[(k * nc + c) * 2 + 1] = J * (Tm[c][0] * gax + Tm[c][1] * gaz);
          }
        }
      // divergence, sign, boundary conditions, scatter
      for (int iz = 0; iz < n; ++iz)
        for (int ix = 0; ix < n; ++ix) {
          const size_t p = P(e, iz, ix);
          T t1[2] = {T(0), T(0)}, t2[2] = {T(0), T(0)};
          for (int l = 0; l < n; ++l)
            for (int c = 0; c < nc; ++c) {
              t1[c] += Fs[((iz * n + l) * nc + c) * 2 + 0] * hpw[ix * n + l];
              t2[c] += Fs[((l * n + ix) * nc + c) * 2 + 1] * hpw[iz * n + l];
            }
          T acc[2];
          for (int c = 0; c < nc; ++c) acc[c] = (w[iz] * t1[c] + w[ix] * t2[c]) * T(-1);
          const uint8_t b = pv.bnd[p];
          const int g = pv.iglob[p];
          if (b & 1) {
            T vel[2];
            for (int c = 0; c < nc; ++c) vel[c] = F.v[static_cast<size_t>(c) * F.nglob + g];
            stacey_terms(m, p, vel, acc);
          }
          if (b & 2)
            for (int c = 0; c < nc; ++c) acc[c] = T(0);
          if (store_stacey && (stacey_store || stacey_store64)) {
            // Forward runs keep the element-local acceleration of every
            // point of a Stacey element (compute_stiffness_interaction.tpp:251-255).
            if (stacey_tagged(e)) {
              const size_t at = (static_cast<size_t>(istep) * pv.nspec * nn + p) * 2;
              for (int c = 0; c < nc; ++c) {
                if (stacey_store64) (*stacey_store64)[at + c] = static_cast<double>(acc[c]);
                else (*stacey_store)[at + c] = static_cast<float>(acc[c]);
              }
            }
          }
          for (int c = 0; c < nc; ++c) {
#pragma omp atomic
            F.a[static_cast<size_t>(c) * F.nglob + g] += acc[c];
          }
        }
    }
  }

  // ---- sources (compute_source_interaction.tpp:77-95) --------------------
  void sources(int m, int istep, int wavefield_sel) {
    Field<T> &F = f[m];
    if (wavefield_sel < 0) return;
    for (int s = 0; s < pv.nsources; ++s) {
      if (pv.src_shot[s] != shot || pv.src_wavefield[s] != wavefield_sel) continue;
      const int e = pv.src_ispec[s];
      if (pv.medium[e] != m) continue;
      for (int iz = 0; iz < n; ++iz)
        for (int ix = 0; ix < n; ++ix) {
          const size_t p = P(e, iz, ix);
          const int g = pv.iglob[p];
          for (int c = 0; c < F.nc; ++c) {
            const T stf = pv.src_stf[(static_cast<size_t>(s) * pv.nstep + istep) * 2 + c];
            const T arr = pv.src_array[((static_cast<size_t>(s) * 2 + c) * n + iz) * n + ix];
            T val = stf * arr;
            if (m == ACOUSTIC) val = stf * arr / static_cast<T>(pv.kappa[p]);
            F.a[static_cast<size_t>(c) * F.nglob + g] += val;
          }
        }
    }
  }

  // Adjoint sources: receiver r injects stf[istep][r][c] * lagrange.
  void adjoint_sources(int m, int istep) {
    if (!adjoint_stf) return;
    Field<T> &F = f[m];
    for (int r = 0; r < pv.nreceivers; ++r) {
      const int e = pv.rec_ispec[r];
      if (pv.medium[e] != m) continue;
      for (int iz = 0; iz < n; ++iz)
        for (int ix = 0; ix < n; ++ix) {
          const size_t p = P(e, iz, ix);
          const int g = pv.iglob[p];
          const T h = pv.rec_lagrange[(static_cast<size_t>(r) * n + iz) * n + ix];
          for (int c = 0; c < F.nc; ++c) {
            const T stf = adjoint_stf[(static_cast<size_t>(istep) * pv.nreceivers + r) * 2 + c];
            T val = stf * h;
            if (m == ACOUSTIC) val = stf * h / static_cast<T>(pv.kappa[p]);
            F.a[static_cast<size_t>(c) * F.nglob + g] += val;
          }
        }
    }
  }

  // ---- coupling (coupled_interface.tpp:55-86) ----------------------------
  void coupling(int m) {
    if (m == ACOUSTIC) {
      Field<T> &S = f[ACOUSTIC];
      const Field<T> &C = f[PSV];
      for (int i = 0; i < pv.ncouple_acoustic; ++i) {
        const int gs = pv.couple_acoustic_self[i], gc = pv.couple_acoustic_other[i];
        const T fac = pv.couple_acoustic_factor[i];
        const T nx = pv.couple_acoustic_nx[i], nz = pv.couple_acoustic_nz[i];
        S.a[gs] += fac * (nx * C.u[gc] + nz * C.u[static_cast<size_t>(C.nglob) + gc]);
      }
    } else if (m == PSV) {
      Field<T> &S = f[PSV];
      const Field<T> &C = f[ACOUSTIC];
      for (int i = 0; i < pv.ncouple_elastic; ++i) {
        const int gs = pv.couple_elastic_self[i], gc = pv.couple_elastic_other[i];
        const T fac = pv.couple_elastic_factor[i];
        const T nx = pv.couple_elastic_nx[i], nz = pv.couple_elastic_nz[i];
        S.a[gs] += fac * nx * C.a[gc];
        S.a[static_cast<size_t>(S.nglob) + gs] += fac * nz * C.a[gc];
      }
    }
  }

  void divide_mass(int m) {
    Field<T> &F = f[m];
    for (size_t i = 0; i < F.a.size(); ++i) F.a[i] = F.a[i] * F.minv[i];
  }

  // update_wavefields<medium>(istep), domain_kernels.hpp:68-126
  int update(int m, int istep, int src_sel) {
    if (elems[m].empty()) return 0;
    coupling(m);
    sources(m, istep, src_sel);
    adjoint_sources(m, istep);
    stiffness(m, istep);
    divide_mass(m);
    return static_cast<int>(elems[m].size());
  }

  // ---- seismograms (compute_seismogram.tpp, wavefield.hpp) ---------------
  template <typename O> void seismograms(O *out, int isig) {
    const int ntypes = pv.nseismogram_types, nrec = pv.nreceivers;
    for (int r = 0; r < nrec; ++r) {
      const int e = pv.rec_ispec[r];
      const int m = pv.medium[e];
      const Field<T> &F = f[m];
      for (int it = 0; it < ntypes; ++it) {
        const int type = pv.seismogram_types[it];
        T acc[2] = {T(0), T(0)};
        // wavefield value at every point of the element
        std::vector<T> wf(static_cast<size_t>(n) * n * 2, T(0));
        const std::vector<T> *src = &F.u;
        if (type == 1) src = &F.v;
        if (type == 2) src = &F.a;
        const bool need_grad = (m == ACOUSTIC && type != 3) || (m == PSV && type == 3);
        if (m == ACOUSTIC && type == 3) src = &F.a;
        if (need_grad) {
          for (int iz = 0; iz < n; ++iz)
            for (int ix = 0; ix < n; ++ix) {
              const size_t p = P(e, iz, ix);
              T dxi[2] = {T(0), T(0)}, dga[2] = {T(0), T(0)};
              for (int l = 0; l < n; ++l)
                for (int c = 0; c < F.nc; ++c) {
                  dxi[c] += hp[ix * n + l] * (*src)[static_cast<size_t>(c) * F.nglob + pv.iglob[P(e, iz, l)]];
                  dga[c] += hp[iz * n + l] * (*src)[static_cast<size_t>(c) * F.nglob + pv.iglob[P(e, l, ix)]];
                }
              const T xix = pv.xix[p], xiz = pv.xiz[p], gax = pv.gammax[p], gaz = pv.gammaz[p];
              T du[2][2];
              for (int c = 0; c < F.nc; ++c) {
                du[c][0] = xix * dxi[c] + gax * dga[c];
                du[c][1] = xiz * dxi[c] + gaz * dga[c];
              }
              const int k = iz * n + ix;
              if (m == ACOUSTIC) {
                const T ri = pv.rho_inverse[p];
                wf[k * 2 + 0] = ri * du[0][0];
                wf[k * 2 + 1] = ri * du[0][1];
              } else {
                const T kappa = pv.kappa[p], mu = pv.mu[p];
                const T l2m = kappa + static_cast<T>(static_cast<float>(4.0 / 3.0)) * mu;
                const T lam = l2m - T(2) * mu;
                wf[k * 2 + 0] = T(-1) * ((lam + static_cast<T>(2.0 / 3.0) * mu) * (du[0][0] + du[1][1]));
                wf[k * 2 + 1] = T(0);
              }
            }
        } else {
          for (int iz = 0; iz < n; ++iz)
            for (int ix = 0; ix < n; ++ix) {
              const int g = pv.iglob[P(e, iz, ix)];
              const int k = iz * n + ix;
              if (m == ACOUSTIC) {  // pressure: -chi_ddot
                wf[k * 2 + 0] = T(-1) * (*src)[g];
                wf[k * 2 + 1] = T(0);
              } else {
                wf[k * 2 + 0] = (*src)[g];
                wf[k * 2 + 1] = F.nc > 1 ? (*src)[static_cast<size_t>(F.nglob) + g] : T(0);
              }
            }
        }
        for (int k = 0; k < n * n; ++k) {
          const T h = pv.rec_lagrange[static_cast<size_t>(r) * n * n + k];
          acc[0] += h * wf[k * 2 + 0];
          acc[1] += h * wf[k * 2 + 1];
        }
        const T s = pv.rec_sin[r], c = pv.rec_cos[r];
        O *o = out + ((static_cast<size_t>(isig) * ntypes + it) * nrec + r) * 2;
        o[0] = static_cast<O>(c * acc[0] - s * acc[1]);
        o[1] = static_cast<O>(s * acc[0] + c * acc[1]);
      }
    }
  }

  // time_marching<forward>::run body (time_marching.tpp:33-89)
  void forward_step(int istep) {
    int dofs = 0, elements = 0;
    for (int m : {ACOUSTIC, PSV, SH}) predictor(m, T(1)), dofs += static_cast<int>(f[m].u.size());
    elements += update(ACOUSTIC, istep, 0);
    corrector(ACOUSTIC, T(1));
    dofs += static_cast<int>(f[ACOUSTIC].u.size());
    elements += update(PSV, istep, 0);
    elements += update(SH, istep, 0);
    corrector(PSV, T(1));
    corrector(SH, T(1));
    dofs += static_cast<int>(f[PSV].u.size() + f[SH].u.size());
    int total_dofs = 0;
    for (int m : {ACOUSTIC, PSV, SH}) total_dofs += 2 * static_cast<int>(f[m].u.size());
    if (dofs != total_dofs || elements != nspec)
      throw std::runtime_error("The time loop has not updated all the degrees of freedom");
  }

  // ---- Frechet kernels (compute_material_derivatives.tpp:84-153 and
  // medium/dim2/*/isotropic/frechet_derivative.hpp), per local point,
  // accumulated in FP64: k[p*3 + 0..2] = (rho, mu, kappa) for elastic,
  // (rho, kappa, sum of rho_kl * kappa_kl) for acoustic.
  // Model derivative of the P-SV Stacey traction (left out of the
  // reference's kernels): kb[p] += -dt w |n| ((s.n^)(v.n^), s.v - (s.n^)(v.n^))
  // at Stacey points, s the adjoint displacement and v the backward
  // wavefield's velocity after its corrector.
  static void stacey_frechet(const Sim &adj, const Sim &bwd, T dt, double *kb) {
    const sfb_problem_view &pv = adj.pv;
    const int n = adj.n;
    for (int e = 0; e < pv.nspec; ++e) {
      if (pv.medium[e] != PSV) continue;
      const Field<T> &FA = adj.f[PSV], &FB = bwd.f[PSV];
      for (int iz = 0; iz < n; ++iz)
        for (int ix = 0; ix < n; ++ix) {
          const size_t p = adj.P(e, iz, ix);
          if (!(pv.bnd[p] & 1)) continue;
          const int g = pv.iglob[p];
          const double nx = pv.bnd_nx[p], nz = pv.bnd_nz[p], we = pv.bnd_w[p];
          const double j = std::sqrt(nx * nx + nz * nz), ux = nx / j, uz = nz / j;
          const double sx = FA.u[g], sz = FA.u[static_cast<size_t>(FA.nglob) + g];
          const double vx = FB.v[g], vz = FB.v[static_cast<size_t>(FB.nglob) + g];
          const double sn = sx * ux + sz * uz, vn = vx * ux + vz * uz;
          const double f = -static_cast<double>(dt) * we * j;
          kb[p * 2 + 0] += f * sn * vn;
          kb[p * 2 + 1] += f * (sx * vx + sz * vz - sn * vn);
        }
    }
  }

  static void frechet(const Sim &adj, const Sim &bwd, T dt, double *k) {
    const sfb_problem_view &pv = adj.pv;
    const int n = adj.n, nn = n * n;
    for (int e = 0; e < pv.nspec; ++e) {
      const int m = pv.medium[e];
      if (m == SH) continue;
      const Field<T> &FA = adj.f[m], &FB = bwd.f[m];
      const int nc = FA.nc;
      for (int iz = 0; iz < n; ++iz)
        for (int ix = 0; ix < n; ++ix) {
          const size_t p = adj.P(e, iz, ix);
          T da[2][2], db[2][2];
          for (int w = 0; w < 2; ++w) {
            const Field<T> &F = w == 0 ? FA : FB;
            T dxi[2] = {T(0), T(0)}, dga[2] = {T(0), T(0)};
            for (int l = 0; l < n; ++l)
              for (int c = 0; c < nc; ++c) {
                dxi[c] += adj.hp[ix * n + l] * F.u[static_cast<size_t>(c) * F.nglob + pv.iglob[adj.P(e, iz, l)]];
                dga[c] += adj.hp[iz * n + l] * F.u[static_cast<size_t>(c) * F.nglob + pv.iglob[adj.P(e, l, ix)]];
              }
            T (*d)[2] = w == 0 ? da : db;
            for (int c = 0; c < nc; ++c) {
              d[c][0] = static_cast<T>(pv.xix[p]) * dxi[c] + static_cast<T>(pv.gammax[p]) * dga[c];
              d[c][1] = static_cast<T>(pv.xiz[p]) * dxi[c] + static_cast<T>(pv.gammaz[p]) * dga[c];
            }
          }
          const int g = pv.iglob[p];
          if (m == PSV) {
            const T kappa0 = pv.kappa[p], mu = pv.mu[p], rho = pv.rho[p];
            const T l2m = kappa0 + static_cast<T>(static_cast<float>(4.0 / 3.0)) * mu;
            const T kappa = l2m - mu;
            const T ad_dsxx = da[0][0], ad_dsxz = T(0.5) * (da[1][0] + da[0][1]), ad_dszz = da[1][1];
            const T b_dsxx = db[0][0], b_dsxz = T(0.5) * (db[1][0] + db[0][1]), b_dszz = db[1][1];
            T kappa_kl = (ad_dsxx + ad_dszz) * (b_dsxx + b_dszz);
            T mu_kl = (ad_dsxx * b_dsxx + ad_dszz * b_dszz + T(2) * ad_dsxz * b_dsxz -
                       static_cast<T>(static_cast<float>(1.0 / 3.0)) * kappa_kl);
            T rho_kl = FA.a[g] * FB.u[g] + FA.a[static_cast<size_t>(FA.nglob) + g] * FB.u[static_cast<size_t>(FB.nglob) + g];
            kappa_kl = T(-1) * kappa * dt * kappa_kl;
            mu_kl = T(-2) * mu * dt * mu_kl;
            rho_kl = T(-1) * rho * dt * rho_kl;
            k[p * 3 + 0] += static_cast<double>(rho_kl);
            k[p * 3 + 1] += static_cast<double>(mu_kl);
            k[p * 3 + 2] += static_cast<double>(kappa_kl);
          } else {
            const T ri = pv.rho_inverse[p], kap = pv.kappa[p];
            const T rho_kl = (da[0][0] * db[0][0] + da[0][1] * db[0][1]) * ri * dt;
            const T kappa_kl = FA.a[g] * FB.u[g] * T(1) / kap * dt;
            k[p * 3 + 0] += static_cast<double>(rho_kl);
            k[p * 3 + 1] += static_cast<double>(kappa_kl);
            // rhop = rho_kl * kappa_kl per step (point/kernels.hpp:189-192)
            k[p * 3 + 2] += static_cast<double>(rho_kl * kappa_kl);
          }
        }
    }
  }
};

// T: arithmetic; O: type of the outputs (seismograms, fields, Stacey store):
// FP32 as the reference writes them, or FP64 for the FP64 oracle's exact
// values.
template <typename T, typename O = float>
int run_forward(const sfb_problem_view *pv, int shot, int nstep, int threads,
                O *seis, O **fields_out, O *stacey_store_out) {
  Sim<T> s(*pv, shot);
  s.threads = threads;
  std::vector<O> store;
  if (stacey_store_out) {
    store.assign(static_cast<size_t>(nstep) * pv->nspec * pv->ngll * pv->ngll * 2, O(0));
    s.store_stacey = true;
    if constexpr (std::is_same<O, double>::value) s.stacey_store64 = &store;
    else s.stacey_store = &store;
  }
  s.init_mass();
  const int nsbs = pv->nstep_between_samples;
  const int max_sig = pv->nstep / nsbs;
  int isig = 0;
  for (int istep = 0; istep < nstep; ++istep) {
    s.forward_step(istep);
    if (istep % nsbs == 0 && isig < max_sig) {
      if (seis) s.seismograms(seis, isig);
      ++isig;
    }
  }
  if (fields_out) {
    int k = 0;
    for (int m : {PSV, SH, ACOUSTIC}) {
      for (auto *vec : {&s.f[m].u, &s.f[m].v, &s.f[m].a, &s.f[m].minv}) {
        if (fields_out[k])
          for (size_t i = 0; i < vec->size(); ++i) fields_out[k][i] = static_cast<O>((*vec)[i]);
        ++k;
      }
    }
  }
  if (stacey_store_out) std::memcpy(stacey_store_out, store.data(), store.size() * sizeof(O));
  return 0;
}


// time_marching<combined>::run (time_marching.tpp:126-247): adjoint wavefield
// forward in reversed time with the adjoint sources, backward wavefield
// reconstructed with -dt from the forward run's last state (`buffer`) with
// Stacey elements replaying the stored element accelerations, Frechet
// kernels accumulated every step.
template <typename T, typename O = float>
int run_combined(const sfb_problem_view *pv, int shot, int nstep, int threads, const float *adjoint_stf,
                 const O *const *buffer, const std::vector<O> &store, double *kernels,
                 O *bseis, double *kb = nullptr) {
  Sim<T> adj(*pv, shot), bwd(*pv, shot);
  adj.threads = bwd.threads = threads;
  adj.adjoint_stf = adjoint_stf;
  bwd.backward = true;
  if constexpr (std::is_same<O, double>::value) bwd.stacey_replay64 = &store;
  else bwd.stacey_replay = &store;
  adj.init_mass();
  bwd.init_mass();
  for (int e = 0; e < pv->nspec; ++e)
    if (pv->medium[e] == SH) throw std::invalid_argument("combined SH runs are not supported by the reference");
  const int nsbs = pv->nstep_between_samples;
  const int max_sig = pv->nstep / nsbs;
  int isig = 0;
  for (int istep = nstep - 1; istep >= 0; --istep) {
    // adjoint time step (forward-style dt), adjoint sources only
    adj.predictor(ACOUSTIC, T(1));
    adj.predictor(PSV, T(1));
    adj.update(ACOUSTIC, istep, -1);
    adj.corrector(ACOUSTIC, T(1));
    adj.update(PSV, istep, -1);
    adj.corrector(PSV, T(1));
    // backward time step (-dt), elastic before acoustic, forward sources
    bwd.predictor(PSV, T(-1));
    bwd.predictor(ACOUSTIC, T(-1));
    bwd.update(PSV, istep, 0);
    bwd.corrector(PSV, T(-1));
    bwd.update(ACOUSTIC, istep, 0);
    bwd.corrector(ACOUSTIC, T(-1));
    if (istep == nstep - 1) {
      int k = 0;
      for (int m : {PSV, SH, ACOUSTIC}) {
        for (auto *vec : {&bwd.f[m].u, &bwd.f[m].v, &bwd.f[m].a}) {
          const O *src = buffer[k++];
          if (src)
            for (size_t i = 0; i < vec->size(); ++i) (*vec)[i] = static_cast<T>(src[i]);
        }
      }
    }
    Sim<T>::frechet(adj, bwd, static_cast<T>(pv->dt), kernels);
    if (kb) Sim<T>::stacey_frechet(adj, bwd, static_cast<T>(pv->dt), kb);
    if (istep % nsbs == 0 && isig < max_sig) {
      if (bseis) bwd.seismograms(bseis, isig);
      ++isig;
    }
  }
  return 0;
}

thread_local std::string g_err;

}  // namespace

// Seismograms of given fields (see oracle_seismograms).
template <typename O>
int seismograms_of_fields(const sfb_problem_view *pv, int precision, const double *const *fields_in, O *seis) {
  auto run = [&](auto zero) -> int {
    using T = decltype(zero);
    Sim<T> s(*pv, 0);
    int k = 0;
    for (int m : {PSV, SH, ACOUSTIC}) {
      for (auto *vec : {&s.f[m].u, &s.f[m].v, &s.f[m].a}) {
        const double *src = fields_in[k++];
        if (src)
          for (size_t i = 0; i < vec->size(); ++i) (*vec)[i] = static_cast<T>(src[i]);
      }
    }
    s.seismograms(seis, 0);
    return 0;
  };
  try {
    if (pv->ngll > 8) throw std::invalid_argument("ngll > 8");
    return precision == 64 ? run(0.0) : run(0.0f);
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

extern "C" {

const char *oracle_last_error() { return g_err.c_str(); }

// Forward run of `shot`, `nstep` steps.  seis: [max_sig_step][ntypes][nrec][2]
// (may be NULL).  fields_out: 12 pointers (u, v, a, minv for P-SV, SH,
// acoustic; each may be NULL) of [ncomp][nglob] floats.  stacey_store_out:
// [nstep][nloc][2] or NULL.  precision: 32 or 64.
int oracle_forward(const sfb_problem_view *pv, int precision, int shot,
                   int nstep, int threads, float *seis, float **fields_out,
                   float *stacey_store_out) {
  try {
    if (pv->ngll > 8) throw std::invalid_argument("ngll > 8");
    if (precision == 64)
      return run_forward<double>(pv, shot, nstep, threads, seis, fields_out, stacey_store_out);
    return run_forward<float>(pv, shot, nstep, threads, seis, fields_out, stacey_store_out);
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

// Combined run of `shot`: adjoint_stf [nstep][nrec][2]; buffer: 9 pointers
// (u, v, a for P-SV, SH, acoustic; [ncomp][nglob] floats, NULL = zero);
// stacey_store [nstep][nloc][2] from oracle_forward; kernels_out
// [nloc][3] FP64 (accumulated into); bseis: backward seismograms or NULL.
int oracle_combined(const sfb_problem_view *pv, int precision, int shot, int nstep, int threads,
                    const float *adjoint_stf, const float *const *buffer, const float *stacey_store,
                    double *kernels_out, float *bseis) {
  try {
    const size_t nloc = static_cast<size_t>(pv->nspec) * pv->ngll * pv->ngll;
    std::vector<float> store(stacey_store, stacey_store + static_cast<size_t>(nstep) * nloc * 2);
    if (precision == 64)
      return run_combined<double>(pv, shot, nstep, threads, adjoint_stf, buffer, store, kernels_out, bseis);
    return run_combined<float>(pv, shot, nstep, threads, adjoint_stf, buffer, store, kernels_out, bseis);
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

// The FP64 oracle with FP64 outputs: the same runs as oracle_forward /
// oracle_combined with precision 64, but seismograms, fields, the Stacey
// store, the backward initial state and the backward seismograms are
// doubles (not rounded to FP32 on the way out).
int oracle_forward_f64(const sfb_problem_view *pv, int shot, int nstep, int threads, double *seis,
                       double **fields_out, double *stacey_store_out) {
  try {
    if (pv->ngll > 8) throw std::invalid_argument("ngll > 8");
    return run_forward<double, double>(pv, shot, nstep, threads, seis, fields_out, stacey_store_out);
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

int oracle_combined_f64(const sfb_problem_view *pv, int shot, int nstep, int threads, const float *adjoint_stf,
                        const double *const *buffer, const double *stacey_store, double *kernels_out,
                        double *bseis, double *stacey_kernels_out) {
  try {
    const size_t nloc = static_cast<size_t>(pv->nspec) * pv->ngll * pv->ngll;
    std::vector<double> store(stacey_store, stacey_store + static_cast<size_t>(nstep) * nloc * 2);
    return run_combined<double, double>(pv, shot, nstep, threads, adjoint_stf, buffer, store, kernels_out, bseis,
                                        stacey_kernels_out);
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

// Seismograms of given fields, one record: what compute_seismograms(0) gives
// on a wavefield loaded from files (the reference's seismogram unit tests,
// tests/unit-tests/seismogram/*/seismogram_tests.cpp).  fields_in: 9
// pointers (u, v, a for P-SV, SH, acoustic; [ncomp][nglob] doubles, NULL =
// zero); seis: [ntypes][nrec][2].
int oracle_seismograms(const sfb_problem_view *pv, int precision, const double *const *fields_in, float *seis) {
  return seismograms_of_fields(pv, precision, fields_in, seis);
}

// The same in FP64 with FP64 outputs.
int oracle_seismograms_f64(const sfb_problem_view *pv, const double *const *fields_in, double *seis) {
  return seismograms_of_fields(pv, 64, fields_in, seis);
}

}  // extern "C"
