// Device-side data and kernel launchers for the SEM time-marching path.
//
// Layout in HBM (device element order = elements sorted by medium, boundary
// elements last within a medium, so each medium is one contiguous range):
//   per local point p = (e * N + iz) * N + ix, SoA float arrays:
//     iglob[p]                        index in the medium's field
//     xix, xiz, gammax, gammaz, jac   geometry
//     mat0, mat1, mat2                P-SV: kappa, mu, rho
//                                     SH:   mu, rho, -
//                                     acoustic: rho_inverse, kappa, -
//   fields, shot-major: field[s][iglob] as float2 (P-SV) or float (SH,
//   acoustic); the inverse mass has no shot index.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sfb {
namespace dev {

enum { MED_PSV = 0, MED_SH = 1, MED_AC = 3 };

struct Static {
  int ngll, nspec;
  const int *iglob;
  const float *xix, *xiz, *gax, *gaz, *jac;
  const float *mat0, *mat1, *mat2;
  const uint8_t *eflag;  // per device element: bit0 Stacey points, bit1 free-surface points
  const uint8_t *bnd;    // per local point
  const float *bnd_nx, *bnd_nz, *bnd_w;
};

struct MediumFields {
  int nglob;    // points in this medium
  int nc;       // components
  int elem_begin, nelem;      // device element range
  int nelem_interior;         // elements [elem_begin, elem_begin+nelem_interior) have no boundary points
  float *u, *v, *a;           // [S][nglob*nc]
  float *minv;                // [nglob*nc]
  double *mass;               // scratch for initialize, [nglob*nc]
};

struct Control {
  int istep;  // step counter advanced on the device by the update kernel
};

struct SourceSet {
  int n;
  const int *elem;       // device element
  const int *shot;
  const int *medium;
  const float *array;    // [n][2][N*N]
  const float *stf;      // [n][nstep][2]
  int nstep;
};

struct ReceiverSet {
  int n;
  const int *elem;       // device element
  const float *lagrange; // [n][N*N]
  const float *sinv, *cosv;
  int ntypes;
  int types[5];
  int max_sig, nsbs;
  float *seis;           // [S][max_sig][ntypes][n][2]
};

struct CouplingSet {
  int n;
  const int *self, *other;
  const float *factor, *nx, *nz;
};

// Stacey replay / store (adjoint reconstruction): element-local
// accelerations of the Stacey elements, [nstep][nstacey][N*N][nc].
struct StaceyStore {
  float *data;
  const int *slot;   // per device element: slot index or -1
  int nstacey;
  int nstep;
  int mode;          // 0 none, 1 store (forward), 2 replay (backward)
};

// ---- launchers (kernels.cu) ----
void set_quadrature(int ngll, const float *hprime, const float *wgll);

void launch_stiffness(int medium, int ngll, const Static &st, const MediumFields &f,
                      int nshots, const StaceyStore &ss, const int *istep_dev,
                      cudaStream_t stream);
void launch_sources(int ngll, const Static &st, const SourceSet &src,
                    MediumFields *fields, int nshots, int medium, const int *istep_dev,
                    int adjoint_only, cudaStream_t stream);
void launch_coupling_acoustic(const CouplingSet &c, const MediumFields &ac,
                              const MediumFields &el, int nshots, cudaStream_t stream);
void launch_coupling_elastic(const CouplingSet &c, const MediumFields &el,
                             const MediumFields &ac, int nshots, int ac_divided,
                             cudaStream_t stream);
// Seismograms at the end of a step.  mode 0: fields hold the final state
// (u, v, a).  mode 1: fused loop, fields hold (u, v*, force) and the final
// velocity/acceleration are formed on the fly.
void launch_receivers(int ngll, const Static &st, const ReceiverSet &rec,
                      const MediumFields *fields, int nshots, float dt2, int mode,
                      const int *istep_dev, cudaStream_t stream);
// Newmark pieces (unfused API) and fused update.
void launch_predictor(const MediumFields &f, int nshots, float dt, float dt2, float dtsq2,
                      cudaStream_t stream);
void launch_corrector(const MediumFields &f, int nshots, float dt2, cudaStream_t stream);
void launch_divide(const MediumFields &f, int nshots, cudaStream_t stream);
// a = force * minv; v += dt2 a; then (last == 0) u += dt v + dtsq2 a,
// v += dt2 a, force = 0.  `ctrl` (may be null) has its step advanced.
void launch_fused_update(const MediumFields &f, int nshots, float dt, float dt2,
                         float dtsq2, int last, Control *ctrl, cudaStream_t stream);
void launch_advance_step(Control *ctrl, cudaStream_t stream);
void launch_mass(int medium, int ngll, const Static &st, const MediumFields &f, float dt,
                 cudaStream_t stream);
void launch_invert_mass(const MediumFields &f, cudaStream_t stream);
void launch_zero(float *p, size_t n, cudaStream_t stream);

}  // namespace dev
}  // namespace sfb
