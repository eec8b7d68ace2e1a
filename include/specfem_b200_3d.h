/* C ABI of the 3D elastic path (hexahedral spectral elements).
 *
 * No counterpart in the reference: its 3D program reads the mesh and stops
 * (src/specfem3d.cpp:49-73).  This path restates the reference's 2D weak
 * form (include/algorithms/gradient.hpp:36-111, divergence.hpp:40-103,
 * medium/dim2/elastic/isotropic/stress.hpp:14-50, core/specfem/point/
 * stress.hpp:117-139, boundary_conditions/stacey/stacey.tpp:41-75,
 * kokkos_kernels/impl/compute_mass_matrix.tpp:80-113, timescheme/
 * newmark.tpp, the Frechet kernels of frechet_derivative.hpp:14-138 and the
 * combined loop of solver/time_marching.tpp:126-247) with a third
 * dimension: NGLL = 5 Gauss-Lobatto-Legendre points per direction,
 * isotropic elastic (kappa, mu, rho; lambda + 2 mu = kappa + 4/3 mu),
 * Newmark explicit in time, Stacey absorbing faces, moment-tensor point
 * sources with Ricker time functions, displacement receivers.
 *
 * Mesh: nx x ny x nz axis-aligned hexahedra over [x0,x1] x [y0,y1] x
 * [z0,z1], z up; element (ex, ey, ez) = (ez * ny + ey) * nx + ex; local
 * point (k, j, i) along (z, y, x), p = e * 125 + (k * 5 + j) * 5 + i.
 * Global points on the (4nx+1) x (4ny+1) x (4nz+1) lattice,
 * g = (gz * (4ny+1) + gy) * (4nx+1) + gx.
 *
 * Absorbing (Stacey) faces: bit f of `absorb` for face f = 0 x-min, 1 x-max,
 * 2 y-min, 3 y-max, 4 z-min (bottom), 5 z-max (top, normally the free
 * surface).  With axis-aligned faces the Stacey traction at a boundary
 * point is -A v with A diagonal (the sum over the point's absorbing element
 * faces of w |J_face| [rho vs + (rho vp - rho vs) n_c^2]).  The combined
 * (adjoint + backward) run replays the tractions the forward run applied at
 * every boundary point.  When the whole run's tractions do not fit in
 * device memory the run is cut into segments: the forward run keeps the
 * state at each segment start (a checkpoint, in device memory when it fits,
 * else in pinned host memory) and the combined run recomputes one segment's
 * forward steps, keeping their tractions, before marching it backwards.
 *
 * All functions return 0 or a negative SFB_E_* status
 * (specfem_b200.h); sfb3_last_error gives the message.
 */
#ifndef SPECFEM_B200_3D_H
#define SPECFEM_B200_3D_H

#include <stddef.h>

#include "specfem_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sfb3_context sfb3_context;

typedef struct sfb3_source {
  int shot;
  double x, y, z;
  /* moment tensor (N m) */
  double mxx, myy, mzz, mxy, mxz, myz;
  double f0, tshift, factor; /* Ricker (the reference's stf, -factor * ricker) */
} sfb3_source;

typedef struct sfb3_desc {
  int nx, ny, nz;
  double x0, x1, y0, y1, z0, z1;
  int absorb;                 /* face bits, see above */
  const float *rho, *vp, *vs; /* per local point [nspec][5][5][5] */
  double dt;
  int nstep, nshots;
  int nsources;
  const sfb3_source *sources;
  int nreceivers;
  const double *receivers;    /* [nreceivers][3] x, y, z; shared by shots */
  int save_boundary_values;   /* allocate the adjoint / backward state */
  int segment_steps;          /* steps per segment; 0 = as many as fit */
  int host_checkpoints;       /* 1: keep checkpoints in pinned host memory */
  int deterministic;          /* 1: bit-reproducible runs (element colours:
                                 one stiffness launch per colour of
                                 hexahedra sharing no point, plain adds;
                                 sources, adjoint sources and mass in a
                                 fixed order) */
} sfb3_desc;

typedef struct sfb3_info {
  int nspec, nglob, nshots, nstep, nreceivers;
  int nboundary_points;       /* global points with an absorbing face */
  int segment_steps, nsegments;
  int checkpoints_on_host;
  double dt, t0;
  size_t device_bytes, host_bytes;
  unsigned long long kernel_launches;
} sfb3_info;

SFB_API int sfb3_create(const sfb3_desc *desc, sfb3_context **out);
SFB_API void sfb3_destroy(sfb3_context *ctx);
SFB_API const char *sfb3_last_error(const sfb3_context *ctx);
SFB_API int sfb3_get_info(const sfb3_context *ctx, sfb3_info *info);
/* Forward run of `nstep` steps (continuing from the steps already run). */
SFB_API int sfb3_run_forward(sfb3_context *ctx, int nstep);
/* Seismograms of `wavefield` (0 forward, 2 backward) for `shot`:
 * [nstep][nreceivers][3] displacement; backward samples in loop order (last
 * step first), as the reference stores them. */
SFB_API int sfb3_get_seismograms(sfb3_context *ctx, int wavefield, int shot, float *host, size_t count);
/* Adjoint sources of `shot` at the receivers: [nstep][nreceivers][3]. */
SFB_API int sfb3_set_adjoint_sources(sfb3_context *ctx, int shot, const float *host, size_t count);
/* Adjoint + backward run over all nstep steps after the whole forward run,
 * Frechet kernels summed over the shots. */
SFB_API int sfb3_run_combined(sfb3_context *ctx);
/* Kernels per local point [nspec][5][5][5], FP64: which = 0 rho, 1 mu,
 * 2 kappa: K_rho = -rho sum dt a_adj . u, K_mu = -2 mu sum dt D_adj : D,
 * K_kappa = -kappa sum dt div u_adj div u (D the deviatoric strain). */
SFB_API int sfb3_get_kernels(sfb3_context *ctx, int which, double *host, size_t count);
/* Field `which` (0 u, 1 v, 2 a) of `wavefield` (0 forward, 1 adjoint,
 * 2 backward) for `shot`, [3][nglob]; which 3: the inverse mass, [3][nglob]. */
SFB_API int sfb3_get_field(sfb3_context *ctx, int wavefield, int which, int shot, float *host, size_t count);
/* Zero every wavefield, the seismograms and the kernels; step count 0. */
SFB_API int sfb3_reset(sfb3_context *ctx);
/* Stiffness / Frechet kernel variant: 0 automatic, 1 one shot per thread,
 * 2 two shots per thread in packed FP32x2 arithmetic (the automatic choice
 * for an even shot count), 3 the same compiled for three resident CTAs per
 * SM.  Odd shot counts always use variant 1.  sfb3_get_variant returns the
 * variant in use. */
SFB_API int sfb3_set_variant(sfb3_context *ctx, int variant);
SFB_API int sfb3_get_variant(const sfb3_context *ctx);
/* Mean device time (ms) of `reps` launches of one kernel on a copy of the
 * forward fields (kept in the adjoint wavefield's buffers, which it
 * overwrites): what 0 stiffness, 1 Newmark update, 2 Frechet kernels,
 * 4 the backward stiffness with the fused Frechet kernels (packed
 * variants); 3 times `reps` whole forward steps, which advance the state;
 * 5 runs the whole combined run (as sfb3_run_combined, `reps` ignored) and
 * gives its mean time per step. */
SFB_API int sfb3_time_kernel(sfb3_context *ctx, int what, int reps, double *mean_ms);

#ifdef __cplusplus
}
#endif

#endif /* SPECFEM_B200_3D_H */
