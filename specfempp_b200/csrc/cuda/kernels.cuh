// Device-side data and kernel launchers for the SEM time-marching path.
//
// Layout in HBM (device element order = elements sorted by medium, boundary
// elements last within a medium, so each medium is one contiguous range):
//   per local point p = (e * N + iz) * N + ix, SoA arrays of `real` (FP32):
//     iglob[p]                        index in the medium's field
//     xix, xiz, gammax, gammaz, jac   geometry
//     mat0, mat1, mat2                P-SV: kappa, mu, rho
//                                     SH:   mu, rho, -
//                                     acoustic: rho_inverse, kappa, -
//   fields, point-major and shot-minor: value (g, s) at g * S + s, as a pair
//   (P-SV) or a scalar (SH, acoustic); the inverse mass has no shot index.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sfb {
namespace dev {

// Arithmetic type of the wavefields, geometry, material and every per-step
// quantity.  The product library is built with FP32 (the reference's
// type_real).  The verification library (SFB_FP64) compiles the same
// generic kernels -- the scalar batched stiffness, sources, coupling,
// receivers, Newmark pieces, the fused update, Frechet kernels and the mass
// matrix -- in FP64, so that the device path can be compared with the FP64
// oracle at FP64 rounding level; the FP32-specific kernels (bulk-copy fed
// row kernels, compact block, packed f32x2) are left out of that build.
#ifdef SFB_FP64
typedef double real;
typedef double2 real2;
typedef double4 real4;
#else
typedef float real;
typedef float2 real2;
typedef float4 real4;
#endif

enum { MED_PSV = 0, MED_SH = 1, MED_AC = 3 };

struct Static {
  int ngll, nspec;
  const int *iglob;
  const real *xix, *xiz, *gax, *gaz, *jac;
  const real *mat0, *mat1, *mat2;
  const uint8_t *eflag;  // per device element: bit0 Stacey points, bit1 free-surface points
  const uint8_t *bnd;    // per local point
  const real *bnd_nx, *bnd_nz, *bnd_w;
  // Packed per-element block for the TMA-fed stiffness kernel:
  // pack[e][8][N*N] = iglob (int bits; FP64 build: the index as a value),
  // xix, xiz, gammax, gammaz, jac, mat0, mat1.
  const real *pack;
  // Compact block of affine elements (constant Jacobian matrix, e.g. the
  // parallelograms of a structured mesh), single-shot contexts only, in
  // chunks of kAffineChunk elements of one medium (affine_chunk_words(N)
  // words each, the last chunk zero-padded): index, mat0, mat1 per point
  // ([3][chunk][N*N]), then xix, xiz, gammax, gammaz, jac ([5][chunk]).
  // affine[m] != 0 when every element of medium m is affine; its chunks
  // start at chunk aff_chunk0[m].
  const float *pack_aff;
  int affine[4];
  int aff_chunk0[4];
  int *err;              // device error flag (bounded waits that expired)
};

struct MediumFields {
  int nglob;    // points in this medium
  int nc;       // components
  int elem_begin, nelem;      // device element range
  int nelem_interior;         // elements [elem_begin, elem_begin+nelem_interior) have no boundary points
  real *u, *v, *a;            // [nglob + nglob % 2][S][nc]
  real *minv;                 // [nglob*nc]
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
  const real *array;     // [n][2][N*N]
  const real *stf;       // [n][nstep][2]
  int nstep;
};

struct ReceiverSet {
  int n;
  const int *elem;       // device element
  const real *lagrange;  // [n][N*N]
  const real *sinv, *cosv;
  int ntypes;
  int types[5];
  int max_sig, nsbs;
  real *seis;            // [S][max_sig][ntypes][n][2]
  // > 0: the backward run of a combined loop of this many steps, whose
  // samples are numbered in loop order (last step first)
  int backward_nstep;
};

struct CouplingSet {
  int n;
  const int *self, *other;
  const real *factor, *nx, *nz;
};

// Stacey replay / store (adjoint reconstruction): element-local
// accelerations of the Stacey elements, [S][nstep][nstacey][N*N][2].
struct StaceyStore {
  real *data;
  const int *slot;   // per device element: slot index or -1
  int nstacey;
  int nstep;
  int mode;          // 0 none, 1 store (forward), 2 replay (backward)
};

// Work folded into the tail of a stiffness launch: the medium's point sources
// and the coupling points where this medium receives from the other one.
struct TailWork {
  SourceSet src;       // only entries whose medium matches are applied
  CouplingSet cp;
  MediumFields other;  // the coupled medium
  int cp_mode;         // 0 none, 1 acoustic <- elastic displacement, 2 elastic <- acoustic acceleration
  int other_divided;   // mode 2: the acoustic array already holds chi_ddot
  // Overlap of the two stiffness launches of a coupled single-shot step
  // (programmatic dependent launch): kOverlapFirst lets the next launch start
  // as soon as every CTA of this one has passed its dependency wait;
  // kOverlapSecond (the elastic launch, whose element loop reads nothing the
  // acoustic launch writes) waits for the acoustic launch only before its
  // tail work, which reads the acoustic force.
  int overlap;
};
constexpr int kOverlapFirst = 1, kOverlapSecond = 2;

// Sources and coupling of one medium in the deterministic assembly mode, as
// an owner-computes map: target point tgt_g[t] receives the entries
// [tgt_begin[t], tgt_begin[t+1]) in that order, each a point source term
// (source i, element point kk: i * N*N + kk >= 0) or a coupling entry
// (-(index + 1)); one thread per (target, shot) sums them and adds the sum
// once, so no two threads add into the same value.
struct DetTail {
  int ntarget;
  const int *tgt_g;
  const int *tgt_begin;
  const int *ent;
};

// Seismograms as a sparse linear map of nodal values, applied inside the
// update kernel: seis[s][isig][slot] += w * field_which(g).  `mask` has one
// bit per point of the medium; `sup_g` lists the tapped points (sorted) and
// [sup_begin[q], sup_begin[q+1]) their entries.
struct ReceiverTaps {
  int nsup;
  const uint32_t *mask;
  const int *sup_g, *sup_begin;
  const int *slot;    // (type * nrec + rec) * 2 + out component
  const int *which;   // field (0 u, 1 v, 2 a) * 2 + input component
  const real *w;
};

// Unsigned 32-bit division by a runtime constant as multiply-high + shift
// (round-up method): q = (umulhi(n, m) + n) >> l for every n < 2^32.
struct FastDiv {
  uint32_t d, m;
  int l;
  static FastDiv make(uint32_t d) {
    FastDiv f{d, 0, 0};
    while ((1ull << f.l) < d) ++f.l;
    f.m = static_cast<uint32_t>(((1ull << 32) * ((1ull << f.l) - d)) / d + 1);
    return f;
  }
#ifdef __CUDACC__
  __device__ __forceinline__ uint32_t div(uint32_t n) const {
    const uint32_t t = __umulhi(n, m);
    return static_cast<uint32_t>((static_cast<uint64_t>(t) + n) >> l);
  }
#endif
};

struct UpdateMedium {
  real *u, *v, *a;
  const real *minv;
  size_t ld2;    // pairs of values of the whole [g][s][c] array
  int nc;        // components per point (1: a pair holds two entries)
  ReceiverTaps taps;
  real *cu, *cv;    // Kahan compensation terms of u and v (same layout), or null
  // forward snapshots for the combined run: slot c (c = 0 .. count-1) holds
  // u at step (c+1)K (written by step (c+1)K - 1) and v half a step later
  // (written by step (c+1)K); null when off
  real *ck_u, *ck_v;
  size_t ck_stride;  // values per slot
};

// Newmark update of element-private points inside the stiffness launch.  A
// GLL point strictly inside an element belongs to that element alone, so
// once the element's force is known the point's corrector and next
// predictor can run in registers without the force ever reaching memory.
// Elements flagged kElemPrivate in `eflag` (no boundary points, no source,
// no receiver) qualify; their (N-2)^2 interior points are numbered after
// every shared point of the P-SV field, which the update kernel covers.
struct FusedUpdate {
  int enabled;
  const real *minv;    // [nglob][nc]
  real *v;             // [g][S][nc]
  real dt, dt2, dtsq2;
  int last;            // 1: finish the step (store a and v, no predictor)
};
constexpr uint8_t kElemPrivate = 4;

// Frechet kernels fused into the batched P-SV backward stiffness launch of
// the combined loop: the launch that gathers the backward displacement and
// forms its gradient also gathers the adjoint displacement and (assembled)
// adjoint force of the same step and adds this step's rho / mu / kappa
// kernels, summed over the launch's shots, to kern[p][3] (FP64).
struct FrechetFuse {
  int enabled;
  real *au;            // adjoint displacement [g][S][2]
  real *aa;            // adjoint force [g][S][2] (times minv = acceleration)
  const real *minv;   // [nglob][2]
  double *kern;        // [nspec * N * N][3]: rho, mu, kappa
  real dt;
  // the adjoint wavefield's element-private points also finish their (+dt)
  // Newmark step here, after their Frechet contribution is taken
  int adjoint_update;
  real *av;            // adjoint velocity [g][S][2]
  real adt, adt2, adtsq2;
  int last;
};

struct UpdateParams {
  UpdateMedium m[3];
  int nm;
  size_t begin[4];  // pair ranges of the media in the flat index space
  int nshots;
  FastDiv sdiv;           // division by nshots
  real dt, dt2, dtsq2;
  int last;               // 1: finish the step (no predictor for the next one)
  Control *ctrl;          // step counter, advanced by the last CTA to finish
  int dir;                // +1 forward in time, -1 for the combined (reversed) loop
  unsigned *done;         // CTA completion counter (zero between launches)
  real *seis;             // [S][max_sig][slots]
  int slots, max_sig, nsbs;
  int nstep;              // steps of the run (numbering of the backward samples)
  int ck_interval, ck_count;  // snapshot cadence K and slots (0: none)
};

// Restore the backward wavefield of the combined run from the forward
// snapshots when the step counter reaches a snapshot step (see UpdateMedium).
struct RestoreParams {
  real *u[3], *v[3];
  const real *ck_u[3], *ck_v[3];
  size_t n[3];        // values per medium field ([g][S][nc] incl. padding)
  size_t ck_stride[3];
  int nm;
  const Control *ctrl;
  int interval, count;
};
void launch_restore(const RestoreParams &p, cudaStream_t stream);

// ---- launchers (kernels.cu) ----
void set_quadrature(int ngll, const real *hprime, const real *wgll);

// `tw` (may be null) is executed in the same launch.  One shot: the
// TMA-fed row kernel; several shots: the shot-parallel kernel.
// Kernel variants of the batched (nshots > 1) stiffness; see launch_shots.
constexpr int kShotsAuto = 0, kShotsPacked = 1, kShotsPair = 2, kShotsSingle = 3;
// Single-shot (nshots == 1) variants: the row kernel with 32- or 16-element
// chunks (NGLL 8: 16 in both) reading the full static block, or (NGLL 5, a
// medium of affine elements) the compact-block kernel.
constexpr int kRowFullChunk = 1, kRowHalfChunk = 2, kRowAffine = 3;
// The variant a pinned one becomes on a medium that is not all affine.
constexpr int row_variant_without_affine(int v) { return v == kRowAffine ? kRowFullChunk : v; }
// Elements per chunk of the compact block, and words per chunk (a multiple
// of 4: 16-byte aligned bulk copies).
constexpr int kAffineChunk = 32;
constexpr int affine_chunk_words(int n) { return kAffineChunk * (3 * n * n + 5); }
void launch_stiffness(int medium, int ngll, const Static &st, const MediumFields &f,
                      int nshots, const StaceyStore &ss, const int *istep_dev,
                      cudaStream_t stream, const TailWork *tw = nullptr,
                      const FusedUpdate *fu = nullptr, int variant = kShotsAuto);
// True when launch_stiffness_frechet applies (P-SV, even nshots > 1, NGLL 5).
bool frechet_fusable(int medium, int ngll, int nshots);
// Backward stiffness of the batched P-SV medium with the Frechet kernels
// fused in (see FrechetFuse).
// fu: element-private points of the backward wavefield finish their (-dt)
// Newmark step in the launch, after their Frechet contribution is taken.
void launch_stiffness_frechet(int ngll, const Static &st, const MediumFields &bwd, int nshots,
                              const StaceyStore &ss, const int *istep_dev, const TailWork &tw,
                              const FrechetFuse &fr, const FusedUpdate &fu, cudaStream_t stream);
// Once per process and device: kernel attributes (dynamic shared memory).
void init_kernel_attributes();

constexpr int kPackFields = 8;
void launch_sources(int ngll, const Static &st, const SourceSet &src,
                    MediumFields *fields, int nshots, int medium, const int *istep_dev,
                    int adjoint_only, cudaStream_t stream);
void launch_coupling_acoustic(const CouplingSet &c, const MediumFields &ac,
                              const MediumFields &el, int nshots, cudaStream_t stream);
void launch_coupling_elastic(const CouplingSet &c, const MediumFields &el,
                             const MediumFields &ac, int nshots, int ac_divided,
                             cudaStream_t stream);
// Deterministic mode: the sources and coupling of `tw` through `dt` (see
// DetTail), after the medium's stiffness launches.
void launch_tail_det(int medium, int ngll, const Static &st, const MediumFields &f, int nshots,
                     const int *istep_dev, const TailWork &tw, const DetTail &dt, cudaStream_t stream);
// Seismograms at the end of a step.  mode 0: fields hold the final state
// (u, v, a).  mode 1: fused loop, fields hold (u, v*, force) and the final
// velocity/acceleration are formed on the fly.
void launch_receivers(int ngll, const Static &st, const ReceiverSet &rec,
                      const MediumFields *fields, int nshots, real dt2, int mode,
                      const int *istep_dev, cudaStream_t stream);
// Newmark pieces (unfused API) and fused update.
// cu, cv: Kahan compensation terms of u and v, or null for the plain update.
void launch_predictor(const MediumFields &f, int nshots, real dt, real dt2, real dtsq2,
                      cudaStream_t stream, real *cu = nullptr, real *cv = nullptr);
void launch_corrector(const MediumFields &f, int nshots, real dt2, cudaStream_t stream);
void launch_divide(const MediumFields &f, int nshots, cudaStream_t stream);
void launch_advance_step(Control *ctrl, cudaStream_t stream);
// Fused divide + corrector (+ predictor of the next step) for every medium in
// one launch, with the seismogram taps.
void launch_update_all(const UpdateParams &p, cudaStream_t stream);
void launch_mass(int medium, int ngll, const Static &st, const MediumFields &f, real dt,
                 cudaStream_t stream);
void launch_invert_mass(const MediumFields &f, cudaStream_t stream);
void launch_zero(real *p, size_t n, cudaStream_t stream);
// Stacey-traction model derivatives of the P-SV medium (see k_stacey_frechet)
// into kb[p][2] (FP64, device element order): dchi/d(rho vp), dchi/d(rho vs).
// vcorr: 0 when bwd.v is the step's final velocity, else the factor of
// force * M^-1 that completes it (-dt/2 for the backward run's update).
void launch_stacey_frechet(int ngll, const Static &st, const MediumFields &adj, const MediumFields &bwd, int nshots,
                           real dt, real vcorr, double *kb, cudaStream_t stream);
// Error word bits: 1 a bounded device wait expired, 2 a non-finite value.
constexpr int kErrWaitTimeout = 1, kErrNonFinite = 2;
// Sets kErrNonFinite in *err when any of p[0, n) is NaN or infinite.
void launch_nonfinite_check(const real *p, size_t n, int *err, cudaStream_t stream);
#ifndef SFB_FP64
void launch_nonfinite_check(const double *p, size_t n, int *err, cudaStream_t stream);
#endif
// Test hook: a bounded mbarrier wait that nothing satisfies, run out after
// `limit_cycles`, recorded in *err as the stiffness kernels record theirs.
void launch_wait_probe(long long limit_cycles, int *err, cudaStream_t stream);
// Frechet kernel accumulation for one medium (P-SV or acoustic) into
// kern[p][3] (FP64, device element order).  a_is_force: the adjoint `a`
// array holds the unassembled force of the fused loop (multiply by M^-1).
void launch_frechet(int medium, int ngll, const Static &st, const MediumFields &adj, const MediumFields &bwd,
                    int nshots, real dt, double *kern, int a_is_force, cudaStream_t stream);

}  // namespace dev
}  // namespace sfb
