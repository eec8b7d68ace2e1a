/*
 * specfem_b200.h -- C ABI of the B200-native SEM time-marching path.
 *
 * The library replaces the device side of SPECFEM++'s 2D time-marching path:
 * `specfem::kokkos_kernels::domain_kernels`, the Newmark `time_scheme`,
 * `specfem::kokkos_kernels::frechet_kernels` and the loop of
 * `specfem::solver::time_marching`.  The reference interfaces are C++ class
 * templates; each entry point below names the member function it stands in
 * for.  All entry points return 0 on success and a negative SFB_E* code on
 * failure; sfb_last_error() gives the message.  Buffers passed in are
 * caller-owned host memory; device memory is owned by the context.  One
 * context = one CUDA stream; a context is not thread-safe.  A context lives
 * on the CUDA device current when it first touches the GPU; the library
 * keeps per-process launch settings (SM count, occupancy) of the first
 * device it sees, so use one process per GPU (the multi-GPU layout of this
 * library).  Work on a context is asynchronous on its stream except where an
 * entry point says it returns host data; the run drivers synchronise before
 * they return.  The time-step kernels are launched with programmatic
 * dependent launch (each waits on its predecessor in the stream before
 * touching a field); the environment variable SFB_PROGRAMMATIC_LAUNCH=0,
 * read once per process, selects plain stream order instead.
 *
 * Integer tags equal the reference's enum ordinals:
 *   medium   (include/enumerations/medium.hpp:39):  0 elastic_psv,
 *            1 elastic_sh, 3 acoustic
 *   boundary (include/enumerations/medium.hpp:61):  0 none,
 *            1 acoustic_free_surface, 2 stacey, 3 composite_stacey_dirichlet
 *   seismogram type (include/enumerations/wavefield.hpp:17): 0 displacement,
 *            1 velocity, 2 acceleration, 3 pressure
 *   wavefield (include/enumerations/wavefield.hpp simulation_field):
 *            0 forward, 1 adjoint, 2 backward
 */
#ifndef SPECFEM_B200_H
#define SPECFEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#define SFB_API extern "C" __attribute__((visibility("default")))
#else
#define SFB_API __attribute__((visibility("default")))
#endif

#define SFB_OK 0
#define SFB_E_INVALID -1     /* bad argument / unsupported configuration      */
#define SFB_E_CUDA -2        /* CUDA runtime error                             */
#define SFB_E_IO -3          /* file not found / unreadable / malformed        */
#define SFB_E_STATE -4       /* call out of order (e.g. step before init)      */
#define SFB_E_ACCOUNTING -5  /* DOF / element accounting mismatch              */
#define SFB_E_NONFINITE -6   /* wavefield watchdog saw NaN/Inf                 */
#define SFB_E_NOMEM -7       /* device allocation failed                       */

#define SFB_MEDIUM_ELASTIC_PSV 0
#define SFB_MEDIUM_ELASTIC_SH 1
#define SFB_MEDIUM_ACOUSTIC 3

#define SFB_WAVEFIELD_FORWARD 0
#define SFB_WAVEFIELD_ADJOINT 1
#define SFB_WAVEFIELD_BACKWARD 2

typedef struct sfb_context sfb_context;

/* ---------------------------------------------------------------------------
 * Problem description for a structured mesh (the benchmark workloads).  The
 * reference builds the same objects from xmeshfem2D output
 * (src/io/mesh/impl/fortran/dim2/mesh.cpp:26) and the YAML source / station
 * files (src/io/sources.cpp:25, src/io/receivers.cpp).
 * ------------------------------------------------------------------------- */
typedef struct sfb_material {
  double rho, vp, vs; /* vs == 0 marks an acoustic material */
} sfb_material;

typedef struct sfb_source_desc {
  int kind;        /* 0 force, 1 moment tensor, 2 user-defined (Lagrange
                      weights in every component, src/source/external.cpp) */
  int shot;        /* shot index in [0, nshots)                              */
  int wavefield;   /* 0: forward (backward in combined runs), 1: adjoint     */
  int stf;         /* 0 Ricker, 1 Dirac, 2 dGaussian, 3 table                */
  double x, z;
  double angle;    /* force direction in degrees (0 = -z, as the reference)  */
  double mxx, mzz, mxz;
  double f0, tshift, factor;
  const float *stf_table; /* stf == 3: [nstep][ncomp] samples, else NULL     */
} sfb_source_desc;

typedef struct sfb_receiver_desc {
  const char *network, *station;
  double x, z, angle;
} sfb_receiver_desc;

typedef struct sfb_structured_desc {
  int nx, nz;                  /* elements along x and z                    */
  double x0, x1, z0, z1;       /* domain                                    */
  int absorb[4];               /* Stacey on bottom, right, top, left        */
  int ngll;                    /* 5 (GLL4)                                  */
  int elastic_sh;              /* 1: elastic elements carry SH waves        */
  int nmaterials;
  const sfb_material *materials;
  const int *element_material; /* [nx*nz], element ispec = iz*nx + ix       */
  /* Optional per-GLL-point model [nx*nz][ngll][ngll] (NULL = per element). */
  const float *gll_rho, *gll_vp, *gll_vs;
  double dt;
  int nstep;
  double t0;                   /* 0: derive from sources (reference rule)   */
  int nshots;                  /* independent wavefields advanced together  */
  int nsources;
  const sfb_source_desc *sources;
  int nreceivers;
  const sfb_receiver_desc *receivers;
  int nseismogram_types;
  const int *seismogram_types;
  int nstep_between_samples;
  int simulation;              /* 0 forward, 1 combined (adjoint+backward)  */
  int save_boundary_values;    /* forward: keep the Stacey replay store     */
} sfb_structured_desc;

/* ---- context life cycle (replaces specfem::compute::assembly) ---------- */

/* Build from a reference YAML parameter file (src/specfem2d.cpp:3-38,
 * src/parameter_parser/setup.cpp): reads the mesh database, sources and
 * stations it names.  `default_file` may be NULL. */
SFB_API int sfb_create_from_yaml(const char *parameter_file,
                                 const char *default_file, sfb_context **out);
SFB_API int sfb_create_structured(const sfb_structured_desc *desc,
                                  sfb_context **out);
SFB_API void sfb_destroy(sfb_context *ctx);
/* Message of the last failure on `ctx` (or of the last failed create when
 * ctx is NULL).  Valid until the next call on the same context. */
SFB_API const char *sfb_last_error(const sfb_context *ctx);

typedef struct sfb_info {
  int ngll, nspec, nshots, nstep, nstep_between_samples, max_sig_step;
  int nglob[4];          /* DOF points per medium tag                        */
  int nelements[4];      /* elements per medium tag                          */
  int nreceivers, nseismogram_types, nsources;
  int simulation;        /* 0 forward, 1 combined                            */
  double dt, t0;
  size_t device_bytes;   /* device memory held by the context                */
  uint64_t kernel_launches; /* kernels this context has launched so far      */
  int stiffness_variant[4]; /* stiffness kernel per medium tag, 0 not chosen
                               yet; nshots > 1: 1 two shots per lane in packed
                               FP32x2, 2 two shots per lane scalar, 3 one shot
                               per lane; nshots == 1: 1 row kernel with
                               32-element chunks, 2 with 16 (NGLL 5), 3 the
                               compact-block kernel of a medium whose
                               elements are all affine (NGLL 5)             */
  int private_points;    /* P-SV points updated inside the batched stiffness
                            launch of the forward run (0: none)             */
  int nadjoint_sources;  /* adjoint sources given in the sources file        */
} sfb_info;
SFB_API int sfb_get_info(const sfb_context *ctx, sfb_info *info);

/* Stiffness kernel of `medium` (values of sfb_info.stiffness_variant;
 * 0 = let the autotuner choose).  The autotuner runs once, when the forward
 * fields are first allocated, and times every variant on this mesh; a
 * variant set before that is kept (the compact-block variant on a medium
 * that is not all affine, or at NGLL 8, becomes variant 1).  No reference
 * counterpart
 * (the reference's chunk size is a compile-time constant). */
SFB_API int sfb_set_stiffness_variant(sfb_context *ctx, int medium, int variant);

/* Deterministic assembly (no reference counterpart; the reference scatters
 * with Kokkos::atomic_add, include/compute/fields/data_access.tpp:683-720,
 * whose summation order changes from run to run).  enable = 1: the
 * elements of each medium are coloured so that no two elements of a colour
 * share a point and each colour is its own stiffness launch, point sources
 * and coupling are summed per target point in a fixed order, seismograms
 * come from the receiver kernel's fixed-order sums and the mass matrix is
 * accumulated colour by colour: the same inputs give bit-identical fields,
 * seismograms and kernels on every run (on the same GPU and build).  The
 * compact block of affine elements is not used in this mode.  Call before
 * the context's first device use; SFB_E_STATE afterwards.  New contexts
 * start in this mode when the environment sets SFB_DETERMINISTIC=1. */
SFB_API int sfb_set_deterministic(sfb_context *ctx, int enable);

/* Kahan-compensated Newmark sums (enable != 0) in the fused forward driver
 * (sfb_run_forward): the corrector and predictor additions to v and u carry
 * their FP32 rounding error forward in two extra device arrays per medium
 * (8 bytes per DOF and shot).  Compensation starts from zero when enabled;
 * the reference-granularity entry points and the combined run are not
 * compensated.  No reference counterpart (the reference sums in plain
 * type_real, newmark.tpp:44-47, 98-105). */
SFB_API int sfb_set_newmark_compensation(sfb_context *ctx, int enable);

/* Forward snapshots for the combined run: every `interval` steps the forward
 * run keeps (u at that step, v half a step later) of every shot in device
 * memory, and the combined run restores the backward wavefield from them
 * when it reaches that step, so the reconstructed backward wavefield carries
 * at most `interval` steps of FP32 reversal error.  0 (default) = pure
 * reconstruction from the last forward state and the Stacey store, the
 * reference's scheme (time_marching.tpp:126-247).  Memory: 2 (nstep - 2) /
 * interval copies of u.  Set before the forward run. */
SFB_API int sfb_set_checkpoint_interval(sfb_context *ctx, int interval);

/* ---- domain_kernels (include/kokkos_kernels/domain_kernels.hpp) -------- */

/* domain_kernels::initialize(dt) (:136-163): mass matrix (FP64 accumulation,
 * FP32 inverse) for every medium of `wavefield`. */
SFB_API int sfb_domain_initialize(sfb_context *ctx, int wavefield, double dt);
/* domain_kernels::update_wavefields<medium>(istep) (:68-126): coupling,
 * sources, stiffness (+ Stacey / free surface), divide by mass.  Writes the
 * number of elements updated. */
SFB_API int sfb_domain_update_wavefields(sfb_context *ctx, int wavefield,
                                         int medium, int istep,
                                         int *elements_updated);
/* domain_kernels::compute_seismograms(isig_step) (:175-186). */
SFB_API int sfb_domain_compute_seismograms(sfb_context *ctx, int wavefield,
                                           int isig_step);

/* ---- time_scheme::newmark (include/timescheme/newmark.tpp) ------------- */

/* apply_predictor_phase_{forward,backward}(medium) (:60-117, :221-242) and
 * apply_corrector_phase_{forward,backward}(medium) (:11-56, :181-199); the
 * backward wavefield uses -dt.  Writes the number of DOFs updated. */
SFB_API int sfb_newmark_predictor(sfb_context *ctx, int wavefield, int medium,
                                  int *dofs_updated);
SFB_API int sfb_newmark_corrector(sfb_context *ctx, int wavefield, int medium,
                                  int *dofs_updated);

/* ---- frechet_kernels::compute_derivatives(dt)
 *      (include/kokkos_kernels/frechet_kernels.hpp:29-49) ---------------- */
SFB_API int sfb_frechet_compute_derivatives(sfb_context *ctx, double dt);

/* ---- solver::time_marching::run (include/solver/time_marching.tpp) ----- */

/* Forward loop, fused: one stiffness launch per medium and one update
 * launch per step, optionally captured once into a CUDA graph
 * (use_graph != 0).  Runs `nstep` steps starting at the context's current
 * step (`time_marching<forward>::run`, :9-124). */
SFB_API int sfb_run_forward(sfb_context *ctx, int nstep, int use_graph);
/* The same loop through the reference-granularity entry points above
 * (predictor / update_wavefields / corrector per medium), with the
 * reference's DOF and element accounting checks (:90-108). */
SFB_API int sfb_run_forward_unfused(sfb_context *ctx, int nstep);

/* Failure reporting (no reference counterpart).  Device kernels record
 * errors in a per-context error word: a bounded device-side wait that
 * expired (every mbarrier wait of the stiffness kernels gives up after
 * about 2 s), and non-finite values seen by the watchdog, which checks the
 * wavefields (and kernels) at the end of every sfb_run_forward /
 * sfb_run_combined and in sfb_synchronize.  The synchronising calls
 * report them (SFB_E_CUDA for a wait, SFB_E_NONFINITE for NaN / Inf); the
 * reference-granularity entry points (sfb_domain_*, sfb_newmark_*,
 * sfb_frechet_compute_derivatives) report, without synchronising, what
 * earlier launches recorded.  Reporting clears the word.
 * sfb_synchronize waits for the context's stream, runs the watchdog over
 * every allocated wavefield and reports. */
SFB_API int sfb_synchronize(sfb_context *ctx);
/* Test hook: enqueue one bounded mbarrier wait that nothing satisfies,
 * giving up after `limit_cycles` GPU clock cycles ([0, 2^32]) and
 * recording the timeout in the error word exactly as the stiffness
 * kernels do; the next reporting call returns SFB_E_CUDA. */
SFB_API int sfb_probe_device_wait(sfb_context *ctx, long long limit_cycles);
/* Combined adjoint + backward loop with Frechet accumulation
 * (`time_marching<combined>::run`, :126-247).  Needs the forward run's last
 * state and Stacey replay store (sfb_copy_forward_to_backward). */
SFB_API int sfb_run_combined(sfb_context *ctx, int nstep, int use_graph);

/* ---- data movement ------------------------------------------------------ */

/* The combined loop's overwrite of the backward wavefield with the forward
 * "buffer" after its first backward step (time_marching.tpp:198-204), for a
 * host loop driving the domain_* entry points: copies this context's forward
 * wavefield (the forward run's final state, or one read back with
 * sfb_read_wavefield) into its backward wavefield. */
SFB_API int sfb_load_backward_from_forward(sfb_context *ctx);

/* Seismograms [max_sig_step][ntypes][nreceivers][2] per shot, in the
 * reference's receiver frame after the angle rotation; `shot` selects the
 * wavefield copy.  count = number of floats the buffer holds. */
SFB_API int sfb_get_seismograms(const sfb_context *ctx, int wavefield,
                                int shot, float *host, size_t count);
/* Field arrays of one medium: which = 0 displacement, 1 velocity,
 * 2 acceleration, 3 inverse mass; layout [ncomp][nglob] for `shot`. */
SFB_API int sfb_get_field(const sfb_context *ctx, int wavefield, int medium,
                          int which, int shot, float *host, size_t count);
SFB_API int sfb_set_field(sfb_context *ctx, int wavefield, int medium,
                          int which, int shot, const float *host,
                          size_t count);
/* The same reads into FP64 host buffers (no reference counterpart): every
 * bit of the device values in the FP64 verification build
 * (libspecfem_b200_fp64.so, the same kernels compiled with FP64
 * arithmetic); widened FP32 values in the product library. */
SFB_API int sfb_get_seismograms_f64(const sfb_context *ctx, int wavefield,
                                    int shot, double *host, size_t count);
SFB_API int sfb_get_field_f64(const sfb_context *ctx, int wavefield,
                              int medium, int which, int shot, double *host,
                              size_t count);
/* Bytes of the library's arithmetic type: 4 for the product library, 8 for
 * the FP64 verification build. */
SFB_API int sfb_real_bytes(void);
/* Replace the adjoint source time functions (combined runs):
 * [nstep][nreceivers][2] for `shot`, receiver r acting at its station. */
SFB_API int sfb_set_adjoint_sources(sfb_context *ctx, int shot,
                                    const float *host, size_t count);
/* Frechet kernels summed over shots, per local point [nspec][ngll][ngll]:
 * which = 0 rho, 1 mu, 2 kappa, 3 rhop, 4 alpha, 5 beta (elastic) or
 * 0 rho, 1 kappa (acoustic points).  FP64.  which = 6, 7 (after a combined
 * run with sfb_set_stacey_kernels): the Stacey-traction derivatives
 * dchi/d(rho vp), dchi/d(rho vs) per P-SV boundary point (zero elsewhere). */
SFB_API int sfb_get_kernels(const sfb_context *ctx, int which, double *host,
                            size_t count);
/* No reference counterpart: also accumulate, in combined runs, the model
 * derivative of the Stacey traction of the P-SV medium, which the
 * reference's kernels leave out (frechet_derivative.hpp:14-138): per
 * boundary point -dt w |n| sum (s_adj.n^)(v.n^) and
 * -dt w |n| sum (s_adj.v - (s_adj.n^)(v.n^)), the derivatives of the misfit
 * with respect to rho vp and rho vs there (read with sfb_get_kernels 6, 7).
 * With them the gradient is the derivative of the discrete misfit on
 * absorbing meshes; without them it is the reference's. */
SFB_API int sfb_set_stacey_kernels(sfb_context *ctx, int enable);
/* Move the forward run's end state and Stacey replay store into the
 * backward wavefield of `dst` (reference: wavefield writer / reader tasks,
 * include/io/wavefield/{writer,reader}.tpp). */
SFB_API int sfb_copy_forward_to_backward(const sfb_context *src,
                                         sfb_context *dst);
/* Write the seismograms as the reference's ASCII traces
 * (src/io/seismogram/writer.cpp:23-88) into `directory`. */
SFB_API int sfb_write_seismograms(const sfb_context *ctx, int wavefield,
                                  int shot, const char *directory);

/* ---- wavefield / kernel files and the whole-run driver ----------------- */

/* Write shot `shot`'s forward state after the whole forward run to
 * <directory>/ForwardWavefield in the reference's ASCII layout
 * (include/io/wavefield/writer.tpp:14-150): Coordinates/<medium>/{X,Z,mapping}
 * and Step<nstep>/<medium>/{Displacement,Velocity,Acceleration} (acoustic:
 * Potential*), plus Step<nstep>/Boundary/Stacey/{IndexMapping,
 * ElementAcceleration}: this library's boundary store (whole-element
 * contributions of the Stacey elements for every step; the reference stores
 * the Stacey traction alone, under other dataset names).  Needs
 * save_boundary_values when the mesh has Stacey edges. */
SFB_API int sfb_write_wavefield(const sfb_context *ctx, int shot, const char *directory);
/* One more step group, StepNNNNNN for the forward steps run so far, in an
 * existing (or new) ForwardWavefield folder, without removing the steps
 * already there: the reference's periodic wavefield writer
 * (include/periodic_tasks/wavefield_writer.hpp; `time_interval` of the
 * parameter file's writer.wavefield, src/parameter_parser/writer/
 * wavefield.cpp:36-66). */
SFB_API int sfb_write_wavefield_step(const sfb_context *ctx, int shot, const char *directory);
/* Read such a folder back as the forward run's final state and boundary
 * store of shot `shot`, so sfb_run_combined can follow (the reference's
 * wavefield reader, include/io/wavefield/reader.tpp). */
SFB_API int sfb_read_wavefield(sfb_context *ctx, int shot, const char *directory);
/* Write the accumulated kernels to <directory>/Kernels/<medium>_isotropic/
 * {X,Z,rho,mu,kappa,rhop,alpha,beta} (acoustic: rho,kappa,rhop,alpha) as the
 * reference's kernel writer does (include/io/kernel/writer.tpp,
 * include/io/impl/medium_writer.tpp), values in the reference's storage
 * order for an element tile of `element_chunk` elements (1 = its CPU
 * build). */
SFB_API int sfb_write_kernels(const sfb_context *ctx, const char *directory, int element_chunk);
/* The model per local point as the reference's property writer and reader
 * store it (include/io/property/{writer,reader}.tpp): <directory>/
 * Properties/<medium>_isotropic/{X,Z,kappa,mu,rho} (acoustic:
 * {X,Z,rho_inverse,kappa}), same element order and tile layout as the
 * kernels.  Reading replaces the context's model (the mass matrix is rebuilt
 * on the next run); a parameter file selects either with
 * databases.writer.properties / databases.reader.properties. */
SFB_API int sfb_write_properties(const sfb_context *ctx, const char *directory, int element_chunk);
SFB_API int sfb_read_properties(sfb_context *ctx, const char *directory, int element_chunk);
/* Run a parameter file end to end as the reference's specfem2d does
 * (src/execute.cpp): forward mode runs, writes seismograms and, when asked,
 * the forward wavefield; combined mode reads the wavefield, runs the
 * adjoint + backward loop with the file's adjoint sources and writes the
 * kernels.  Errors: sfb_last_error(NULL). */
SFB_API int sfb_execute(const char *parameter_file, const char *default_file);
/* The same with the parameter and default dictionaries as YAML text, as the
 * reference's Python entry point takes them (specfempp_core._execute,
 * src/python/core.cpp:46-66); paths inside are relative to the working
 * directory. */
SFB_API int sfb_execute_text(const char *parameter_yaml, const char *default_yaml);
SFB_API int sfb_create_from_yaml_text(const char *parameter_yaml,
                                      const char *default_yaml,
                                      sfb_context **out);

/* Replace the source time function of source `isource` ([nstep][2] samples,
 * the second column only used by two-component media).  The reference's
 * counterpart is an `external` source time function
 * (src/source_time_function/external.cpp). */
SFB_API int sfb_set_source_time_function(sfb_context *ctx, int isource,
                                         const float *host, size_t count);

/* ---- measurement hooks (no reference counterpart) ----------------------- */

/* The CUDA stream all work of `ctx` is enqueued on (cudaStream_t). */
SFB_API int sfb_get_stream(const sfb_context *ctx, void **stream);
/* Launch the stiffness kernel of `medium` (forward wavefield) `reps` times on
 * the context stream between two CUDA events and report the mean duration in
 * milliseconds.  The force accumulator is cleared afterwards, so a run can
 * follow. */
SFB_API int sfb_time_stiffness(sfb_context *ctx, int medium, int reps,
                               double *mean_ms);

/* Replace the model, per local point [nspec][ngll][ngll] (density, P and S
 * velocity; S ignored in acoustic elements), as the reference's property
 * reader does (include/io/property/reader.tpp:17-44).  Fields are not
 * touched; the mass matrix is rebuilt on the next run. */
SFB_API int sfb_set_model(sfb_context *ctx, const float *rho, const float *vp,
                          const float *vs, size_t count);
/* Zero every wavefield, the seismograms, the Stacey store and the Frechet
 * kernels, and rewind the step counters (a new simulation on the same
 * mesh). */
SFB_API int sfb_reset(sfb_context *ctx);

/* ---- problem export (host arrays; valid while the context lives) ------- */

/* Flat host view of the assembled problem, for checkers and tools that need
 * the same discrete inputs the device kernels read. */
typedef struct sfb_problem_view {
  int ngll, nspec, nshots, nstep, nstep_between_samples;
  double dt, t0;
  const double *xi, *wgll, *hprime; /* [ngll], [ngll], [ngll*ngll] l_j'(xi_i) */
  const int *medium;                /* [nspec]                                */
  const int *iglob;                 /* [nloc] index in own medium's field    */
  int nglob[4];
  const float *xix, *xiz, *gammax, *gammaz, *jacobian;   /* [nloc] */
  const float *kappa, *mu, *rho, *rho_inverse;           /* [nloc] */
  const uint8_t *bnd;               /* [nloc] bit0 Stacey, bit1 free surface */
  const float *bnd_nx, *bnd_nz, *bnd_w;                  /* [nloc] */
  int ncouple_acoustic, ncouple_elastic;
  const int *couple_acoustic_self, *couple_acoustic_other; /* iglob pairs    */
  const float *couple_acoustic_factor, *couple_acoustic_nx, *couple_acoustic_nz;
  const int *couple_elastic_self, *couple_elastic_other;
  const float *couple_elastic_factor, *couple_elastic_nx, *couple_elastic_nz;
  int nsources;
  const int *src_ispec, *src_shot, *src_wavefield;       /* [nsources]      */
  const float *src_array;           /* [nsources][2][ngll][ngll]             */
  const float *src_stf;             /* [nsources][nstep][2]                  */
  int nreceivers;
  const int *rec_ispec;             /* [nreceivers]                          */
  const float *rec_lagrange;        /* [nreceivers][ngll][ngll]              */
  const float *rec_sin, *rec_cos;   /* [nreceivers]                          */
  int nseismogram_types;
  const int *seismogram_types;
} sfb_problem_view;
SFB_API int sfb_get_problem_view(const sfb_context *ctx,
                                 sfb_problem_view *view);

/* ---- assembly without device allocation -------------------------------- */

/* No counterpart in the reference.  Assembles the mass matrix of one medium
 * in FP64 and writes its FP32 inverse, for callers that cannot allocate
 * device memory where they need it: a host framework that hands out every
 * device buffer from its own pool and forbids plugins from calling
 * cudaMalloc, or a real-time loop that must not touch the allocator (a
 * cudaMalloc can synchronise the device).  The caller passes device inputs
 * (per local point of the medium's `nelem` elements, point
 * p = (e * ngll + iz) * ngll + ix: the medium-local point index, the
 * Jacobian, the material -- P-SV: kappa, mu, rho; SH: mu, rho, unused;
 * acoustic: rho_inverse, kappa, unused -- and optionally the Stacey tags /
 * normals / weights, NULL for none), the host GLL weights, and the device
 * output minv[npoints * ncomp] (components interleaved).  Work is enqueued
 * on `stream` (a cudaStream_t, NULL for the default stream).
 * The only scratch is a fixed FP64 device array of SFB_NOALLOC_MAX_DOFS
 * entries (16 MiB) plus one error word, which every GPU loading the library
 * holds until exit; npoints * ncomp above that limit is rejected with
 * SFB_E_INVALID.  The first call on a device looks up the array's address
 * (cudaGetSymbolAddress), so make it before any stream capture; a device
 * reset after it is not supported.  All calls on a device share the array:
 * each call clears what it uses, and calls that overlap on the GPU race.  A
 * point index outside [0, npoints) is skipped on the device and the whole
 * output of that call is set to NaN.  Errors found on the host are reported
 * through sfb_noalloc_last_error(). */
#define SFB_NOALLOC_MAX_DOFS (1 << 21)
SFB_API int sfb_assemble_inverse_mass_noalloc(
    int medium, int ngll, int nelem, int npoints, const int *iglob,
    const float *jacobian, const float *mat0, const float *mat1,
    const float *mat2, const uint8_t *bnd, const float *bnd_nx,
    const float *bnd_nz, const float *bnd_w, const double *wgll, double dt,
    float *minv, void *stream);
SFB_API const char *sfb_noalloc_last_error(void);

#endif /* SPECFEM_B200_H */
