/* C++ adapter over the C ABI of specfem_b200.h with the shapes of the
 * reference's hot-path classes, so that a time loop written like
 * specfem::solver::time_marching (include/solver/time_marching.tpp:9-247)
 * drives the B200 kernels unchanged:
 *
 *   domain_kernels_b200<W>   specfem::kokkos_kernels::domain_kernels
 *                            (include/kokkos_kernels/domain_kernels.hpp:32-195):
 *                            initialize(dt), update_wavefields<medium>(istep)
 *                            returning the elements updated,
 *                            compute_seismograms(isig_step)
 *   newmark_b200             specfem::time_scheme::newmark
 *                            (include/timescheme/newmark.hpp,
 *                            timescheme.hpp:119-171): apply_{predictor,
 *                            corrector}_phase_{forward,backward}(medium)
 *                            returning the degrees of freedom updated,
 *                            iterate_forward / iterate_backward, the
 *                            seismogram cadence
 *   frechet_kernels_b200     specfem::kokkos_kernels::frechet_kernels
 *                            (include/kokkos_kernels/frechet_kernels.hpp:29-49):
 *                            compute_derivatives(dt)
 *
 * Header only; link against libspecfem_b200.so.  Every call that the
 * library reports as failed throws specfem_b200::error with the library's
 * status code and message.
 */
#ifndef SPECFEM_B200_HPP
#define SPECFEM_B200_HPP

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "specfem_b200.h"

namespace specfem_b200 {

/* The reference's medium and wavefield tags (enum ordinals of
 * include/enumerations/material_definitions.hpp and simulation_field). */
enum class medium_tag : int { elastic_psv = SFB_MEDIUM_ELASTIC_PSV, elastic_sh = SFB_MEDIUM_ELASTIC_SH,
                              acoustic = SFB_MEDIUM_ACOUSTIC };
enum class wavefield : int { forward = SFB_WAVEFIELD_FORWARD, adjoint = SFB_WAVEFIELD_ADJOINT,
                             backward = SFB_WAVEFIELD_BACKWARD };
enum class simulation : int { forward = 0, combined = 1 };

struct error : std::runtime_error {
  int code;
  error(int c, const std::string &msg) : std::runtime_error(msg), code(c) {}
};

inline void check(const sfb_context *ctx, int rc) {
  if (rc != SFB_OK) {
    const char *msg = sfb_last_error(ctx);
    throw error(rc, msg ? msg : "specfem_b200 error");
  }
}

/* Owns one library context (the reference's compute::assembly and the
 * objects read with it). */
class context {
 public:
  static context from_yaml(const std::string &parameter_file, const std::string &default_file = "") {
    sfb_context *c = nullptr;
    check(nullptr, sfb_create_from_yaml(parameter_file.c_str(), default_file.empty() ? nullptr : default_file.c_str(),
                                        &c));
    return context(c);
  }
  context(context &&o) noexcept : ctx_(o.ctx_) { o.ctx_ = nullptr; }
  context &operator=(context &&o) noexcept {
    std::swap(ctx_, o.ctx_);
    return *this;
  }
  context(const context &) = delete;
  context &operator=(const context &) = delete;
  ~context() {
    if (ctx_) sfb_destroy(ctx_);
  }
  sfb_context *get() const { return ctx_; }
  sfb_info info() const {
    sfb_info i;
    check(ctx_, sfb_get_info(ctx_, &i));
    return i;
  }
  /* assembly.get_total_degrees_of_freedom(): sum over media of nglob * ncomp */
  int total_degrees_of_freedom() const {
    const sfb_info i = info();
    return 2 * i.nglob[SFB_MEDIUM_ELASTIC_PSV] + i.nglob[SFB_MEDIUM_ELASTIC_SH] + i.nglob[SFB_MEDIUM_ACOUSTIC];
  }
  /* assembly.get_total_number_of_elements() */
  int total_number_of_elements() const { return info().nspec; }

 private:
  explicit context(sfb_context *c) : ctx_(c) {}
  sfb_context *ctx_;
};

template <wavefield W> class domain_kernels_b200 {
 public:
  explicit domain_kernels_b200(const context &c) : ctx_(c.get()) {}
  void initialize(double dt) { check(ctx_, sfb_domain_initialize(ctx_, static_cast<int>(W), dt)); }
  template <medium_tag M> int update_wavefields(int istep) {
    int n = 0;
    check(ctx_, sfb_domain_update_wavefields(ctx_, static_cast<int>(W), static_cast<int>(M), istep, &n));
    return n;
  }
  void compute_seismograms(int isig_step) {
    check(ctx_, sfb_domain_compute_seismograms(ctx_, static_cast<int>(W), isig_step));
  }

 private:
  sfb_context *ctx_;
};

class newmark_b200 {
 public:
  /* forward simulations: the forward phase acts on the forward wavefield;
   * combined simulations: on the adjoint wavefield, and the backward phase
   * on the backward wavefield (include/timescheme/newmark.tpp). */
  newmark_b200(const context &c, simulation type) : ctx_(c.get()), type_(type) {
    const sfb_info i = c.info();
    nstep_ = i.nstep;
    dt_ = i.dt;
    nsbs_ = i.nstep_between_samples;
  }
  int get_max_timestep() const { return nstep_; }
  double get_timestep() const { return dt_; }
  int apply_predictor_phase_forward(medium_tag m) { return call(sfb_newmark_predictor, forward_field(), m); }
  int apply_corrector_phase_forward(medium_tag m) { return call(sfb_newmark_corrector, forward_field(), m); }
  int apply_predictor_phase_backward(medium_tag m) { return call(sfb_newmark_predictor, SFB_WAVEFIELD_BACKWARD, m); }
  int apply_corrector_phase_backward(medium_tag m) { return call(sfb_newmark_corrector, SFB_WAVEFIELD_BACKWARD, m); }
  /* (istep, dt) pairs: forward 0 .. nstep-1, backward nstep-1 .. 0, both
   * with the time step dt (timescheme.hpp:119-146) */
  std::vector<std::pair<int, double>> iterate_forward() const {
    std::vector<std::pair<int, double>> r;
    for (int i = 0; i < nstep_; ++i) r.emplace_back(i, dt_);
    return r;
  }
  std::vector<std::pair<int, double>> iterate_backward() const {
    std::vector<std::pair<int, double>> r;
    for (int i = nstep_ - 1; i >= 0; --i) r.emplace_back(i, dt_);
    return r;
  }
  bool compute_seismogram(int istep) const { return istep % nsbs_ == 0 && seismogram_step_ < nstep_ / nsbs_; }
  int get_seismogram_step() const { return seismogram_step_; }
  void increment_seismogram_step() { ++seismogram_step_; }

 private:
  int forward_field() const { return type_ == simulation::forward ? SFB_WAVEFIELD_FORWARD : SFB_WAVEFIELD_ADJOINT; }
  int call(int (*fn)(sfb_context *, int, int, int *), int w, medium_tag m) {
    int n = 0;
    check(ctx_, fn(ctx_, w, static_cast<int>(m), &n));
    return n;
  }
  sfb_context *ctx_;
  simulation type_;
  int nstep_ = 0, nsbs_ = 1, seismogram_step_ = 0;
  double dt_ = 0;
};

class frechet_kernels_b200 {
 public:
  explicit frechet_kernels_b200(const context &c) : ctx_(c.get()) {}
  void compute_derivatives(double dt) { check(ctx_, sfb_frechet_compute_derivatives(ctx_, dt)); }

 private:
  sfb_context *ctx_;
};

}  // namespace specfem_b200

#endif /* SPECFEM_B200_HPP */
