// The reference's time loops (include/solver/time_marching.tpp:9-124 forward,
// :126-247 combined) written against the C++ adapter of include/
// specfem_b200.hpp, with the reference's degree-of-freedom and element
// accounting after every step.  Test driver:
//
//   time_marching_b200 forward  <parameter file> <seismogram directory>
//   time_marching_b200 combined <parameter file> <forward wavefield directory>
//                               <kernel directory> <seismogram directory>
//   time_marching_b200 info     <parameter file>        (no device use)
//
// `combined` reads the forward wavefield a forward run wrote, runs the
// adjoint + backward loop with the parameter file's adjoint sources and
// writes the kernels and the backward seismograms.  Exit status 0 on success; a failed
// accounting check or library error prints the message and exits 1.
#include <cstdio>
#include <sstream>
#include <stdexcept>
#include <string>

#include "../../include/specfem_b200.hpp"

using namespace specfem_b200;

namespace {

void accounting(int dofs, int want_dofs, int elements, int want_elements) {
  if (dofs != want_dofs) {
    std::ostringstream m;
    m << "The time loop has not updated all the degrees of freedom. Only " << dofs << " out of " << want_dofs
      << " degrees of freedom have been updated.";
    throw std::runtime_error(m.str());
  }
  if (elements != want_elements) {
    std::ostringstream m;
    m << "The time loop has not updated all the elements. Only " << elements << " out of " << want_elements
      << " elements have been updated.";
    throw std::runtime_error(m.str());
  }
}

constexpr auto acoustic = medium_tag::acoustic;
constexpr auto elastic_psv = medium_tag::elastic_psv;
constexpr auto elastic_sh = medium_tag::elastic_sh;

void run_forward(const context &ctx) {
  domain_kernels_b200<wavefield::forward> kernels(ctx);
  newmark_b200 ts(ctx, simulation::forward);
  kernels.initialize(ts.get_timestep());
  const int total_dofs = 2 * ctx.total_degrees_of_freedom();
  const int total_elements = ctx.total_number_of_elements();
  for (const auto &step : ts.iterate_forward()) {
    const int istep = step.first;
    int dofs = 0, elements = 0;
    dofs += ts.apply_predictor_phase_forward(acoustic);
    dofs += ts.apply_predictor_phase_forward(elastic_psv);
    dofs += ts.apply_predictor_phase_forward(elastic_sh);
    elements += kernels.update_wavefields<acoustic>(istep);
    dofs += ts.apply_corrector_phase_forward(acoustic);
    elements += kernels.update_wavefields<elastic_psv>(istep);
    elements += kernels.update_wavefields<elastic_sh>(istep);
    dofs += ts.apply_corrector_phase_forward(elastic_psv);
    dofs += ts.apply_corrector_phase_forward(elastic_sh);
    if (ts.compute_seismogram(istep)) {
      kernels.compute_seismograms(ts.get_seismogram_step());
      ts.increment_seismogram_step();
    }
    accounting(dofs, total_dofs, elements, total_elements);
  }
  check(ctx.get(), sfb_synchronize(ctx.get()));
}

void run_combined(const context &ctx) {
  domain_kernels_b200<wavefield::adjoint> adjoint_kernels(ctx);
  domain_kernels_b200<wavefield::backward> backward_kernels(ctx);
  frechet_kernels_b200 frechet_kernels(ctx);
  newmark_b200 ts(ctx, simulation::combined);
  adjoint_kernels.initialize(ts.get_timestep());
  backward_kernels.initialize(ts.get_timestep());
  const int nstep = ts.get_max_timestep();
  const int total_dofs = 4 * ctx.total_degrees_of_freedom();
  const int total_elements = 2 * ctx.total_number_of_elements();
  for (const auto &step : ts.iterate_backward()) {
    const int istep = step.first;
    const double dt = step.second;
    int dofs = 0, elements = 0;
    dofs += ts.apply_predictor_phase_forward(acoustic);
    dofs += ts.apply_predictor_phase_forward(elastic_psv);
    dofs += ts.apply_predictor_phase_forward(elastic_sh);
    elements += adjoint_kernels.update_wavefields<acoustic>(istep);
    dofs += ts.apply_corrector_phase_forward(acoustic);
    elements += adjoint_kernels.update_wavefields<elastic_psv>(istep);
    elements += adjoint_kernels.update_wavefields<elastic_sh>(istep);
    dofs += ts.apply_corrector_phase_forward(elastic_psv);
    dofs += ts.apply_corrector_phase_forward(elastic_sh);
    dofs += ts.apply_predictor_phase_backward(elastic_psv);
    dofs += ts.apply_predictor_phase_backward(acoustic);
    elements += backward_kernels.update_wavefields<elastic_psv>(istep);
    elements += backward_kernels.update_wavefields<elastic_sh>(istep);
    dofs += ts.apply_corrector_phase_backward(elastic_psv);
    dofs += ts.apply_corrector_phase_backward(elastic_sh);
    elements += backward_kernels.update_wavefields<acoustic>(istep);
    dofs += ts.apply_corrector_phase_backward(acoustic);
    if (istep == nstep - 1) check(ctx.get(), sfb_load_backward_from_forward(ctx.get()));
    frechet_kernels.compute_derivatives(dt);
    if (ts.compute_seismogram(istep)) {
      backward_kernels.compute_seismograms(ts.get_seismogram_step());
      ts.increment_seismogram_step();
    }
    accounting(dofs, total_dofs, elements, total_elements);
  }
  check(ctx.get(), sfb_synchronize(ctx.get()));
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s forward|combined|info <parameter file> [directories]\n", argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  try {
    context ctx = context::from_yaml(argv[2]);
    const sfb_info info = ctx.info();
    if (mode == "info") {
      std::printf("nspec %d nstep %d dofs %d\n", info.nspec, info.nstep, ctx.total_degrees_of_freedom());
      return 0;
    }
    if (mode == "forward" && argc >= 4) {
      run_forward(ctx);
      check(ctx.get(), sfb_write_seismograms(ctx.get(), SFB_WAVEFIELD_FORWARD, 0, argv[3]));
      return 0;
    }
    if (mode == "combined" && argc >= 6) {
      check(ctx.get(), sfb_read_wavefield(ctx.get(), 0, argv[3]));
      run_combined(ctx);
      check(ctx.get(), sfb_write_kernels(ctx.get(), argv[4], 1));
      check(ctx.get(), sfb_write_seismograms(ctx.get(), SFB_WAVEFIELD_BACKWARD, 0, argv[5]));
      return 0;
    }
    std::fprintf(stderr, "bad arguments\n");
    return 2;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}
