// Adjoint / Frechet entry points (combined simulation).
#include "../../../include/specfem_b200.h"

SFB_API int sfb_frechet_compute_derivatives(sfb_context *, double) { return SFB_E_STATE; }
SFB_API int sfb_run_combined(sfb_context *, int, int) { return SFB_E_STATE; }
SFB_API int sfb_set_adjoint_sources(sfb_context *, int, const float *, size_t) { return SFB_E_STATE; }
SFB_API int sfb_get_kernels(const sfb_context *, int, double *, size_t) { return SFB_E_STATE; }
SFB_API int sfb_copy_forward_to_backward(const sfb_context *, sfb_context *) { return SFB_E_STATE; }
