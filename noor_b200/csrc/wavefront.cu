// Persistent wavefront integrator (placeholder entry points until the
// wavefront kernels land).
#include "host_common.h"
#include "runtime.h"

namespace nb {
void wavefront_release(Context& C) { (void)C; }
}  // namespace nb

extern "C" int noor_wavefront_render(const noor_wf_frame* frames, uint32_t n_frames, const noor_wf_params* params) {
    (void)frames; (void)n_frames; (void)params;
    return set_error(NOOR_ERR_UNSUPPORTED, "wavefront integrator not built yet");
}
extern "C" int noor_wavefront_autotune(const noor_wf_frame* frames, uint32_t n_frames, noor_wf_params* best,
                                       float* best_ms) {
    (void)frames; (void)n_frames; (void)best; (void)best_ms;
    return set_error(NOOR_ERR_UNSUPPORTED, "wavefront integrator not built yet");
}
extern "C" int noor_adjoint_forward(const noor_adjoint_desc* desc, float* d_image) {
    (void)desc; (void)d_image;
    return set_error(NOOR_ERR_UNSUPPORTED, "adjoint not built yet");
}
extern "C" int noor_adjoint_backward(const noor_adjoint_desc* desc, const float* d_grad_image, float* d_grad_albedo,
                                     float* d_grad_roughness, float* d_grad_env) {
    (void)desc; (void)d_grad_image; (void)d_grad_albedo; (void)d_grad_roughness; (void)d_grad_env;
    return set_error(NOOR_ERR_UNSUPPORTED, "adjoint not built yet");
}
