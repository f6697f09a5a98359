// Entry points whose device code lives elsewhere are declared in yr.h;
// this file holds the ones not yet implemented, which fail loudly.
#include "scene.h"

extern "C" {
YR_API uint32_t yr_param_count(const yr_scene *scene) { return 0; }
YR_API yr_status yr_params_get(const yr_scene *scene, float *params) { return YR_ERR_UNSUPPORTED; }
YR_API yr_status yr_params_set(yr_scene *scene, const float *params) { return YR_ERR_UNSUPPORTED; }
YR_API yr_status yr_backward(yr_scene *scene, const yr_backward_desc *desc, float *dparams, float *loss_out,
                             void *stream) {
    return YR_ERR_UNSUPPORTED;
}
}
