// unet.cu — learned initial guess for the Poisson solve (placeholder until the
// conv kernels land): reports that no network is available.
#include "internal.cuh"

namespace fopis {
void unet_free(Ctx& c) { c.unet = nullptr; }
int unet_set_training(Ctx& c, int enable, double lr) {
    (void)c; (void)enable; (void)lr;
    throw ApiError{FOPIS_ERR_STATE, "learned guess not built"};
}
int unet_get_state(Ctx& c, double* loss, int64_t* steps) {
    (void)c;
    if (loss) *loss = 0.0;
    if (steps) *steps = 0;
    return FOPIS_OK;
}
int unet_predict(Ctx& c) { (void)c; return 0; }
void unet_observe(Ctx& c) { (void)c; }
}  // namespace fopis
