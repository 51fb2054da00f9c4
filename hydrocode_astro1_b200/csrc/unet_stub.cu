// unet_stub.cu -- placeholder for the learned warm start.
#include "hc_internal.cuh"
void hc_unet_free(void *) {}
extern "C" int hc_unet_param_count(void) { return 0; }
extern "C" int hc_unet_load(hc_ctx *, const uint16_t *, int) { return HC_ERR_STATE; }
extern "C" int hc_unet_load_file(hc_ctx *, const char *) { return HC_ERR_STATE; }
