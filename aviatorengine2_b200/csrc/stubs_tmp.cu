// Entry points whose families are not built yet report so loudly.
#include "fast.h"
namespace ae {
}
extern "C" int ae_any_hit(ae_ctx *, const ae_ray *, const float *, uint32_t, uint8_t *) { return AE_ERR_STATE; }
extern "C" int ae_refit_instances(ae_ctx *, const ae_instance *, uint32_t) { return AE_ERR_STATE; }
