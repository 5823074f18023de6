// Temporary: families not yet built report so loudly.
#include "fast.h"
namespace ae {
void destroy_wavefront(Ctx *) {}
void destroy_deferred(Ctx *) {}
int render_deferred(Ctx *c, const ae_gbuffer *) { return c->fail(AE_ERR_STATE, "deferred resolve not built"); }
int render_wavefront(Ctx *c) { return c->fail(AE_ERR_STATE, "wavefront not built"); }
int read_image_extra(Ctx *c, int which, void *, size_t) { return c->fail(AE_ERR_INVALID, "unknown image %d", which); }
}
extern "C" int ae_build_gbuffer(ae_ctx *) { return AE_ERR_STATE; }
extern "C" int ae_any_hit(ae_ctx *, const ae_ray *, const float *, uint32_t, uint8_t *) { return AE_ERR_STATE; }
extern "C" int ae_refit_instances(ae_ctx *, const ae_instance *, uint32_t) { return AE_ERR_STATE; }
