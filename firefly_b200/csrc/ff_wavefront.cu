// ff_wavefront.cu — wavefront stages (filled in next).
#include "ff_internal.h"

extern "C" {

ff_status ff_render(ff_context* ctx, ff_scene* scene, const ff_render_settings* settings, ff_film* film,
                    ff_render_stats* stats)
{
    (void)scene; (void)settings; (void)film; (void)stats;
    if (!ctx) return FF_ERR_INVALID_ARG;
    ctx->last_error = "ff_render is not available in this build";
    return FF_ERR_UNSUPPORTED;
}

ff_status ff_scene_read_env_tables(const ff_scene* scene, double* marginal, double* conditional, float* pdf,
                                   double* pdf_denom)
{
    (void)scene; (void)marginal; (void)conditional; (void)pdf; (void)pdf_denom;
    return FF_ERR_UNSUPPORTED;
}

}
