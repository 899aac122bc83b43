// ff_envmap.cu — environment-map importance tables (filled in next).
#include "ff_internal.h"

void ff_build_env_tables(ff_context* ctx, ff_scene* s) { (void)ctx; (void)s; }

extern "C" ff_status ff_scene_read_env_tables(const ff_scene* scene, double* marginal, double* conditional, float* pdf,
                                              double* pdf_denom)
{
    (void)scene; (void)marginal; (void)conditional; (void)pdf; (void)pdf_denom;
    return FF_ERR_UNSUPPORTED;
}
