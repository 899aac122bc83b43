// ff_envmap.cu — environment-map importance tables (filled in with the wavefront stages).
#include "ff_internal.h"

void ff_build_env_tables(ff_context* ctx, ff_scene* s) { (void)ctx; (void)s; }
