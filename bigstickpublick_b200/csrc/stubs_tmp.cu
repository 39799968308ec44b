#include "bsg_internal.h"
extern "C" int bsg_grad(bsg_ctx *ctx, const double *, int, double *, double *, double *, double *, double *) { return bsg::set_err(ctx, BSG_ERR_UNSUPPORTED, "grad not built"); }
