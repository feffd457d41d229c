// Discrete adjoint (gradient) path: placeholder entry point until the adjoint kernels land.
#include <cstring>

#include "../../include/eikcuda.h"
#include "runtime.hpp"

using namespace eik;

extern "C" int eik_gradient(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc,
                            const int64_t* rec_off, const double* rec, const double* pickobs,
                            const double* stdobs, int32_t whichgrad, const eik_extra* ep, double* gradvel,
                            double* gradsrc, double* misfit, eik_stats* stats) {
  (void)model; (void)nsrc; (void)coordsrc; (void)rec_off; (void)rec; (void)pickobs; (void)stdobs;
  (void)whichgrad; (void)ep; (void)gradvel; (void)gradsrc; (void)misfit; (void)stats;
  return fail(ctx, EIK_ERR_UNSUPPORTED, "eik_gradient: not built yet");
}
