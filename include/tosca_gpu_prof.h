/*
 * tosca_gpu_prof.h -- instrumentation of the B200 TOSCA time-step library.
 *
 * No counterpart in the reference: TOSCA times whole stages with PetscTime
 * prints. When enabled, the library brackets its main kernels with CUDA events
 * on the context's stream and accumulates per-kernel launch counts and device
 * milliseconds; tg_prof_get reads one accumulated record.
 */
#ifndef TOSCA_GPU_PROF_H
#define TOSCA_GPU_PROF_H

#include "tosca_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

tg_status tg_prof_enable(tg_ctx *ctx, int32_t on);
tg_status tg_prof_reset(tg_ctx *ctx);
int32_t   tg_prof_count(tg_ctx *ctx);
/* name: caller buffer of >= 64 bytes */
tg_status tg_prof_get(tg_ctx *ctx, int32_t index, char *name, int64_t *launches, double *milliseconds);

#ifdef __cplusplus
}
#endif

#endif
