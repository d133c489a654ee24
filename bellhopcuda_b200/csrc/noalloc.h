// Interface between the context runtime (api.cu) and the allocation-free
// entry point (noalloc.cu).
#pragma once
#include <cuda_runtime.h>

#include "../../include/bhcb.h"
#include "bhcb_internal.h"

namespace bhcb {

struct NoAllocJob {   // one field of a prepared context
    GroupDev group;   // host copy of the trace group that owns the field
    double freq;
    int precision, gaussian, coherent;
    int nsz, nrzp, nrr, sm_count;
    int device;       // the context's GPU: its stream, tables and buffers live there
    cudaStream_t stream;
};

// Describe field (env, ifreq) of a prepared context; reads prepared state only
// (no allocation). Returns a bhcb status and sets *why on failure.
int noalloc_job_from_ctx(bhcb_ctx *ctx, int32_t env, int32_t ifreq, NoAllocJob *job, const char **why);

} // namespace bhcb
