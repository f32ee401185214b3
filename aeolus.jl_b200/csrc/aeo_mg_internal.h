// aeo_mg_internal.h -- the multigrid-preconditioned CG handle as the pressure
// solver of the stepping engine (C++ linkage, not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include "../../include/aeolus_b200_mgpcg.h"

// the handle's device right-hand side b and solution x (nx*ny*nz FP64 each)
aeo_status aeo_mg_buffers(aeo_mg* h, double** b, double** x);
// x = A^-1 b (zero first guess), enqueued on s: no host synchronisation
aeo_status aeo_mg_launch(aeo_mg* h, cudaStream_t s);
// x = A^-1 b enqueued on s; when s is capturing, the solve's nodes (its
// conditional CG loop included) are captured into s's graph
aeo_status aeo_mg_enqueue(aeo_mg* h, cudaStream_t s);
// the work queued on the handle's own stream precedes what s runs next
aeo_status aeo_mg_order_before(aeo_mg* h, cudaStream_t s);
// the statistics of the last solve (synchronises the device)
aeo_status aeo_mg_read_stats(aeo_mg* h, aeo_mg_stats* o);
// kernels one solve of `iterations` CG iterations launches (graph nodes)
int aeo_mg_launches_per_solve(const aeo_mg* h, int iterations);
