// A simulator's shot as resumable work units (used by the shot server).
// Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/tti_capi.h"

namespace tti {

// tti_sim_create with every device allocation of the simulator (and of its
// model upload) taken from `pool` (nullptr: the device's default pool).
int sim_create_in_pool(const tti_sim_config* cfg, cudaMemPool_t pool, tti_sim** out);

// Observed traces (nt*nrec, host) for the adjoint's residual; nullptr = zero.
int shot_upload_observed(tti_sim* s, const float* host_obs);
// Reset the state and start at forward step 0 (fused, snapshots, model set).
int shot_begin(tti_sim* s);
// Enqueue up to max_units units on st (capturable); *done = units enqueued.
int shot_advance(tti_sim* s, cudaStream_t st, int64_t max_units, int64_t* done);
int64_t shot_units_left(const tti_sim* s);
bool shot_done(const tti_sim* s);
cudaStream_t shot_stream(const tti_sim* s);
// Synthetic traces of the last forward pass (nt*nrec) to host memory.
int shot_read_traces(tti_sim* s, float* host);
// After the enqueued work has completed: the status of its kernels.
int shot_end(tti_sim* s);

} // namespace tti
