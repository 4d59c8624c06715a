// qk_dist.h -- one batch priced across several GPUs, one rank per GPU.
//
// A plan's tiles are independent given their Philox counters, so a batch
// shards at tile granularity: every rank holds the same plan, simulates a
// contiguous range of its tiles balanced by path-steps (Plan::shard_bounds),
// and the ranges' tile partials are exchanged with one NCCL broadcast per
// rank, grouped into a single collective step on the plan's stream.  Every
// rank then runs the finalize kernel over all options: the partials and the
// merge order are those of a single-GPU execute, so the sharded results equal
// the unsharded ones bit for bit, on every rank.
//
// NCCL is loaded at run time (dlopen of libnccl.so.2, or QK_B200_NCCL_PATH):
// the library has no link-time dependency on it, and without it the calls
// here return QK_ERR_RUNTIME_INIT with "nccl unavailable: ...".
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

struct qk_dist;

namespace qkb {

class Plan;

// This rank's share of `plan` on `stream` (null: the plan's stream): the
// simulate kernels over its tile range, the grouped broadcast of every
// rank's range, the finalize kernel over all options.  Returns a QK_* code
// with the thread's error message set.
int32_t dist_execute(Plan& plan, qk_dist* d, cudaStream_t stream, const char* where);

}  // namespace qkb
