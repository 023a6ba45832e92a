// Host-side launchers of the step kernels (eb_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include "eb_types.h"

namespace eb {
void launch_update(const PopDev &P, const NetDev &N, int rel, cudaStream_t st);
constexpr int kPostThreads = 256;  // plastic synapses per post-STDP work item
void launch_push(const PopDev &P, const NetDev &N, int rel, double inv_dt, int blocks, int threads, cudaStream_t st);
void launch_input_push(const NetDev &N, int rel, double inv_dt, int blocks, int threads, cudaStream_t st);
void launch_post_stdp(const PopDev &P, const NetDev &N, int rel, int max_chunks, int blocks, cudaStream_t st);
void launch_advance(int64_t *step, int K, cudaStream_t st);
}  // namespace eb
