// Host-side launchers of the step kernels (eb_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include "eb_types.h"

namespace eb {
// Steps rel+1 .. rel+nsteps after the device step counter.  push_inv_dt > 0: the
// update kernel also fans out the spikes (no launch_push).  With nsteps > 1 the
// population spike list is not kept (the eager post-synaptic and separate fan-out
// kernels cannot follow such a launch).
void launch_update(const PopDev &P, const NetDev &N, int rel, int nsteps, double push_inv_dt, cudaStream_t st);
// Kernel attributes the update launches need (once per device, before launching).
cudaError_t prepare_update_kernels();
constexpr int kPostThreads = 256;  // plastic synapses per post-STDP work item
void launch_push(const PopDev &P, const NetDev &N, int rel, double inv_dt, int blocks, int threads, cudaStream_t st);
void launch_input_push(const NetDev &N, int rel, int nsteps, double inv_dt, int blocks, int threads, cudaStream_t st);
void launch_post_stdp(const PopDev &P, const NetDev &N, int rel, int max_chunks, int blocks, cudaStream_t st);
// Deferred post-synaptic STDP: apply the spikes noted since the last flush to the
// synapses of every neuron with more than keep of them (3 launches).
void launch_flush_post(const PopDev &P, const NetDev &N, int max_chunks, uint32_t keep, int blocks, cudaStream_t st);
void launch_advance(int64_t *step, int K, cudaStream_t st);

constexpr int kMaxPersistPops = 16;
// Host-built description of one network for the persistent kernel.
struct PersistInfo {
    int n_pops;                       // model populations (PopDev array order)
    int has_inputs, inputs_concurrent;
    unsigned has_out, has_plastic;    // bit q: population q
    int post_chunks[kMaxPersistPops];
    double inv_dt;
    int order[kMaxPersistPops];       // phase-A population order (wide populations first)
    int n_wide;                       // number of wide populations at the front of order
    unsigned *bar;                    // grid barrier words (generation, root, group counters)
    unsigned long long *queue;        // item counters [step parity][phase], 128 bytes apart
    unsigned long long *tl;           // optional timeline [tl_steps][4][grid] (globaltimer ns)
    int tl_steps;
    unsigned long long spin_limit;    // polls of a grid-barrier wait before it reports a timeout
    int withhold;                     // block 0 does not arrive at barriers (exercises the timeout)
};
constexpr unsigned long long kBarrierSpinLimit = 1ull << 24;
int persist_class_of(int kind, int integ);
int persistent_blocks_per_sm(int cls);
cudaError_t launch_persistent(int cls, const PopDev *pops, const PersistInfo &I, const NetDev &N, int K, int grid,
                              cudaStream_t st);
}  // namespace eb
