/*
 * edlut_b200 -- C ABI of the B200 time-driven simulation path.
 *
 * Plain C types only (no CUDA or torch types): a host program, a C++ neuron-model
 * plugin, ctypes or any other FFI binds these symbols from libedlut_b200.so.
 * All functions return EB_OK (0) or a negative EB_ERR_* code; eb_last_error()
 * returns a message for the calling thread's last failure.  No C++ exception
 * crosses this boundary and no function calls exit().
 *
 * References are paths in the EDLUT reference tree, relative to its Kernel/
 * directory.
 *
 * Device-resident network: populations, synapses, STDP rules,
 *     input spikes and K-step runs all on the GPU.  Replaces the per-step host work
 *     of the reference engine for time-driven networks: TimeEventUpdateNeurons
 *     (src/simulation/TimeEventUpdateNeurons.cpp:82-116), TimeDrivenInternalSpike
 *     (src/spike/TimeDrivenInternalSpike.cpp:182-253), PropagatedSpikeGroup delivery
 *     (src/spike/PropagatedSpikeGroup.cpp:112-149) and the STDP hooks
 *     (src/learning_rules/STDPWeightChange.cpp:43-76).
 */
#ifndef EDLUT_B200_H
#define EDLUT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EB_OK 0
#define EB_ERR_ARG (-1)        /* bad argument */
#define EB_ERR_CUDA (-2)       /* CUDA runtime failure */
#define EB_ERR_STATE (-3)      /* call made in the wrong phase (e.g. run before finalize) */
#define EB_ERR_OVERFLOW (-4)   /* an arrival bucket, spike list or recording buffer overflowed */
#define EB_ERR_PARSE (-5)      /* .cfg / network / weights / input file error */
#define EB_ERR_UNSUPPORTED (-6)/* model, integrator or synapse type outside this path */
#define EB_ERR_NOMEM (-7)      /* device allocation failed */
#define EB_ERR_NUMERIC (-8)    /* BDF Newton matrix singular (the reference exits the process) */

/* Neuron model kinds: the reference names LIFTimeDrivenModel[_GPU],
 * AdExTimeDrivenModel[_GPU], HHTimeDrivenModel[_GPU] and InputSpikeNeuronModel
 * (src/neuron_model/NeuronModelFactory.cu:85-91,221-257). */
#define EB_INPUT 0
#define EB_LIF 1
#define EB_ADEX 2
#define EB_HH 3
/* PoissonGeneratorDeviceVector (src/neuron_model/PoissonGeneratorDeviceVector.cpp):
 * params = {frequency in Hz}; it samples every 0.1 ms, so the network's other
 * populations must use that step. */
#define EB_POISSON 4
/* Integration methods "Euler", "RK2", "RK4", "BDF"
 * (src/integration_method/IntegrationMethodFactory_GPU_C_INTERFACE.cu:54-97). */
#define EB_EULER 0
#define EB_RK2 1
#define EB_RK4 2
#define EB_BDF 3

typedef struct eb_ctx eb_ctx;

/* Last error message of the calling thread ("" if none). */
const char *eb_last_error(void);
/* Library version string. */
const char *eb_version(void);

/* ----------------------------------------------------------- lifecycle --- */
/* Create a context on CUDA device `device`.  `stream` is a cudaStream_t passed as a
 * pointer (NULL: the library creates its own).  Replaces the per-queue
 * cudaSetDevice + InitializeStatesGPU set-up, src/neuron_model/LIFTimeDrivenModel_GPU_C_INTERFACE.cu:139-194. */
int eb_ctx_create(int device, void *stream, eb_ctx **out);
int eb_ctx_destroy(eb_ctx *ctx);

/* ------------------------------------------------------------- network --- */
/* Append a population (one layer line of the network file, Network::ParseNet,
 * src/spike/Network.cpp:448-484).  params: the model's .cfg values in file order
 * (e.g. LIF: e_exc e_inh e_leak v_thr c_m tau_exc tau_inh tau_ref g_leak tau_nmda,
 * LIFTimeDrivenModel::ParseNeuronModel); dt_s the integration step in seconds as
 * parsed (float).  Input populations (EB_INPUT) take no params.  *out_first gets
 * the population's first global neuron index. */
int eb_add_population(eb_ctx *ctx, int kind, int64_t n, int integrator, int bdf_order,
                      float dt_s, const float *params, int n_params, int64_t *out_first);
/* Additive STDP rule "STDP" with its .cfg values max_LTP tau_LTP max_LTD tau_LTD
 * (taus in seconds), STDPWeightChange::ParseLearningRule,
 * src/learning_rules/STDPWeightChange.cpp:78-99.  *out_rule gets its index. */
int eb_add_stdp_rule(eb_ctx *ctx, float max_ltp, float tau_ltp, float max_ltd, float tau_ltd,
                     int *out_rule);
/* Synapses in network-file order (Network::CreateConnections,
 * src/spike/Network.cpp:790-1014): source, target, delay (s, float as parsed; rounded
 * like RoundPropagationDelay, :1311-1317), type (0 AMPA, 1 GABA, 2 NMDA), weight,
 * max weight, learning rule (-1: none).  May be called once. */
int eb_set_connectivity(eb_ctx *ctx, int64_t m, const int64_t *src, const int64_t *tgt,
                        const float *delay_s, const int32_t *type, const float *weight,
                        const float *max_weight, const int32_t *rule);
/* Per-target bucket capacity limit (arrivals one neuron can take in one step);
 * default min(in-degree x multiplicity, 8192). */
int eb_set_bucket_limit(eb_ctx *ctx, uint32_t max_per_target, uint32_t input_multiplicity);
/* Populations whose largest in-degree exceeds `indegree` (default 1024) update
 * with a block per neuron, the others with a thread per neuron; both give the
 * same results.  0: a block per neuron whenever one step can bring more than 16
 * arrivals to a neuron.  Before eb_finalize. */
int eb_set_wide_indegree(eb_ctx *ctx, int64_t indegree);
/* Build the device network: sort synapses (qsort_inters order,
 * src/spike/Network.cpp:45-68), build source-major and target-major tables, allocate
 * state, buckets and tables.  *out_sorted_perm (m entries, optional) receives the
 * reference's synapse order as original indices. */
int eb_finalize(eb_ctx *ctx, int64_t *out_sorted_perm);
/* Load a reference network file + weights file (Network::ParseNet,
 * src/spike/Network.cpp:422-704); equivalent to the calls above.  Model .cfg paths
 * are resolved like the reference (relative to the current directory, ".cfg" added). */
int eb_load_network_files(eb_ctx *ctx, const char *network_file, const char *weights_file);

/* --------------------------------------------------------------- inputs --- */
/* Spikes of input neurons (InputSpikeNeuronModel), times in seconds as float like
 * FileInputSpikeDriver (src/communication/FileInputSpikeDriver.cpp:45-78) or the
 * ArrayInputSpikeDriver.  Times must not precede the current simulation time. */
int eb_inject_spikes(eb_ctx *ctx, int64_t n, const float *time_s, const int64_t *cell);
/* Load an input-spike file in the reference format. */
int eb_load_input_file(eb_ctx *ctx, const char *input_file);

/* ----------------------------------------------------------------- run --- */
/* Advance n_steps integration steps (each: deliveries, neuron updates, spikes, STDP),
 * replaying captured CUDA graphs of `graph_steps` steps (0: default 512; 1: plain
 * launches; a shorter remainder of 8 steps or more gets a graph of its own).  In a
 * graph each population is a chain of launches, each running up to 8 steps when
 * the delays allow.  Blocks until done.  Replaces the per-step
 * TimeEventUpdateNeurons / TimeDrivenInternalSpike / PropagatedSpikeGroup cycle. */
int eb_run(eb_ctx *ctx, int64_t n_steps);
int eb_set_graph_steps(eb_ctx *ctx, int graph_steps);
/* on != 0: run all phases of up to 1000 steps in one cooperative persistent
 * kernel with bounded grid barriers where the device and network allow (<= 16
 * model populations).  0 (default): per-step kernels replayed as CUDA graphs,
 * which is faster on B200 for the networks measured (a grid barrier over all
 * SMs costs more than the launches it replaces). */
int eb_set_persistent(eb_ctx *ctx, int on);
/* The persistent kernel's grid barriers wait at most spin_limit polls (default
 * 2^24, about a second) before the kernel records a timeout and ends; the run then
 * returns EB_ERR_CUDA, the barrier counters are reset, and the context stays usable
 * (restore a snapshot: the run stopped part-way).  withhold_first_block != 0 makes
 * block 0 skip its barrier arrivals, so every wait runs out: a way to exercise that
 * failure path without a fault. */
int eb_set_barrier_wait(eb_ctx *ctx, uint64_t spin_limit, int withhold_first_block);
/* Timeline of the persistent kernel for the first `steps` steps of each launch:
 * globaltimer (ns) per step, per mark (0 start, 1 phase-A barrier arrival,
 * 2 phase-A barrier exit, 3 phase-B barrier arrival, 4 end of the block's first
 * phase-A item, 5 number of phase-A items of the block) and per block:
 * out[(step * 6 + mark) * grid + block]; *grid receives the block count. */
int eb_set_timeline(eb_ctx *ctx, int steps);
int eb_get_timeline(eb_ctx *ctx, int *grid, unsigned long long *out);
/* Enqueue n_steps on the context stream without synchronizing (error flags are
 * checked by the next eb_sync / eb_run). */
int eb_run_async(eb_ctx *ctx, int64_t n_steps);
int eb_sync(eb_ctx *ctx);

/* -------------------------------------------------------------- outputs --- */
/* Recording buffer capacity in spikes (default 16M). */
int eb_set_record_capacity(eb_ctx *ctx, int64_t cap);
/* Drain recorded spikes (1-based step index, global neuron), sorted by (step, neuron);
 * the ArrayOutputSpikeDriver::GetBufferedSpikes counterpart
 * (src/communication/ArrayOutputSpikeDriver.cpp:56-80).  With cap too small, returns
 * EB_ERR_OVERFLOW and *n the required size without draining. */
int eb_get_spikes(eb_ctx *ctx, int64_t cap, int64_t *n, int64_t *step, int64_t *cell);
/* Drain recorded spikes (as eb_get_spikes) into a text file in the reference's
 * output format, FileOutputSpikeDriver::WriteSpike
 * (src/communication/FileOutputSpikeDriver.cpp:40-46, the -of option): one
 * "%f\t%li" line per spike with the update time of its step and the neuron,
 * sorted by (step, neuron), for the populations whose output flag is set (the
 * output column of the network file's layer line; eb_add_population: set).
 * append != 0 appends to the file.  Spikes of input neurons, which the caller
 * supplied, are not recorded and not written. */
int eb_write_spikes(eb_ctx *ctx, const char *path, int append);
/* Enable conductance types of population `pop` (mask: bit 0 AMPA, 1 GABA, 2 NMDA)
 * beyond those its synapses enable -- for populations that receive arrivals
 * folded in from outside (eb_fold_arrivals), such as the neuron-model plugins of a
 * host engine that delivers spikes itself.  The models integrate and decay the
 * enabled types only, as the reference CPU models do
 * (src/neuron_model/LIFTimeDrivenModel.cpp:209-241).  Before eb_finalize. */
int eb_enable_conductances(eb_ctx *ctx, int pop, int mask);
/* Device address of state variable `var` (order as eb_get_state) of population
 * `pop`, or NULL when the variable is not stored; valid until eb_ctx_destroy.  For
 * device-side ops on the state between runs, e.g. eb_fold_arrivals into the
 * conductances. */
int eb_population_state(eb_ctx *ctx, int pop, int var, float **device_ptr);
/* Output flag of population `pop` (eb_add_population order). */
int eb_set_output(eb_ctx *ctx, int pop, int on);
/* State-monitor flag of population `pop` (the log column of the network file's
 * layer line; eb_add_population: clear).  Takes effect at the next
 * eb_open_monitor; input populations are never monitored, as in the reference
 * (src/spike/Network.cpp:1102-1108). */
int eb_set_monitor(eb_ctx *ctx, int pop, int on);
/* Write the states of the monitored neurons to a text file in the reference's
 * state-monitor format, FileOutputSpikeDriver::WriteState
 * (src/communication/FileOutputSpikeDriver.cpp:48-62, the -logp option), as every
 * following eb_run advances: one "%f\t%li" + "\t%1.12f" x (variables + 3) line
 * (time, neuron, the model's state variables, last-update time 0 and -1 -1 for a
 * time-driven model) at each delivery into a monitored neuron, after the weight
 * is added (src/spike/PropagatedSpikeGroup.cpp:73-85, PropagatedSpike.cpp:74-84),
 * and after each step a line per monitored neuron that spiked, then one per
 * monitored neuron (src/spike/TimeDrivenInternalSpike.cpp:66-72,113-131).  Runs
 * advance in chunks of `chunk_steps` steps (0: sized from the monitored
 * neurons); `delivery_capacity` bounds the deliveries into monitored neurons per
 * chunk (0: 1M; more returns EB_ERR_OVERFLOW).  After eb_finalize; eb_run_async
 * is refused while the file is open. */
int eb_open_monitor(eb_ctx *ctx, const char *path, int64_t chunk_steps, int64_t delivery_capacity);
/* Flush and close the state-monitor file (also done by eb_ctx_destroy). */
int eb_close_monitor(eb_ctx *ctx);
/* Write the weights in network-file order in the reference's weights-file format,
 * Network::SaveWeights (src/spike/Network.cpp:1165-1202, the -sf option): runs of
 * equal weights as "%i %g" lines.  The file loads back with eb_load_network_files. */
int eb_save_weights(eb_ctx *ctx, const char *path);
/* Update time of step k (double seconds, accumulated like the reference). */
int eb_step_time(eb_ctx *ctx, int64_t k, double *t);
/* State variable `var` (model order: V first, then the other differential variables,
 * then gE, gI, gNMDA) of neurons [first, first+n). */
int eb_get_state(eb_ctx *ctx, int64_t first, int64_t n, int var, float *out);
int eb_set_state(eb_ctx *ctx, int64_t first, int64_t n, int var, const float *in);
/* Record all state variables of neurons [first, first+n) after each of the next
 * `steps` steps: layout [steps][n][8] floats. */
int eb_set_trace(eb_ctx *ctx, int64_t first, int64_t n, int64_t steps);
int eb_get_trace(eb_ctx *ctx, float *out);
/* Weights in network-file order (Network::SaveWeights, src/spike/Network.cpp:1165-1202). */
int eb_get_weights(eb_ctx *ctx, float *w);
int eb_set_weights(eb_ctx *ctx, const float *w);
/* Steps done, spikes emitted, synaptic events delivered. */
int eb_get_counters(eb_ctx *ctx, int64_t *steps, int64_t *spikes, int64_t *events);
/* Seed of the reference's random generators (RandomGenerator::srand,
 * include/simulation/RandomGenerator.h:61-64; EDLUTKernel uses 1, the default).
 * It fixes the Poisson generators' sequences; call before eb_finalize. */
int eb_set_random_seed(eb_ctx *ctx, uint32_t seed);
/* Per-neuron frequencies (Hz) of Poisson generator neurons first .. first+n-1,
 * the vector parameter PoissonGeneratorDeviceVector::SetSpecificNeuronParameters
 * sets (src/neuron_model/PoissonGeneratorDeviceVector.cpp:142-155).  Before or
 * after eb_finalize. */
int eb_set_poisson_rates(eb_ctx *ctx, int64_t first, int64_t n, const float *rates_hz);
/* Synaptic events delivered into population `pop` (index in eb_add_population order). */
int eb_get_population_events(eb_ctx *ctx, int pop, int64_t *events);
/* Device memory held by the context, bytes. */
int eb_device_bytes(eb_ctx *ctx, int64_t *bytes);

/* The context's CUDA stream (cudaStream_t as a pointer), for callers that order
 * their own work or CUDA events against the simulation. */
int eb_stream(eb_ctx *ctx, void **stream);
/* Move the input spikes and step tables of the next n_steps to the device now, so
 * a following eb_run of those steps does no host-to-device copy. */
int eb_prestage(eb_ctx *ctx, int64_t n_steps);
/* Per-kernel timing: with on != 0, each run is one captured graph of its steps, the
 * same launches as the run path (per-population chains, several steps per launch
 * where the delays allow), with CUDA event records around every kernel on the
 * stream it runs on; eb_get_profile returns, per (kernel kind, population), the
 * launch count and total milliseconds.  kind: 0 input fan-out, 1 neuron update,
 * 2 post-synaptic STDP, 3 spike fan-out, 4 deferred post-synaptic STDP flush;
 * pop: population index (-1: none). */
int eb_set_profile(eb_ctx *ctx, int on);
int eb_get_profile(eb_ctx *ctx, int cap, int *n, int *kind, int *pop, int64_t *launches, double *total_ms);
/* Number of library kernels launched so far (nodes of a replayed graph counted per replay). */
int eb_launch_count(eb_ctx *ctx, int64_t *launches);

/* ------------------------------------------------------ delivery op ---- */
/* Fold a batch of n synaptic arrivals into conductance arrays in the reference's
 * delivery order, on the device (stream: cudaStream_t as a pointer; enqueued, not
 * synchronized).  All array arguments are device pointers.  Arrival i adds weight[i]
 * to g_exc / g_inh / g_nmda (type[i] 0 / 1 / 2) of neuron target[i] < n_targets;
 * per target the additions happen in order of (time[i], i) (time may be NULL: batch
 * order), so the float sums round like the reference CPU models, which add each
 * arrival straight into the conductance (NeuronModel::ProcessInputSpike,
 * src/neuron_model/LIFTimeDrivenModel.cpp:77-83, event order
 * src/spike/PropagatedSpikeGroup.cpp:112-149).  Replaces the per-arrival host
 * accumulation of the GPU models (src/neuron_model/LIFTimeDrivenModel_GPU_C_INTERFACE.cu:66-70).
 * Scratch memory is allocated per call on the stream (cudaMallocAsync).
 * n_targets <= 1048576. */
int eb_fold_arrivals(void *stream, int64_t n, const int32_t *target, const int8_t *type,
                     const float *weight, const double *time, int64_t n_targets,
                     float *g_exc, float *g_inh, float *g_nmda);
/* The same fold without any allocation, for callers that cannot allocate device
 * memory while they run (a closed-loop real-time controller whose step deadline
 * must not contain allocator calls, or a host engine that claims all device memory
 * at start-up).  No counterpart in the reference.  Its scratch is a fixed array in
 * the library's device image (about 7 MiB, held on every GPU that loads the library
 * until exit), so one call takes at most 262144 arrivals and 262144 targets; larger
 * batches return EB_ERR_ARG.  It runs on the calling thread's current device; the
 * first call on a device looks up that array's address (cudaGetSymbolAddress) and
 * should come before any stream capture.  All calls share the array: calls whose
 * GPU work overlaps (other streams or threads on the same device) race. */
int eb_fold_arrivals_noalloc(void *stream, int64_t n, const int32_t *target, const int8_t *type,
                             const float *weight, const double *time, int64_t n_targets,
                             float *g_exc, float *g_inh, float *g_nmda);

/* ---------------------------------------------------- checkpoint/resume --- */
/* Copy the whole dynamic state (neurons, BDF history, arrival buckets, weights,
 * plasticity traces, step counter) into an internal snapshot slot / restore it. */
int eb_snapshot(eb_ctx *ctx, int slot);
int eb_restore(eb_ctx *ctx, int slot);

/* ------------------------------------------------------ batched sweep --- */
/* Many independent LIF networks of uneven size advanced by one persistent kernel
 * (the parameter-sweep use: the reference runs one Simulation per parameter set,
 * Simulation::RunSimulation, src/simulation/Simulation.cpp:285-320, each with
 * its own network file; the reference README describes sweeps of several hundred
 * million 5k-neuron simulations).  Network i: n LIF neurons (neurons [0, n_exc) excitatory
 * sources, AMPA; [n_exc, n) inhibitory, GABA) and n_in input neurons (sources
 * n .. n+n_in-1, AMPA) driven by given spike times; every source connects to
 * every neuron with probability p through one delay, weights uniform in
 * [0, w_max) of the source's class, drawn on the device from a hash of (seed,
 * network, source, target).  Each network's spikes equal a run of the same
 * network (eb_sweep_get_synapses, LIF layer first, inputs after) on the plain
 * path.  Up to 65535 networks of at most 16384 neurons; Euler, RK2 or RK4. */
typedef struct eb_sweep eb_sweep;
int eb_sweep_create(int device, int n_networks, int integrator, float dt_s, float delay_s, uint64_t seed,
                    eb_sweep **out);
int eb_sweep_destroy(eb_sweep *h);
/* lif_params: the 10 LIFTimeDrivenModel .cfg values in file order
 * (LIFTimeDrivenModel::ParseNeuronModel, src/neuron_model/LIFTimeDrivenModel.cpp:459-540). */
int eb_sweep_set_network(eb_sweep *h, int i, int n, int n_in, int n_exc, const float *lif_params, float p,
                         float w_exc_max, float w_inh_max, float w_in_max);
/* Input spikes of network i: times in seconds, cells in [0, n_in). */
int eb_sweep_set_inputs(eb_sweep *h, int i, int64_t n, const float *time_s, const int32_t *cell);
/* Generate connectivity and allocate everything for up to n_steps_max steps;
 * the spike record holds max_rate_hz mean firing per network. */
int eb_sweep_build(eb_sweep *h, int64_t n_steps_max, float max_rate_hz);
/* Back to step 0 (initial state, empty records). */
int eb_sweep_reset(eb_sweep *h);
/* Threads per CTA (128/256/512/1024; neurons per thread follow) and steps per
 * kernel launch; 0 keeps the current value. */
int eb_sweep_configure(eb_sweep *h, int block, int steps_per_launch);
/* Time trial_steps from the initial state for each launch configuration, keep
 * the fastest, leave the sweep reset. */
int eb_sweep_autotune(eb_sweep *h, int64_t trial_steps, int *best_block, int *best_spl, float *best_ms);
/* Advance every network n_steps (whole chunks replay one CUDA graph). */
int eb_sweep_run(eb_sweep *h, int64_t n_steps);
int eb_sweep_run_async(eb_sweep *h, int64_t n_steps);
int eb_sweep_sync(eb_sweep *h);
/* Spikes of network i as (1-based step, neuron), sorted; size query with cap 0. */
int eb_sweep_get_spikes(eb_sweep *h, int i, int64_t cap, int64_t *n, int32_t *step, int32_t *cell);
int eb_sweep_spike_counts(eb_sweep *h, int64_t *counts);
/* Synapses of network i in delivery order (source, then target). */
int eb_sweep_get_synapses(eb_sweep *h, int i, int64_t cap, int64_t *m, int32_t *src, int32_t *tgt, float *w);
/* var 0 V, 1 gAMPA, 2 gGABA of the n neurons of network i. */
int eb_sweep_get_state(eb_sweep *h, int i, int var, float *out);
int eb_sweep_info(eb_sweep *h, int64_t *synapses, int64_t *device_bytes, int64_t *events, int *block,
                  int *steps_per_launch, int *grid);
int eb_sweep_stream(eb_sweep *h, void **stream);
/* Explicit connectivity of network i (after eb_sweep_set_network, before build):
 * m synapses source -> target (sources as above, at most one synapse per pair)
 * with weights, in the caller's order; the network then has no hash synapses. */
int eb_sweep_set_synapses(eb_sweep *h, int i, int64_t m, const int32_t *src, const int32_t *tgt, const float *w);
/* New .cfg parameters of network i (before or after build; a built sweep uses
 * them from its next launch, and the initial V = E_leak from its next reset). */
int eb_sweep_set_params(eb_sweep *h, int i, const float *lif_params);
/* All synaptic weights, networks in order, each network's synapses in its
 * eb_sweep_set_synapses order (hash networks: the delivery order).  w is device
 * memory when on_device != 0. */
int eb_sweep_set_weights(eb_sweep *h, const float *w, int on_device);
int eb_sweep_get_weights(eb_sweep *h, float *w, int on_device);
/* Record V after every step of m neurons per network (idx[n_networks][m], local
 * indices); eb_sweep_get_trace copies [n_networks][steps run][m]. */
int eb_sweep_set_observed(eb_sweep *h, int m, const int32_t *idx);
int eb_sweep_get_trace(eb_sweep *h, float *out, int on_device);
/* Save the whole state every `every` (1..255) steps during runs (0: off). */
int eb_sweep_set_checkpoints(eb_sweep *h, int every);

/* ---------------------------------------------------------------- adjoint --- */
/* Gradients of a loss L(trace) with respect to every network's g_leak, E_leak,
 * tau_exc (AMPA), tau_inh (GABA) and every weight, for the run just made from
 * step 0 with checkpoints (reset, set_checkpoints, run).  grad_trace = dL/dtrace,
 * [n_networks][steps run][m] (device memory when gt_on_device != 0); grad_w gets
 * dL/dw in eb_sweep_set_weights order (device memory when gw_on_device != 0);
 * grad_params gets [n_networks][4] on the host.  Discrete adjoint of the forward
 * as computed: spike times are the update steps at which V crosses v_thr, so the
 * threshold crossing enters through the reset V <- E_leak (the adjoint of V is
 * cut and its value goes to E_leak).  Each segment between checkpoints is
 * recomputed once.  No counterpart in the reference. Leaves the sweep needing
 * eb_sweep_reset. */
int eb_sweep_adjoint(eb_sweep *h, const float *grad_trace, int gt_on_device, float *grad_w, int gw_on_device,
                     double *grad_params);

#ifdef __cplusplus
}
#endif
#endif /* EDLUT_B200_H */
