/*
 * nestgpu.h -- C ABI of the B200 (sm_100a) engine for NEST's per-min_delay
 * simulation cycle: node update, spike gather/delivery into ring buffers, and
 * the spike_recorder sink.
 *
 * Plain C: pointers, sizes and status codes only.  Host buffers are owned by
 * the caller and copied; an engine owns all device memory it allocates.  One
 * engine is driven by one host thread at a time (the ABI is not re-entrant per
 * engine); different engines may be driven from different threads.
 *
 * Each entry point replaces a piece of the reference's node/kernel interface;
 * the reference location is given beside it (paths inside nest-simulator).
 */
#ifndef NESTGPU_H
#define NESTGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NG_ABI_VERSION 1

/* status codes (0 = success) */
#define NG_OK 0
#define NG_ERR_ARG -1          /* bad argument (BadProperty / BadParameter in the reference) */
#define NG_ERR_CUDA -2         /* CUDA runtime error or no usable device */
#define NG_ERR_STATE -3        /* call not valid in the engine's current state (KernelException) */
#define NG_ERR_NUMERIC -4      /* NumericalInstability (aeif_cond_alpha.cpp:481-490) */
#define NG_ERR_MEMORY -5       /* device allocation failed */
#define NG_ERR_CAPACITY -6     /* a device list overflowed (spike list, trace buffer) */
#define NG_ERR_UNKNOWN_NAME -7 /* unknown parameter/state name (UnaccessedDictionaryEntry) */

/* neuron models on the path */
#define NG_IAF_PSC_DELTA 0   /* models/iaf_psc_delta.{h,cpp} */
#define NG_IAF_PSC_EXP 1     /* models/iaf_psc_exp.{h,cpp} */
#define NG_AEIF_COND_ALPHA 2 /* models/aeif_cond_alpha.{h,cpp} */
#define NG_IAF_PSC_ALPHA 3   /* models/iaf_psc_alpha.{h,cpp} */

/* arithmetic forms */
#define NG_FP64 0 /* plain: FP64 state and FP64 ring buffers (red.global.add.f64) */
#define NG_FP32 1 /* precision form: FP32 state, int64 fixed-point ring buffers */

#define NG_MAX_BLOCKS 8

typedef struct ng_engine ng_engine;

/* Network-wide settings, fixed for the engine's lifetime.  A network is a
 * list of model blocks; neuron indices 0..n_neurons-1 run block by block. */
typedef struct
{
  int32_t device;          /* CUDA device ordinal */
  int32_t precision;       /* NG_FP64 or NG_FP32 */
  double h;                /* resolution [ms]: Time::get_resolution().get_ms() (nest_time.h:330) */
  double tics_per_ms;      /* Time tics per ms, 1000 by default (nest_time.cpp:43) */
  int32_t min_delay;       /* steps; slice length (connection_manager.cpp:485-530) */
  int32_t max_delay;       /* steps; the engine's rings hold max_delay slots (ring_buffer.cpp:25-46
                              holds min_delay + max_delay: the reference delivers before it updates) */
  int32_t n_blocks;
  int32_t block_model[ NG_MAX_BLOCKS ];
  int64_t block_size[ NG_MAX_BLOCKS ];
  int64_t n_generators;    /* extra spike sources after the neurons (spike_generator ports) */
  int64_t spike_log_capacity; /* device spike-log entries between drains, 0 = automatic */
  int64_t start_step;      /* absolute step of the engine's first slice origin (SimulationManager clock_) */
  /* serving: networks are added and removed while the engine runs (ng_net_*);
   * block_size[0] is then the neuron capacity of the pool */
  int32_t serving;
  int32_t max_networks;    /* serving: network slots */
  int64_t edge_capacity;   /* serving: edge pool, padding included */
  double max_abs_weight;   /* serving, FP32 form: largest |weight| (sets the fixed-point scale) */
  int32_t ring32;          /* serving, FP32 form: 32-bit fixed-point ring cells (half the atomic width)
                              instead of 64-bit; needs ring_bound */
  double ring_bound;       /* with ring32: largest sum of |weight| over one neuron's in-edges; sets the
                              scale so that no ring cell can overflow, checked for every admitted network */
  int64_t tile_capacity;   /* serving: entries of the segment tables of target-tiled delivery (0: off);
                              a pairwise_bernoulli network of n neurons needs n * (ceil(n / t) + 1): tiles of
                              t targets, about a multiple of the SM count S of them, t = min(T, ceil(n / (r S))
                              rounded up to 32), r = ceil(n / (T S)), T = min(1024, 163840 / (min(max_delay, 32)
                              * 2 * e) rounded down to 32), e = 4 for 32-bit rings, else 8 */
} ng_config;

/* Counters and timings of an engine. */
typedef struct
{
  int64_t clock_steps;       /* simulated steps so far (SimulationManager::get_time) */
  int64_t slices;            /* completed min_delay slices */
  int64_t spikes;            /* neuron spikes emitted (local_spike_counter) */
  int64_t syn_events;        /* recurrent synaptic events delivered: sum of out-degree x multiplicity */
  int64_t drive_events;      /* Poisson drive spikes (sum of multiplicities) */
  double update_ms;          /* device time in node-update kernels (profiling on) */
  double deliver_ms;         /* device time in delivery kernels (profiling on) */
  int64_t update_launches;
  int64_t deliver_launches;
  double simulate_ms;        /* host wall time inside ng_simulate */
  int64_t gather_slices;     /* serving, FP32 form: (network, slice) pairs delivered by the per-target gather */
  double wait_ms;            /* host time waiting for the device at the end of a group */
  double drain_ms;           /* host time draining spike logs and trace rows */
} ng_stats;

/* Version of this ABI (NG_ABI_VERSION). */
int ng_abi_version( void );

/* Message of the last error on this host thread (empty if none). */
const char* ng_last_error( void );

/* Number of usable CUDA devices. */
int ng_device_count( int32_t* n );

/* Create an engine: allocates state, ring buffers and spike lists on the
 * device.  Replaces NodeManager::prepare_nodes + Node::init_buffers_
 * (nestkernel/node_manager.cpp:590-596, node.cpp:75-86) and
 * EventDeliveryManager::init_moduli (event_delivery_manager.cpp:251-278). */
int ng_create( const ng_config* cfg, ng_engine** out );

/* Free all device memory of the engine. */
int ng_destroy( ng_engine* eng );

/* Set `count` values of a parameter or state variable for neurons
 * first..first+count-1 of block `block`.  Names and units are the model's
 * internal representation (models/iaf_psc_delta.cpp:94-200 keeps V_m, V_th,
 * V_reset, V_min relative to E_L: names V_m_rel, V_th_rel, ...).  Replaces
 * Node::set_status (nestkernel/node.h:420) for the model's Parameters_ and
 * State_.  `r` is the refractory step counter. */
int ng_set_var( ng_engine* eng, int32_t block, const char* name, const double* values, int64_t first, int64_t count );

/* Read back a parameter or state variable.  Replaces Node::get_status
 * (nestkernel/node.h:404) for State_ values. */
int ng_get_var( ng_engine* eng, int32_t block, const char* name, double* out, int64_t first, int64_t count );

/* Connectivity as CSR over sources 0..n_src-1 (neurons first, then
 * generator ports): targets are neuron indices, weights in the model's units,
 * delays in steps (min_delay <= d <= max_delay).  Replaces the per-thread
 * Connector<static_synapse> tables walked by ConnectionManager::send
 * (connection_manager.h:910-917, connector_base.h:398-434,
 * models/static_synapse.h:161-170). */
int ng_set_connections( ng_engine* eng, int64_t n_src, const int64_t* row_ptr, const int32_t* target,
  const double* weight, const int32_t* delay_steps );

/* The same connectivity as unordered (source, target, weight, delay) lists;
 * the engine groups them by source (counting sort, edge order kept within a
 * source) -- the order in which Connector::send walks a source's run of
 * connections (connector_base.h:398-434). */
int ng_set_connections_coo( ng_engine* eng, int64_t n_src, int64_t nnz, const int32_t* source, const int32_t* target,
  const double* weight, const int32_t* delay_steps );

/* stdp_pl_synapse_hom connections (models/stdp_pl_synapse_hom.h) as a CSR
 * over neuron sources 0..n_src-1: targets, initial weights (>= 0), delays
 * in steps, and the common properties lambda, alpha, mu, tau_plus.  Each
 * presynaptic spike updates its connections' weights -- facilitation by
 * the target's spikes since the source's previous spike, depression by the
 * target's trace -- before it reaches the ring buffer
 * (stdp_pl_synapse_hom::send, :255-298); targets keep the spike history
 * and trace of ArchivingNode (nestkernel/archiving_node.cpp, their
 * "tau_minus" set with ng_set_var, default 20 ms).  Static engines with
 * iaf_psc_delta / iaf_psc_exp / iaf_psc_alpha targets and min_delay <= 32
 * steps; a history holds 64 spikes per neuron (NG_ERR_CAPACITY if a
 * presynaptic neuron stays silent for longer than its targets' last 64). */
int ng_set_plastic_connections( ng_engine* eng, int64_t n_src, const int64_t* row_ptr, const int32_t* target,
  const double* weight, const int32_t* delay_steps, double lambda, double alpha, double mu, double tau_plus );

/* Current weights of the plastic connections, in their CSR order (n = their count). */
int ng_get_plastic_weights( ng_engine* eng, double* out, int64_t n );

/* Spikes of generator ports: emission step t_e (spike stamp minus one) and
 * source index (>= n_neurons), sorted by step.  Replaces
 * spike_generator::update (models/spike_generator.cpp:320-388). */
int ng_set_spike_schedule( ng_engine* eng, int64_t n, const int64_t* emit_step, const int32_t* source );

/* Poisson drive per neuron: rate [Hz] (<= 0: none), weight, delay [steps];
 * a generator draw happens at steps t_g with start < t_g <= stop and arrives
 * at t_g + delay.  Replaces poisson_generator::update/event_hook
 * (models/poisson_generator.cpp:125-148) with a counter-based Philox4x32-10
 * stream keyed by `seed`. */
int ng_set_poisson( ng_engine* eng, const double* rate_hz, const double* weight, const int32_t* delay_steps,
  int64_t start_step, int64_t stop_step, uint64_t seed );

/* Which sources (length n_src) have their spikes logged for recorders.
 * Replaces the device targets of TargetTableDevices::send_to_device
 * (nestkernel/target_table_devices_impl.h:76-91). */
int ng_set_recording( ng_engine* eng, const uint8_t* flags );

/* Record the state variables `vars[0..n_vars-1]` of the listed neurons at
 * every step whose stamp (step + 1) is a multiple of interval_steps.
 * Replaces the UniversalDataLogger of a multimeter
 * (nestkernel/universal_data_logger_impl.h:142-180). */
int ng_set_trace( ng_engine* eng, int64_t n_idx, const int32_t* neuron, int32_t n_vars, const char* const* vars,
  int32_t interval_steps );

/* Advance the network by n_steps steps: node updates, delivery of each
 * completed slice into the ring buffers, spike logging.  Partial slices are
 * handled as SimulationManager::update_ does (simulation_manager.cpp:842-1189).
 * Replaces SimulationManager::run (simulation_manager.cpp:614-671). */
int ng_simulate( ng_engine* eng, int64_t n_steps );

/* ng_simulate that returns while the last group of steps still runs on the
 * device; the spikes it logs are drained by the next simulate call (while
 * that call's first group runs) or by ng_sync.  Every entry point that reads
 * results or changes the engine drains first, except ng_net_add,
 * ng_net_poll, ng_net_capacity, ng_spike_count / ng_get_spikes (the spikes
 * drained so far), and ng_net_spikes / ng_net_remove of a network that ended
 * before that group began.  The engine-side counterpart
 * of repeated Run(t) calls between Prepare() and Cleanup()
 * (pynest/nest/lib/hl_api_simulation.py:66-130), which return when the
 * steps are done. */
int ng_simulate_async( ng_engine* eng, int64_t n_steps );

/* Steps [from, to) of the slice that starts at step `origin` -- the call a
 * NEST node receives once per slice, Node::update(Time const& origin, long
 * from, long to) (nestkernel/node.h:297, called by SimulationManager::
 * update_, simulation_manager.cpp:1062-1071).  The engine must stand at
 * origin + from (NG_ERR_STATE otherwise); a call with to == min_delay
 * closes the slice (its delivery runs).  Asynchronous: the steps of
 * successive calls are appended to one group on the device and the host
 * does not wait; their spikes are drained when the group fills the spike
 * log, or by ng_sync or any call that reads or changes the engine. */
int ng_update( ng_engine* eng, int64_t origin, int32_t from, int32_t to );

/* Wait for the steps of ng_simulate_async or ng_update and drain their spikes. */
int ng_sync( ng_engine* eng );

/* Number of logged spikes waiting to be drained. */
int ng_spike_count( ng_engine* eng, int64_t* n );

/* Drain up to `cap` logged spikes as (source, stamp step) in emission order
 * per drain; *n_out receives the count copied.  Replaces
 * RecordingBackendMemory::write (recording_backend_memory.cpp:104-112). */
int ng_get_spikes( ng_engine* eng, int32_t* source, int64_t* stamp, int64_t cap, int64_t* n_out );

/* Number of trace rows waiting and the drain: a row holds n_vars x n_idx
 * values (variable-major); row k has stamp first_stamp + k * interval_steps. */
int ng_trace_count( ng_engine* eng, int64_t* n_rows, int64_t* first_stamp );
int ng_get_trace( ng_engine* eng, double* out, int64_t max_rows, int64_t* n_rows_out );

/* Counters and timings. */
int ng_get_stats( ng_engine* eng, ng_stats* out );

/* Time each kernel launch with CUDA events (adds a small overhead). */
int ng_set_profiling( ng_engine* eng, int32_t on );

/* Run every following launch of this engine on the given cudaStream_t
 * (NULL: the engine's own stream). */
int ng_set_stream( ng_engine* eng, void* cuda_stream );

/* Capture full slices as CUDA graphs of `slices_per_graph` slices (0: off). */
int ng_set_graph_slices( ng_engine* eng, int32_t slices_per_graph );

/* ---------------------------------------------------------------------
 * Launch configuration and the autotuner.  No counterpart in the reference
 * (its OpenMP loop has no launch shapes to choose).  By default an engine
 * tunes itself on the first call long enough to afford the trials: it runs
 * the network's own next slices (real steps of the call) under each
 * candidate, timed with CUDA events -- the node-update kernel (one thread
 * per neuron gathering 4 or 8 lags of inputs at a time, or the two-phase
 * kernel with 256- or 128-thread CTAs), the resident delivery CTAs per SM,
 * and the edge chunks a delivery warp takes per descriptor load -- and keeps
 * the fastest.  The choice is cached for the process by network shape and
 * activity (precision, models, log2 of the neuron count, of the mean
 * out-degree and of the spikes per neuron-step, min_delay, delivery form),
 * so an engine of the same kind starts with it.  Every candidate computes
 * the same result.
 * --------------------------------------------------------------------- */
#define NG_TUNE_MAX_CANDIDATES 32
typedef struct
{
  int32_t mode;            /* 0: fixed, 1: autotuned */
  int32_t state;           /* 0: not tuned yet, 1: measured, 2: from the process cache, 3: fixed */
  int32_t update_variant;  /* 0/1/6: one thread per neuron (4/8/2 lags of inputs at a time), 2/3:
                              two-phase (256/128-thread CTAs), 4: aeif_cond_alpha's RKF45 kernel,
                              5: the persistent slice kernel */
  int32_t deliver_per_sm;  /* resident delivery CTAs per SM */
  int32_t deliver_group;   /* edge chunks per delivery warp and descriptor load */
  int32_t cache_hit;
  int32_t rate_bucket;     /* floor(log2(spikes per 1000 neuron-steps)) measured at tuning */
  int32_t n_candidates;    /* trials below, in the order they ran */
  int32_t cand_variant[ NG_TUNE_MAX_CANDIDATES ];
  int32_t cand_per_sm[ NG_TUNE_MAX_CANDIDATES ];
  int32_t cand_group[ NG_TUNE_MAX_CANDIDATES ];
  double cand_us_per_slice[ NG_TUNE_MAX_CANDIDATES ]; /* device time per min_delay slice */
  int64_t trial_steps;     /* steps of one timed trial */
} ng_tuning;

/* mode 1: autotune at the next long enough call (process cache first);
 * mode 2: the same, measuring even where the cache has an entry; mode 0:
 * fixed configuration -- update_variant (0..3, 5, 6; -1: by network size),
 * delivery CTAs per SM and chunks per warp (-1: defaults). */
int ng_set_tuning( ng_engine* eng, int32_t mode, int32_t update_variant, int32_t deliver_ctas_per_sm,
  int32_t deliver_chunks_per_warp );

/* The configuration in force and the autotuner's trials. */
int ng_get_tuning( ng_engine* eng, ng_tuning* out );

/* Engine options: "late_delivery" (1/0: edges of delay >= 2 min_delay
 * delivered on a second stream beside the next slice's update),
 * "late_ctas_per_sm", "aeif_binning" (1/0, default 0: aeif_cond_alpha
 * neurons ordered by their last RKF45 step size before each slice, so a
 * warp's neurons need similar numbers of sub-steps; measured 7 % slower on a
 * 50,000-neuron network, whose slice time is its slowest neuron's sub-step
 * chain), and for serving engines in the FP32 form, before any
 * network is admitted, "gather" (1/0: the per-target gather of hot
 * fixed_indegree networks) and "gather_frac" (the share of a network's
 * neurons spiking in a slice from which its next slice gathers). */
int ng_set_option( ng_engine* eng, const char* name, double value );

/* FP64 coefficients the engine computed for a neuron (testing hook):
 * writes up to `cap` values in the model's order, *n_out the count.  For
 * iaf_psc_delta: P33, P30, RefractoryCounts; iaf_psc_exp: P11ex, P11in, P22,
 * P21ex, P21in, P20, RefractoryCounts (models/iaf_psc_exp.cpp:244-285);
 * iaf_psc_alpha: P11ex, P11in, P21ex, P21in, P30, P31ex, P32ex, P31in, P32in,
 * expm1(-h/tau_m), EPSC and IPSC initial values, RefractoryCounts
 * (models/iaf_psc_alpha.cpp, pre_run_hook). */
int ng_debug_coefficients( ng_engine* eng, int32_t block, int64_t index, double* out, int32_t cap, int32_t* n_out );

/* ---------------------------------------------------------------------
 * Serving: independent networks admitted into and retired from one engine
 * while it runs (continuous batching).  All networks share the engine's
 * model (block 0), resolution and min/max delay; each has its own clock
 * origin, duration and drive seed.  A network draws the same drive and
 * produces the same spikes wherever and whenever it is admitted (its Philox
 * counters use network-local neuron indices and steps; the FP32 form's
 * int64 ring sums are order independent).  No counterpart in the reference,
 * which runs one network per kernel.
 * --------------------------------------------------------------------- */

/* fixed_indegree connectivity drawn on the device (nestkernel/conn_builder.cpp
 * FixedInDegreeBuilder, with a Philox stream instead of the reference's RNG):
 * every target gets k_exc sources from neurons [0, n_exc) and k_inh from
 * [n_exc, n), weights w_exc / w_inh, one delay. */
typedef struct
{
  int64_t n_exc;
  int32_t k_exc, k_inh;
  double w_exc, w_inh;
  int32_t delay_steps;
  int32_t allow_autapses;
  uint64_t seed;
} ng_fixed_indegree;

/* pairwise_bernoulli connectivity drawn on the device (nestkernel/conn_builder.h:716
 * BernoulliBuilder, with a Philox stream): the network's neurons form
 * populations in order; a (source, target) pair of populations (i, j) is
 * connected with probability p[i * NG_MAX_POPS + j]; weights and delays are
 * normal per source type (index 1: excitatory population, 0: inhibitory),
 * delays clipped to [h, d_max_ms] and rounded to steps. */
#define NG_MAX_POPS 16
typedef struct
{
  int32_t n_pops;
  int64_t pop_size[ NG_MAX_POPS ];
  int32_t pop_exc[ NG_MAX_POPS ];
  double p[ NG_MAX_POPS * NG_MAX_POPS ];
  double w_mean[ 2 ], w_sd[ 2 ];
  double d_mean_ms[ 2 ], d_sd_ms[ 2 ];
  double d_max_ms;
  int32_t allow_autapses;
  uint64_t seed;
} ng_pairwise_bernoulli;

typedef struct
{
  int64_t n;                        /* neurons */
  int64_t steps;                    /* steps to simulate from admission */
  uint64_t seed;                    /* Philox key of the network's drive */
  int32_t record;                   /* log the network's spikes */
  int32_t n_vars;                   /* per-neuron parameter/state arrays (model's internal names) */
  const char* const* var_names;
  const double* const* var_values;
  int64_t nnz;                      /* explicit edges (local neuron indices), or ... */
  const int32_t* source;
  const int32_t* target;
  const double* weight;
  const int32_t* delay_steps;
  const ng_fixed_indegree* build;   /* ... connectivity drawn on the device (nnz ignored) */
  const double* poisson_rate;       /* per neuron [Hz] (NULL: no drive) */
  const double* poisson_weight;
  const int32_t* poisson_delay;
  const ng_pairwise_bernoulli* build_pb; /* or pairwise_bernoulli connectivity drawn on the device */
} ng_net_desc;

/* Admit a network at the current clock (a slice boundary).  Returns
 * NG_ERR_CAPACITY, and changes nothing, when its neurons or edges do not
 * fit the free pool right now (admission by device-memory footprint). */
int ng_net_add( ng_engine* eng, const ng_net_desc* desc, int32_t* net_id );

/* Steps simulated so far and whether the network has reached its duration. */
int ng_net_poll( ng_engine* eng, int32_t net_id, int64_t* steps_done, int32_t* finished );

/* Drain the network's logged spikes: local neuron index and local stamp (at
 * most cap of them; source == NULL: *n_out = the number held, nothing drained). */
int ng_net_spikes( ng_engine* eng, int32_t net_id, int32_t* source, int64_t* stamp, int64_t cap, int64_t* n_out );

/* Read a state variable of the network's neurons (length n). */
int ng_net_get_var( ng_engine* eng, int32_t net_id, const char* name, double* out );

/* The network's connections in network-local ids, grouped by source
 * (GetConnections, nestkernel/nest.cpp:get_connections, with the fields
 * source, target, weight, delay of nestkernel/connection_manager.cpp:
 * get_connections).  With source == NULL only *n_out (the count) is set;
 * otherwise cap must hold all of them. */
int ng_net_get_connections( ng_engine* eng, int32_t net_id, int32_t* source, int32_t* target, double* weight,
  int32_t* delay_steps, int64_t cap, int64_t* n_out );

/* Retire the network and free its neurons, edges and slot. */
int ng_net_remove( ng_engine* eng, int32_t net_id );

/* Free neurons and edges of the pool (largest free runs). */
int ng_net_capacity( ng_engine* eng, int64_t* free_neurons, int64_t* free_edges );

/* ---------------------------------------------------------------------
 * Allocation-free entry point.  No counterpart in the reference.
 *
 * For callers that may not allocate device memory on the path that steps a
 * network: a host framework that owns all device memory through its own
 * allocator or pool and forbids foreign allocations, or a closed-loop
 * controller that steps a small network every control tick and cannot take
 * an allocation's implicit synchronisation and latency.  It simulates a
 * small iaf_psc_delta network in the plain FP64 form (the same arithmetic as
 * ng_simulate) from inputs and into outputs that the caller owns in device
 * memory, and calls no cudaMalloc, cudaFree or other allocating routine.
 *
 * Its ring buffer, spike list and counters live in one file-scope device
 * array of NG_NOALLOC_SCRATCH_BYTES that every GPU which loads the library
 * holds until the process exits.  Networks whose scratch
 * ((min_delay + max_delay) * n * 8 + n * min_delay * 8 bytes + 256) does not
 * fit are rejected with NG_ERR_CAPACITY.  A call with continue_run = 0
 * starts a fresh run: it zeroes the ring and counters, and start_step must
 * be a multiple of min_delay.  A call with continue_run = 1 goes on with the
 * run of the previous call on this device (same n, min_delay, max_delay, and
 * start_step equal to where that call stopped, which may be inside a
 * slice): the spikes still pending in the ring and the open slice's spike
 * list are kept, so a chain of calls gives the same result as one call over
 * the same steps.  Every call shares the one array, so calls that overlap on
 * the GPU race: serialise them (one stream, or events).  The first call on a
 * device looks up the array's device address with that device current; make
 * that first call before any stream capture.  The call is asynchronous on
 * `cuda_stream`; spikes beyond out_cap are counted in *out_count but not
 * written.  The kernels check every edge they walk: an edge whose target is
 * not in [0, n) or whose delay is not in [min_delay, max_delay] is skipped
 * and counted in *out_skipped (so no write ever leaves the ring); row_ptr
 * must be non-decreasing with row_ptr[n] edges in target/weight/delay.
 * --------------------------------------------------------------------- */
#define NG_NOALLOC_SCRATCH_BYTES ( 16u << 20 )

typedef struct
{
  int64_t n;                  /* neurons */
  int32_t min_delay;          /* steps */
  int32_t max_delay;          /* steps */
  int64_t start_step;         /* absolute step of the first step: a multiple of min_delay for a fresh run,
                                 the previous call's end for a continued one */
  const double* P33;          /* per neuron: exp(-h / tau_m) */
  const double* P30;          /* per neuron: 1 / C_m * (1 - P33) * tau_m */
  const double* V_th_rel;     /* per neuron, relative to E_L */
  const double* V_reset_rel;  /* per neuron, relative to E_L */
  const double* V_min_rel;    /* per neuron, relative to E_L */
  const double* I_e;          /* per neuron [pA] */
  const int32_t* refr_counts; /* per neuron: refractory steps */
  double* V_m_rel;            /* in/out: membrane potential relative to E_L */
  int32_t* r;                 /* in/out: refractory step counter */
  const int64_t* row_ptr;     /* CSR over the n neurons (n + 1 entries) */
  const int32_t* target;      /* edge target neuron */
  const double* weight;       /* edge weight [mV] */
  const int32_t* delay;       /* edge delay [steps], min_delay <= d <= max_delay */
  int32_t* out_src;           /* out: spike sources */
  int64_t* out_stamp;         /* out: spike stamps (emission step + 1) */
  int64_t out_cap;            /* capacity of out_src / out_stamp */
  unsigned long long* out_count; /* out: number of spikes emitted in this call */
  int32_t continue_run;       /* 0: fresh run; 1: continue the previous call's run on this device */
  int32_t reserved;           /* must be 0 */
  unsigned long long* out_skipped; /* out (may be NULL): edges skipped for an out-of-range target or delay */
} ng_noalloc_net;

/* Simulate n_steps of `net` with no memory allocation (see above). */
int ng_simulate_noalloc( const ng_noalloc_net* net, int64_t n_steps, void* cuda_stream );

#ifdef __cplusplus
}
#endif
#endif
