/*
 * bsnn.h -- C-ABI of libbsnn, the B200-native (sm_100a) engine for the per-step hot path of the
 * paulazoo/example-cuda-spiking-nn simulator ("buryn").
 *
 * The entry points below replace the reference's component constructors and its step loop:
 * the host builds a network with the same parameter PODs the reference uses
 * (NeuronGroupParams, ConnectionParams, PlasticityParams: identical field names, order and
 * layout), then advances it with bsnn_step / bsnn_run, which execute exactly what
 * System::step_the_clock (cpp_src/core/system.cpp:43-63) executes: neuron evolve, the four
 * propagations, stimulus, plasticity and monitor historicize, fused into one persistent
 * sm_100a kernel per call.
 *
 * Conventions
 *  - Every call returns a bsnn_status; on failure bsnn_last_error(sim) (or bsnn_last_error(NULL)
 *    for failures before a sim exists) holds a message.  The status codes map onto the
 *    exception types the reference throws (cpp_src/gpu_core/cuda_utils.h:10-20).
 *  - Plain pointers and sizes only; all host arrays are copied in at the call.
 *  - Calls on one bsnn_sim are not thread-safe; different sims may be driven from different
 *    host threads.  Each sim owns one CUDA stream.
 *  - Neuron indices are global ("offset + local id") exactly as in the reference's
 *    GpuSimulationState, where the excitatory group sits at offset 0 and the inhibitory group
 *    at offset num_excitatory_neurons.
 */
#ifndef BSNN_H
#define BSNN_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BSNN_API __attribute__((visibility("default")))
#else
#define BSNN_API
#endif

typedef struct bsnn_sim bsnn_sim; /* opaque; one simulated network on one GPU */

typedef int32_t bsnn_status;
#define BSNN_OK 0
#define BSNN_ERR_INVALID_ARGUMENT 1 /* reference: std::invalid_argument                          */
#define BSNN_ERR_OUT_OF_RANGE 2     /* reference: std::out_of_range                               */
#define BSNN_ERR_RUNTIME 3          /* reference: std::runtime_error                              */
#define BSNN_ERR_CUDA 4             /* reference: cuda_check -> std::runtime_error                */
#define BSNN_ERR_DEVICE_TIMEOUT 5   /* a bounded device-side wait gave up (kernel returned early) */
#define BSNN_ERR_STATE 6            /* call made in the wrong lifecycle state                     */

/* Plasticity kinds (TripletPlasticity / IstdpPlasticity / StdpPlasticity classes). */
#define BSNN_PLASTICITY_TRIPLET 1 /* cpp_src/plasticities/triplet_plasticity.h:10-27 (normalising form) */
#define BSNN_PLASTICITY_ISTDP 2   /* cpp_src/plasticities/istdp_plasticity.h:14-27                     */
#define BSNN_PLASTICITY_STDP 3    /* cpp_src/plasticities/stdp_plasticity.h:14-27                      */

/* Background-noise source for the per-neuron Poisson shot noise. */
#define BSNN_NOISE_PHILOX 0 /* counter-based Philox4x32-10 keyed by (rng_seed, neuron, step)         */
#define BSNN_NOISE_OFF 1    /* all Poisson counts are 0 (same as mean_background_* == 0)             */
#define BSNN_NOISE_REPLAY 2 /* counts supplied by bsnn_set_noise_replay (e.g. recorded elsewhere)    */

/* Fields for bsnn_read_state / bsnn_write_state. */
#define BSNN_FIELD_MEMBRANE_POTENTIALS 1     /* float [N_total]                                        */
#define BSNN_FIELD_G_EXCITATORY 2            /* float [N_total]                                        */
#define BSNN_FIELD_G_INHIBITORY 3            /* float [N_total]                                        */
#define BSNN_FIELD_I_STIMULUS 4              /* float [N_total]                                        */
#define BSNN_FIELD_REFRACTORY_COUNTER 5      /* uint32 [N_total]                                       */
#define BSNN_FIELD_SPIKES 6                  /* uint32 [N_total] (0/1)                                 */
#define BSNN_FIELD_BG_G_EXCITATORY 7         /* float [N_total]                                        */
#define BSNN_FIELD_BG_G_INHIBITORY 8         /* float [N_total]                                        */
#define BSNN_FIELD_BG_E_R_TRACES 9           /* float [N_total]                                        */
#define BSNN_FIELD_BG_E_D_TRACES 10          /* float [N_total]                                        */
#define BSNN_FIELD_BG_I_R_TRACES 11          /* float [N_total]                                        */
#define BSNN_FIELD_BG_I_D_TRACES 12          /* float [N_total]                                        */
#define BSNN_FIELD_CONN_R_TRACES 13          /* float [N_pre] of connection `index`                    */
#define BSNN_FIELD_CONN_D_TRACES 14          /* float [N_pre] of connection `index`                    */
#define BSNN_FIELD_CONN_SUMMED 15            /* float [N_pre] x = d - r of connection `index`          */
#define BSNN_FIELD_PLAST_PRE_TRACES 16       /* float [N_pre] of plasticity `index`                    */
#define BSNN_FIELD_PLAST_POST_TRACES 17      /* float [N_post] of plasticity `index`                   */
#define BSNN_FIELD_PLAST_TRIPLET_PRE 18      /* float [N_pre] of plasticity `index`                    */
#define BSNN_FIELD_PLAST_TRIPLET_POST 19     /* float [N_post] of plasticity `index`                   */
#define BSNN_FIELD_PLAST_PRE_WEIGHT_SUMS 20  /* float [N_pre] normalisation targets of plasticity     */
/* Row-scaled weight forms only (read-only; `index` = connection): */
#define BSNN_FIELD_CONN_ROW_SCALE 21         /* float [N_pre] normalisation scale s (weight = s * master) */
#define BSNN_FIELD_CONN_ROW_MASTER_SUM 22    /* float [N_pre] sum of the row's FP32 masters              */
#define BSNN_FIELD_CONN_ROW_QUANT_SCALE 23   /* float [N_pre] FP8 copy: value = e4m3 * scale             */

/* Weight storage forms (bsnn_set_weight_format).  No reference counterpart: the reference stores
 * FP32 weights and rescales every normalised row each step (BSNN_WEIGHTS_F32 keeps exactly that).
 * The other forms keep an FP32 master m per weight of every connection and a per-row
 * normalisation scale s (weight = s * m), so the triplet normalisation rewrites one number per
 * row; the propagation reads a copy of the masters in the given type (FP8: E4M3 times a per-row
 * scale fixed at upload), and weight updates refresh the entries they change. */
#define BSNN_WEIGHTS_F32 0           /* the reference's arithmetic                              */
#define BSNN_WEIGHTS_F32_ROWSCALED 1 /* FP32 masters, lazy row scale, FP32 GEMV copy            */
#define BSNN_WEIGHTS_BF16 2          /* GEMV copy in BF16 (round to nearest even)               */
#define BSNN_WEIGHTS_FP8_E4M3 3      /* GEMV copy in FP8 E4M3 (satfinite) with per-row scales   */

/*
 * Parameter PODs.  Field names, order and types are those of the reference structs, so a
 * reference NeuronGroupParams / ConnectionParams / PlasticityParams object can be passed by
 * address.  (The reference gives C++ default member initialisers; C has none, so the C++
 * facade in this package supplies the same defaults.)
 */

/* cpp_src/neuron_groups/neuron_group_params.h:7-31 */
typedef struct bsnn_neuron_group_params {
    float timestep;
    float g_leak;
    float membrane_capacitance;
    float depolarization_slope_factor;
    float v_effective_spike_threshold;
    float v_excitatory_reversal;
    float v_inhibitory_reversal;
    float v_threshold;
    float v_reset;
    float v_rest;
    uint32_t refractory_steps;
    bool is_inhibitory;
    float mean_background_excitatory_spikes;
    float mean_background_inhibitory_spikes;
    float background_excitatory_postsynaptic_r_trace_decay;
    float background_excitatory_postsynaptic_d_trace_decay;
    float background_inhibitory_postsynaptic_r_trace_decay;
    float background_inhibitory_postsynaptic_d_trace_decay;
    float background_excitatory_scaling_factor;
    float background_inhibitory_scaling_factor;
    uint32_t offset;
    uint32_t num_neurons;
} bsnn_neuron_group_params;

/* cpp_src/connections/connection_params.h:7-14 */
typedef struct bsnn_connection_params {
    float timestep;
    float decay_time;
    float rise_time;
    float postsynaptic_kernel_normalization_value;
    uint32_t weight_matrix_idx;
} bsnn_connection_params;

/* cpp_src/plasticities/plasticity_params.h:7-20 */
typedef struct bsnn_plasticity_params {
    float ltp_A;
    float ltd_A;
    float ltp_B;
    float ltd_B;
    float pre_trace_decay;
    float post_trace_decay;
    float triplet_pre_trace_decay;
    float triplet_post_trace_decay;
    float weight_min;
    float weight_max;
    uint32_t plasticity_offset;
} bsnn_plasticity_params;

/* Constructor arguments of GpuSimulationState (cpp_src/gpu_core/gpu_simulation_state.h:21-25)
 * plus the two globals of cpp_src/core/buryn_definitions.h:11-13 the reference reads. */
typedef struct bsnn_state_desc {
    uint32_t total_simulation_length;
    uint32_t num_excitatory_neurons;
    uint32_t num_inhibitory_neurons;
    uint32_t num_stimulus_events;
    uint32_t num_plasticities;
    uint32_t recording_interval_steps; /* buryn::recording_interval_steps; 0 means 10000 */
    int32_t rng_seed;                  /* buryn::rng_seed */
    int32_t device;                    /* CUDA device ordinal */
} bsnn_state_desc;

typedef struct bsnn_info {
    uint32_t total_neurons;
    uint32_t num_groups;
    uint32_t num_connections;
    uint32_t num_plasticities;
    uint32_t num_monitors;
    uint32_t grid_ctas;        /* persistent CTAs (one per SM)                          */
    uint32_t block_threads;    /* threads per CTA                                       */
    uint32_t steps_per_launch; /* steps one persistent launch covers inside bsnn_run    */
    uint64_t steps_done;       /* steps executed so far (the stimulus / noise cursor)   */
    uint64_t device_bytes;     /* bytes held in the device arena                        */
    uint64_t weight_bytes;     /* bytes of weight storage                               */
    uint64_t kernel_launches;  /* persistent-kernel launches issued so far              */
    uint64_t smem_bytes;       /* dynamic shared memory per CTA                         */
    uint64_t resident_bytes;   /* weight bytes per CTA kept in shared memory per launch */
} bsnn_info;

/* ---- lifecycle --------------------------------------------------------------------------- */

/* Replaces GpuSimulationState::GpuSimulationState (cpp_src/gpu_core/gpu_simulation_state.cu:8-28). */
BSNN_API bsnn_status bsnn_create(const bsnn_state_desc* desc, bsnn_sim** out_sim);
/* Replaces GpuSimulationState::~GpuSimulationState (cpp_src/gpu_core/gpu_simulation_state.cu:31-33). */
BSNN_API bsnn_status bsnn_destroy(bsnn_sim* sim);
/* Message of the last failed call on `sim` (or of the calling thread when sim == NULL). */
BSNN_API const char* bsnn_last_error(const bsnn_sim* sim);
BSNN_API bsnn_status bsnn_get_info(const bsnn_sim* sim, bsnn_info* out);
/* Version string of the library build. */
BSNN_API const char* bsnn_version(void);

/* ---- components (each mirrors one reference constructor) --------------------------------- */

/* NeuronGroup::NeuronGroup (cpp_src/neuron_groups/neuron_group.cpp:4-17): uploads v = v_rest and
 * zero for every other per-neuron field of the slice [offset, offset + num_neurons). */
BSNN_API bsnn_status bsnn_add_neuron_group(bsnn_sim* sim, const bsnn_neuron_group_params* params,
                                           uint32_t* out_group);

/* Connection::Connection (cpp_src/connections/connection.cpp:3-23): `weights` is the
 * pre x post matrix in row-major order (weights[pre * num_post + post]), as
 * Connection::initialize_data flattens it (cpp_src/connections/connection.cpp:27-42).
 * Negative weights are rejected (gpu_simulation_state.cu:221-229). */
BSNN_API bsnn_status bsnn_add_connection(bsnn_sim* sim, uint32_t pre_group, uint32_t post_group,
                                         const float* weights, const bsnn_connection_params* params,
                                         uint32_t* out_connection);

/* Stimulus::Stimulus (cpp_src/stimuli/stimulus.cpp:3-17): per-step event counts and the flat,
 * time-ordered event arrays; events add `delta` to i_stimulus[offset + id]. */
BSNN_API bsnn_status bsnn_add_stimulus(bsnn_sim* sim, const uint32_t* timestep_event_count,
                                       uint32_t num_timesteps, const uint32_t* neuron_ids,
                                       const uint32_t* post_group_offsets, const float* amplitude_changes,
                                       uint32_t num_events);

/* TripletPlasticity / IstdpPlasticity / StdpPlasticity constructors
 * (cpp_src/plasticities/triplet_plasticity.cpp:3-12, istdp_plasticity.cpp:3-12,
 * stdp_plasticity.cpp:3-12).  For the triplet rule the normalisation targets are the initial
 * column sums of the weight matrix (triplet_plasticity.cpp:21-31). */
BSNN_API bsnn_status bsnn_add_plasticity(bsnn_sim* sim, int32_t kind, uint32_t connection,
                                         const bsnn_plasticity_params* params, uint32_t* out_plasticity);

/* SpikeRecorder::SpikeRecorder (cpp_src/monitors/spike_recorder.cpp:3-14): a device ring of
 * `recording_interval_steps` slots holding the group's spikes of each step. */
BSNN_API bsnn_status bsnn_add_spike_recorder(bsnn_sim* sim, uint32_t group, uint32_t recording_interval_steps,
                                             uint32_t* out_monitor);

/* VoltageRecorder::VoltageRecorder (cpp_src/monitors/voltage_recorder.cpp:3-28): ring of the
 * selected neurons' membrane potentials (an empty selection records the whole group). */
BSNN_API bsnn_status bsnn_add_voltage_recorder(bsnn_sim* sim, uint32_t group, const uint32_t* selected_neurons,
                                               uint32_t num_selected, uint32_t recording_interval_steps,
                                               uint32_t* out_monitor);

/* ---- noise ---------------------------------------------------------------------------------- */

BSNN_API bsnn_status bsnn_set_noise_mode(bsnn_sim* sim, int32_t mode);
/* counts[(s * N_total + neuron) * 2 + channel] for steps s = 0 .. num_steps-1 counted from the
 * sim's first step; channel 0 = excitatory, 1 = inhibitory.  Steps past num_steps draw 0. */
BSNN_API bsnn_status bsnn_set_noise_replay(bsnn_sim* sim, const uint8_t* counts, uint32_t num_steps);
/* Weight storage form (BSNN_WEIGHTS_*), before the first step.  No reference counterpart. */
BSNN_API bsnn_status bsnn_set_weight_format(bsnn_sim* sim, int32_t format);

/* ---- the hot path --------------------------------------------------------------------------- */

/* System::step_the_clock(clock_step) (cpp_src/core/system.cpp:43-63): one step of every phase.
 * Returns after the work is queued; errors of the kernel surface at the next synchronising
 * call (bsnn_synchronize, reads). */
BSNN_API bsnn_status bsnn_step(bsnn_sim* sim, uint32_t clock_step);
/* The step loop of System::run (cpp_src/core/system.cpp:65-84) without its callbacks and
 * recording: steps first_clock_step .. first_clock_step + num_steps - 1, as CUDA-graph replays
 * of the persistent kernel. */
BSNN_API bsnn_status bsnn_run(bsnn_sim* sim, uint32_t first_clock_step, uint32_t num_steps);
/* Waits for queued work and reports a device-side error (barrier timeout) if one occurred. */
BSNN_API bsnn_status bsnn_synchronize(bsnn_sim* sim);
/* The sim's CUDA stream (a cudaStream_t), for callers that time or order work around it. */
BSNN_API bsnn_status bsnn_get_stream(const bsnn_sim* sim, void** out_stream);
/* Steps per persistent launch used by bsnn_run (default 1000; 1..65536). */
BSNN_API bsnn_status bsnn_set_steps_per_launch(bsnn_sim* sim, uint32_t steps);
/* Error contract of cpp_src/gpu_core/cuda_utils.h:10-20 for the persistent kernel's own waits.
 * Every device-side wait (the grid barrier between steps, the staging copies) gives up after
 * `nanoseconds` (default 2 s; 1 us .. 60 s): the kernel then records the failure and returns, the
 * call that ran it (or bsnn_synchronize) returns BSNN_ERR_DEVICE_TIMEOUT, and later calls on that
 * sim return BSNN_ERR_STATE.  Other sims on the device are unaffected. */
BSNN_API bsnn_status bsnn_set_device_wait_limit(bsnn_sim* sim, uint64_t nanoseconds);
/* Test switch, no reference counterpart: CTA `cta` of the persistent grid does not arrive at the
 * grid barrier that ends internal step `step` (steps counted from 0 since creation), so every
 * CTA's bounded wait runs out.  It exercises the timeout path above without a fault; finalises
 * the network.  BSNN_ERR_OUT_OF_RANGE for a cta outside the grid. */
BSNN_API bsnn_status bsnn_debug_skip_arrival(bsnn_sim* sim, uint32_t cta, uint64_t step);
/* Measurement aid, no reference counterpart: the latency floor of one clock step of this network.
 * Runs the step's communication skeleton alone -- every CTA stores its partial-sum slots, crosses
 * the grid barrier and gathers its own columns from every slot, with the same grid, block and plan
 * as bsnn_step / bsnn_run -- for num_steps steps after a warm-up launch, and writes its mean time
 * per step (microseconds, CUDA events on the sim's stream).  The simulation's state is unchanged.
 * Finalises the network. */
BSNN_API bsnn_status bsnn_measure_exchange_floor(bsnn_sim* sim, uint32_t num_steps, float* out_us_per_step);

/* ---- state access (GpuSimulationState download helpers) ------------------------------------ */

/* Checkpoint / resume (no reference counterpart): the whole device state and the clock cursor to
 * a binary file, and back into a simulation built from the same components in the same order,
 * with the same weight form, on the same kind of GPU (checked; BSNN_ERR_INVALID_ARGUMENT
 * otherwise).  Files written by text monitors are not part of a checkpoint. */
BSNN_API bsnn_status bsnn_save_checkpoint(bsnn_sim* sim, const char* path);
BSNN_API bsnn_status bsnn_load_checkpoint(bsnn_sim* sim, const char* path);

/* Copies `count` elements starting at `offset` of a field (BSNN_FIELD_*) to host memory.
 * `index` selects the connection / plasticity for the per-component fields. */
BSNN_API bsnn_status bsnn_read_state(bsnn_sim* sim, int32_t field, uint32_t index, uint32_t offset,
                                     uint32_t count, void* host_out);
/* Overwrites elements of a per-neuron field (test set-up; same fields as bsnn_read_state). */
BSNN_API bsnn_status bsnn_write_state(bsnn_sim* sim, int32_t field, uint32_t index, uint32_t offset,
                                      uint32_t count, const void* host_in);
/* GpuSimulationState::download_weight_matrix (cpp_src/gpu_core/gpu_simulation_state.cu:287-306):
 * row-major pre x post matrix of a connection. */
BSNN_API bsnn_status bsnn_read_weights(bsnn_sim* sim, uint32_t connection, float* host_out);
/* Row-scaled forms: the propagation's copy of the masters, row-major pre x post, as stored
 * (4-byte floats, 2-byte BF16 or 1-byte E4M3 elements).  No reference counterpart. */
BSNN_API bsnn_status bsnn_read_weight_copy(bsnn_sim* sim, uint32_t connection, void* host_out);
/* GpuSimulationState::download_and_flush_spike_history (gpu_simulation_state.cu:239-261):
 * writes the spike ring of a spike recorder in the reference layout
 * host_out[neuron * interval + slot] (0/1) and, when `flush` is non-zero, zeroes the ring. */
BSNN_API bsnn_status bsnn_read_spike_history(bsnn_sim* sim, uint32_t monitor, uint32_t* host_out, int32_t flush);
/* Same ring as packed bits, time-major: host_out[slot * words + w], words = ceil(N_group / 32);
 * bit b of word w is neuron 32 * w + b of the group.  This is what the device stores. */
BSNN_API bsnn_status bsnn_read_spike_bits(bsnn_sim* sim, uint32_t monitor, uint32_t* host_out, int32_t flush);
/* GpuSimulationState::download_and_flush_membrane_potential_history (gpu_simulation_state.cu:263-285),
 * restricted to the recorder's selected neurons: host_out[k * interval + slot] for the k-th
 * selected neuron. */
BSNN_API bsnn_status bsnn_read_voltage_history(bsnn_sim* sim, uint32_t monitor, float* host_out, int32_t flush);
/* Device address of a field (for the C++ facade's *View structs); read-only use. */
BSNN_API bsnn_status bsnn_get_device_pointer(const bsnn_sim* sim, int32_t field, uint32_t index, void** out);

/* ---- recording to text files (Monitor::record) --------------------------------------------- */

/* Output file of a spike or voltage recorder: the output_filepath of SpikeRecorder /
 * VoltageRecorder (cpp_src/monitors/spike_recorder.cpp:3-14, voltage_recorder.cpp:3-28).  A spike
 * recorder's file is truncated now and gets the header "clock_step, neuron_ids"; a voltage recorder
 * writes one file per recorded step, named by inserting "_step<N>" before the ".txt" that `path`
 * must contain (else BSNN_ERR_OUT_OF_RANGE).  A file that cannot be opened is skipped, as the
 * reference skips output when its stream is not good(). */
BSNN_API bsnn_status bsnn_set_monitor_output(bsnn_sim* sim, uint32_t monitor, const char* path);
/* WeightRecorder (cpp_src/monitors/weight_recorder.cpp:3-51): at recorded clock steps that are
 * multiples of 100,000, writes "<path with _step<N>>" holding "pre_neuron_id, post_neuron_id,
 * weight" and every (pre, post) triple, zeros included.  May be added at any time. */
BSNN_API bsnn_status bsnn_add_weight_recorder(bsnn_sim* sim, uint32_t connection, const char* path);
/* Monitor::record(clock_step) of every recorder with an output (spike_recorder.cpp:40-60,
 * voltage_recorder.cpp:54-78, weight_recorder.cpp:25-51), in the reference's formats and labels:
 * the rings are copied out and flushed before the call returns; the text is formatted and written
 * by a writer thread of the sim, so stepping can continue meanwhile. */
BSNN_API bsnn_status bsnn_record(bsnn_sim* sim, uint32_t clock_step);
/* Waits until every record queued so far is written and flushed. */
BSNN_API bsnn_status bsnn_flush_records(bsnn_sim* sim);
/* System::run(total_clock_steps) (cpp_src/core/system.cpp:65-84) without step callbacks: clock
 * steps 0 .. total-1, with bsnn_record after every step that is a multiple of the state's
 * recording_interval_steps.  With progress output on (bsnn_set_progress_output) it prints the
 * reference's line "Completed clock step: <step> | elapsed: <seconds>s" on stdout after each of
 * those records (system.cpp:78-81), the seconds counted from the start of the call. */
BSNN_API bsnn_status bsnn_run_system(bsnn_sim* sim, uint32_t total_clock_steps);
/* Turns bsnn_run_system's progress line on (enabled != 0) or off (the default). */
BSNN_API bsnn_status bsnn_set_progress_output(bsnn_sim* sim, int32_t enabled);
/* GpuSimulationState::memory_report (cpp_src/gpu_core/gpu_simulation_state.cu:308-364): writes
 * "Total GPU Memory Allocated: <bytes> bytes (<MB> MB)" with this sim's device arena into `buf`
 * (NUL-terminated; BSNN_ERR_OUT_OF_RANGE when `capacity` is too small).  The reference allocates
 * in its constructor; bsnn allocates when the network is complete, so this call finalises the
 * network first (as the first bsnn_step or bsnn_run would): add every component before it. */
BSNN_API bsnn_status bsnn_memory_report(bsnn_sim* sim, char* buf, uint64_t capacity);

/* ---- one connection on caller-owned device buffers ------------------------------------------ */

/* cpp_src/connections/connection_view.h:8-31, same field names, order and layout, so the address of
 * a reference ConnectionView can be passed as is.  The pointers are device pointers into the
 * caller's buffers: weight_matrix is row-major [pre][post], the trace arrays and `spikes` are
 * [pre_group_num_neurons] (the reference points `spikes` at d_spikes + pre_group_offset,
 * connection.cpp:85), and the conductance arrays are [post_group_num_neurons].  The offsets and
 * weight_matrix_idx are bookkeeping and are not read; cublas_handle is ignored. */
typedef struct bsnn_connection_view {
    float postsynaptic_r_trace_decay;
    float postsynaptic_d_trace_decay;
    float postsynaptic_kernel_normalization_value;
    bool pre_group_is_inhibtory;
    uint32_t weight_matrix_idx;
    uint32_t pre_group_offset;
    uint32_t post_group_offset;
    uint32_t pre_group_num_neurons;
    uint32_t post_group_num_neurons;
    float* weight_matrix;
    float* postsynaptic_r_traces;
    float* postsynaptic_d_traces;
    float* summed_postsynaptic_conductances;
    float* post_group_g_excitatory;
    float* post_group_g_inhibitory;
    uint32_t* spikes;
    void* cublas_handle;
} bsnn_connection_view;

/* kernel_connection_propagate_launch (cpp_src/connections/kernel_connection_propagate.cu:64-111):
 * decays the r and d traces, adds the normalisation value on a presynaptic spike, writes
 * x = d - r into summed_postsynaptic_conductances, then adds W^T x into post_group_g_inhibitory
 * when the presynaptic group is inhibitory, else into post_group_g_excitatory (the cublasSgemv
 * with alpha = beta = 1).  Runs on the current CUDA device; `stream` is a cudaStream_t (NULL =
 * the legacy default stream).  The work is queued and the call returns: where the reference
 * blocks on cudaDeviceSynchronize, synchronise the stream.  GEMV scratch of splits x N_post
 * floats comes from cudaMallocAsync on `stream` and is freed in stream order.  Errors: null view
 * or pointer, or an empty connection -> BSNN_ERR_INVALID_ARGUMENT; failed launch -> BSNN_ERR_CUDA
 * (message in bsnn_last_error(NULL)). */
BSNN_API bsnn_status bsnn_connection_propagate(const bsnn_connection_view* view, void* stream);

/* No counterpart in the reference.  The same work as bsnn_connection_propagate, but the call
 * allocates no device memory: the GEMV scratch is a fixed module-scope device array of
 * 1,048,576 floats (4 MiB) per device, so post_group_num_neurons above 1,048,576 is rejected with
 * BSNN_ERR_OUT_OF_RANGE before anything is queued.  It is for callers that must not allocate per
 * call, e.g. a step loop inside an application whose device memory is already claimed by its own
 * caching allocator (PyTorch's), where a cudaMallocAsync can fail or grow a pool mid-run.
 *  - Result: the same bits as bsnn_connection_propagate whenever both split the rows into the same
 *    number of chunks, which holds for every post_group_num_neurons up to the limit on a 148-SM
 *    B200.  On a GPU where the allocating path's chunks x post_group_num_neurons would not fit the
 *    array, fewer chunks are used and the conductances agree with it to float rounding only.
 *  - The first call on each device does a one-time set-up with that device current (looking up the
 *    array's device address with cudaGetSymbolAddress, which may load this library's device code);
 *    make that first call before any stream capture.  A failed set-up returns BSNN_ERR_CUDA.  The
 *    address is kept with the context it came from and looked up again when the device's current
 *    context changes (after cudaDeviceReset, for instance); the call that does so is a set-up call.
 *  - Nothing has to start at zero: each call writes every scratch value it reads.
 *  - All calls on one device share the array: calls that overlap in time (on different streams or
 *    from different host threads) race and give wrong results.  Order them (one stream, or events). */
BSNN_API bsnn_status bsnn_connection_propagate_noalloc(const bsnn_connection_view* view, void* stream);

/* ---- network generation on the GPU (a flagged alternative to cpp_src/generation/generate_weights.cpp:10-103)
 * The reference's rule (candidates off the diagonal when excluded and within max_distance on the
 * periodic layout; existence with probability multiplier [x exp(-d^2/S)]; value max_weight [x the
 * same Gaussian]) with counter-based Philox draws per (seed, pre, post) instead of one mt19937
 * stream: the candidate sets equal the reference's, the matrix equals it in distribution, not bit
 * for bit (the host generator in bsnn_generate.hpp is the byte-identical one).  uniform_values
 * draws each existing weight from U[0, max_weight_value). */
typedef struct bsnn_weight_generation_params {
    float max_weight_value;
    float max_distance;
    float spread_scale;
    float probability_multiplier;
    float x_location_length;
    float y_location_length;
    int32_t weight_value_normal_dropoff;
    int32_t probabilistic_normal_not_uniform;
    int32_t no_diagonal_connections;
    int32_t uniform_values;
} bsnn_weight_generation_params;

/* pre_xy / post_xy: (x, y) per neuron; w_out: host memory for n_pre * n_post floats, row-major. */
BSNN_API bsnn_status bsnn_generate_distance_weights(const float* pre_xy, uint32_t n_pre, const float* post_xy,
                                                    uint32_t n_post, const bsnn_weight_generation_params* params,
                                                    uint64_t seed, int32_t device, float* w_out);

/* ---- the batched form (no reference counterpart) ---------------------------------------------
 * Many independent networks ("instances") of uneven size, without plasticity, stepped together by
 * one persistent launch.  Each instance is the reference's two-group network (E group, I group,
 * connections E->E, E->I, I->E, I->I, one stimulus, background noise) with its own neuron-group
 * parameters, seed and stimulus; instances of one size class share one weight set, stored once in
 * BF16, so the class's propagation is a GEMM on the tensor cores (BF16 weights, traces split into
 * BF16 high and low parts, FP32 accumulation).  Needs an sm_100 GPU. */
typedef struct bsnn_batch bsnn_batch;

typedef struct bsnn_batch_info {
    uint32_t num_classes;
    uint32_t num_instances;
    uint32_t num_neurons;      /* over all instances                                      */
    uint32_t num_units;        /* GEMM work units per step                                */
    uint32_t grid_ctas;
    uint32_t block_threads;
    uint64_t steps_done;
    uint64_t device_bytes;
    uint64_t weight_bytes;     /* BF16 weight tiles, padding included                     */
    uint64_t kernel_launches;
    uint64_t smem_bytes;
    uint32_t state_in_smem;    /* 1: each CTA's neuron state stays in shared memory      */
    uint32_t operand_stages;   /* shared-memory operand stages of the GEMM ring           */
    int32_t form;              /* BSNN_BATCH_FORM_*                                       */
} bsnn_batch_info;

BSNN_API bsnn_status bsnn_batch_create(int32_t device, bsnn_batch** out_batch);
BSNN_API bsnn_status bsnn_batch_destroy(bsnn_batch* batch);
BSNN_API const char* bsnn_batch_last_error(const bsnn_batch* batch);
/* A size class: weight matrices row-major [pre][post] (non-negative FP32, stored as BF16) and the
 * connection parameters of its excitatory-presynaptic (E->E, E->I) and inhibitory-presynaptic
 * (I->E, I->I) connections.  At most 8 classes. */
BSNN_API bsnn_status bsnn_batch_add_class(bsnn_batch* batch, uint32_t num_excitatory, uint32_t num_inhibitory,
                                          const float* w_ee, const float* w_ei, const float* w_ie, const float* w_ii,
                                          const bsnn_connection_params* excitatory_pre,
                                          const bsnn_connection_params* inhibitory_pre, uint32_t* out_class);
/* An instance of a class (at most 128 per class): its two groups' parameters (num_neurons must
 * match the class; offset is ignored), its noise seed (rng_seed of the single-network form) and
 * its stimulus as per-step event counts, each event an (instance-local neuron, amplitude change). */
BSNN_API bsnn_status bsnn_batch_add_instance(bsnn_batch* batch, uint32_t class_index,
                                             const bsnn_neuron_group_params* excitatory_group,
                                             const bsnn_neuron_group_params* inhibitory_group, int32_t rng_seed,
                                             const uint32_t* stimulus_counts, uint32_t stimulus_steps,
                                             const uint32_t* stimulus_neurons, const float* stimulus_deltas,
                                             uint32_t num_events, uint32_t* out_instance);
BSNN_API bsnn_status bsnn_batch_set_noise(bsnn_batch* batch, int32_t on);
BSNN_API bsnn_status bsnn_batch_set_steps_per_launch(bsnn_batch* batch, uint32_t steps);
/* How the kernel orders a clock step's work (before the first step; results are bit-identical):
 * FLOW runs each size class as its own chain, its GEMM units starting when its neurons are
 * stepped and its neurons when its units are done, neuron updates and GEMMs overlapping inside a
 * CTA; PHASED steps all neurons, then runs all GEMM units, with a grid barrier after each. */
#define BSNN_BATCH_FORM_FLOW 0
#define BSNN_BATCH_FORM_PHASED 1
BSNN_API bsnn_status bsnn_batch_set_form(bsnn_batch* batch, int32_t form);
/* Bound of the batch kernel's device-side waits (default 2 s; 1 us .. 60 s), as
 * bsnn_set_device_wait_limit. */
BSNN_API bsnn_status bsnn_batch_set_device_wait_limit(bsnn_batch* batch, uint64_t nanoseconds);
BSNN_API bsnn_status bsnn_batch_run(bsnn_batch* batch, uint32_t num_steps);
BSNN_API bsnn_status bsnn_batch_synchronize(bsnn_batch* batch);
BSNN_API bsnn_status bsnn_batch_get_stream(const bsnn_batch* batch, void** out_stream);
/* One instance's per-neuron field (BSNN_FIELD_* per-neuron fields; CONN_* = the neuron's own
 * presynaptic traces), E neurons then I neurons. */
BSNN_API bsnn_status bsnn_batch_read_state(bsnn_batch* batch, uint32_t instance, int32_t field, void* host_out);
/* Spikes since creation, host_out[2 * instance + 0 / 1] for the E / I group. */
BSNN_API bsnn_status bsnn_batch_read_spike_counts(bsnn_batch* batch, uint64_t* host_out);
BSNN_API bsnn_status bsnn_batch_get_info(bsnn_batch* batch, bsnn_batch_info* out);

/* The autotuner's choice: GEMM unit size (K tiles of 64 presynaptic neurons per unit), operand
 * ring depth, how many candidates were timed, and the clock-step times of the choice and of the
 * default shapes. */
typedef struct bsnn_batch_tuning {
    uint32_t k_tiles_per_unit;
    uint32_t operand_stages;
    uint32_t candidates;
    float us_per_step;
    float default_us_per_step;
} bsnn_batch_tuning;

/* Before the first step: times candidate unit sizes and ring depths over trial_steps clock steps
 * each on the device and keeps the fastest (the batch stays at step 0).  out may be null. */
BSNN_API bsnn_status bsnn_batch_autotune(bsnn_batch* batch, uint32_t trial_steps, bsnn_batch_tuning* out);
/* Applies shapes an earlier autotune found (0 fields keep the defaults), before the first step. */
BSNN_API bsnn_status bsnn_batch_set_tuning(bsnn_batch* batch, const bsnn_batch_tuning* tuning);

/* ---- the differentiation form (no reference counterpart) -------------------------------------
 * A surrogate-gradient adjoint of the two-group network with frozen weights: the forward pass is
 * the reference's step without plasticity (FP32), checkpointed every checkpoint_interval steps;
 * the backward pass replays each segment and propagates adjoints back through time, with the
 * spike's derivative replaced by the fast sigmoid 1 / (1 + |u - v_th| / surrogate_beta)^2 (0 turns
 * it off) and the reset not differentiated.  The loss is
 *   rate_weight / T * sum_t (rho_t - rho*_t)^2 + voltage_weight / T * sum_t (vbar_{t+1} - v*_t)^2,
 * rho the excitatory population rate (Hz) smoothed with time constant rate_tau, vbar the mean
 * excitatory membrane potential; the gradients are dL/dW_EE and dL/dg_leak (g_leak shared by the
 * two groups).  Needs only plain CUDA. */
typedef struct bsnn_adjoint bsnn_adjoint;

typedef struct bsnn_adjoint_desc {
    uint32_t num_excitatory;
    uint32_t num_inhibitory;
    uint32_t num_steps;
    uint32_t checkpoint_interval;
    int32_t rng_seed;
    int32_t noise_on;
    float rate_tau;        /* s  */
    float surrogate_beta;  /* V  */
    float rate_weight;
    float voltage_weight;
} bsnn_adjoint_desc;

BSNN_API bsnn_status bsnn_adjoint_create(const bsnn_adjoint_desc* desc, const bsnn_neuron_group_params* excitatory_group,
                                         const bsnn_neuron_group_params* inhibitory_group,
                                         const bsnn_connection_params* excitatory_pre,
                                         const bsnn_connection_params* inhibitory_pre, const float* w_ee,
                                         const float* w_ei, const float* w_ie, const float* w_ii,
                                         const uint32_t* stimulus_counts, uint32_t stimulus_steps,
                                         const uint32_t* stimulus_neurons, const float* stimulus_deltas,
                                         uint32_t num_events, int32_t device, bsnn_adjoint** out_adjoint);
BSNN_API bsnn_status bsnn_adjoint_destroy(bsnn_adjoint* adjoint);
BSNN_API const char* bsnn_adjoint_last_error(const bsnn_adjoint* adjoint);
/* The stream the passes run on (cudaStream_t), and the number of kernels run so far (the kernels
 * of the captured per-segment graphs included). */
BSNN_API bsnn_status bsnn_adjoint_get_stream(bsnn_adjoint* adjoint, void** out_stream);
BSNN_API bsnn_status bsnn_adjoint_kernel_launches(bsnn_adjoint* adjoint, uint64_t* out);
/* New E->E weights (row-major [E][E]; null keeps them) and g_leak (NaN keeps it). */
BSNN_API bsnn_status bsnn_adjoint_set_params(bsnn_adjoint* adjoint, const float* w_ee, float g_leak);
/* Forward pass over num_steps: targets of num_steps values (voltage_target may be null when
 * voltage_weight is 0); optional outputs: the loss, rho_t and vbar_{t+1}. */
BSNN_API bsnn_status bsnn_adjoint_forward(bsnn_adjoint* adjoint, const float* rate_target, const float* voltage_target,
                                          float* loss_out, float* rate_out, float* mean_voltage_out);
/* Gradients of the last forward pass's loss: dL/dW_EE (row-major [E][E]) and dL/dg_leak. */
BSNN_API bsnn_status bsnn_adjoint_backward(bsnn_adjoint* adjoint, float* grad_w_ee, double* grad_g_leak);

#ifdef __cplusplus
}
#endif

#endif /* BSNN_H */
