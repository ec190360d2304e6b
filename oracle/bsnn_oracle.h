/*
 * bsnn_oracle.h -- CPU oracle for the per-step hot path (TEST INFRASTRUCTURE ONLY).
 *
 * A sequential CPU restatement of what the reference's CUDA kernels compute for
 * System::step_the_clock (cpp_src/core/system.cpp:43-63), kernel by kernel in launch order.
 * It exists to check libbsnn: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  The product path never calls it.
 *
 * Precision: OR_PREC_F32 repeats the reference's FP32 arithmetic statement by statement
 * (compiled without FP contraction); OR_PREC_F64 runs the same model in double precision with
 * the same float-valued parameters, as the reference point for reduced-precision error.
 *
 * Parity pinning: the reference ships no tests, fixtures or golden vectors.  This oracle is
 * pinned (1) by hand-derived known-answer cases in tests/golden (single neuron, trace impulse
 * response, refractory timing, stimulus on/off, single-pair plasticity updates, the
 * column-sum normalisation quirk), (2) by Philox4x32-10 known-answer vectors, and (3) by
 * dumps of the reference's own CUDA build run on a B200 (oracle/ref_harness, outputs under
 * tests/golden/ref_*).
 *
 * The API mirrors include/bsnn.h (same parameter structs, same field codes) so a test can drive
 * both with one description.
 */
#ifndef BSNN_ORACLE_H
#define BSNN_ORACLE_H

#include "../include/bsnn.h"

#ifdef __cplusplus
extern "C" {
#endif

#define OR_PREC_F32 32
#define OR_PREC_F64 64

typedef struct or_sim or_sim;

BSNN_API or_sim* or_create(const bsnn_state_desc* desc, int32_t precision);
BSNN_API void or_destroy(or_sim* s);
BSNN_API const char* or_last_error(const or_sim* s);
BSNN_API int32_t or_add_neuron_group(or_sim* s, const bsnn_neuron_group_params* p, uint32_t* out);
BSNN_API int32_t or_add_connection(or_sim* s, uint32_t pre, uint32_t post, const float* w,
                                   const bsnn_connection_params* p, uint32_t* out);
BSNN_API int32_t or_add_stimulus(or_sim* s, const uint32_t* counts, uint32_t n_steps, const uint32_t* ids,
                                 const uint32_t* offsets, const float* deltas, uint32_t n_events);
BSNN_API int32_t or_add_plasticity(or_sim* s, int32_t kind, uint32_t conn, const bsnn_plasticity_params* p,
                                   uint32_t* out);
BSNN_API int32_t or_add_spike_recorder(or_sim* s, uint32_t group, uint32_t interval, uint32_t* out);
BSNN_API int32_t or_add_voltage_recorder(or_sim* s, uint32_t group, const uint32_t* ids, uint32_t n_ids,
                                         uint32_t interval, uint32_t* out);
BSNN_API int32_t or_set_noise_mode(or_sim* s, int32_t mode);
BSNN_API int32_t or_set_noise_replay(or_sim* s, const uint8_t* counts, uint32_t n_steps);
BSNN_API int32_t or_step(or_sim* s, uint32_t clock_step);
BSNN_API int32_t or_run(or_sim* s, uint32_t first_clock_step, uint32_t n_steps);
/* Advances the step counter and the stimulus cursors by n steps without simulating them (for
 * tests that copy a device state into the oracle at step n). */
BSNN_API int32_t or_skip_steps(or_sim* s, uint32_t n);
/* Same field codes as bsnn_read_state; values converted to float (uint32 fields as uint32). */
BSNN_API int32_t or_read_state(or_sim* s, int32_t field, uint32_t index, uint32_t offset, uint32_t count,
                               void* out);
/* Same, as double (exact state of the F64 oracle). */
BSNN_API int32_t or_read_state_f64(or_sim* s, int32_t field, uint32_t index, uint32_t offset, uint32_t count,
                                   double* out);
BSNN_API int32_t or_write_state(or_sim* s, int32_t field, uint32_t index, uint32_t offset, uint32_t count,
                                const void* in);
BSNN_API int32_t or_read_weights(or_sim* s, uint32_t conn, float* out);
BSNN_API int32_t or_write_weights(or_sim* s, uint32_t conn, const float* in);
BSNN_API int32_t or_read_weights_f64(or_sim* s, uint32_t conn, double* out);
BSNN_API int32_t or_read_spike_history(or_sim* s, uint32_t mon, uint32_t* out, int32_t flush);
BSNN_API int32_t or_read_voltage_history(or_sim* s, uint32_t mon, float* out, int32_t flush);
/* Poisson counts the oracle drew at its last step: out[neuron * 2 + channel]. */
BSNN_API int32_t or_last_noise_counts(or_sim* s, uint8_t* out);

/* Philox4x32-10 block function and the Poisson sampler, exposed for known-answer tests. */
BSNN_API void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
BSNN_API uint32_t or_poisson(float exp_neg_mean, uint32_t seed, uint32_t neuron, uint64_t step, uint32_t channel);

/* One connection's propagation on host arrays (kernel_connection_propagate_launch,
 * cpp_src/connections/kernel_connection_propagate.cu:8-46, 64-111): r, d and x [n_pre] are updated
 * in place and g [n_post] += W^T x with W row-major [n_pre][n_post], dot products in double. */
BSNN_API void or_connection_propagate(float r_decay, float d_decay, float norm, uint32_t n_pre, uint32_t n_post,
                                      const float* w, float* r, float* d, float* x, float* g,
                                      const uint32_t* spikes);

#ifdef __cplusplus
}
#endif

#endif /* BSNN_ORACLE_H */
