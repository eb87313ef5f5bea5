/*
 * nest_oracle.h -- CPU restatement of NEST's per-min_delay simulation cycle.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA engine is
 * compared against; nothing in the product links, loads or calls it.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * It restates, in plain C with FP64 arithmetic and no FP contraction, what
 * the reference computes on this path:
 *   - iaf_psc_delta::pre_run_hook / update  (models/iaf_psc_delta.cpp:234-329)
 *   - iaf_psc_exp::pre_run_hook / update    (models/iaf_psc_exp.cpp:244-348)
 *   - IAFPropagator / IAFPropagatorExp      (libnestutil/iaf_propagator.cpp:42-75,
 *                                            libnestutil/iaf_propagator.h:152-159)
 *   - aeif_cond_alpha dynamics / update     (models/aeif_cond_alpha.cpp:74-126, 450-533)
 *     with an adaptive Runge-Kutta-Fehlberg 4(5) step following GSL's
 *     documented rkf45 / control_yp / evolve_apply behaviour (GSL is an
 *     external dependency of the reference, not vendored).
 *   - ring-buffer delivery: slot = (t_emit + d) mod (min_delay + max_delay)
 *     (nestkernel/event.h:1006-1013, event_delivery_manager.cpp:251-303,
 *     ring_buffer.h:169-181)
 *   - spike_recorder: stamp = t_emit + 1 (models/spike_recorder.cpp:100-112)
 *   - poisson_generator drive: a draw per target per generator step t_g with
 *     start < t_g <= stop, arriving at t_g + d (models/poisson_generator.cpp:
 *     125-148, nestkernel/stimulation_device.cpp:47-57).  The draw itself uses
 *     a counter-based Philox4x32-10 stream and inversion over a CDF table, so the
 *     drive is statistically (not bitwise) equal to the reference's
 *     std::poisson_distribution over mt19937_64.
 *
 * Parity status: pinned bit-exactly to the reference's own spike raster and
 * final V_m on the golden fixtures in tests/golden/ (generated by running the
 * reference), and to the reference's propagator code compiled from
 * libnestutil sources (oracle/build_ref.sh).
 */
#ifndef NEST_ORACLE_H
#define NEST_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_IAF_PSC_DELTA = 0, ORC_IAF_PSC_EXP = 1, ORC_AEIF_COND_ALPHA = 2, ORC_IAF_PSC_ALPHA = 3 };

typedef struct orc_net orc_net;

/* h in ms; delays in steps; ring length L = min_delay + max_delay. */
orc_net* orc_create( int model, int64_t n, double h, int32_t min_delay, int32_t max_delay );
void orc_destroy( orc_net* net );
const char* orc_error( void );

/* Set a per-neuron parameter or state array (length n) by name.  Names are
 * the model's internal representation (e.g. V_m_rel = V_m - E_L for the iaf
 * models), see nest_oracle.c for the list. */
int orc_set( orc_net* net, const char* name, const double* values );
int orc_get( orc_net* net, const char* name, double* out );

/* Connectivity in CSR over sources 0..n_src-1 (the first n are the neurons,
 * the rest are spike-generator sources).  Delays in steps. */
int orc_set_csr( orc_net* net, int64_t n_src, const int64_t* row_ptr, const int32_t* tgt, const double* w,
  const int32_t* d, int nthreads );

/* Spikes of generator sources: emission step t_e (stamp - 1) and source. */
int orc_set_sched( orc_net* net, int64_t n, const int64_t* step, const int32_t* src );

/* Poisson drive per neuron (rate <= 0: none). start/stop in steps (exclusive
 * start, inclusive stop, as NEST's StimulationDevice). */
int orc_set_poisson( orc_net* net, const double* rate_hz, const double* w, const int32_t* d, int64_t start_step,
  int64_t stop_step, uint64_t seed );

/* Which sources are logged to the spike log (length n_src; NULL = all). */
int orc_set_record( orc_net* net, const uint8_t* flags );

/* Record an internal state variable of the listed neurons after every step. */
int orc_set_trace( orc_net* net, int64_t n_idx, const int32_t* idx, const char* var );

/* Advance the network by n_steps (any count; partial slices are handled as
 * NEST does).  nthreads <= 0 uses all OpenMP threads. */
int orc_run( orc_net* net, int64_t n_steps, int nthreads );

int64_t orc_n_spikes( orc_net* net );
/* Copy out the spike log (source, stamp step) in emission order. */
int64_t orc_get_spikes( orc_net* net, int32_t* src, int64_t* stamp, int64_t cap );
int64_t orc_n_trace( orc_net* net );
int64_t orc_get_trace( orc_net* net, double* out, int64_t cap );
int64_t orc_clock( orc_net* net );
int64_t orc_syn_events( orc_net* net );

/* Propagator restatement (libnestutil/iaf_propagator.cpp) for pinning. */
double orc_iaf_propagator_exp( double tau_syn, double tau_m, double c_m, double h );
/* stdp_pl_synapse_hom connections (models/stdp_pl_synapse_hom.h) as a CSR over
 * neuron sources, with the common properties lambda, alpha, mu, tau_plus;
 * the postsynaptic neurons' tau_minus is the variable "tau_minus" */
int orc_set_plastic( orc_net* net, int64_t n_src, const int64_t* row_ptr, const int32_t* tgt, const double* w,
  const int32_t* d, double lambda, double alpha, double mu, double tau_plus );
int orc_get_plastic( orc_net* net, double* w );
/* IAFPropagatorAlpha::evaluate (libnestutil/iaf_propagator.cpp:95-118): out[0] = P31, out[1] = P32 */
void orc_iaf_propagator_alpha( double tau_syn, double tau_m, double c_m, double h, double* out );

/* Philox4x32-10 block (Salmon et al., SC'11) for known-answer tests. */
void orc_philox4x32( const uint32_t ctr[ 4 ], const uint32_t key[ 2 ], int rounds, uint32_t out[ 4 ] );

/* Poisson draw by inversion (CDF table, or the walk from the mode for long tables). */
int64_t orc_poisson_draw( double lambda, double u );

#ifdef __cplusplus
}
#endif
#endif
