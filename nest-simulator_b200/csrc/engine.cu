// engine.cu -- host side of the slice engine and the extern "C" ABI of
// include/nestgpu.h.
//
// The host computes every FP64 coefficient with the C library's exp/expm1
// by the same formulas as the reference's pre_run_hook functions, dedupes
// them into coefficient classes, and uploads them; the device never
// recomputes them.  The slice driver mirrors SimulationManager::update_
// (nestkernel/simulation_manager.cpp:842-1189): node updates over the lags of
// a slice, then delivery of the slice's spikes; partial slices are allowed.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <chrono>
#include <string>
#include <unordered_map>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <new>

#include "../../include/nestgpu.h"
#include "ng_kernels.cuh"
#include "ng_persistent.cuh"
#include "ng_serving.cuh"
#include "ng_stdp.cuh"

using namespace ng;

namespace
{

thread_local std::string g_err;

int
fail( int code, const std::string& msg )
{
  g_err = msg;
  return code;
}

#define CU( call )                                                                                       \
  do                                                                                                     \
  {                                                                                                      \
    cudaError_t e_ = ( call );                                                                           \
    if ( e_ != cudaSuccess )                                                                             \
      return fail( e_ == cudaErrorMemoryAllocation ? NG_ERR_MEMORY : NG_ERR_CUDA,                        \
        std::string( #call ) + ": " + cudaGetErrorString( e_ ) );                                        \
  } while ( 0 )

enum VarKind
{
  PARAM = 0,
  STATE = 1,
  REFR = 2,
  ISTEP = 3
};

struct VarSpec
{
  const char* name;
  int kind;
  int slot;
};

// Internal representation of each model's Parameters_ and State_.
const VarSpec DELTA_VARS[] = { { "tau_m", PARAM, 0 }, { "C_m", PARAM, 1 }, { "t_ref", PARAM, 2 },
  { "V_th_rel", PARAM, 3 }, { "V_reset_rel", PARAM, 4 }, { "V_min_rel", PARAM, 5 }, { "V_m_rel", STATE, 0 },
  { "y0", STATE, 1 }, { "I_e", STATE, 2 }, { "r", REFR, 0 }, { nullptr, 0, 0 } };
const VarSpec EXP_VARS[] = { { "tau_m", PARAM, 0 }, { "C_m", PARAM, 1 }, { "t_ref", PARAM, 2 },
  { "V_th_rel", PARAM, 3 }, { "V_reset_rel", PARAM, 4 }, { "tau_syn_ex", PARAM, 5 }, { "tau_syn_in", PARAM, 6 },
  { "V_m_rel", STATE, 0 }, { "I_syn_ex", STATE, 1 }, { "I_syn_in", STATE, 2 }, { "i_0", STATE, 3 },
  { "i_1", STATE, 4 }, { "I_e", STATE, 5 }, { "r", REFR, 0 }, { nullptr, 0, 0 } };
const VarSpec AEIF_VARS[] = { { "V_peak", PARAM, 0 }, { "V_reset", PARAM, 1 }, { "t_ref", PARAM, 2 },
  { "g_L", PARAM, 3 }, { "C_m", PARAM, 4 }, { "E_ex", PARAM, 5 }, { "E_in", PARAM, 6 }, { "E_L", PARAM, 7 },
  { "Delta_T", PARAM, 8 }, { "tau_w", PARAM, 9 }, { "a", PARAM, 10 }, { "b", PARAM, 11 }, { "V_th", PARAM, 12 },
  { "tau_syn_ex", PARAM, 13 }, { "tau_syn_in", PARAM, 14 }, { "gsl_error_tol", PARAM, 15 }, { "V_m", STATE, 0 },
  { "dg_ex", STATE, 1 }, { "g_ex", STATE, 2 }, { "dg_in", STATE, 3 }, { "g_in", STATE, 4 }, { "w", STATE, 5 },
  { "I_e", STATE, 6 }, { "r", REFR, 0 }, { "integration_step", ISTEP, 0 }, { nullptr, 0, 0 } };

// iaf_psc_alpha: the state in iaf_psc_exp's slot layout (V_m, I_syn_ex,
// I_syn_in, then the derivatives dI_ex, dI_in of the alpha currents, I_e)
const VarSpec ALPHA_VARS[] = { { "tau_m", PARAM, 0 }, { "C_m", PARAM, 1 }, { "t_ref", PARAM, 2 },
  { "V_th_rel", PARAM, 3 }, { "V_reset_rel", PARAM, 4 }, { "tau_syn_ex", PARAM, 5 }, { "tau_syn_in", PARAM, 6 },
  { "V_min_rel", PARAM, 7 }, { "V_m_rel", STATE, 0 }, { "I_syn_ex", STATE, 1 }, { "I_syn_in", STATE, 2 },
  { "dI_syn_ex", STATE, 3 }, { "dI_syn_in", STATE, 4 }, { "I_e", STATE, 5 }, { "r", REFR, 0 }, { nullptr, 0, 0 } };

const VarSpec*
vars_of( int model )
{
  return model == NG_IAF_PSC_DELTA ? DELTA_VARS
    : model == NG_IAF_PSC_EXP      ? EXP_VARS
    : model == NG_IAF_PSC_ALPHA    ? ALPHA_VARS
                                   : AEIF_VARS;
}
int
n_params( int model )
{
  return model == NG_IAF_PSC_DELTA ? 6 : model == NG_IAF_PSC_EXP ? 7 : model == NG_IAF_PSC_ALPHA ? 8 : 16;
}
int
n_states( int model )
{
  return model == NG_IAF_PSC_DELTA ? 3 : model == NG_IAF_PSC_EXP ? 6 : model == NG_IAF_PSC_ALPHA ? 6 : 7;
}
// the coefficient row index of RefractoryCounts
int
refr_index( int model )
{
  return model == NG_IAF_PSC_DELTA ? 5 : model == NG_IAF_PSC_EXP ? 8 : model == NG_IAF_PSC_ALPHA ? 15 : 18;
}
// models whose input splits into excitatory/inhibitory channels by the weight's sign
bool
sign_channels( int model )
{
  return model == NG_IAF_PSC_EXP || model == NG_IAF_PSC_ALPHA;
}
const VarSpec*
find_var( int model, const char* name )
{
  for ( const VarSpec* v = vars_of( model ); v->name; ++v )
    if ( std::strcmp( v->name, name ) == 0 )
      return v;
  return nullptr;
}

// Reference defaults (Parameters_::Parameters_ / State_::State_ of each model).
void
default_params( int model, std::vector< double >& p )
{
  if ( model == NG_IAF_PSC_DELTA )
    p = { 10.0, 250.0, 2.0, -55.0 - ( -70.0 ), -70.0 - ( -70.0 ), -1.7976931348623157e308 };
  else if ( model == NG_IAF_PSC_EXP )
    p = { 10.0, 250.0, 2.0, -55.0 - ( -70.0 ), -70.0 - ( -70.0 ), 2.0, 2.0 };
  else if ( model == NG_IAF_PSC_ALPHA )
    p = { 10.0, 250.0, 2.0, -55.0 - ( -70.0 ), -70.0 - ( -70.0 ), 2.0, 2.0, -HUGE_VAL };
  else
    p = { 0.0, -60.0, 0.0, 30.0, 281.0, 0.0, -85.0, -70.6, 2.0, 144.0, 4.0, 80.5, -50.4, 0.2, 2.0, 1e-6 };
}
double
default_state( int model, int slot )
{
  if ( model == NG_AEIF_COND_ALPHA && slot == 0 )
    return -70.6;
  return 0.0;
}

// IAFPropagatorExp::evaluate (libnestutil/iaf_propagator.cpp:42-75,
// iaf_propagator.h:152-159): P32 with the singular tau_m ~ tau_syn branch.
double
propagator_exp( double tau_syn, double tau_m, double c_m, double h )
{
  const double beta = tau_syn * tau_m / ( tau_m - tau_syn );
  const double gamma = beta / c_m;
  const double inv_tau_syn = 1 / tau_syn;
  const double inv_tau_m = 1 / tau_m;
  const double inv_c_m = 1 / c_m;
  const double inv_beta = ( tau_m - tau_syn ) / ( tau_syn * tau_m );
  const double exp_h_tau_syn = std::exp( -h * inv_tau_syn );
  const double expm1_h_tau = std::expm1( h * inv_beta );
  const double P32 = gamma * exp_h_tau_syn * expm1_h_tau;
  if ( std::isnormal( P32 ) and P32 > 0 )
    return P32;
  const double exp_h_tau = std::exp( -h * inv_tau_m );
  return h * inv_c_m * exp_h_tau;
}

// IAFPropagatorAlpha::evaluate (libnestutil/iaf_propagator.cpp:95-118, with
// the P32 of :56-75 and NUMERICAL_STABILITY_FACTOR_ = 1e-7,
// iaf_propagator.h:66): (P31, P32), each with its singular tau_m ~ tau_syn
// form.  The same formulas and operation order (bit-equal coefficients).
void
propagator_alpha( double tau_syn, double tau_m, double c_m, double h, double* P31, double* P32 )
{
  const double h_min_regular = 1e-7 * tau_m * tau_m / std::abs( tau_m - tau_syn );
  const double beta = tau_syn * tau_m / ( tau_m - tau_syn );
  const double gamma = beta / c_m;
  const double inv_tau_syn = 1 / tau_syn;
  const double inv_tau_m = 1 / tau_m;
  const double inv_c_m = 1 / c_m;
  const double inv_beta = ( tau_m - tau_syn ) / ( tau_syn * tau_m );
  const double exp_h_tau_syn = std::exp( -h * inv_tau_syn );
  const double expm1_h_tau = std::expm1( h * inv_beta );
  double p32 = gamma * exp_h_tau_syn * expm1_h_tau;
  double exp_h_tau = std::nan( "" );
  if ( !( std::isnormal( p32 ) and p32 > 0 ) )
  {
    exp_h_tau = std::exp( -h * inv_tau_m );
    p32 = h * inv_c_m * exp_h_tau;
  }
  *P32 = p32;
  if ( h > h_min_regular )
  {
    *P31 = gamma * exp_h_tau_syn * ( beta * expm1_h_tau - h );
    return;
  }
  if ( std::isnan( exp_h_tau ) )
    exp_h_tau = std::exp( -h * inv_tau_m );
  *P31 = 0.5 * h * h * inv_c_m * exp_h_tau;
}

// Poisson table (lambda, p_m, F_m, m) for inversion from the mode.
double4
poisson_table( double lambda )
{
  if ( !( lambda > 0.0 ) )
    return make_double4( 0.0, 1.0, 1.0, 0.0 );
  const double m = std::floor( lambda );
  const double pm = std::exp( -lambda + m * std::log( lambda ) - std::lgamma( m + 1.0 ) );
  double p = std::exp( -lambda ), F = p;
  for ( long long k = 1; k <= ( long long ) m; ++k )
  {
    p = p * lambda / ( double ) k;
    F += p;
  }
  return make_double4( lambda, pm, F, m );
}

// CDF table of Poisson(lambda): cdf[k] = P(X <= k), summed upward in FP64,
// up to 1 - cdf < 1e-17 or 256 entries; the last entry is set to 1 so the
// search always ends.  Returns false when the table would be too long.
// Stored as thresholds floor(cdf[k] * 2^53): a uniform u = m * 2^-53 (m a
// 53-bit integer) exceeds cdf[k] exactly when m exceeds the threshold.
bool
poisson_cdf_table( double lambda, std::vector< uint64_t >& cdf )
{
  cdf.clear();
  if ( lambda > 100.0 )
    return false;
  const auto thr = []( double F ) { return ( uint64_t ) std::floor( F * 9007199254740992.0 ); };
  double p = std::exp( -lambda ), F = p;
  cdf.push_back( thr( F ) );
  for ( int k = 1; k < 256; ++k )
  {
    p = p * lambda / ( double ) k;
    F += p;
    cdf.push_back( thr( F ) );
    if ( 1.0 - F < 1e-17 && ( double ) k > lambda )
      break;
  }
  if ( 1.0 - F > 1e-15 )
    return false;
  cdf.back() = thr( 1.0 );
  return true;
}

struct DevBuf
{
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct ng_engine
{
  ng_config cfg {};
  int prec = NG_FP64;
  size_t rsz = 8;  // bytes per state element
  double h = 0.1;
  int64_t tics_per_step = 100;
  int64_t N = 0, n_src = 0;
  int L = 0, C = 2;
  int sms = 148;
  cudaStream_t own = nullptr, stream = nullptr;

  struct Blk
  {
    int model = 0;
    int64_t off = 0, n = 0;
    std::vector< std::vector< double > > par;  // [param][neuron]
    bool dirty = true;
    DevBuf st[ MAX_STATE ], r, istep, cls, ctab;
    DevBuf perm, bins;  // aeif: substep-binned thread order and its counting-sort counters
    int64_t n_classes = 0;
    std::vector< double > host_ctab;
    std::vector< int32_t > host_cls;
  };
  std::vector< Blk > blk;

  DevBuf ring, row_beg, row_len, real_deg, tdc, w, ent, log, rec, pois, pois_w, pois_d, pois_ref, pois_cdf, trace_col,
    trace, sched_step, sched_src, ctl, row_ue, row_ls, ent_late;
  int32_t tbits = 1;
  int ring_bytes = 8;  // 4: 32-bit fixed-point ring cells (serving, FP32 form)
  uint32_t tmask = 1, dmask = 0;
  double fx_inv = 1.0;
  int64_t nnz_padded = 0, ent_cap = 0, log_cap = 0, n_sched = 0, n_rec = 0;
  int64_t chunks_all_src = 0, chunks_max_gen = 0;  // for the delivery work capacity
  int has_pois = 0;
  int64_t pois_start = 0, pois_stop = INT64_MAX;
  uint32_t key0 = 0, key1 = 0;
  int32_t n_trace_idx = 0, trace_interval = 1, n_trace_vars = 0;
  int8_t trace_slot[ MAX_STATE ] = { 0, 0, 0, 0, 0, 0, 0, 0 };
  int64_t trace_rows_cap = 0;
  std::vector< int64_t > host_sched_step;

  // clock: absolute step = slice origin + from
  int64_t origin = 0;
  int32_t from = 0;
  int64_t slices = 0;

  // drained output
  std::vector< int32_t > out_src;
  std::vector< int64_t > out_stamp;
  std::vector< double > out_trace;
  int64_t trace_first_stamp = -1;
  int64_t next_trace_stamp_row = 0;  // absolute row index (stamp / interval) of the next row expected

  Ctl* host_ctl = nullptr;  // pinned, one per log half
  cudaEvent_t group_done[ 2 ] = { nullptr, nullptr };
  cudaStream_t copy_stream = nullptr;
  uint2* pinned_log = nullptr;
  size_t pinned_log_bytes = 0;
  // pinned staging of an admission's per-neuron uploads (ng_net_add): kept
  // across calls, so an admission neither pins nor first-touches fresh host
  // memory; reused only after the admission stream has drained
  char* adm_pin = nullptr;
  size_t adm_pin_bytes = 0;
  ng_stats stats {};
  int profiling = 0;
  int graph_slices = 0;
  // instantiated graphs of k full slices (k in {graph_slices, 16, 4, 1}),
  // plain or with an event pair around every kernel (profiling)
  struct GraphEntry
  {
    int slices = 0;
    bool prof = false;
    int64_t gen = -1;
    cudaGraphExec_t exec = nullptr;
    std::vector< cudaEvent_t > ev;
  };
  std::vector< GraphEntry > graphs;
  int64_t generation = 0;
  std::vector< uint8_t > rec_host;
  double log_per_step = 1.0;  // bound on recorded neuron spikes per step (refractoriness)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector< DevBuf* > all;
  int deliver_ctas = 0, deliver_per_sm = 4;

  // ---- late delivery: the edges of delay >= 2 min_delay of a slice's
  // spikes are delivered on a second stream while the next slice updates
  // (its update reads no ring slot they reach); the slice after that waits
  // for them.  Rows hold their shorter-delay edges first (row_ue, row_ls).
  cudaStream_t late_stream = nullptr;
  // admissions prepare a network's region (state, tables, graph) on their own
  // stream while the slices already enqueued run; only the activation of the
  // network is ordered behind them
  cudaStream_t adm_stream = nullptr;
  cudaEvent_t ev_adm = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_late[ 2 ] = { nullptr, nullptr };
  bool late_pending[ 2 ] = { false, false };
  bool late_env = true;
  int32_t late_min_cur = INT32_MAX;  // in force: 2 min_delay, or INT32_MAX (off)
  int late_ctas = 1, late_per_sm = 2;

  // rows are split by delay class when the ring can hold such edges and the
  // target-tiled delivery (which needs target-sorted rows) is off
  bool
  late_possible() const
  {
    return !tiled_on && cfg.max_delay >= 2 * cfg.min_delay;
  }

  int32_t
  late_thr() const
  {
    return late_possible() ? 2 * cfg.min_delay : INT32_MAX;
  }

  // off while a network uses the per-target gather: its plain ring updates
  // must not meet a late delivery's atomics on the same cells (a network can
  // turn from scatter to gather between two slices)
  int32_t
  late_target() const
  {
    if ( !late_possible() || !late_env )
      return INT32_MAX;
    if ( gather_on )
      for ( size_t id = 0; id < nets.size(); ++id )
        if ( nets[ id ].used && host_g[ id ].ke + host_g[ id ].ki > 0 )
          return INT32_MAX;
    return 2 * cfg.min_delay;
  }

  // a network with a per-target gather table is admitted: the gather kernel
  // is launched every slice (it needs whole SMs, so it would also wait for
  // any delivery still running)
  bool gather_live = false;

  void
  refresh_late()
  {
    const int32_t v = late_target();
    bool gl = false;
    if ( gather_on )
      for ( size_t id = 0; id < nets.size(); ++id )
        gl = gl || ( nets[ id ].used && host_g[ id ].ke + host_g[ id ].ki > 0 );
    if ( v != late_min_cur || gl != gather_live )
    {
      late_min_cur = v;
      gather_live = gl;
      ++generation;
    }
    late_ctas = std::max( 1, std::min( deliver_ctas, sms * std::min( late_per_sm, deliver_per_sm ) ) );
  }

  // ---- serving: networks added to and removed from the running engine
  bool serving = false;
  DevBuf d_nid, d_step0, d_until, d_off, d_key, sc_src, sc_cnt, sc_fill, sc_beg, sc_plen, sc_total, sc_sb, sc_bound;
  std::vector< int32_t > nid_host;
  // Spikes of a serving network: the raw log entries of each group, as
  // grouped by network on the device, decoded only when they are read.
  struct RawBlock
  {
    int64_t clock = 0;  // log base (stamp offset) of the group
    uint2* e = nullptr;
    int64_t n = 0;
    int64_t m = 0;      // spikes (multiplicities summed)
  };

  static void
  free_blocks( std::vector< RawBlock >& bs )
  {
    for ( auto& b : bs )
      std::free( b.e );
    bs.clear();
  }

  struct NetInfo
  {
    bool used = false;
    int64_t off = 0, n = 0, e0 = 0, ne = 0, step0 = 0, until = 0;
    int64_t g0 = -1, gn = 0;  // gather table run
    int64_t s0 = -1, sn = 0;  // segment table run (target-tiled delivery)
    bool rec = false;
    double log_rate = 0.0;
    std::vector< RawBlock > blocks;  // logged spikes, group by group
    int64_t held = 0;                // spikes held (multiplicities counted)
    int64_t first = 0;               // entries of blocks[0] already drained
  };
  std::vector< NetInfo > nets;
  std::map< int64_t, int64_t > free_neurons, free_edges;  // run start -> length
  // per-target gather of fixed_indegree networks (precision form)
  bool gather_on = false;
  float gather_frac = 0.08f;
  DevBuf gmask, gin, net_g, net_mode, net_spk;
  DevBuf log_sorted, log_cnt, log_off;  // spike log grouped by network (two halves)
  // target-tiled delivery of pairwise_bernoulli networks
  bool tiled_on = false;
  int tile_t = 0;
  size_t tile_smem = 0;
  DevBuf seg, net_t;
  std::map< int64_t, int64_t > free_seg;
  std::vector< TileNet > host_t;
  long long* host_off = nullptr;        // pinned, 2 x (max_networks + 1)
  std::map< int64_t, int64_t > free_gin;
  std::vector< GatherNet > host_g;
  std::unordered_map< std::string, int32_t > cls_ids;     // engine-wide coefficient classes
  int64_t cls_cap = 0, cdf_cap = 0;
  std::vector< uint64_t > cdf_host;
  std::unordered_map< double, int2 > cdf_tables;
  int fx_S = 0;

  static bool
  take_run( std::map< int64_t, int64_t >& fl, int64_t len, int64_t* start )
  {
    if ( len == 0 )
    {
      *start = 0;
      return true;
    }
    for ( auto it = fl.begin(); it != fl.end(); ++it )
      if ( it->second >= len )
      {
        *start = it->first;
        const int64_t rest = it->second - len, s2 = it->first + len;
        fl.erase( it );
        if ( rest > 0 )
          fl[ s2 ] = rest;
        return true;
      }
    return false;
  }

  static void
  give_run( std::map< int64_t, int64_t >& fl, int64_t start, int64_t len )
  {
    if ( len <= 0 )
      return;
    auto it = fl.emplace( start, len ).first;
    auto nx = std::next( it );
    if ( nx != fl.end() && it->first + it->second == nx->first )
    {
      it->second += nx->second;
      fl.erase( nx );
    }
    if ( it != fl.begin() )
    {
      auto pv = std::prev( it );
      if ( pv->first + pv->second == it->first )
      {
        pv->second += it->second;
        fl.erase( it );
      }
    }
  }

  // pools of a serving engine: every array sized for the capacity up front,
  // so admitting or retiring a network changes no device pointer and the
  // captured slice graphs stay valid
  int
  setup_serving()
  {
    int rc;
    const int64_t E = cfg.edge_capacity;
    const int nmax = cfg.max_networks;
    nets.assign( ( size_t ) nmax, NetInfo() );
    nid_host.assign( ( size_t ) N, -1 );
    if ( ( rc = alloc( d_nid, ( size_t ) N * 4 ) ) )
      return rc;
    k_fill_i32<<< ( unsigned ) ( ( N + 255 ) / 256 ), 256, 0, stream >>>( ( int32_t* ) d_nid.p, N, -1 );
    if ( ( rc = alloc( d_step0, ( size_t ) nmax * 8 ) ) || ( rc = alloc( d_until, ( size_t ) nmax * 8 ) )
      || ( rc = alloc( d_off, ( size_t ) nmax * 8 ) ) || ( rc = alloc( d_key, ( size_t ) nmax * 8 ) ) )
      return rc;
    if ( ( rc = alloc( tdc, ( size_t ) E * 4 ) ) || ( rc = alloc( w, ( size_t ) E * ( prec == NG_FP64 ? 8 : 4 ) ) ) )
      return rc;
    Blk& b = blk[ 0 ];
    cls_cap = 1 << 16;
    if ( ( rc = alloc( b.ctab, ( size_t ) cls_cap * CT_STRIDE * 8 ) ) || ( rc = alloc( b.cls, ( size_t ) N * 4 ) ) )
      return rc;
    b.host_cls.assign( ( size_t ) N, 0 );
    b.dirty = false;
    cdf_cap = 1 << 20;
    if ( ( rc = alloc( pois_cdf, ( size_t ) cdf_cap * 8 ) ) || ( rc = alloc( pois_ref, ( size_t ) N * 8 ) )
      || ( rc = alloc( pois, ( size_t ) N * sizeof( double4 ) ) ) || ( rc = alloc( pois_w, ( size_t ) N * 8 ) )
      || ( rc = alloc( pois_d, ( size_t ) N * 4 ) ) )
      return rc;
    has_pois = 1;
    if ( ( rc = alloc( rec, ( size_t ) N ) ) )
      return rc;
    rec_host.assign( ( size_t ) N, 0 );
    free_neurons.clear();
    free_edges.clear();
    free_neurons[ 0 ] = N;
    free_edges[ 0 ] = E;
    // per-target gather: precision form, current-based models, slices of at most 16 steps
    // (ng_set_option "gather" turns it off, "gather_frac" sets the switch point)
    gather_on = prec != NG_FP64 && b.model != NG_AEIF_COND_ALPHA && cfg.min_delay <= 16 && nmax <= 1024;
    if ( gather_on )
    {
      if ( cudaFuncSetAttribute( k_gather, cudaFuncAttributeMaxDynamicSharedMemorySize, ( int ) G_SMEM ) != cudaSuccess )
        return fail( NG_ERR_CUDA, "serving: cannot reserve shared memory for the per-target gather" );
      if ( ( rc = alloc( gmask, ( size_t ) N * 4 ) ) || ( rc = alloc( gin, ( size_t ) E * 2 ) )
        || ( rc = alloc( net_g, ( size_t ) nmax * sizeof( GatherNet ) ) ) || ( rc = alloc( net_mode, ( size_t ) nmax * 4 ) )
        || ( rc = alloc( net_spk, ( size_t ) nmax * 4 ) ) )
        return rc;
      CU( cudaMemsetAsync( gmask.p, 0, ( size_t ) N * 4, stream ) );
      CU( cudaMemsetAsync( net_g.p, 0, ( size_t ) nmax * sizeof( GatherNet ), stream ) );
      CU( cudaMemsetAsync( net_mode.p, 0, ( size_t ) nmax * 4, stream ) );
      CU( cudaMemsetAsync( net_spk.p, 0, ( size_t ) nmax * 4, stream ) );
      host_g.assign( ( size_t ) nmax, GatherNet {} );
      free_gin.clear();
      free_gin[ 0 ] = E;
    }
    // target-tiled delivery: a window of a tile's ring cells in 160 KiB of shared memory
    if ( cfg.tile_capacity > 0 && b.model != NG_AEIF_COND_ALPHA && nmax <= 1024 )
    {
      const size_t esz = ( size_t ) ring_bytes;
      const size_t W = ( size_t ) std::min( L, TILE_W );
      tile_t = ( int ) std::min< size_t >( 1024, ( 163840 / ( W * 2 * esz ) ) / 32 * 32 );
      if ( tile_t >= 32 )
      {
        tiled_on = true;
        tile_smem = W * C * tile_t * esz;
        cudaError_t ce;
        if ( prec == NG_FP64 )
          ce = cudaFuncSetAttribute( k_deliver_tiled< double, false >, cudaFuncAttributeMaxDynamicSharedMemorySize,
            ( int ) tile_smem );
        else if ( ring_bytes == 4 )
          ce = cudaFuncSetAttribute( k_deliver_tiled< int32_t, true >, cudaFuncAttributeMaxDynamicSharedMemorySize,
            ( int ) tile_smem );
        else
          ce = cudaFuncSetAttribute( k_deliver_tiled< long long, true >, cudaFuncAttributeMaxDynamicSharedMemorySize,
            ( int ) tile_smem );
        if ( ce != cudaSuccess )
          return fail( NG_ERR_CUDA, "serving: cannot reserve shared memory for the tiled delivery" );
        if ( ( rc = alloc( seg, ( size_t ) cfg.tile_capacity * 4 ) )
          || ( rc = alloc( net_t, ( size_t ) nmax * sizeof( TileNet ) ) ) )
          return rc;
        host_t.assign( ( size_t ) nmax, TileNet {} );
        free_seg.clear();
        free_seg[ 0 ] = cfg.tile_capacity;
      }
    }
    chunks_all_src = E / CHUNK_EDGES + N;
    if ( ( rc = resize_work() ) )
      return rc;
    // one fixed-point scale for every network (FP32 form)
    // 32-bit rings: the scale keeps the largest possible cell sum inside 31 bits
    const double mx = ring_bytes == 4 ? cfg.ring_bound : cfg.max_abs_weight > 0 ? cfg.max_abs_weight : 1e4;
    fx_S = ( int ) std::floor( std::log2( 2147483647.0 / mx ) );
    fx_S = std::max( -30, std::min( fx_S, 60 ) );
    fx_inv = prec == NG_FP64 ? 1.0 : std::ldexp( 1.0, -fx_S );
    log_per_step = 1.0;
    serving = true;
    ++generation;
    CU( cudaStreamSynchronize( stream ) );
    return NG_OK;
  }

  // Rows [n0, n0 + n) of a network drawn on the device, edges [e0, e0 + ne):
  // each row's edges of delay < 2 min_delay first, through a temporary copy
  // (without the memory for it, both deliveries walk the whole rows).
  int
  split_rows( int64_t n, int64_t n0, int64_t e0, int64_t ne )
  {
    if ( n <= 0 )
      return NG_OK;
    const size_t wsz = prec == NG_FP64 ? 8 : 4;
    void* st = nullptr;
    void* sw = nullptr;
    const unsigned gn = ( unsigned ) ( ( n + 255 ) / 256 );
    if ( ne > 0 && cudaMalloc( &st, ( size_t ) ne * 4 ) == cudaSuccess
      && cudaMalloc( &sw, ( size_t ) ne * wsz ) == cudaSuccess )
    {
      const unsigned g = ( unsigned ) ( ( n * 32 + 255 ) / 256 );
      if ( wsz == 8 )
        k_row_split< double ><<< g, 256, 0, stream >>>( n, n0, e0, ( const int64_t* ) row_beg.p,
          ( const int32_t* ) row_len.p, ( const int32_t* ) real_deg.p, ( const uint32_t* ) tdc.p, ( const double* ) w.p,
          ( uint32_t* ) st, ( double* ) sw, late_thr(), tbits, dmask, ( int32_t* ) row_ue.p, ( int32_t* ) row_ls.p );
      else
        k_row_split< int32_t ><<< g, 256, 0, stream >>>( n, n0, e0, ( const int64_t* ) row_beg.p,
          ( const int32_t* ) row_len.p, ( const int32_t* ) real_deg.p, ( const uint32_t* ) tdc.p, ( const int32_t* ) w.p,
          ( uint32_t* ) st, ( int32_t* ) sw, late_thr(), tbits, dmask, ( int32_t* ) row_ue.p, ( int32_t* ) row_ls.p );
      cudaError_t ce = cudaGetLastError();
      if ( ce == cudaSuccess )
        ce = cudaMemcpyAsync( ( uint32_t* ) tdc.p + e0, st, ( size_t ) ne * 4, cudaMemcpyDeviceToDevice, stream );
      if ( ce == cudaSuccess )
        ce = cudaMemcpyAsync( ( char* ) w.p + ( size_t ) e0 * wsz, sw, ( size_t ) ne * wsz, cudaMemcpyDeviceToDevice,
          stream );
      if ( ce == cudaSuccess )
        ce = cudaStreamSynchronize( stream );
      cudaFree( st );
      cudaFree( sw );
      if ( ce != cudaSuccess )
        return fail( NG_ERR_CUDA, std::string( "row split: " ) + cudaGetErrorString( ce ) );
      return NG_OK;
    }
    cudaGetLastError();  // a failed allocation leaves no sticky error
    if ( st )
      cudaFree( st );
    k_row_uniform<<< gn, 256, 0, stream >>>( n, n0, ( const int32_t* ) row_len.p, ne > 0 ? 2 : 1,
      ( int32_t* ) row_ue.p, ( int32_t* ) row_ls.p );
    CU( cudaGetLastError() );
    return NG_OK;
  }

  // channel word and stored weight of an edge into the block-0 model
  void
  edge_word( double wv, uint32_t* ch, double* we ) const
  {
    const int model = blk[ 0 ].model;
    *ch = 0;
    *we = wv;
    if ( sign_channels( model ) )
      *ch = wv > 0 ? 0u : 1u;
    else if ( model == NG_AEIF_COND_ALPHA && !( wv > 0.0 ) )
    {
      *ch = 1u;
      *we = -wv;
    }
  }

  int
  grow( DevBuf& b, size_t bytes )
  {
    if ( b.bytes >= bytes )
      return NG_OK;
    return alloc( b, bytes );
  }

  // admission scratch: grown to the next power of two (at least 1 MiB), so a
  // stream of networks of growing size reallocates -- and, through cudaFree,
  // waits for the running slices -- a few times, not at every new maximum
  int
  grow_scratch( DevBuf& b, size_t bytes )
  {
    if ( b.bytes >= bytes )
      return NG_OK;
    size_t want = ( size_t ) 1 << 20;
    while ( want < bytes )
      want <<= 1;
    return alloc( b, want );
  }

  // delivery work per slice: every source spiking at every lag, each spike
  // queueing ceil(padded degree / 128) chunks, plus the generator spikes
  int
  resize_work()
  {
    int64_t need = ( int64_t ) cfg.min_delay * chunks_all_src + n_sched * chunks_max_gen + 1024;
    need = std::min< int64_t >( need, 1ll << 28 );
    if ( need <= ent_cap && ( !late_possible() || ent_late.bytes >= 2 * ( size_t ) ent_cap * sizeof( int4 ) ) )
      return NG_OK;
    ent_cap = std::max( need, ent_cap );
    ++generation;
    int rc = alloc( ent, ( size_t ) ent_cap * sizeof( int4 ) );
    if ( rc == NG_OK && late_possible() )
      rc = alloc( ent_late, 2 * ( size_t ) ent_cap * sizeof( int4 ) );
    return rc;
  }
  // ---- launch configuration: chosen by the autotuner (measured on the
  // network's own first slices, cached per network shape and activity for
  // the process) or fixed through ng_set_tuning.  Every choice computes the
  // same result (the kernels share their arithmetic and its order).
  int tune_mode = 1;         // 0: fixed, 1: autotune (process cache first), 2: autotune, cache ignored
  int tune_state = 0;        // 0: pending, 1: measured, 2: from the process cache, 3: fixed
  int upd_variant = -1;      // iaf update kernel: 0/1/6 one thread per neuron (4/8/2 lags of inputs
                             // at a time), 2/3 two-phase (256/128 threads), 5 the persistent slice
                             // kernel (update and delivery of many slices in one launch); -1: by
                             // network size (serving engines: 6)
  DevBuf pk;                 // grid-barrier state of the persistent slice kernel
  // ---- stdp_pl_synapse_hom connections (ng_set_plastic_connections)
  bool plastic_on = false;
  DevBuf pl_row, pl_tgt, pl_dly, pl_w, pl_Kplus, pl_tlast, pl_ninc, pl_tauinv, pl_Kminus, pl_last, pl_hist_t, pl_hist_K,
    pl_hist_n, pl_hist_lo, pl_drop_t, pl_drop_K, pl_nflush, pl_in_row, pl_in_edge, pl_in_src, pl_wrun, pl_tab_fin,
    pl_tab_km;
  int64_t pl_nnz = 0, pl_nsrc = 0;
  double pl_dmax_ms = 0;
  int32_t pl_dconst = -1;  // the plastic delay when all are equal
  double pl_lambda = 0.1, pl_alpha = 1.0, pl_mu = 0.4, pl_tau_plus = 20.0;
  std::vector< double > tau_minus_host;  // per neuron, the postsynaptic trace's time constant (ArchivingNode)
  int pk_occ = -1;           // its resident CTAs per SM (-1: not known yet)
  int pk_occ_mg = 0;         // ... and the multi-group form's
  int occ_deliver = 8;       // resident k_deliver CTAs per SM (occupancy bound)
  int deliver_group = 4;     // edge chunks one delivery warp takes per descriptor load
  int64_t deliver_want = 1;  // delivery CTAs the graph can keep busy (its chunks / 64)
  int rate_bucket = -1;
  int64_t trial_steps = 0;
  bool aeif_binning = false;  // order aeif threads by RKF45 step size (ng_set_option "aeif_binning"; off: measured slower)
  struct TuneCand
  {
    int variant, per_sm, group;
    double us;
  };
  std::vector< TuneCand > tune_log;

  // the update kernel a block of n neurons runs before (or without) tuning
  static int
  default_variant( int64_t n )
  {
    return n >= 20000 ? 0 : 2;
  }

  // ... on this engine: a serving engine (whose pool of many small networks
  // is never tuned: its chunks are too short for the trials) takes the
  // one-thread kernel with 2 lags of inputs at a time, whose smaller code
  // measured faster there than 4 lags at a time (update -16 % on the serving
  // sweep; the kernel is bound by instruction issue and fetch, not memory)
  int
  engine_default_variant( int64_t n ) const
  {
    return serving ? 6 : default_variant( n );
  }

  void
  apply_deliver()
  {
    deliver_ctas = ( int ) std::max< int64_t >( 1, std::min< int64_t >( deliver_want, ( int64_t ) sms * deliver_per_sm ) );
    refresh_late();
    ++generation;
  }

  ~ng_engine()
  {
    cudaSetDevice( cfg.device );
    drop_graphs();
    for ( auto& b : blk )
    {
      for ( auto& s : b.st )
        cudaFree( s.p );
      cudaFree( b.r.p );
      cudaFree( b.istep.p );
      cudaFree( b.cls.p );
      cudaFree( b.ctab.p );
      cudaFree( b.perm.p );
      cudaFree( b.bins.p );
    }
    DevBuf* bufs[] = { &ring, &row_beg, &row_len, &real_deg, &tdc, &w, &ent, &log, &rec, &pois, &pois_w, &pois_d,
      &pois_ref, &pois_cdf, &trace_col, &trace, &sched_step, &sched_src, &ctl, &d_nid, &d_step0, &d_until, &d_off,
      &d_key, &sc_src, &sc_cnt, &sc_fill, &sc_beg, &sc_plen, &sc_total, &sc_sb, &gmask, &gin, &net_g, &net_mode,
      &net_spk, &log_sorted, &log_cnt, &log_off, &sc_bound, &seg, &net_t, &row_ue, &row_ls, &ent_late, &pk, &pl_row,
      &pl_tgt, &pl_dly, &pl_w, &pl_Kplus, &pl_tlast, &pl_ninc, &pl_tauinv, &pl_Kminus, &pl_last, &pl_hist_t, &pl_hist_K,
      &pl_hist_n, &pl_hist_lo, &pl_drop_t, &pl_drop_K, &pl_nflush, &pl_in_row, &pl_in_edge, &pl_in_src, &pl_wrun,
      &pl_tab_fin, &pl_tab_km };
    for ( DevBuf* b : bufs )
      cudaFree( b->p );
    if ( host_ctl )
      cudaFreeHost( host_ctl );
    if ( pinned_log )
      cudaFreeHost( pinned_log );
    if ( adm_pin )
      cudaFreeHost( adm_pin );
    for ( auto& nw : nets )
      free_blocks( nw.blocks );
    if ( host_off )
      cudaFreeHost( host_off );
    for ( auto& ev : group_done )
      if ( ev )
        cudaEventDestroy( ev );
    if ( copy_stream )
      cudaStreamDestroy( copy_stream );
    if ( late_stream )
      cudaStreamDestroy( late_stream );
    if ( adm_stream )
      cudaStreamDestroy( adm_stream );
    if ( ev_adm )
      cudaEventDestroy( ev_adm );
    for ( cudaEvent_t ev : { ev_fork, ev_late[ 0 ], ev_late[ 1 ] } )
      if ( ev )
        cudaEventDestroy( ev );
    if ( ev0 )
      cudaEventDestroy( ev0 );
    if ( ev1 )
      cudaEventDestroy( ev1 );
    if ( own )
      cudaStreamDestroy( own );
  }

  int
  alloc( DevBuf& b, size_t bytes )
  {
    cudaFree( b.p );
    b.p = nullptr;
    b.bytes = 0;
    if ( bytes == 0 )
      return NG_OK;
    CU( cudaMalloc( &b.p, bytes ) );
    b.bytes = bytes;
    CU( cudaMemsetAsync( b.p, 0, bytes, stream ) );
    return NG_OK;
  }

  int
  upload( DevBuf& b, const void* src, size_t bytes )
  {
    int rc = alloc( b, bytes );
    if ( rc )
      return rc;
    if ( bytes )
      CU( cudaMemcpyAsync( b.p, src, bytes, cudaMemcpyHostToDevice, stream ) );
    return NG_OK;
  }

  int
  block_of( int64_t i ) const
  {
    for ( size_t k = 0; k < blk.size(); ++k )
      if ( i >= blk[ k ].off && i < blk[ k ].off + blk[ k ].n )
        return ( int ) k;
    return -1;
  }

  int64_t
  ms_to_steps( double ms ) const
  {
    // Time( Time::ms( t ) ).get_steps() (nestkernel/nest_time.h:306-311, 508-521)
    const int64_t tics = ( int64_t ) ( ms * cfg.tics_per_ms + 0.5 );
    return ( int64_t ) ( ( double ) ( tics + tics_per_step - 1 ) * ( 1. / ( double ) tics_per_step ) );
  }

  // pre_run_hook restatements -> coefficient rows (FP64), deduped into classes
  // pre_run_hook restatement for neuron i of block b: one coefficient row
  int
  coef_row( const Blk& b, int64_t i, double* row ) const
  {
  std::fill( row, row + CT_STRIDE, 0.0 );
  const auto& P = b.par;
  if ( b.model == NG_IAF_PSC_DELTA )
  {
    const double tau_m = P[ 0 ][ i ], c_m = P[ 1 ][ i ];
    if ( !( c_m > 0 ) || !( tau_m > 0 ) || P[ 2 ][ i ] < 0 )
      return fail( NG_ERR_ARG, "iaf_psc_delta: C_m and tau_m must be > 0, t_ref >= 0" );
    if ( P[ 4 ][ i ] >= P[ 3 ][ i ] )
      return fail( NG_ERR_ARG, "Reset potential must be smaller than threshold." );
    row[ 0 ] = std::exp( -h / tau_m );
    row[ 1 ] = 1 / c_m * ( 1 - row[ 0 ] ) * tau_m;
    row[ 2 ] = P[ 3 ][ i ];
    row[ 3 ] = P[ 4 ][ i ];
    row[ 4 ] = P[ 5 ][ i ];
    row[ 5 ] = ( double ) ms_to_steps( P[ 2 ][ i ] );
  }
  else if ( b.model == NG_IAF_PSC_ALPHA )
  {
    // iaf_psc_alpha::pre_run_hook (models/iaf_psc_alpha.cpp), same order
    const double tau_m = P[ 0 ][ i ], c_m = P[ 1 ][ i ], tex = P[ 5 ][ i ], tin = P[ 6 ][ i ];
    if ( !( c_m > 0 ) )
      return fail( NG_ERR_ARG, "Capacitance must be > 0." );
    if ( !( tau_m > 0 ) )
      return fail( NG_ERR_ARG, "Membrane time constant must be > 0." );
    if ( !( tex > 0 ) || !( tin > 0 ) )
      return fail( NG_ERR_ARG, "All synaptic time constants must be > 0." );
    if ( P[ 2 ][ i ] < 0 )
      return fail( NG_ERR_ARG, "Refractory time must not be negative." );
    if ( P[ 4 ][ i ] >= P[ 3 ][ i ] )
      return fail( NG_ERR_ARG, "Reset potential must be smaller than threshold." );
    row[ 0 ] = std::exp( -h / tex );  // P11ex = P22ex
    row[ 1 ] = std::exp( -h / tin );  // P11in = P22in
    row[ 9 ] = std::expm1( -h / tau_m );
    row[ 4 ] = -tau_m / c_m * std::expm1( -h / tau_m );  // P30
    row[ 2 ] = h * row[ 0 ];                               // P21ex
    row[ 3 ] = h * row[ 1 ];                               // P21in
    propagator_alpha( tex, tau_m, c_m, h, &row[ 5 ], &row[ 6 ] );
    propagator_alpha( tin, tau_m, c_m, h, &row[ 7 ], &row[ 8 ] );
    row[ 10 ] = 1.0 * M_E / tex;
    row[ 11 ] = 1.0 * M_E / tin;
    row[ 12 ] = P[ 3 ][ i ];
    row[ 13 ] = P[ 4 ][ i ];
    row[ 14 ] = P[ 7 ][ i ];
    row[ 15 ] = ( double ) ms_to_steps( P[ 2 ][ i ] );
  }
  else if ( b.model == NG_IAF_PSC_EXP )
  {
    const double tau_m = P[ 0 ][ i ], c_m = P[ 1 ][ i ], tex = P[ 5 ][ i ], tin = P[ 6 ][ i ];
    if ( !( c_m > 0 ) || !( tau_m > 0 ) || !( tex > 0 ) || !( tin > 0 ) || P[ 2 ][ i ] < 0 )
      return fail( NG_ERR_ARG, "iaf_psc_exp: capacitance and time constants must be > 0, t_ref >= 0" );
    if ( P[ 4 ][ i ] >= P[ 3 ][ i ] )
      return fail( NG_ERR_ARG, "Reset potential must be smaller than threshold." );
    const double P11ex = std::exp( -h / tex );
    const double P11in = std::exp( -h / tin );
    const double P22 = std::exp( -h / tau_m );
    row[ 0 ] = P22;
    row[ 1 ] = propagator_exp( tex, tau_m, c_m, h );
    row[ 2 ] = propagator_exp( tin, tau_m, c_m, h );
    row[ 3 ] = tau_m / c_m * ( 1.0 - P22 );
    row[ 4 ] = P11ex;
    row[ 5 ] = P11in;
    row[ 6 ] = P[ 3 ][ i ];
    row[ 7 ] = P[ 4 ][ i ];
    row[ 8 ] = ( double ) ms_to_steps( P[ 2 ][ i ] );
    row[ 9 ] = 1. - P11ex;
  }
  else
  {
    for ( int k = 0; k < 15; ++k )
      row[ k ] = P[ k == 0 ? 0 : k == 1 ? 1 : k + 1 ][ i ];
    // order: V_peak, V_reset, g_L, C_m, E_ex, E_in, E_L, Delta_T, tau_w, a, b, V_th, tau_ex, tau_in, tol
    row[ 14 ] = P[ 15 ][ i ];
    const double Vpeak = P[ 0 ][ i ], Vreset = P[ 1 ][ i ], Vth = P[ 12 ][ i ], DT = P[ 8 ][ i ];
    if ( Vreset >= Vpeak )
      return fail( NG_ERR_ARG, "Ensure that: V_reset < V_peak ." );
    if ( DT < 0. )
      return fail( NG_ERR_ARG, "Delta_T must be positive." );
    if ( Vpeak < Vth )
      return fail( NG_ERR_ARG, "V_peak >= V_th required." );
    if ( !( P[ 4 ][ i ] > 0 ) )
      return fail( NG_ERR_ARG, "Capacitance must be strictly positive." );
    if ( !( P[ 13 ][ i ] > 0 ) || !( P[ 14 ][ i ] > 0 ) || !( P[ 9 ][ i ] > 0 ) )
      return fail( NG_ERR_ARG, "All time constants must be strictly positive." );
    if ( !( P[ 15 ][ i ] > 0 ) )
      return fail( NG_ERR_ARG, "The gsl_error_tol must be strictly positive." );
    if ( P[ 2 ][ i ] < 0 )
      return fail( NG_ERR_ARG, "Refractory time cannot be negative." );
    row[ 15 ] = 1.0 * M_E / P[ 13 ][ i ];
    row[ 16 ] = 1.0 * M_E / P[ 14 ][ i ];
    row[ 17 ] = DT > 0. ? Vpeak : Vth;
    row[ 18 ] = ( double ) ms_to_steps( P[ 2 ][ i ] );
  }
  return NG_OK;
  }

  int
  build_classes( Blk& b )
  {
    std::unordered_map< std::string, int32_t > ids;
    b.host_ctab.clear();
    b.host_cls.assign( ( size_t ) b.n, 0 );
    double row[ CT_STRIDE ];
    for ( int64_t i = 0; i < b.n; ++i )
    {
      int rc = coef_row( b, i, row );
      if ( rc )
        return rc;
      std::string key( reinterpret_cast< const char* >( row ), sizeof( row ) );
      auto it = ids.find( key );
      int32_t id;
      if ( it == ids.end() )
      {
        id = ( int32_t ) ids.size();
        ids.emplace( std::move( key ), id );
        b.host_ctab.insert( b.host_ctab.end(), row, row + CT_STRIDE );
      }
      else
      {
        id = it->second;
      }
      b.host_cls[ ( size_t ) i ] = id;
    }
    b.n_classes = ( int64_t ) ids.size();
    int rc = upload( b.ctab, b.host_ctab.data(), b.host_ctab.size() * sizeof( double ) );
    if ( rc )
      return rc;
    rc = upload( b.cls, b.host_cls.data(), b.host_cls.size() * sizeof( int32_t ) );
    if ( rc )
      return rc;
    b.dirty = false;
    ++generation;
    return NG_OK;
  }

  Net
  net() const
  {
    Net d {};
    d.N = N;
    d.n_src = n_src;
    d.L = L;
    d.C = C;
    d.min_delay = cfg.min_delay;
    d.tbits = tbits;
    d.tmask = tmask;
    d.dmask = dmask;
    d.ring = ring.p;
    d.ring32 = ring_bytes == 4 ? 1 : 0;
    d.fx_inv = fx_inv;
    d.row_beg = ( const int64_t* ) row_beg.p;
    d.row_len = ( const int32_t* ) row_len.p;
    d.real_deg = ( const int32_t* ) real_deg.p;
    d.late_min = late_min_cur;
    d.row_ue = ( const int32_t* ) row_ue.p;
    d.row_ls = ( const int32_t* ) row_ls.p;
    d.ent_late = ( int4* ) ent_late.p;
    d.edge_tdc = ( const uint32_t* ) tdc.p;
    d.edge_w = w.p;
    d.ent = ( int4* ) ent.p;
    d.ent_cap = ent_cap;
    d.log = ( uint2* ) log.p;
    d.log_cap = log_cap;
    d.rec = ( const uint8_t* ) rec.p;
    d.pois = ( const double4* ) pois.p;
    d.pois_w = ( const double* ) pois_w.p;
    d.pois_d = ( const int32_t* ) pois_d.p;
    d.pois_cdf_ref = ( const int2* ) pois_ref.p;
    d.pois_cdf = ( const uint64_t* ) pois_cdf.p;
    d.pois_start = pois_start;
    d.pois_stop = pois_stop;
    d.key0 = key0;
    d.key1 = key1;
    d.has_pois = has_pois;
    d.trace_col = n_trace_idx > 0 ? ( const int32_t* ) trace_col.p : nullptr;
    d.trace = ( double* ) trace.p;
    d.n_trace_idx = n_trace_idx;
    d.trace_interval = trace_interval;
    d.n_trace_vars = n_trace_vars;
    for ( int k = 0; k < MAX_STATE; ++k )
      d.trace_slot[ k ] = trace_slot[ k ];
    d.trace_rows = trace_rows_cap;
    d.nid = serving ? ( const int32_t* ) d_nid.p : nullptr;
    d.net_step0 = ( const long long* ) d_step0.p;
    d.net_until = ( const long long* ) d_until.p;
    d.net_off = ( const long long* ) d_off.p;
    d.net_key = ( const uint2* ) d_key.p;
    if ( serving )
      d.n_nets = cfg.max_networks;
    if ( tiled_on )
    {
      d.net_t = ( const TileNet* ) net_t.p;
      d.seg = ( const int32_t* ) seg.p;
      d.tile_t = tile_t;
    }
    if ( plastic_on )
      d.gmask = ( uint32_t* ) gmask.p;  // the update writes each neuron's lag bits of the slice
    if ( gather_on )
    {
      d.gmask = ( uint32_t* ) gmask.p;
      d.gin = ( const uint16_t* ) gin.p;
      d.net_g = ( const GatherNet* ) net_g.p;
      d.net_mode = ( int* ) net_mode.p;
      d.net_spk = ( unsigned* ) net_spk.p;
      d.n_nets = cfg.max_networks;
      d.gather_frac = gather_frac;
    }
    d.sched_step = ( const int64_t* ) sched_step.p;
    d.sched_src = ( const int32_t* ) sched_src.p;
    d.n_sched = n_sched;
    d.deliver_group = deliver_group;
    d.ctl = ( Ctl* ) ctl.p;
    return d;
  }

  Block
  dblock( const Blk& b ) const
  {
    Block k {};
    k.off = b.off;
    k.n = b.n;
    k.model = b.model;
    k.cls = ( const int32_t* ) b.cls.p;
    k.ctab = ( const double* ) b.ctab.p;
    for ( int s = 0; s < MAX_STATE; ++s )
      k.s[ s ] = b.st[ s ].p;
    k.r = ( int32_t* ) b.r.p;
    k.istep = ( double* ) b.istep.p;
    k.perm = ( aeif_binning && b.perm.p ) ? ( const int32_t* ) b.perm.p : nullptr;
    return k;
  }

  void
  launch_update( const Net& d, int from_, int to_ )
  {
    for ( size_t k = 0; k < blk.size(); ++k )
    {
      const Blk& b = blk[ k ];
      const int sched = ( k == 0 ) ? 1 : 0;
      const Block db = dblock( b );
      if ( b.model == NG_AEIF_COND_ALPHA )
      {
        if ( db.perm )
        {
          // threads ordered by the neurons' last RKF45 step size (k_aeif_bin_*)
          const unsigned gb = ( unsigned ) std::max< int64_t >( 1, std::min< int64_t >( ( b.n + 255 ) / 256, 2 * sms ) );
          cudaMemsetAsync( b.bins.p, 0, 2 * AEIF_BINS * sizeof( unsigned ), stream );
          k_aeif_bin_count<<< gb, 256, 0, stream >>>( ( const double* ) b.istep.p, b.n, h, ( unsigned* ) b.bins.p );
          k_aeif_bin_scatter<<< gb, 256, 0, stream >>>( ( const double* ) b.istep.p, b.n, h, ( unsigned* ) b.bins.p,
            ( int32_t* ) b.perm.p );
        }
        // CTAs of 2 warps, registers capped for 12 warps per SM (the RKF45 state and
        // tableau need ~170 registers; more warps hide the FP64 latency)
        const unsigned grid = ( unsigned ) std::max< int64_t >( 1, ( b.n + 63 ) / 64 );
        if ( prec == NG_FP64 )
          k_update_aeif< double, false ><<< grid, 64, 0, stream >>>( d, db, from_, to_, sched, h );
        else
          k_update_aeif< float, true ><<< grid, 64, 0, stream >>>( d, db, from_, to_, sched, h );
      }
      else
      {
        launch_iaf( d, db, b.model, from_, to_, sched );
      }
    }
  }

  template < typename Real, bool FIX, int MODEL >
  void
  launch_iaf_g( const Net& d, const Block& db, int from_, int to_, int sched )
  {
    const int span = to_ - from_;
    // the tuned (or default) kernel; one thread per neuron for 1-2 step
    // slices and for engines with the per-target gather or the target-tiled
    // delivery (the lag bits are written there)
    int v = upd_variant >= 0 ? upd_variant : engine_default_variant( db.n );
    if ( span <= 2 || gather_on || tiled_on || plastic_on )
      v = ( v == 1 || v == 6 ) ? v : 0;
    if ( v <= 1 || v == 6 )
    {
      // CTAs of 4 warps: a large network's grid is resident in one wave
      const unsigned grid = ( unsigned ) std::max< int64_t >( 1, ( db.n + 127 ) / 128 );
      if ( span == 1 )
        k_update_iaf< Real, FIX, MODEL, 1 ><<< grid, 128, 0, stream >>>( d, db, from_, to_, sched );
      else if ( v == 0 )
        k_update_iaf< Real, FIX, MODEL, 4 ><<< grid, 128, 0, stream >>>( d, db, from_, to_, sched );
      else if ( v == 6 )
        k_update_iaf< Real, FIX, MODEL, 2 ><<< grid, 128, 0, stream >>>( d, db, from_, to_, sched );
      else
        k_update_iaf< Real, FIX, MODEL, 8 ><<< grid, 128, 0, stream >>>( d, db, from_, to_, sched );
    }
    else
    {
      const unsigned grid = ( unsigned ) std::max< int64_t >( 1, ( db.n + P2_NB - 1 ) / P2_NB );
      if ( v == 2 )
        k_update_iaf2< Real, FIX, MODEL, 256, 32 ><<< grid, 256, 0, stream >>>( d, db, from_, to_, sched );
      else
        k_update_iaf2< Real, FIX, MODEL, 128, 16 ><<< grid, 128, 0, stream >>>( d, db, from_, to_, sched );
    }
  }

  void
  launch_iaf( const Net& d, const Block& db, int model, int from_, int to_, int sched )
  {
    if ( model == NG_IAF_PSC_DELTA )
    {
      if ( prec == NG_FP64 )
        launch_iaf_g< double, false, NG_IAF_PSC_DELTA >( d, db, from_, to_, sched );
      else
        launch_iaf_g< float, true, NG_IAF_PSC_DELTA >( d, db, from_, to_, sched );
    }
    else if ( model == NG_IAF_PSC_ALPHA )
    {
      if ( prec == NG_FP64 )
        launch_iaf_g< double, false, NG_IAF_PSC_ALPHA >( d, db, from_, to_, sched );
      else
        launch_iaf_g< float, true, NG_IAF_PSC_ALPHA >( d, db, from_, to_, sched );
    }
    else
    {
      if ( prec == NG_FP64 )
        launch_iaf_g< double, false, NG_IAF_PSC_EXP >( d, db, from_, to_, sched );
      else
        launch_iaf_g< float, true, NG_IAF_PSC_EXP >( d, db, from_, to_, sched );
    }
  }

  template < typename Real, bool FIX, int MODEL >
  const void*
  pk_func( bool mg ) const
  {
    return mg ? reinterpret_cast< const void* >( &k_run_slices_mg< Real, FIX, MODEL > )
              : reinterpret_cast< const void* >( &k_run_slices< Real, FIX, MODEL > );
  }

  // the persistent kernel: one resident wave holding every neuron's state in
  // registers (k_run_slices), or the multi-group form for larger networks
  const void*
  pk_kernel( bool mg ) const
  {
    const int m = blk[ 0 ].model;
    if ( prec == NG_FP64 )
      return m == NG_IAF_PSC_DELTA ? pk_func< double, false, NG_IAF_PSC_DELTA >( mg )
        : m == NG_IAF_PSC_EXP      ? pk_func< double, false, NG_IAF_PSC_EXP >( mg )
                                   : pk_func< double, false, NG_IAF_PSC_ALPHA >( mg );
    return m == NG_IAF_PSC_DELTA ? pk_func< float, true, NG_IAF_PSC_DELTA >( mg )
      : m == NG_IAF_PSC_EXP      ? pk_func< float, true, NG_IAF_PSC_EXP >( mg )
                                 : pk_func< float, true, NG_IAF_PSC_ALPHA >( mg );
  }

  bool
  pk_multi_group() const
  {
    return N > ( int64_t ) pk_occ * sms * PK_NB;
  }

  // the persistent slice kernel applies: one iaf block of a static engine,
  // no traces or scheduled generator spikes (whose bookkeeping is per
  // launch), a device that supports cooperative launches
  bool
  persistent_ok()
  {
    if ( serving || blk.size() != 1 || blk[ 0 ].model == NG_AEIF_COND_ALPHA || n_sched > 0 || n_trace_idx > 0
      || gather_on || tiled_on || plastic_on || nnz_padded <= 0 )
      return false;
    if ( pk_occ < 0 )
    {
      int coop = 0, occ = 0, occ_mg = 0;
      cudaDeviceGetAttribute( &coop, cudaDevAttrCooperativeLaunch, cfg.device );
      if ( !coop || cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, pk_kernel( false ), PK_THREADS, 0 ) != cudaSuccess
        || cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ_mg, pk_kernel( true ), PK_THREADS, 0 ) != cudaSuccess )
        occ = occ_mg = 0;
      cudaGetLastError();
      pk_occ = occ;
      pk_occ_mg = occ_mg;
      if ( occ > 0 && occ_mg > 0 && !pk.p && alloc( pk, sizeof( PkCtl ) ) != NG_OK )
        pk_occ = 0;
    }
    return pk_occ > 0 && ( !pk_multi_group() || pk_occ_mg > 0 );
  }

  // k full slices in one cooperative launch; the grid covers the neurons
  // (32 per CTA) and at least one CTA per SM (every CTA takes part in the
  // delivery)
  int
  launch_persistent( const Net& d, int k )
  {
    Net dd = d;
    dd.late_min = INT32_MAX;  // every edge at its slice's close
    Block db = dblock( blk[ 0 ] );
    const bool mg = pk_multi_group();
    const int64_t need = ( N + PK_NB - 1 ) / PK_NB;
    const int64_t cap = ( int64_t ) ( mg ? pk_occ_mg : pk_occ ) * sms;
    const unsigned grid = ( unsigned ) std::min< int64_t >( cap, std::max< int64_t >( need, sms ) );
    PkCtl* pkc = ( PkCtl* ) pk.p;
    CU( cudaMemsetAsync( pk.p, 0, sizeof( PkCtl ), stream ) );
    void* args[] = { &dd, &db, &k, &pkc };
    CU( cudaLaunchCooperativeKernel( pk_kernel( mg ), dim3( grid ), dim3( PK_THREADS ), args, 0, stream ) );
    return NG_OK;
  }

  int
  upload_tau_minus()
  {
    if ( !plastic_on )
      return NG_OK;  // uploaded with the plastic connections
    cudaSetDevice( cfg.device );
    std::vector< double > inv( ( size_t ) N );
    for ( int64_t i = 0; i < N; ++i )
      inv[ ( size_t ) i ] = 1. / tau_minus_host[ ( size_t ) i ];
    CU( cudaMemcpyAsync( pl_tauinv.p, inv.data(), inv.size() * 8, cudaMemcpyHostToDevice, stream ) );
    CU( cudaStreamSynchronize( stream ) );
    return NG_OK;
  }

  StdpNet
  stdp() const
  {
    StdpNet p {};
    p.row = ( const int64_t* ) pl_row.p;
    p.tgt = ( const int32_t* ) pl_tgt.p;
    p.dly = ( const int32_t* ) pl_dly.p;
    p.w = ( double* ) pl_w.p;
    p.w_run = ( double* ) pl_wrun.p;
    p.Kplus = ( double* ) pl_Kplus.p;
    p.tlast = ( double* ) pl_tlast.p;
    p.n_src = pl_nsrc;
    p.n_inc = ( const uint8_t* ) pl_ninc.p;
    p.tau_minus_inv = ( const double* ) pl_tauinv.p;
    p.Kminus = ( double* ) pl_Kminus.p;
    p.last_spike = ( double* ) pl_last.p;
    p.hist_t = ( double* ) pl_hist_t.p;
    p.hist_K = ( double* ) pl_hist_K.p;
    p.hist_n = ( int64_t* ) pl_hist_n.p;
    p.hist_lo = ( int64_t* ) pl_hist_lo.p;
    p.drop_t = ( double* ) pl_drop_t.p;
    p.drop_K = ( double* ) pl_drop_K.p;
    p.n_flush = ( int32_t* ) pl_nflush.p;
    p.in_row = ( const int64_t* ) pl_in_row.p;
    p.in_edge = ( const uint32_t* ) pl_in_edge.p;
    p.in_src = ( const int32_t* ) pl_in_src.p;
    p.dmax_ms = pl_dmax_ms;
    p.dconst = pl_dconst;
    p.tab_fin = ( int32_t* ) pl_tab_fin.p;
    p.tab_km = ( double* ) pl_tab_km.p;
    p.lambda = pl_lambda;
    p.alpha = pl_alpha;
    p.mu = pl_mu;
    p.tau_plus_inv = 1. / pl_tau_plus;
    p.ms_per_tic = 1. / cfg.tics_per_ms;
    p.tics_per_step = tics_per_step;
    p.sign_channels = sign_channels( blk[ 0 ].model ) ? 1 : 0;
    return p;
  }

  void
  launch_deliver( const Net& d )
  {
    if ( plastic_on )
    {
      // plastic connections of the closing slice: the presynaptic spikes (which
      // read only earlier slices' postsynaptic spikes), then the histories
      const StdpNet p = stdp();
      const unsigned ga = ( unsigned ) std::max< int64_t >( 1, std::min< int64_t >( ( N + 255 ) / 256, 4 * sms ) );
      const unsigned gd = ( unsigned ) std::max< int64_t >( 1, std::min< int64_t >( pl_nsrc, 8 * sms ) );
      if ( pl_dconst >= 0 )
      {
        const int64_t q = N * cfg.min_delay;
        k_stdp_arrivals<<< ( unsigned ) std::max< int64_t >( 1, std::min< int64_t >( ( q + 255 ) / 256, 8 * sms ) ), 256, 0,
          stream >>>( d, p );
      }
      if ( prec == NG_FP64 )
        k_stdp_deliver< false ><<< gd, 256, 0, stream >>>( d, p );
      else
        k_stdp_deliver< true ><<< gd, 256, 0, stream >>>( d, p );
      k_stdp_archive<<< ga, 256, 0, stream >>>( d, p );
      k_stdp_flush<<< ( unsigned ) std::max< int64_t >( 1, std::min< int64_t >( N, 8 * sms ) ), 256, 0, stream >>>( d, p );
    }
    if ( gather_live )
      k_gather<<< ( unsigned ) sms, G_THREADS, G_SMEM, stream >>>( d );
    if ( tiled_on )
    {
      if ( prec == NG_FP64 )
        k_deliver_tiled< double, false ><<< ( unsigned ) sms, 1024, tile_smem, stream >>>( d );
      else if ( ring_bytes == 4 )
        k_deliver_tiled< int32_t, true ><<< ( unsigned ) sms, 1024, tile_smem, stream >>>( d );
      else
        k_deliver_tiled< long long, true ><<< ( unsigned ) sms, 1024, tile_smem, stream >>>( d );
    }
    const unsigned grid = ( unsigned ) deliver_ctas;
    if ( prec == NG_FP64 )
      k_deliver< false, false ><<< grid, 256, 0, stream >>>( d );
    else
      k_deliver< true, false ><<< grid, 256, 0, stream >>>( d );
  }

  // the late delivery of the slice whose update was launched last
  void
  launch_late( const Net& d, cudaStream_t s )
  {
    const unsigned grid = ( unsigned ) late_ctas;
    if ( prec == NG_FP64 )
      k_deliver< false, true ><<< grid, 256, 0, s >>>( d );
    else
      k_deliver< true, true ><<< grid, 256, 0, s >>>( d );
  }

  // before a slice's update (slice parity j): the late delivery of two
  // slices back, which read the list this update appends to, has finished
  void
  late_wait( int j )
  {
    if ( late_pending[ j ] )
    {
      cudaStreamWaitEvent( stream, ev_late[ j ], 0 );
      late_pending[ j ] = false;
    }
  }

  // after a slice's update: its late delivery on the second stream
  void
  late_fork( const Net& d, int j )
  {
    cudaEventRecord( ev_fork, stream );
    cudaStreamWaitEvent( late_stream, ev_fork, 0 );
    launch_late( d, late_stream );
    cudaEventRecord( ev_late[ j ], late_stream );
    late_pending[ j ] = true;
  }

  void
  late_join()
  {
    late_wait( 0 );
    late_wait( 1 );
  }

  int
  run_slice_range( const Net& d, int from_, int to_ )
  {
    const bool late = d.late_min != INT32_MAX;
    const int par = ( int ) ( slices & 1 );
    if ( late && from_ == 0 )
      late_wait( par );
    if ( profiling )
      CU( cudaEventRecord( ev0, stream ) );
    launch_update( d, from_, to_ );
    CU( cudaGetLastError() );
    if ( profiling )
    {
      CU( cudaEventRecord( ev1, stream ) );
      CU( cudaEventSynchronize( ev1 ) );
      float ms = 0;
      CU( cudaEventElapsedTime( &ms, ev0, ev1 ) );
      stats.update_ms += ms;
    }
    stats.update_launches += ( int64_t ) blk.size();
    if ( to_ == cfg.min_delay )
    {
      // profiling: the late delivery runs after the slice-close one, timed with it
      if ( late && !profiling )
        late_fork( d, par );
      if ( profiling )
        CU( cudaEventRecord( ev0, stream ) );
      launch_deliver( d );
      if ( late && profiling )
        launch_late( d, stream );
      CU( cudaGetLastError() );
      if ( profiling )
      {
        CU( cudaEventRecord( ev1, stream ) );
        CU( cudaEventSynchronize( ev1 ) );
        float ms = 0;
        CU( cudaEventElapsedTime( &ms, ev0, ev1 ) );
        stats.deliver_ms += ms;
      }
      stats.deliver_launches += 1;
    }
    return NG_OK;
  }

  void
  drop_graphs()
  {
    for ( auto& g : graphs )
    {
      if ( g.exec )
        cudaGraphExecDestroy( g.exec );
      for ( cudaEvent_t ev : g.ev )
        cudaEventDestroy( ev );
    }
    graphs.clear();
  }

  int
  get_graph( const Net& d, int k, bool prof, GraphEntry** out )
  {
    for ( auto& g : graphs )
      if ( g.slices == k && g.prof == prof && g.gen == generation )
      {
        *out = &g;
        return NG_OK;
      }
    // stale graphs of an older configuration are rebuilt
    for ( auto it = graphs.begin(); it != graphs.end(); )
    {
      if ( it->gen != generation )
      {
        if ( it->exec )
          cudaGraphExecDestroy( it->exec );
        for ( cudaEvent_t ev : it->ev )
          cudaEventDestroy( ev );
        it = graphs.erase( it );
      }
      else
        ++it;
    }
    GraphEntry g;
    g.slices = k;
    g.prof = prof;
    g.gen = generation;
    if ( prof )
    {
      g.ev.resize( ( size_t ) 4 * k );
      for ( auto& ev : g.ev )
        CU( cudaEventCreate( &ev ) );
    }
    cudaGraph_t cg;
    CU( cudaStreamBeginCapture( stream, cudaStreamCaptureModeThreadLocal ) );
    // event record nodes inside the graph (external events) bracket every
    // kernel; late deliveries fork to the second stream and join before the
    // graph ends (profiling: they run after the slice-close delivery)
    const bool late = d.late_min != INT32_MAX;
    for ( int sl = 0; sl < k; ++sl )
    {
      if ( late )
        late_wait( sl & 1 );
      if ( prof )
        cudaEventRecordWithFlags( g.ev[ 4 * sl + 0 ], stream, cudaEventRecordExternal );
      launch_update( d, 0, cfg.min_delay );
      if ( prof )
      {
        cudaEventRecordWithFlags( g.ev[ 4 * sl + 1 ], stream, cudaEventRecordExternal );
        cudaEventRecordWithFlags( g.ev[ 4 * sl + 2 ], stream, cudaEventRecordExternal );
      }
      if ( late && !prof )
        late_fork( d, sl & 1 );
      launch_deliver( d );
      if ( late && prof )
        launch_late( d, stream );
      if ( prof )
        cudaEventRecordWithFlags( g.ev[ 4 * sl + 3 ], stream, cudaEventRecordExternal );
    }
    late_join();
    CU( cudaStreamEndCapture( stream, &cg ) );
    cudaError_t e = cudaGraphInstantiate( &g.exec, cg, 0 );
    cudaGraphDestroy( cg );
    if ( e != cudaSuccess )
      return fail( NG_ERR_CUDA, std::string( "cudaGraphInstantiate: " ) + cudaGetErrorString( e ) );
    graphs.push_back( std::move( g ) );
    *out = &graphs.back();
    return NG_OK;
  }

  // enqueue n steps without host synchronisation (except when profiling)
  int
  enqueue_steps( int64_t n )
  {
    const Net d = net();
    while ( n > 0 )
    {
      if ( from == 0 && upd_variant == 5 && n >= cfg.min_delay && persistent_ok() )
      {
        const int k = ( int ) std::min< int64_t >( n / cfg.min_delay, 1 << 20 );
        late_join();
        if ( profiling )
          CU( cudaEventRecord( ev0, stream ) );
        int rc = launch_persistent( d, k );
        if ( rc )
          return rc;
        if ( profiling )
        {
          // the fused kernel's time is counted as node update
          CU( cudaEventRecord( ev1, stream ) );
          CU( cudaEventSynchronize( ev1 ) );
          float ms = 0;
          CU( cudaEventElapsedTime( &ms, ev0, ev1 ) );
          stats.update_ms += ms;
        }
        const int64_t st = ( int64_t ) k * cfg.min_delay;
        origin += st;
        slices += k;
        n -= st;
        stats.update_launches += 1;
        continue;
      }
      if ( from == 0 && graph_slices > 0 && n >= cfg.min_delay )
      {
        // largest graph chunk that fits: graph_slices, 16, 4 or 1 slices
        const int64_t full = n / cfg.min_delay;
        int k = 1;
        for ( int cand : { graph_slices, 16, 4 } )
          if ( cand <= graph_slices && cand <= full && cand > k )
            k = cand;
        late_join();  // a graph starts with no late delivery outstanding
        GraphEntry* g = nullptr;
        int rc = get_graph( d, k, profiling != 0, &g );
        if ( rc )
          return rc;
        CU( cudaGraphLaunch( g->exec, stream ) );
        if ( profiling )
        {
          CU( cudaStreamSynchronize( stream ) );
          for ( int sl = 0; sl < k; ++sl )
          {
            float a = 0, b2 = 0;
            CU( cudaEventElapsedTime( &a, g->ev[ 4 * sl + 0 ], g->ev[ 4 * sl + 1 ] ) );
            CU( cudaEventElapsedTime( &b2, g->ev[ 4 * sl + 2 ], g->ev[ 4 * sl + 3 ] ) );
            stats.update_ms += a;
            stats.deliver_ms += b2;
          }
        }
        const int64_t st = ( int64_t ) k * cfg.min_delay;
        origin += st;
        slices += k;
        n -= st;
        stats.update_launches += ( int64_t ) k * ( int64_t ) blk.size();
        stats.deliver_launches += k;
        continue;
      }
      const int to_ = ( int ) std::min< int64_t >( from + n, cfg.min_delay );
      int rc = run_slice_range( d, from, to_ );
      if ( rc )
        return rc;
      n -= to_ - from;
      if ( to_ == cfg.min_delay )
      {
        origin += cfg.min_delay;
        from = 0;
        slices += 1;
      }
      else
      {
        from = to_;
      }
    }
    late_join();
    return NG_OK;
  }

  // bound on recorded neuron spikes per step: a neuron with refractory
  // count R emits at most one logged entry per R + 1 steps
  void
  update_log_bound()
  {
    double bound = 0.0;
    for ( const auto& b : blk )
    {
      const int ri = refr_index( b.model );
      for ( int64_t j = 0; j < b.n; ++j )
      {
        const int64_t i = b.off + j;
        if ( rec_host.empty() || !rec_host[ ( size_t ) i ] )
          continue;
        const double R = b.host_cls.empty() ? 0.0 : b.host_ctab[ ( size_t ) b.host_cls[ ( size_t ) j ] * CT_STRIDE + ri ];
        bound += 1.0 / ( R + 1.0 );
      }
    }
    log_per_step = std::max( bound, 1.0 );
  }

  int
  prepare()
  {
    bool rebuilt = false;
    for ( auto& b : blk )
      if ( b.dirty && !serving )
      {
        int rc = build_classes( b );
        if ( rc )
          return rc;
        rebuilt = true;
      }
    if ( ( rebuilt || log_bound_dirty ) && !serving )
    {
      update_log_bound();
      log_bound_dirty = false;
    }
    return NG_OK;
  }
  bool log_bound_dirty = true;

  // one group: set ctl, enqueue, sync, drain
  // A group of steps runs on the device while the host drains the previous
  // group's spike log: the groups alternate between the two log halves.
  struct GroupInfo
  {
    int64_t clock = 0, row0 = 0, end = 0;
  };

  int
  begin_group( int sel, GroupInfo& gi )
  {
    gi.clock = origin + from;
    gi.row0 = ( gi.clock + 1 + trace_interval - 1 ) / trace_interval;
    k_set_ctl<<< 1, 1, 0, stream >>>( ( Ctl* ) ctl.p, gi.clock, gi.row0, 1, sel );
    CU( cudaGetLastError() );
    return NG_OK;
  }

  int
  launch_group( int64_t n, int sel, GroupInfo& gi )
  {
    int rc = begin_group( sel, gi );
    if ( rc )
      return rc;
    if ( ( rc = enqueue_steps( n ) ) )
      return rc;
    return end_group( sel, gi );
  }

  // the group's end: its spike log grouped (serving), the control block
  // copied back, the event the drain waits for
  int
  end_group( int sel, GroupInfo& gi )
  {
    int rc = NG_OK;
    gi.end = origin + from;
    if ( serving )
    {
      const int nn = cfg.max_networks;
      if ( log_sorted.bytes < 2 * ( size_t ) log_cap * sizeof( uint2 ) )
      {
        if ( ( rc = alloc( log_sorted, 2 * ( size_t ) log_cap * sizeof( uint2 ) ) ) || ( rc = alloc( log_cnt, ( size_t ) nn * 4 ) )
          || ( rc = alloc( log_off, 2 * ( size_t ) ( nn + 1 ) * 8 ) ) )
          return rc;
        if ( !host_off && cudaMallocHost( &host_off, 2 * ( size_t ) ( nn + 1 ) * 8 ) != cudaSuccess )
          return fail( NG_ERR_MEMORY, "cannot allocate pinned host memory for the spike log offsets" );
      }
      // the counters double as the scatter's fill counters: zero them each group
      CU( cudaMemsetAsync( log_cnt.p, 0, ( size_t ) nn * 4, stream ) );
      const uint2* half = ( const uint2* ) log.p + ( sel ? log_cap : 0 );
      long long* off = ( long long* ) log_off.p + ( size_t ) sel * ( nn + 1 );
      k_log_count<<< ( unsigned ) ( 2 * sms ), 256, 0, stream >>>( ( const Ctl* ) ctl.p, half, log_cap, nn,
        ( unsigned* ) log_cnt.p );
      k_log_offsets<<< 1, 1024, 0, stream >>>( ( unsigned* ) log_cnt.p, off, nn );
      k_log_scatter<<< ( unsigned ) ( 2 * sms ), 256, 0, stream >>>( ( const Ctl* ) ctl.p, half, log_cap, nn, off,
        ( unsigned* ) log_cnt.p, ( uint2* ) log_sorted.p + ( sel ? log_cap : 0 ) );
      CU( cudaGetLastError() );
      CU( cudaMemcpyAsync( host_off + ( size_t ) sel * ( nn + 1 ), off, ( size_t ) ( nn + 1 ) * 8, cudaMemcpyDeviceToHost,
        stream ) );
    }
    CU( cudaMemcpyAsync( host_ctl + sel, ctl.p, sizeof( Ctl ), cudaMemcpyDeviceToHost, stream ) );
    CU( cudaEventRecord( group_done[ sel ], stream ) );
    return NG_OK;
  }

  int
  grow_pinned( size_t bytes )
  {
    if ( bytes <= pinned_log_bytes )
      return NG_OK;
    if ( pinned_log )
      cudaFreeHost( pinned_log );
    pinned_log = nullptr;
    pinned_log_bytes = 0;
    if ( cudaMallocHost( &pinned_log, bytes ) != cudaSuccess )
      return fail( NG_ERR_MEMORY, "cannot allocate pinned host memory for the spike log" );
    pinned_log_bytes = bytes;
    return NG_OK;
  }

  int
  grow_adm_pin( size_t bytes )
  {
    if ( bytes <= adm_pin_bytes )
      return NG_OK;
    const size_t want = std::max( { bytes, 2 * adm_pin_bytes, ( size_t ) 4 << 20 } );
    if ( adm_pin )
      cudaFreeHost( adm_pin );
    adm_pin = nullptr;
    adm_pin_bytes = 0;
    if ( cudaMallocHost( &adm_pin, want ) != cudaSuccess )
      return fail( NG_ERR_MEMORY, "cannot allocate pinned host memory for admissions" );
    adm_pin_bytes = want;
    return NG_OK;
  }

  int
  drain_group( int sel, const GroupInfo& gi )
  {
    const auto w0 = std::chrono::steady_clock::now();
    CU( cudaEventSynchronize( group_done[ sel ] ) );
    const auto w1 = std::chrono::steady_clock::now();
    stats.wait_ms += std::chrono::duration< double, std::milli >( w1 - w0 ).count();
    struct Tally
    {
      ng_stats& st;
      std::chrono::steady_clock::time_point t;
      ~Tally()
      {
        st.drain_ms += std::chrono::duration< double, std::milli >( std::chrono::steady_clock::now() - t ).count();
      }
    } tally { stats, w1 };
    const Ctl& c = host_ctl[ sel ];
    if ( c.err & ERR_NUMERIC )
      return fail( NG_ERR_NUMERIC, "NumericalInstability: aeif_cond_alpha state exploded (V_m < -1e3 or |w| > 1e6)" );
    if ( c.err & ERR_STDP_HISTORY )
      return fail( NG_ERR_CAPACITY, "stdp_pl_synapse_hom: more than " + std::to_string( STDP_HIST - 32 )
          + " postsynaptic spikes of one neuron within max_delay (its spike history ring is full)" );
    if ( c.err & ERR_BARRIER )
      return fail( NG_ERR_CUDA, "persistent slice kernel: a grid barrier gave up waiting (a CTA did not arrive)" );
    if ( c.err & ( ERR_SPIKE_LIST | ERR_LOG | ERR_TRACE ) )
      return fail( NG_ERR_CAPACITY, "device spike list, spike log or trace buffer overflowed (err word "
          + std::to_string( c.err ) + ")" );
    // (serving: the entries grouped by network, all with a valid id)
    const int64_t nl = serving ? std::min< int64_t >( ( int64_t ) c.log_count,
                                   host_off[ ( size_t ) sel * ( cfg.max_networks + 1 ) + cfg.max_networks ] )
                               : ( int64_t ) c.log_count;
    if ( nl > 0 )
    {
      int rc = grow_pinned( ( size_t ) nl * sizeof( uint2 ) );
      if ( rc )
        return rc;
      // the copy engine fetches this half while the next group computes
      const uint2* src_half = ( const uint2* ) ( serving ? log_sorted.p : log.p ) + ( sel ? log_cap : 0 );
      CU( cudaMemcpyAsync( pinned_log, src_half, sizeof( uint2 ) * ( size_t ) nl, cudaMemcpyDeviceToHost, copy_stream ) );
      CU( cudaStreamSynchronize( copy_stream ) );
      const uint2* ent = pinned_log;
      if ( serving )
      {
        // one block per network: its entries are contiguous
        const long long* off = host_off + ( size_t ) sel * ( cfg.max_networks + 1 );
        for ( int id = 0; id < cfg.max_networks; ++id )
        {
          const int64_t cnt = off[ id + 1 ] - off[ id ];
          NetInfo& nw = nets[ ( size_t ) id ];
          if ( cnt <= 0 || !nw.used )
            continue;
          RawBlock rb;
          rb.clock = gi.clock;
          rb.n = cnt;
          rb.e = static_cast< uint2* >( std::malloc( ( size_t ) cnt * sizeof( uint2 ) ) );
          if ( !rb.e )
            return fail( NG_ERR_MEMORY, "out of host memory for the spike log" );
          std::memcpy( rb.e, ent + off[ id ], ( size_t ) cnt * sizeof( uint2 ) );
          int64_t m = 0;
          for ( int64_t k = 0; k < cnt; ++k )
            m += rb.e[ k ].y >> 24;
          rb.m = m;
          nw.held += m;
          nw.blocks.push_back( rb );
        }
      }
      else
      {
        int64_t tot = 0;
        for ( int64_t k = 0; k < nl; ++k )
          tot += ent[ k ].y >> 24;
        size_t p = out_src.size();
        out_src.resize( p + ( size_t ) tot );
        out_stamp.resize( p + ( size_t ) tot );
        for ( int64_t k = 0; k < nl; ++k )
        {
          const int64_t stamp = gi.clock + ( int64_t ) ( ent[ k ].y & 0xFFFFFFu );
          for ( uint32_t m = ent[ k ].y >> 24; m > 0; --m, ++p )
          {
            out_src[ p ] = ( int32_t ) ent[ k ].x;
            out_stamp[ p ] = stamp;
          }
        }
      }
    }
    // the trace rows of this group (tracing runs the groups one at a time)
    if ( n_trace_idx > 0 )
    {
      const int64_t row_end = gi.end / trace_interval;  // last complete row index
      const int64_t rows = row_end - gi.row0 + 1;
      if ( rows > 0 )
      {
        const size_t cnt = ( size_t ) rows * ( size_t ) n_trace_idx * ( size_t ) n_trace_vars;
        const size_t old = out_trace.size();
        out_trace.resize( old + cnt );
        CU( cudaMemcpy( out_trace.data() + old, trace.p, cnt * sizeof( double ), cudaMemcpyDeviceToHost ) );
        if ( trace_first_stamp < 0 )
          trace_first_stamp = gi.row0 * trace_interval;
      }
    }
    stats.spikes = ( int64_t ) c.n_spikes;
    stats.syn_events = ( int64_t ) c.syn_events;
    stats.drive_events = ( int64_t ) c.drive_events;
    stats.gather_slices = ( int64_t ) c.gathered;
    return NG_OK;
  }

  // a group launched by an asynchronous simulate and not drained yet
  int pend_sel = -1;
  GroupInfo pend_gi;

  // ---- slice-aligned calls (ng_update): the steps of successive calls are
  // appended to one open group, which is closed (and becomes the pending
  // group) when it reaches the spike log's capacity or when anything reads
  // or changes the engine
  int og_sel = -1;
  GroupInfo og_gi;
  int64_t og_steps = 0, og_max = 0;

  int
  close_group()
  {
    if ( og_sel < 0 )
      return NG_OK;
    const int sel = og_sel;
    og_sel = -1;
    int rc = end_group( sel, og_gi );
    if ( rc )
      return rc;
    if ( pend_sel >= 0 )
    {
      const int s = pend_sel;
      pend_sel = -1;
      if ( ( rc = drain_group( s, pend_gi ) ) )
        return rc;
    }
    pend_sel = sel;
    pend_gi = og_gi;
    return NG_OK;
  }

  int
  sync_pending()
  {
    if ( og_sel >= 0 )
    {
      const int rc = close_group();
      if ( rc )
        return rc;
    }
    if ( pend_sel < 0 )
      return NG_OK;
    const int s = pend_sel;
    pend_sel = -1;
    return drain_group( s, pend_gi );
  }

  // largest group (in steps) the spike log and the trace buffer hold
  int
  group_max( int64_t* gmax_out )
  {
    int64_t by_log = ( int64_t ) std::floor( ( double ) ( log_cap - n_sched - n_rec ) / log_per_step );
    if ( by_log < 1 )
      return fail( NG_ERR_CAPACITY, "spike log capacity too small for one step" );
    int64_t gmax = std::min< int64_t >( by_log, ( 1 << 24 ) - 2 );
    if ( n_trace_idx > 0 )
      gmax = std::min< int64_t >( gmax, ( trace_rows_cap - 1 ) * trace_interval );
    if ( gmax < 1 )
      return fail( NG_ERR_CAPACITY, "trace buffer too small" );
    *gmax_out = gmax;
    return NG_OK;
  }

  // steps [from_, to_) of the open slice (Node::update(origin, from, to)),
  // enqueued without waiting for the device
  int
  update_range( int from_, int to_ )
  {
    int rc;
    if ( og_sel < 0 )
    {
      if ( ( rc = prepare() ) || ( rc = group_max( &og_max ) ) )
        return rc;
      og_max = std::max< int64_t >( 1, og_max );
      og_sel = pend_sel == 0 ? 1 : 0;
      og_steps = 0;
      if ( ( rc = begin_group( og_sel, og_gi ) ) )
      {
        og_sel = -1;
        return rc;
      }
    }
    if ( ( rc = enqueue_steps( to_ - from_ ) ) )
      return rc;
    og_steps += to_ - from_;
    stats.clock_steps = origin + from;
    stats.slices = slices;
    if ( og_steps + cfg.min_delay > og_max )
      rc = close_group();
    return rc;
  }

  // ---- autotuner.  The trials run the network's own next slices (real
  // steps of the call: every candidate computes the same result), each as
  // one group timed with CUDA events on the engine's stream: first the
  // current configuration (which also measures the activity), then the
  // update kernels, the delivery CTAs per SM and the chunks per delivery
  // warp, one knob at a time with the others at their best so far.  Each
  // candidate runs an untimed group first (its slice graphs are captured
  // there) and a timed one.  The winner is cached for the process by
  // network shape and activity (precision, models, log2 of N, of the mean
  // out-degree and of the spikes per neuron-step, min_delay, late
  // delivery, gather and tiled delivery), so a later engine of the same kind
  // starts with it.
  struct TuneKey
  {
    std::string k;
  };
  static std::mutex& tune_mutex()
  {
    static std::mutex m;
    return m;
  }
  static std::map< std::string, TuneCand >& tune_cache()
  {
    static std::map< std::string, TuneCand > c;
    return c;
  }

  std::string
  tune_key( int rb ) const
  {
    int models = 0;
    for ( const auto& b : blk )
      models |= 1 << b.model;
    int64_t nn = 0, ne = 0;
    for ( const auto& nw : nets )
    {
      nn += nw.used ? nw.n : 0;
      ne += nw.used ? nw.ne : 0;
    }
    const int64_t n_live = serving ? std::max< int64_t >( 1, nn ) : N;
    const int64_t edges = serving ? ne : nnz_padded;
    const double deg = ( double ) std::max< int64_t >( 1, edges ) / ( double ) std::max< int64_t >( 1, n_live );
    char buf[ 160 ];
    std::snprintf( buf, sizeof( buf ), "p%d m%d n%d k%d r%d md%d L%d late%d g%d t%d s%d", prec, models,
      ( int ) std::floor( std::log2( ( double ) n_live ) ), ( int ) std::floor( std::log2( deg ) ), rb, cfg.min_delay,
      L, late_min_cur != INT32_MAX ? 1 : 0, gather_on ? 1 : 0, tiled_on ? 1 : 0, serving ? 1 : 0 );
    return buf;
  }

  void
  apply_cand( const TuneCand& c )
  {
    upd_variant = c.variant;
    deliver_group = c.group;
    deliver_per_sm = c.per_sm;
    apply_deliver();
  }

  // one group of `steps` steps with the current configuration: device time [us]
  int
  timed_group( int64_t steps, double* us, int64_t* spikes )
  {
    GroupInfo gi;
    CU( cudaEventRecord( ev0, stream ) );
    int rc = launch_group( steps, 0, gi );
    if ( rc )
      return rc;
    CU( cudaEventRecord( ev1, stream ) );
    const int64_t s0 = stats.spikes;
    if ( ( rc = drain_group( 0, gi ) ) )
      return rc;
    float ms = 0;
    CU( cudaEventSynchronize( ev1 ) );  // the drain may have waited on an earlier point of the stream
    CU( cudaEventElapsedTime( &ms, ev0, ev1 ) );
    *us = 1e3 * ms;
    if ( spikes )
      *spikes = stats.spikes - s0;
    return NG_OK;
  }

  int
  autotune( int64_t& n, int64_t gmax )
  {
    const int64_t md = cfg.min_delay;
    bool iaf = false;
    for ( const auto& b : blk )
      iaf = iaf || b.model != NG_AEIF_COND_ALPHA;
    std::vector< int > variants;
    if ( iaf )
    {
      variants = { 0, 1, 6 };
      if ( md >= 3 && !gather_on && !tiled_on && !plastic_on )
      {
        variants.push_back( 2 );
        variants.push_back( 3 );
      }
      if ( persistent_ok() )
        variants.push_back( 5 );
    }
    std::vector< int > per_sm;
    for ( int p : { 1, 2, 4, 8 } )
      if ( p <= occ_deliver )
        per_sm.push_back( p );
    if ( per_sm.back() != occ_deliver )
      per_sm.push_back( occ_deliver );
    const std::vector< int > groups = { 1, 2, 4, 8 };
    if ( variants.empty() )
      variants.push_back( upd_variant >= 0 ? upd_variant : 0 );
    const int64_t n_cand = ( int64_t ) ( variants.size() + per_sm.size() + groups.size() );
    // slices per trial group: ~256 steps (long enough for event timing),
    // fewer when the probe (3 groups) and the trials (2 groups each) would
    // not fit the call's steps, at least 4; within the spike log.  A call
    // too short for that leaves the tuning to a longer one.
    const int64_t S = std::min( { std::max< int64_t >( 4, ( 256 + md - 1 ) / md ), n / ( ( 3 + 2 * n_cand ) * md ),
      gmax / md } );
    if ( S < 4 )
      return NG_OK;
    const int64_t steps = S * md;
    const int v0 = upd_variant >= 0 ? upd_variant : ( iaf ? engine_default_variant( blk[ 0 ].n ) : 0 );
    TuneCand best { v0, deliver_per_sm, deliver_group, 1e300 };
    tune_log.clear();
    int rc;
    // a group with the current configuration: its spikes give the activity
    // bucket (its time is not compared: a network's first slices often hold
    // a transient burst)
    int64_t spk = 0;
    for ( int k = 0; k < 3; ++k )
    {
      double probe_us = 0;
      int64_t sk = 0;
      if ( ( rc = timed_group( steps, &probe_us, &sk ) ) )
        return rc;
      spk += sk;
      n -= steps;
    }
    trial_steps = steps;
    int64_t n_live = N;
    if ( serving )
    {
      n_live = 0;
      for ( const auto& nw : nets )
        n_live += nw.used ? nw.n : 0;
      n_live = std::max< int64_t >( 1, n_live );
    }
    const double per_kstep = 1e3 * ( double ) spk / ( ( double ) n_live * ( double ) ( 3 * steps ) );
    rate_bucket = per_kstep > 0 ? ( int ) std::floor( std::log2( per_kstep ) ) : -99;
    const std::string key = tune_key( rate_bucket );
    if ( tune_mode == 1 )
    {
      std::lock_guard< std::mutex > lock( tune_mutex() );
      auto it = tune_cache().find( key );
      if ( it != tune_cache().end() )
      {
        apply_cand( it->second );
        tune_state = 2;
        return NG_OK;
      }
    }
    auto trial = [ & ]( TuneCand c, double* us ) -> int {
      apply_cand( c );
      double warm = 0;
      int r = timed_group( steps, &warm, nullptr );
      if ( r == NG_OK )
        r = timed_group( steps, us, nullptr );
      n -= 2 * steps;
      return r;
    };
    for ( int pass = 0; pass < 3; ++pass )
    {
      if ( pass > 0 && best.variant == 5 )
        break;  // the persistent kernel delivers inside itself: the delivery launch shape is unused
      const std::vector< int >& opts = pass == 0 ? variants : pass == 1 ? per_sm : groups;
      TuneCand round_best = best;
      for ( int o : opts )
      {
        TuneCand c = best;
        if ( pass == 0 )
          c.variant = o;
        else if ( pass == 1 )
          c.per_sm = o;
        else
          c.group = o;
        if ( pass > 0 && c.variant == best.variant && c.per_sm == best.per_sm && c.group == best.group )
          continue;  // measured in an earlier pass
        if ( ( rc = trial( c, &c.us ) ) )
          return rc;
        tune_log.push_back( c );
        if ( c.us < round_best.us )
          round_best = c;
      }
      best = round_best;
    }
    apply_cand( best );
    tune_state = 1;
    {
      std::lock_guard< std::mutex > lock( tune_mutex() );
      tune_cache()[ key ] = best;
    }
    return NG_OK;
  }

  // keep: leave the last group running and undrained (asynchronous form);
  // a group left so by an earlier call is drained while this call's first
  // group runs
  int
  simulate( int64_t n, bool keep = false )
  {
    auto t0 = std::chrono::steady_clock::now();
    int rc = close_group();  // steps of slice-aligned calls still open
    if ( rc )
      return rc;
    if ( ( rc = prepare() ) )
      return rc;
    // group size: bounded by the spike-log and trace capacities
    // over S steps a recorded neuron logs at most S / (R + 1) + 1 entries
    int64_t by_log = ( int64_t ) std::floor( ( double ) ( log_cap - n_sched - n_rec ) / log_per_step );
    if ( by_log < 1 )
      return fail( NG_ERR_CAPACITY, "spike log capacity too small for one step" );
    int64_t gmax = std::min< int64_t >( by_log, ( 1 << 24 ) - 2 );
    if ( n_trace_idx > 0 )
      gmax = std::min< int64_t >( gmax, ( trace_rows_cap - 1 ) * trace_interval );
    if ( gmax < 1 )
      return fail( NG_ERR_CAPACITY, "trace buffer too small" );
    // keep groups to whole graph chunks where possible
    const int64_t chunk = graph_slices > 0 ? ( int64_t ) graph_slices * cfg.min_delay : cfg.min_delay;
    if ( gmax > chunk )
      gmax = ( gmax / chunk ) * chunk;
    // groups alternate between the log halves; the host drains one group
    // while the device runs the next (one at a time when tracing).  A call
    // is cut into at least 4 groups where it is long enough, so only the
    // last quarter's drain is not hidden behind device work.
    const bool overlap = n_trace_idx == 0;
    // (an asynchronous call needs no split: its group's drain overlaps the
    // next call's group)
    if ( overlap && graph_slices >= 16 && !keep )
    {
      const int64_t q = 16 * ( int64_t ) cfg.min_delay;
      const int64_t quarter = ( ( n / 4 + q - 1 ) / q ) * q;
      if ( quarter >= q && quarter < gmax )
        gmax = quarter;
    }
    // the autotuner runs on the first long enough call, at a slice boundary,
    // with no group in flight and no tracing or profiling
    bool live = nnz_padded > 0;
    if ( serving )
    {
      live = false;
      for ( const auto& nw : nets )
        live = live || ( nw.used && nw.ne > 0 );
    }
    if ( tune_mode != 0 && tune_state == 0 && pend_sel < 0 && from == 0 && n_trace_idx == 0 && !profiling && live )
    {
      rc = autotune( n, gmax );
      if ( rc )
      {
        cudaStreamSynchronize( stream );
        return rc;
      }
    }
    int pending = pend_sel;
    GroupInfo gi[ 2 ];
    if ( pending >= 0 )
      gi[ pending ] = pend_gi;
    pend_sel = -1;
    while ( n > 0 )
    {
      const int64_t g = std::min( n, gmax );
      const int sel = pending == 0 ? 1 : 0;
      rc = launch_group( g, sel, gi[ sel ] );
      if ( rc == NG_OK && pending >= 0 )
        rc = drain_group( pending, gi[ pending ] );
      pending = sel;
      if ( rc == NG_OK && !overlap )
      {
        rc = drain_group( pending, gi[ pending ] );
        pending = -1;
      }
      if ( rc )
      {
        cudaStreamSynchronize( stream );
        return rc;
      }
      n -= g;
    }
    if ( pending >= 0 )
    {
      if ( keep && overlap )
      {
        pend_sel = pending;
        pend_gi = gi[ pending ];
      }
      else if ( ( rc = drain_group( pending, gi[ pending ] ) ) )
        return rc;
    }
    stats.clock_steps = origin + from;
    stats.slices = slices;
    stats.simulate_ms += std::chrono::duration< double, std::milli >( std::chrono::steady_clock::now() - t0 ).count();
    return NG_OK;
  }
};

// error text of entry points compiled in other files of the library
void
ng_internal_set_error( const char* msg )
{
  g_err = msg;
}

// Entry points that read results or change the engine first drain a group
// left running by ng_simulate_async.
#define SETTLE( e )                                                                                                   \
  do                                                                                                                 \
  {                                                                                                                  \
    if ( ( e ) && ( ( e )->pend_sel >= 0 || ( e )->og_sel >= 0 ) )                                                  \
    {                                                                                                                \
      const int rc_settle = ( e )->sync_pending();                                                                   \
      if ( rc_settle )                                                                                               \
        return rc_settle;                                                                                            \
    }                                                                                                                \
  } while ( 0 )

extern "C" {

int
ng_abi_version( void )
{
  return NG_ABI_VERSION;
}

const char*
ng_last_error( void )
{
  return g_err.c_str();
}

int
ng_device_count( int32_t* n )
{
  int c = 0;
  cudaError_t e = cudaGetDeviceCount( &c );
  if ( e != cudaSuccess )
  {
    *n = 0;
    return fail( NG_ERR_CUDA, std::string( "cudaGetDeviceCount: " ) + cudaGetErrorString( e ) );
  }
  *n = c;
  return NG_OK;
}

int
ng_create( const ng_config* cfg, ng_engine** out )
{
  if ( !cfg || !out )
    return fail( NG_ERR_ARG, "ng_create: null argument" );
  *out = nullptr;
  if ( cfg->precision != NG_FP64 && cfg->precision != NG_FP32 )
    return fail( NG_ERR_ARG, "ng_create: precision must be NG_FP64 or NG_FP32" );
  if ( !( cfg->h > 0 ) || !( cfg->tics_per_ms > 0 ) )
    return fail( NG_ERR_ARG, "ng_create: resolution and tics_per_ms must be > 0" );
  if ( cfg->min_delay < 1 || cfg->max_delay < cfg->min_delay )
    return fail( NG_ERR_ARG, "ng_create: need 1 <= min_delay <= max_delay (steps)" );
  if ( cfg->n_blocks < 1 || cfg->n_blocks > NG_MAX_BLOCKS )
    return fail( NG_ERR_ARG, "ng_create: n_blocks out of range" );
  int64_t N = 0;
  for ( int k = 0; k < cfg->n_blocks; ++k )
  {
    if ( cfg->block_model[ k ] < 0 || cfg->block_model[ k ] > 3 || cfg->block_size[ k ] < 0 )
      return fail( NG_ERR_ARG, "ng_create: bad block model or size" );
    N += cfg->block_size[ k ];
  }
  if ( N < 1 || N >= ( 1ll << 30 ) || cfg->n_generators < 0 )
    return fail( NG_ERR_ARG, "ng_create: neuron count out of range" );
  int ndev = 0;
  if ( cudaGetDeviceCount( &ndev ) != cudaSuccess || ndev == 0 )
    return fail( NG_ERR_CUDA, "ng_create: no CUDA device available (the engine has no CPU fallback)" );
  if ( cfg->device < 0 || cfg->device >= ndev )
    return fail( NG_ERR_ARG, "ng_create: device ordinal out of range" );
  CU( cudaSetDevice( cfg->device ) );
  auto* e = new ng_engine();
  e->cfg = *cfg;
  e->prec = cfg->precision;
  e->rsz = e->prec == NG_FP64 ? 8 : 4;
  // Time::set_resolution: tics per step rounded, h = MS_PER_TIC * tics (nest_time.cpp:88-104)
  e->tics_per_step = ( int64_t ) std::floor( cfg->tics_per_ms * cfg->h + 0.5 );
  if ( e->tics_per_step < 1 )
  {
    delete e;
    return fail( NG_ERR_ARG, "ng_create: resolution below one tic" );
  }
  e->h = ( 1 / cfg->tics_per_ms ) * ( double ) e->tics_per_step;
  e->N = N;
  e->n_src = N + cfg->n_generators;
  e->tau_minus_host.assign( ( size_t ) N, 20.0 );  // ArchivingNode default
  e->L = std::max( cfg->min_delay, cfg->max_delay );  // update-then-deliver order: max_delay slots suffice
  if ( cfg->start_step < 0 )
  {
    delete e;
    return fail( NG_ERR_ARG, "ng_create: start_step must be >= 0" );
  }
  e->origin = cfg->start_step;
  cudaDeviceProp prop;
  if ( cudaGetDeviceProperties( &prop, cfg->device ) == cudaSuccess )
    e->sms = prop.multiProcessorCount;
  int rc = NG_OK;
  auto bail = [ & ]( int code ) {
    delete e;
    return code;
  };
  // the engine's own stream outranks the late deliveries: the update CTAs
  // are placed first where both wait for SM slots
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange( &lo, &hi );
  if ( cudaStreamCreateWithPriority( &e->own, cudaStreamNonBlocking, hi ) != cudaSuccess )
    return bail( fail( NG_ERR_CUDA, "cudaStreamCreate failed" ) );
  e->stream = e->own;
  {
    if ( cudaStreamCreateWithPriority( &e->late_stream, cudaStreamNonBlocking, lo ) != cudaSuccess
      || cudaEventCreateWithFlags( &e->ev_fork, cudaEventDisableTiming ) != cudaSuccess
      || cudaEventCreateWithFlags( &e->ev_late[ 0 ], cudaEventDisableTiming ) != cudaSuccess
      || cudaEventCreateWithFlags( &e->ev_late[ 1 ], cudaEventDisableTiming ) != cudaSuccess
      || cudaStreamCreateWithFlags( &e->adm_stream, cudaStreamNonBlocking ) != cudaSuccess
      || cudaEventCreateWithFlags( &e->ev_adm, cudaEventDisableTiming ) != cudaSuccess )
      return bail( fail( NG_ERR_CUDA, "ng_create: late-delivery stream or event creation failed" ) );
  }
  cudaEventCreate( &e->ev0 );
  cudaEventCreate( &e->ev1 );
  if ( cudaMallocHost( &e->host_ctl, 2 * sizeof( Ctl ) ) != cudaSuccess )
    return bail( fail( NG_ERR_MEMORY, "cudaMallocHost failed" ) );
  std::memset( e->host_ctl, 0, 2 * sizeof( Ctl ) );
  if ( cudaEventCreateWithFlags( &e->group_done[ 0 ], cudaEventDisableTiming ) != cudaSuccess
    || cudaEventCreateWithFlags( &e->group_done[ 1 ], cudaEventDisableTiming ) != cudaSuccess
    || cudaStreamCreateWithFlags( &e->copy_stream, cudaStreamNonBlocking ) != cudaSuccess )
    return bail( fail( NG_ERR_CUDA, "ng_create: event or stream creation failed" ) );
  int64_t off = 0;
  for ( int k = 0; k < cfg->n_blocks; ++k )
  {
    ng_engine::Blk b;
    b.model = cfg->block_model[ k ];
    b.off = off;
    b.n = cfg->block_size[ k ];
    off += b.n;
    std::vector< double > dp;
    default_params( b.model, dp );
    b.par.resize( ( size_t ) n_params( b.model ) );
    for ( int p = 0; p < n_params( b.model ); ++p )
      b.par[ p ].assign( ( size_t ) b.n, dp[ p ] );
    e->blk.push_back( std::move( b ) );
  }
  for ( auto& b : e->blk )
  {
    for ( int s = 0; s < n_states( b.model ); ++s )
    {
      if ( ( rc = e->alloc( b.st[ s ], ( size_t ) b.n * e->rsz ) ) )
        return bail( rc );
      const double dv = default_state( b.model, s );
      if ( dv != 0.0 )
      {
        std::vector< char > tmp( ( size_t ) b.n * e->rsz );
        for ( int64_t i = 0; i < b.n; ++i )
        {
          if ( e->rsz == 8 )
            reinterpret_cast< double* >( tmp.data() )[ i ] = dv;
          else
            reinterpret_cast< float* >( tmp.data() )[ i ] = ( float ) dv;
        }
        if ( ( rc = e->upload( b.st[ s ], tmp.data(), tmp.size() ) ) )
          return bail( rc );
      }
    }
    if ( ( rc = e->alloc( b.r, ( size_t ) b.n * sizeof( int32_t ) ) ) )
      return bail( rc );
    if ( b.model == NG_AEIF_COND_ALPHA )
    {
      std::vector< double > hs( ( size_t ) b.n, e->h );
      if ( ( rc = e->upload( b.istep, hs.data(), hs.size() * sizeof( double ) ) ) )
        return bail( rc );
      if ( ( rc = e->alloc( b.perm, ( size_t ) std::max< int64_t >( b.n, 1 ) * sizeof( int32_t ) ) )
        || ( rc = e->alloc( b.bins, 2 * AEIF_BINS * sizeof( unsigned ) ) ) )
        return bail( rc );
    }
  }
  // ring [L][C][N]
  if ( cfg->ring32 && !( cfg->serving && cfg->precision == NG_FP32 && cfg->ring_bound > 0 ) )
    return bail( fail( NG_ERR_ARG, "ng_create: ring32 needs a serving engine in the FP32 form and a ring_bound" ) );
  e->ring_bytes = cfg->ring32 ? 4 : 8;
  if ( ( rc = e->alloc( e->ring, ( size_t ) e->L * e->C * ( size_t ) N * e->ring_bytes ) ) )
    return bail( rc );
  // empty CSR: every source has no edges
  if ( ( rc = e->alloc( e->row_beg, ( size_t ) e->n_src * sizeof( int64_t ) ) ) )
    return bail( rc );
  if ( ( rc = e->alloc( e->row_len, ( size_t ) e->n_src * sizeof( int32_t ) ) ) )
    return bail( rc );
  if ( ( rc = e->alloc( e->real_deg, ( size_t ) e->n_src * sizeof( int32_t ) ) ) )
    return bail( rc );
  if ( ( rc = e->alloc( e->row_ue, ( size_t ) e->n_src * sizeof( int32_t ) ) )
    || ( rc = e->alloc( e->row_ls, ( size_t ) e->n_src * sizeof( int32_t ) ) ) )
    return bail( rc );
  if ( ( rc = e->alloc( e->tdc, 16 ) ) || ( rc = e->alloc( e->w, 32 ) ) )
    return bail( rc );
  e->tbits = 1;
  while ( ( 1ll << e->tbits ) < N )
    ++e->tbits;
  if ( e->tbits > 30 )
    return bail( fail( NG_ERR_ARG, "ng_create: too many neurons for the packed edge format" ) );
  e->tmask = ( 1u << e->tbits ) - 1u;
  const int dbits = 31 - e->tbits;
  e->dmask = ( 1u << dbits ) - 1u;
  if ( ( int64_t ) cfg->max_delay > ( int64_t ) e->dmask )
    return bail( fail( NG_ERR_ARG, "ng_create: max_delay does not fit the packed edge format for this network size" ) );
  if ( e->L >= 65536 )
    return bail( fail( NG_ERR_ARG, "ng_create: max_delay must be below 65536 steps" ) );
  e->ent_cap = 1024;
  if ( ( rc = e->alloc( e->ent, ( size_t ) e->ent_cap * sizeof( int4 ) ) ) )
    return bail( rc );
  e->log_cap = cfg->spike_log_capacity > 0 ? cfg->spike_log_capacity
                                           : std::max< int64_t >( 1 << 22, 64 * e->n_src );
  e->log_cap = std::min< int64_t >( e->log_cap, 1ll << 28 );
  if ( ( rc = e->alloc( e->log, 2 * ( size_t ) e->log_cap * sizeof( uint2 ) ) ) )
    return bail( rc );
  // pinned staging for the spike-log drain, sized once for a typical group
  if ( e->grow_pinned( ( size_t ) std::min< int64_t >( e->log_cap, 1ll << 24 ) * sizeof( uint2 ) ) )
    return bail( NG_ERR_MEMORY );
  if ( ( rc = e->alloc( e->rec, ( size_t ) e->n_src ) ) )
    return bail( rc );
  if ( ( rc = e->alloc( e->ctl, sizeof( Ctl ) ) ) )
    return bail( rc );
  {
    const long long o = ( long long ) cfg->start_step;
    if ( cudaMemcpyAsync( ( char* ) e->ctl.p + offsetof( Ctl, origin ), &o, sizeof( o ), cudaMemcpyHostToDevice,
           e->stream )
      != cudaSuccess )
      return bail( fail( NG_ERR_CUDA, "ng_create: control block upload failed" ) );
  }
  e->deliver_ctas = 1;
  {
    // resident delivery CTAs per SM (the kernel splits its work over the warps of one wave)
    int occ = 0;
    if ( e->prec == NG_FP64 )
      cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, k_deliver< false, false >, 256, 0 );
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, k_deliver< true, false >, 256, 0 );
    e->occ_deliver = std::max( 1, std::min( occ, 8 ) );
    e->deliver_per_sm = e->occ_deliver;
  }
  if ( cfg->serving )
  {
    if ( cfg->n_blocks != 1 || cfg->n_generators != 0 || cfg->edge_capacity < 4 || cfg->max_networks < 1
      || cfg->max_networks > ( 1 << ( 32 - LOG_ID_SHIFT ) ) )
      return bail( fail( NG_ERR_ARG, "ng_create: serving needs one model block, no generators, an edge capacity "
                                     "and 1 to 1024 network slots" ) );
    if ( ( rc = e->setup_serving() ) )
      return bail( rc );
    e->deliver_want = INT64_MAX;
    e->deliver_ctas = e->sms * e->deliver_per_sm;
  }
  e->refresh_late();
  if ( cudaStreamSynchronize( e->stream ) != cudaSuccess )
    return bail( fail( NG_ERR_CUDA, "ng_create: device initialisation failed" ) );
  *out = e;
  return NG_OK;
}

int
ng_destroy( ng_engine* eng )
{
  delete eng;
  return NG_OK;
}

static int
check_range( ng_engine* e, int32_t block, int64_t first, int64_t count )
{
  if ( !e )
    return fail( NG_ERR_ARG, "null engine" );
  if ( block < 0 || block >= ( int32_t ) e->blk.size() )
    return fail( NG_ERR_ARG, "block index out of range" );
  if ( first < 0 || count < 0 || first + count > e->blk[ block ].n )
    return fail( NG_ERR_ARG, "neuron range out of bounds" );
  return NG_OK;
}

int
ng_set_var( ng_engine* e, int32_t block, const char* name, const double* values, int64_t first, int64_t count )
{
  SETTLE( e );
  int rc = check_range( e, block, first, count );
  if ( rc )
    return rc;
  if ( !name || ( count > 0 && !values ) )
    return fail( NG_ERR_ARG, "ng_set_var: null argument" );
  auto& b = e->blk[ block ];
  if ( std::strcmp( name, "tau_minus" ) == 0 )
  {
    // ArchivingNode's tau_minus (archiving_node.cpp:232-245), for postsynaptic traces of STDP
    for ( int64_t k = 0; k < count; ++k )
      if ( !( values[ k ] > 0.0 ) )
        return fail( NG_ERR_ARG, "All time constants must be strictly positive." );
    std::copy( values, values + count, e->tau_minus_host.begin() + b.off + first );
    return e->upload_tau_minus();
  }
  const VarSpec* v = find_var( b.model, name );
  if ( !v )
    return fail( NG_ERR_UNKNOWN_NAME, std::string( "unknown variable '" ) + name + "' for this model" );
  cudaSetDevice( e->cfg.device );
  if ( count == 0 )
    return NG_OK;
  if ( v->kind == PARAM )
  {
    std::copy( values, values + count, b.par[ v->slot ].begin() + first );
    b.dirty = true;
    return NG_OK;
  }
  if ( v->kind == REFR )
  {
    std::vector< int32_t > tmp( ( size_t ) count );
    for ( int64_t i = 0; i < count; ++i )
      tmp[ i ] = ( int32_t ) values[ i ];
    CU( cudaMemcpyAsync( ( int32_t* ) b.r.p + first, tmp.data(), tmp.size() * 4, cudaMemcpyHostToDevice, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
    return NG_OK;
  }
  if ( v->kind == ISTEP )
  {
    CU( cudaMemcpyAsync( ( double* ) b.istep.p + first, values, ( size_t ) count * 8, cudaMemcpyHostToDevice, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
    return NG_OK;
  }
  if ( e->rsz == 8 )
  {
    CU( cudaMemcpyAsync( ( double* ) b.st[ v->slot ].p + first, values, ( size_t ) count * 8, cudaMemcpyHostToDevice,
      e->stream ) );
  }
  else
  {
    std::vector< float > tmp( ( size_t ) count );
    for ( int64_t i = 0; i < count; ++i )
      tmp[ i ] = ( float ) values[ i ];
    CU( cudaMemcpyAsync( ( float* ) b.st[ v->slot ].p + first, tmp.data(), tmp.size() * 4, cudaMemcpyHostToDevice,
      e->stream ) );
  }
  CU( cudaStreamSynchronize( e->stream ) );
  return NG_OK;
}

int
ng_get_var( ng_engine* e, int32_t block, const char* name, double* out, int64_t first, int64_t count )
{
  SETTLE( e );
  int rc = check_range( e, block, first, count );
  if ( rc )
    return rc;
  if ( !name || ( count > 0 && !out ) )
    return fail( NG_ERR_ARG, "ng_get_var: null argument" );
  auto& b = e->blk[ block ];
  if ( std::strcmp( name, "tau_minus" ) == 0 )
  {
    std::copy( e->tau_minus_host.begin() + b.off + first, e->tau_minus_host.begin() + b.off + first + count, out );
    return NG_OK;
  }
  const VarSpec* v = find_var( b.model, name );
  if ( !v )
    return fail( NG_ERR_UNKNOWN_NAME, std::string( "unknown variable '" ) + name + "' for this model" );
  cudaSetDevice( e->cfg.device );
  if ( count == 0 )
    return NG_OK;
  if ( v->kind == PARAM )
  {
    std::copy( b.par[ v->slot ].begin() + first, b.par[ v->slot ].begin() + first + count, out );
    return NG_OK;
  }
  if ( v->kind == REFR )
  {
    std::vector< int32_t > tmp( ( size_t ) count );
    CU( cudaMemcpyAsync( tmp.data(), ( int32_t* ) b.r.p + first, tmp.size() * 4, cudaMemcpyDeviceToHost, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
    for ( int64_t i = 0; i < count; ++i )
      out[ i ] = tmp[ i ];
    return NG_OK;
  }
  if ( v->kind == ISTEP )
  {
    CU( cudaMemcpyAsync( out, ( double* ) b.istep.p + first, ( size_t ) count * 8, cudaMemcpyDeviceToHost, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
    return NG_OK;
  }
  if ( e->rsz == 8 )
  {
    CU( cudaMemcpyAsync( out, ( double* ) b.st[ v->slot ].p + first, ( size_t ) count * 8, cudaMemcpyDeviceToHost,
      e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
  }
  else
  {
    std::vector< float > tmp( ( size_t ) count );
    CU( cudaMemcpyAsync( tmp.data(), ( float* ) b.st[ v->slot ].p + first, tmp.size() * 4, cudaMemcpyDeviceToHost,
      e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
    for ( int64_t i = 0; i < count; ++i )
      out[ i ] = tmp[ i ];
  }
  return NG_OK;
}

int
ng_set_connections( ng_engine* e, int64_t n_src, const int64_t* row_ptr, const int32_t* target, const double* weight,
  const int32_t* delay_steps )
{
  SETTLE( e );
  if ( !e || !row_ptr )
    return fail( NG_ERR_ARG, "ng_set_connections: null argument" );
  if ( n_src != e->n_src )
    return fail( NG_ERR_ARG, "ng_set_connections: n_src must equal n_neurons + n_generators" );
  const int64_t nnz = row_ptr[ n_src ];
  if ( row_ptr[ 0 ] != 0 || nnz < 0 || ( nnz > 0 && ( !target || !weight || !delay_steps ) ) )
    return fail( NG_ERR_ARG, "ng_set_connections: bad CSR" );
  cudaSetDevice( e->cfg.device );
  std::vector< int64_t > prow( ( size_t ) n_src + 1, 0 );
  std::vector< int32_t > rdeg( ( size_t ) n_src, 0 );
  for ( int64_t s = 0; s < n_src; ++s )
  {
    const int64_t deg = row_ptr[ s + 1 ] - row_ptr[ s ];
    if ( deg < 0 || deg > INT32_MAX )
      return fail( NG_ERR_ARG, "ng_set_connections: row pointers must be non-decreasing" );
    rdeg[ s ] = ( int32_t ) deg;
    prow[ s + 1 ] = prow[ s ] + ( ( deg + 3 ) & ~3ll );
  }
  const int64_t np = prow[ n_src ];
  // the edges are packed on the device: copy the caller's arrays as they are
  int rc;
  DevBuf d_rp, d_prow, d_tgt, d_w, d_d, d_scr;
  auto free_tmp = [ & ]() {
    for ( DevBuf* b : { &d_rp, &d_prow, &d_tgt, &d_w, &d_d, &d_scr } )
      cudaFree( b->p );
  };
  PackSpec ps {};
  ps.n_blocks = ( int ) e->blk.size();
  for ( int k = 0; k < ps.n_blocks; ++k )
  {
    ps.bend[ k ] = e->blk[ k ].off + e->blk[ k ].n;
    ps.model[ k ] = e->blk[ k ].model;
  }
  ps.N = e->N;
  ps.min_d = e->cfg.min_delay;
  ps.max_d = e->cfg.max_delay;
  ps.tbits = e->tbits;
  if ( ( rc = e->upload( d_rp, row_ptr, ( size_t ) ( n_src + 1 ) * 8 ) ) || ( rc = e->upload( d_prow, prow.data(), prow.size() * 8 ) )
    || ( rc = e->upload( d_tgt, target, ( size_t ) nnz * 4 ) ) || ( rc = e->upload( d_w, weight, ( size_t ) nnz * 8 ) )
    || ( rc = e->upload( d_d, delay_steps, ( size_t ) nnz * 4 ) ) || ( rc = e->alloc( d_scr, 16 ) ) )
  {
    free_tmp();
    return rc;
  }
  unsigned long long host_scr[ 2 ] = { 0ull, 0ull };
  if ( nnz > 0 )
  {
    const unsigned g = ( unsigned ) std::min< int64_t >( ( nnz + 255 ) / 256, ( int64_t ) e->sms * 16 );
    k_edge_check<<< g, 256, 0, e->stream >>>( nnz, ( const int32_t* ) d_tgt.p, ( const double* ) d_w.p,
      ( const int32_t* ) d_d.p, ps, ( unsigned long long* ) d_scr.p, ( int* ) ( ( unsigned long long* ) d_scr.p + 1 ) );
    CU( cudaGetLastError() );
    CU( cudaMemcpyAsync( host_scr, d_scr.p, 16, cudaMemcpyDeviceToHost, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
  }
  const int bad = ( int ) ( host_scr[ 1 ] & 0xffffffffull );
  if ( bad )
  {
    free_tmp();
    if ( bad & 1 )
      return fail( NG_ERR_ARG, "ng_set_connections: target out of range" );
    if ( bad & 2 )
      return fail( NG_ERR_ARG, "ng_set_connections: delay outside [min_delay, max_delay]" );
    return fail( NG_ERR_ARG, "ng_set_connections: weight not finite" );
  }
  double maxabs = 0.0;
  std::memcpy( &maxabs, &host_scr[ 0 ], 8 );
  {
    std::vector< int32_t > plen( ( size_t ) n_src );
    for ( int64_t sidx = 0; sidx < n_src; ++sidx )
      plen[ sidx ] = ( int32_t ) ( prow[ sidx + 1 ] - prow[ sidx ] );
    if ( ( rc = e->upload( e->row_beg, prow.data(), ( size_t ) n_src * sizeof( int64_t ) ) )
      || ( rc = e->upload( e->row_len, plen.data(), plen.size() * sizeof( int32_t ) ) )
      || ( rc = e->upload( e->real_deg, rdeg.data(), rdeg.size() * sizeof( int32_t ) ) ) )
    {
      free_tmp();
      return rc;
    }
    CU( cudaStreamSynchronize( e->stream ) );  // the host vectors go out of scope
  }
  const bool fx = e->prec != NG_FP64;
  // int32 fixed point with a power-of-two scale: |w| * 2^S < 2^31
  int S = 0;
  if ( fx && maxabs > 0 )
  {
    S = ( int ) std::floor( std::log2( 2147483647.0 / maxabs ) );
    S = std::max( -30, std::min( S, 60 ) );
    while ( S > -30 && std::ldexp( maxabs, S ) >= 2147483647.0 )
      --S;
  }
  const size_t np4 = ( size_t ) std::max< int64_t >( np, 4 );
  if ( ( rc = e->alloc( e->tdc, np4 * sizeof( uint32_t ) ) ) || ( rc = e->alloc( e->w, np4 * ( fx ? 4 : 8 ) ) ) )
  {
    free_tmp();
    return rc;
  }
  if ( n_src > 0 && nnz > 0 )
  {
    const unsigned g = ( unsigned ) ( ( n_src * 32 + 255 ) / 256 );
    k_pack_edges<<< g, 256, 0, e->stream >>>( n_src, ( const long long* ) d_rp.p, ( const long long* ) d_prow.p,
      ( const int32_t* ) d_tgt.p, ( const double* ) d_w.p, ( const int32_t* ) d_d.p, ps, fx ? 1 : 0, std::ldexp( 1.0, S ),
      ( uint32_t* ) e->tdc.p, e->w.p, e->late_thr(), ( int32_t* ) e->row_ue.p, ( int32_t* ) e->row_ls.p );
    CU( cudaGetLastError() );
  }
  else
  {
    CU( cudaMemsetAsync( e->row_ue.p, 0, e->row_ue.bytes, e->stream ) );
    CU( cudaMemsetAsync( e->row_ls.p, 0, e->row_ls.bytes, e->stream ) );
  }
  CU( cudaStreamSynchronize( e->stream ) );
  free_tmp();
  e->fx_inv = fx ? std::ldexp( 1.0, -S ) : 1.0;
  e->nnz_padded = np;
  e->chunks_all_src = 0;
  e->chunks_max_gen = 0;
  for ( int64_t sidx = 0; sidx < n_src; ++sidx )
  {
    const int64_t nch = ( prow[ sidx + 1 ] - prow[ sidx ] + CHUNK_EDGES - 1 ) / CHUNK_EDGES;
    if ( sidx < e->N )
      e->chunks_all_src += nch;
    else
      e->chunks_max_gen = std::max( e->chunks_max_gen, nch );
  }
  if ( ( rc = e->resize_work() ) )
    return rc;
  // delivery grid: up to one wave of resident CTAs, fewer for small graphs
  e->deliver_want = std::max< int64_t >( 1, e->chunks_all_src / 64 );
  e->apply_deliver();
  CU( cudaStreamSynchronize( e->stream ) );
  return NG_OK;
}

int
ng_set_connections_coo( ng_engine* e, int64_t n_src, int64_t nnz, const int32_t* source, const int32_t* target,
  const double* weight, const int32_t* delay_steps )
{
  SETTLE( e );
  if ( !e || nnz < 0 || ( nnz > 0 && ( !source || !target || !weight || !delay_steps ) ) )
    return fail( NG_ERR_ARG, "ng_set_connections_coo: bad argument" );
  if ( n_src != e->n_src )
    return fail( NG_ERR_ARG, "ng_set_connections_coo: n_src must equal n_neurons + n_generators" );
  std::vector< int64_t > row( ( size_t ) n_src + 1, 0 );
  for ( int64_t k = 0; k < nnz; ++k )
  {
    const int32_t s = source[ k ];
    if ( s < 0 || s >= n_src )
      return fail( NG_ERR_ARG, "ng_set_connections_coo: source out of range" );
    ++row[ ( size_t ) s + 1 ];
  }
  for ( int64_t s = 0; s < n_src; ++s )
    row[ s + 1 ] += row[ s ];
  std::vector< int64_t > pos( row.begin(), row.end() - 1 );
  std::vector< int32_t > tg( ( size_t ) std::max< int64_t >( nnz, 1 ) );
  std::vector< double > ww( ( size_t ) std::max< int64_t >( nnz, 1 ) );
  std::vector< int32_t > dd( ( size_t ) std::max< int64_t >( nnz, 1 ) );
  for ( int64_t k = 0; k < nnz; ++k )
  {
    const int64_t j = pos[ source[ k ] ]++;
    tg[ j ] = target[ k ];
    ww[ j ] = weight[ k ];
    dd[ j ] = delay_steps[ k ];
  }
  return ng_set_connections( e, n_src, row.data(), tg.data(), ww.data(), dd.data() );
}

int
ng_set_plastic_connections( ng_engine* e, int64_t n_src, const int64_t* row_ptr, const int32_t* target,
  const double* weight, const int32_t* delay_steps, double lambda, double alpha, double mu, double tau_plus )
{
  SETTLE( e );
  if ( !e || !row_ptr || n_src < 0 || n_src > ( e ? e->N : 0 ) )
    return fail( NG_ERR_ARG, "ng_set_plastic_connections: sources are neurons 0..n_src-1, n_src <= neurons" );
  if ( e->serving )
    return fail( NG_ERR_STATE, "ng_set_plastic_connections: plastic connections run in a static engine" );
  for ( const auto& b : e->blk )
    if ( b.model == NG_AEIF_COND_ALPHA || sign_channels( b.model ) != sign_channels( e->blk[ 0 ].model ) )
      return fail( NG_ERR_ARG, "ng_set_plastic_connections: targets are iaf_psc_delta, iaf_psc_exp or iaf_psc_alpha "
                               "neurons with one input rule" );
  if ( e->cfg.min_delay > 32 )
    return fail( NG_ERR_ARG, "ng_set_plastic_connections: needs min_delay <= 32 steps" );
  if ( !( tau_plus > 0 ) )
    return fail( NG_ERR_ARG, "tau_plus must be > 0" );
  const int64_t nnz = row_ptr[ n_src ];
  if ( row_ptr[ 0 ] != 0 || nnz < 0 || ( nnz > 0 && ( !target || !weight || !delay_steps ) ) )
    return fail( NG_ERR_ARG, "ng_set_plastic_connections: bad CSR" );
  if ( nnz >= ( int64_t ) 0xffffffffll )
    return fail( NG_ERR_ARG, "ng_set_plastic_connections: at most 2^32 - 1 plastic connections" );
  std::vector< uint8_t > ninc( ( size_t ) e->N, 0 );
  for ( int64_t s2 = 0; s2 < n_src; ++s2 )
    if ( row_ptr[ s2 + 1 ] < row_ptr[ s2 ] )
      return fail( NG_ERR_ARG, "ng_set_plastic_connections: row pointers must not decrease" );
  for ( int64_t k = 0; k < nnz; ++k )
  {
    if ( target[ k ] < 0 || target[ k ] >= e->N )
      return fail( NG_ERR_ARG, "ng_set_plastic_connections: target out of range" );
    if ( delay_steps[ k ] < e->cfg.min_delay || delay_steps[ k ] > e->cfg.max_delay )
      return fail( NG_ERR_ARG, "ng_set_plastic_connections: delay outside [min_delay, max_delay]" );
    if ( !( weight[ k ] >= 0.0 ) )
      return fail( NG_ERR_ARG, "stdp_pl_synapse_hom: weights must be >= 0 (the power law of the facilitation)" );
    ninc[ ( size_t ) target[ k ] ] = 1;
  }
  // the target-major index (the flush walks a neuron's incoming connections)
  const size_t N = ( size_t ) e->N;
  std::vector< int64_t > in_row( N + 1, 0 );
  for ( int64_t k = 0; k < nnz; ++k )
    ++in_row[ ( size_t ) target[ k ] + 1 ];
  for ( size_t i = 0; i < N; ++i )
    in_row[ i + 1 ] += in_row[ i ];
  std::vector< uint32_t > in_edge( ( size_t ) std::max< int64_t >( nnz, 1 ) );
  std::vector< int32_t > in_src( ( size_t ) std::max< int64_t >( nnz, 1 ) );
  {
    std::vector< int64_t > fill( in_row.begin(), in_row.end() - 1 );
    int32_t dmax = 0, dmin = INT32_MAX;
    for ( int64_t s2 = 0; s2 < n_src; ++s2 )
      for ( int64_t k = row_ptr[ s2 ]; k < row_ptr[ s2 + 1 ]; ++k )
      {
        const int64_t q = fill[ ( size_t ) target[ k ] ]++;
        in_edge[ ( size_t ) q ] = ( uint32_t ) k;
        in_src[ ( size_t ) q ] = ( int32_t ) s2;
        dmax = std::max( dmax, delay_steps[ k ] );
        dmin = std::min( dmin, delay_steps[ k ] );
      }
    e->pl_dmax_ms = ( double ) dmax * ( ( double ) e->tics_per_step / e->cfg.tics_per_ms );
    e->pl_dconst = ( nnz > 0 && dmin == dmax ) ? dmax : -1;
  }
  cudaSetDevice( e->cfg.device );
  int rc;
  std::vector< double > inv( N );
  for ( size_t i = 0; i < N; ++i )
    inv[ i ] = 1. / e->tau_minus_host[ i ];
  static const int64_t zero[ 1 ] = { 0 };  // the one cell of an empty plastic table
  if ( ( rc = e->upload( e->pl_row, row_ptr, ( size_t ) ( n_src + 1 ) * 8 ) )
    || ( rc = e->upload( e->pl_tgt, nnz ? ( const void* ) target : zero, ( size_t ) std::max< int64_t >( nnz, 1 ) * 4 ) )
    || ( rc = e->upload( e->pl_dly, nnz ? ( const void* ) delay_steps : zero, ( size_t ) std::max< int64_t >( nnz, 1 ) * 4 ) )
    || ( rc = e->upload( e->pl_w, nnz ? ( const void* ) weight : zero, ( size_t ) std::max< int64_t >( nnz, 1 ) * 8 ) )
    || ( rc = e->upload( e->pl_wrun, nnz ? ( const void* ) weight : zero, ( size_t ) std::max< int64_t >( nnz, 1 ) * 8 ) )
    || ( rc = e->alloc( e->pl_Kplus, ( size_t ) std::max< int64_t >( n_src, 1 ) * 8 ) )
    || ( rc = e->alloc( e->pl_tlast, ( size_t ) std::max< int64_t >( n_src, 1 ) * 8 ) )
    || ( rc = e->upload( e->pl_ninc, ninc.data(), N ) ) || ( rc = e->upload( e->pl_tauinv, inv.data(), N * 8 ) )
    || ( rc = e->alloc( e->pl_Kminus, N * 8 ) ) || ( rc = e->alloc( e->pl_last, N * 8 ) )
    || ( rc = e->alloc( e->pl_hist_t, N * STDP_HIST * 8 ) ) || ( rc = e->alloc( e->pl_hist_K, N * STDP_HIST * 8 ) )
    || ( rc = e->alloc( e->pl_hist_n, N * 8 ) ) || ( rc = e->alloc( e->pl_hist_lo, N * 8 ) )
    || ( rc = e->alloc( e->pl_drop_t, N * 8 ) ) || ( rc = e->alloc( e->pl_drop_K, N * 8 ) )
    || ( rc = e->alloc( e->pl_nflush, N * 4 ) ) || ( rc = e->upload( e->pl_in_row, in_row.data(), ( N + 1 ) * 8 ) )
    || ( rc = e->upload( e->pl_in_edge, in_edge.data(), in_edge.size() * 4 ) )
    || ( rc = e->upload( e->pl_in_src, in_src.data(), in_src.size() * 4 ) ) )
    return rc;
  if ( !e->gmask.p && ( rc = e->alloc( e->gmask, N * 4 ) ) )
    return rc;
  if ( e->pl_dconst >= 0 )
  {
    const size_t q = N * ( size_t ) e->cfg.min_delay;
    if ( ( rc = e->alloc( e->pl_tab_fin, q * 4 ) ) || ( rc = e->alloc( e->pl_tab_km, q * 8 ) ) )
      return rc;
  }
  e->pl_nnz = nnz;
  e->pl_nsrc = n_src;
  e->pl_lambda = lambda;
  e->pl_alpha = alpha;
  e->pl_mu = mu;
  e->pl_tau_plus = tau_plus;
  e->plastic_on = true;
  ++e->generation;
  CU( cudaStreamSynchronize( e->stream ) );
  return NG_OK;
}

int
ng_get_plastic_weights( ng_engine* e, double* out, int64_t n )
{
  SETTLE( e );
  if ( !e || ( n > 0 && !out ) )
    return fail( NG_ERR_ARG, "ng_get_plastic_weights: null argument" );
  if ( n != e->pl_nnz )
    return fail( NG_ERR_ARG, "ng_get_plastic_weights: n must be the number of plastic connections" );
  cudaSetDevice( e->cfg.device );
  if ( n > 0 )
  {
    CU( cudaMemcpyAsync( out, e->pl_w.p, ( size_t ) n * 8, cudaMemcpyDeviceToHost, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
  }
  return NG_OK;
}

int
ng_set_spike_schedule( ng_engine* e, int64_t n, const int64_t* emit_step, const int32_t* source )
{
  SETTLE( e );
  if ( !e || n < 0 || ( n > 0 && ( !emit_step || !source ) ) )
    return fail( NG_ERR_ARG, "ng_set_spike_schedule: bad argument" );
  cudaSetDevice( e->cfg.device );
  for ( int64_t i = 0; i < n; ++i )
  {
    if ( i > 0 && emit_step[ i ] < emit_step[ i - 1 ] )
      return fail( NG_ERR_ARG, "ng_set_spike_schedule: steps must be sorted" );
    if ( source[ i ] < 0 || source[ i ] >= e->n_src )
      return fail( NG_ERR_ARG, "ng_set_spike_schedule: source out of range" );
  }
  int rc;
  if ( ( rc = e->upload( e->sched_step, emit_step, ( size_t ) n * sizeof( int64_t ) ) ) )
    return rc;
  if ( ( rc = e->upload( e->sched_src, source, ( size_t ) n * sizeof( int32_t ) ) ) )
    return rc;
  e->n_sched = n;
  // the delivery work must also hold the generator spikes of one slice
  if ( ( rc = e->resize_work() ) )
    return rc;
  if ( e->log_cap < 2 * n + 4 * e->n_src )
  {
    e->log_cap = 2 * n + 4 * e->n_src;
    if ( ( rc = e->alloc( e->log, 2 * ( size_t ) e->log_cap * sizeof( uint2 ) ) ) )
      return rc;
  }
  // consume entries already in the past
  const int64_t clock = e->origin + e->from;
  int64_t pos = 0;
  while ( pos < n && emit_step[ pos ] < clock )
    ++pos;
  CU( cudaMemcpyAsync( ( char* ) e->ctl.p + offsetof( Ctl, sched_pos ), &pos, sizeof( long long ),
    cudaMemcpyHostToDevice, e->stream ) );
  CU( cudaStreamSynchronize( e->stream ) );
  ++e->generation;
  return NG_OK;
}

int
ng_set_poisson( ng_engine* e, const double* rate_hz, const double* weight, const int32_t* delay_steps,
  int64_t start_step, int64_t stop_step, uint64_t seed )
{
  SETTLE( e );
  if ( !e || !rate_hz || !weight || !delay_steps )
    return fail( NG_ERR_ARG, "ng_set_poisson: null argument" );
  cudaSetDevice( e->cfg.device );
  const int64_t n = e->N;
  std::vector< double4 > tab( ( size_t ) n );
  std::vector< int2 > ref( ( size_t ) n, make_int2( 0, 0 ) );
  std::vector< uint64_t > cdf;
  std::unordered_map< double, int2 > tables;  // one CDF table per distinct lambda
  bool any = false;
  for ( int64_t i = 0; i < n; ++i )
  {
    if ( rate_hz[ i ] > 0 && ( delay_steps[ i ] < e->cfg.min_delay || delay_steps[ i ] > e->cfg.max_delay ) )
      return fail( NG_ERR_ARG, "ng_set_poisson: delay outside [min_delay, max_delay]" );
    // lambda = h * rate * 1e-3 (models/poisson_generator.cpp:114)
    const double lam = rate_hz[ i ] > 0 ? e->h * rate_hz[ i ] * 1e-3 : 0.0;
    tab[ i ] = poisson_table( lam );
    if ( !( lam > 0 ) )
      continue;
    any = true;
    auto it = tables.find( lam );
    if ( it == tables.end() )
    {
      int2 r2 = make_int2( ( int ) cdf.size(), -1 );
      std::vector< uint64_t > t2;
      if ( poisson_cdf_table( lam, t2 ) )
      {
        r2.y = ( int ) t2.size();
        cdf.insert( cdf.end(), t2.begin(), t2.end() );
      }
      it = tables.emplace( lam, r2 ).first;
    }
    ref[ i ] = it->second;
  }
  if ( cdf.empty() )
    cdf.push_back( 1ull << 53 );
  int rc;
  if ( ( rc = e->upload( e->pois, tab.data(), tab.size() * sizeof( double4 ) ) ) )
    return rc;
  if ( ( rc = e->upload( e->pois_ref, ref.data(), ref.size() * sizeof( int2 ) ) ) )
    return rc;
  if ( ( rc = e->upload( e->pois_cdf, cdf.data(), cdf.size() * sizeof( uint64_t ) ) ) )
    return rc;
  if ( ( rc = e->upload( e->pois_w, weight, ( size_t ) n * sizeof( double ) ) ) )
    return rc;
  if ( ( rc = e->upload( e->pois_d, delay_steps, ( size_t ) n * sizeof( int32_t ) ) ) )
    return rc;
  e->has_pois = any ? 1 : 0;
  e->pois_start = start_step;
  e->pois_stop = stop_step;
  e->key0 = ( uint32_t ) seed;
  e->key1 = ( uint32_t ) ( seed >> 32 );
  CU( cudaStreamSynchronize( e->stream ) );
  ++e->generation;
  return NG_OK;
}

int
ng_set_recording( ng_engine* e, const uint8_t* flags )
{
  SETTLE( e );
  if ( !e || !flags )
    return fail( NG_ERR_ARG, "ng_set_recording: null argument" );
  cudaSetDevice( e->cfg.device );
  int64_t nr = 0;
  for ( int64_t i = 0; i < e->n_src; ++i )
    nr += flags[ i ] ? 1 : 0;
  std::vector< uint8_t > f( flags, flags + e->n_src );
  e->rec_host = f;
  e->log_bound_dirty = true;
  int rc = e->upload( e->rec, f.data(), f.size() );
  if ( rc )
    return rc;
  e->n_rec = nr;
  CU( cudaStreamSynchronize( e->stream ) );
  ++e->generation;
  return NG_OK;
}

int
ng_set_trace( ng_engine* e, int64_t n_idx, const int32_t* neuron, int32_t n_vars, const char* const* vars,
  int32_t interval_steps )
{
  SETTLE( e );
  if ( !e || n_idx < 0 || ( n_idx > 0 && ( !neuron || !vars || n_vars < 1 ) ) || interval_steps < 1
    || n_vars > MAX_STATE || n_vars < 0 )
    return fail( NG_ERR_ARG, "ng_set_trace: bad argument" );
  cudaSetDevice( e->cfg.device );
  std::vector< int32_t > col( ( size_t ) e->N, -1 );
  int model = -1;
  for ( int64_t k = 0; k < n_idx; ++k )
  {
    const int32_t i = neuron[ k ];
    if ( i < 0 || i >= e->N || col[ i ] >= 0 )
      return fail( NG_ERR_ARG, "ng_set_trace: neuron index out of range or repeated" );
    col[ i ] = ( int32_t ) k;
    const int bk = e->block_of( i );
    if ( model >= 0 && e->blk[ bk ].model != model )
      return fail( NG_ERR_ARG, "ng_set_trace: traced neurons must share one model" );
    model = e->blk[ bk ].model;
  }
  int8_t slots[ MAX_STATE ] = { 0, 0, 0, 0, 0, 0, 0, 0 };
  if ( n_idx > 0 )
  {
    for ( int32_t v = 0; v < n_vars; ++v )
    {
      const VarSpec* vs = vars[ v ] ? find_var( model, vars[ v ] ) : nullptr;
      if ( !vs || vs->kind != STATE )
        return fail( NG_ERR_UNKNOWN_NAME, std::string( "ng_set_trace: '" ) + ( vars[ v ] ? vars[ v ] : "(null)" )
            + "' is not a recordable state of this model" );
      slots[ v ] = ( int8_t ) vs->slot;
    }
  }
  int rc = e->upload( e->trace_col, col.data(), col.size() * sizeof( int32_t ) );
  if ( rc )
    return rc;
  e->n_trace_idx = n_idx > 0 ? ( int32_t ) n_idx : 0;
  e->n_trace_vars = n_idx > 0 ? n_vars : 0;
  std::copy( slots, slots + MAX_STATE, e->trace_slot );
  e->trace_interval = interval_steps;
  // rows held per group: bounded to 256 MB
  const int64_t per_row = std::max< int64_t >( 1, n_idx * std::max< int32_t >( 1, n_vars ) ) * 8;
  e->trace_rows_cap = std::max< int64_t >( 2, std::min< int64_t >( ( 256ll << 20 ) / per_row, 1 << 20 ) );
  if ( n_idx > 0 && ( rc = e->alloc( e->trace, ( size_t ) ( e->trace_rows_cap * per_row ) ) ) )
    return rc;
  e->out_trace.clear();
  e->trace_first_stamp = -1;
  CU( cudaStreamSynchronize( e->stream ) );
  ++e->generation;
  return NG_OK;
}

int
ng_simulate( ng_engine* e, int64_t n_steps )
{
  if ( !e || n_steps < 0 )
    return fail( NG_ERR_ARG, "ng_simulate: bad argument" );
  CU( cudaSetDevice( e->cfg.device ) );
  try
  {
    return e->simulate( n_steps );
  }
  catch ( const std::bad_alloc& )
  {
    cudaStreamSynchronize( e->stream );
    return fail( NG_ERR_MEMORY, "ng_simulate: out of host memory" );
  }
}

int
ng_simulate_async( ng_engine* e, int64_t n_steps )
{
  if ( !e || n_steps < 0 )
    return fail( NG_ERR_ARG, "ng_simulate_async: bad argument" );
  CU( cudaSetDevice( e->cfg.device ) );
  try
  {
    return e->simulate( n_steps, true );
  }
  catch ( const std::bad_alloc& )
  {
    cudaStreamSynchronize( e->stream );
    return fail( NG_ERR_MEMORY, "ng_simulate_async: out of host memory" );
  }
}

int
ng_update( ng_engine* e, int64_t origin, int32_t from, int32_t to )
{
  if ( !e )
    return fail( NG_ERR_ARG, "ng_update: null engine" );
  if ( e->serving )
    return fail( NG_ERR_STATE, "ng_update: serving engines advance with ng_simulate" );
  if ( from < 0 || to <= from || to > e->cfg.min_delay )
    return fail( NG_ERR_ARG, "ng_update: need 0 <= from < to <= min_delay" );
  if ( origin != e->origin || from != e->from )
    return fail( NG_ERR_STATE, "ng_update: the engine stands at slice origin " + std::to_string( e->origin ) + ", lag "
        + std::to_string( e->from ) + " (called with " + std::to_string( origin ) + ", " + std::to_string( from ) + ")" );
  CU( cudaSetDevice( e->cfg.device ) );
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = e->update_range( from, to );
  e->stats.simulate_ms += std::chrono::duration< double, std::milli >( std::chrono::steady_clock::now() - t0 ).count();
  return rc;
}

int
ng_sync( ng_engine* e )
{
  if ( !e )
    return fail( NG_ERR_ARG, "ng_sync: null engine" );
  CU( cudaSetDevice( e->cfg.device ) );
  SETTLE( e );
  return NG_OK;
}

int
ng_spike_count( ng_engine* e, int64_t* n )
{
  if ( !e || !n )
    return fail( NG_ERR_ARG, "ng_spike_count: null argument" );
  *n = ( int64_t ) e->out_src.size();
  return NG_OK;
}

int
ng_get_spikes( ng_engine* e, int32_t* source, int64_t* stamp, int64_t cap, int64_t* n_out )
{
  if ( !e || !n_out || cap < 0 || ( cap > 0 && ( !source || !stamp ) ) )
    return fail( NG_ERR_ARG, "ng_get_spikes: bad argument" );
  const int64_t k = std::min< int64_t >( cap, ( int64_t ) e->out_src.size() );
  std::copy( e->out_src.begin(), e->out_src.begin() + k, source );
  std::copy( e->out_stamp.begin(), e->out_stamp.begin() + k, stamp );
  e->out_src.erase( e->out_src.begin(), e->out_src.begin() + k );
  e->out_stamp.erase( e->out_stamp.begin(), e->out_stamp.begin() + k );
  *n_out = k;
  return NG_OK;
}

int
ng_trace_count( ng_engine* e, int64_t* n_rows, int64_t* first_stamp )
{
  SETTLE( e );
  if ( !e || !n_rows || !first_stamp )
    return fail( NG_ERR_ARG, "ng_trace_count: null argument" );
  const int64_t w = ( int64_t ) e->n_trace_idx * e->n_trace_vars;
  *n_rows = w > 0 ? ( int64_t ) e->out_trace.size() / w : 0;
  *first_stamp = e->trace_first_stamp;
  return NG_OK;
}

int
ng_get_trace( ng_engine* e, double* out, int64_t max_rows, int64_t* n_rows_out )
{
  SETTLE( e );
  if ( !e || !n_rows_out || max_rows < 0 || ( max_rows > 0 && !out ) )
    return fail( NG_ERR_ARG, "ng_get_trace: bad argument" );
  if ( e->n_trace_idx == 0 )
  {
    *n_rows_out = 0;
    return NG_OK;
  }
  const int64_t w = ( int64_t ) e->n_trace_idx * e->n_trace_vars;
  const int64_t rows = std::min< int64_t >( max_rows, ( int64_t ) e->out_trace.size() / w );
  const size_t cnt = ( size_t ) ( rows * w );
  std::copy( e->out_trace.begin(), e->out_trace.begin() + cnt, out );
  e->out_trace.erase( e->out_trace.begin(), e->out_trace.begin() + cnt );
  if ( rows > 0 )
    e->trace_first_stamp += rows * e->trace_interval;
  if ( e->out_trace.empty() )
    e->trace_first_stamp = -1;
  *n_rows_out = rows;
  return NG_OK;
}

int
ng_get_stats( ng_engine* e, ng_stats* out )
{
  SETTLE( e );
  if ( !e || !out )
    return fail( NG_ERR_ARG, "ng_get_stats: null argument" );
  e->stats.clock_steps = e->origin + e->from;
  e->stats.slices = e->slices;
  *out = e->stats;
  return NG_OK;
}

int
ng_set_profiling( ng_engine* e, int32_t on )
{
  SETTLE( e );
  if ( !e )
    return fail( NG_ERR_ARG, "null engine" );
  e->profiling = on ? 1 : 0;
  return NG_OK;
}

int
ng_set_stream( ng_engine* e, void* cuda_stream )
{
  SETTLE( e );
  if ( !e )
    return fail( NG_ERR_ARG, "null engine" );
  e->stream = cuda_stream ? ( cudaStream_t ) cuda_stream : e->own;
  e->drop_graphs();
  return NG_OK;
}

int
ng_set_graph_slices( ng_engine* e, int32_t slices_per_graph )
{
  SETTLE( e );
  if ( !e || slices_per_graph < 0 || slices_per_graph > 4096 )
    return fail( NG_ERR_ARG, "ng_set_graph_slices: bad argument" );
  e->graph_slices = slices_per_graph;
  ++e->generation;
  return NG_OK;
}

int
ng_set_tuning( ng_engine* e, int32_t mode, int32_t update_variant, int32_t deliver_ctas_per_sm,
  int32_t deliver_chunks_per_warp )
{
  if ( !e )
    return fail( NG_ERR_ARG, "null engine" );
  if ( mode < 0 || mode > 2 || update_variant < -1 || update_variant > 6 || update_variant == 4 || deliver_ctas_per_sm < -1
    || deliver_ctas_per_sm == 0 || deliver_chunks_per_warp < -1 || deliver_chunks_per_warp == 0
    || deliver_chunks_per_warp > 32 )
    return fail( NG_ERR_ARG, "ng_set_tuning: mode 0..2, update_variant -1, 0..3, 5 or 6, per-SM CTAs and chunks per warp "
                             "-1 or >= 1" );
  int rc = e->sync_pending();
  if ( rc )
    return rc;
  cudaSetDevice( e->cfg.device );
  e->tune_mode = mode;
  if ( mode == 0 )
  {
    e->upd_variant = update_variant;
    e->deliver_per_sm = deliver_ctas_per_sm > 0 ? std::min( deliver_ctas_per_sm, e->occ_deliver ) : e->occ_deliver;
    e->deliver_group = deliver_chunks_per_warp > 0 ? deliver_chunks_per_warp : 4;
    e->tune_state = 3;
  }
  else
  {
    e->tune_state = 0;  // measured again at the next long enough call
  }
  e->tune_log.clear();
  e->apply_deliver();
  return NG_OK;
}

int
ng_get_tuning( ng_engine* e, ng_tuning* out )
{
  if ( !e || !out )
    return fail( NG_ERR_ARG, "null argument" );
  std::memset( out, 0, sizeof( *out ) );
  out->mode = e->tune_mode == 0 ? 0 : 1;
  out->state = e->tune_state;
  bool iaf = false;
  for ( const auto& b : e->blk )
    iaf = iaf || b.model != NG_AEIF_COND_ALPHA;
  out->update_variant = !iaf ? 4 : e->upd_variant >= 0 ? e->upd_variant : e->engine_default_variant( e->blk[ 0 ].n );
  out->deliver_per_sm = e->deliver_per_sm;
  out->deliver_group = e->deliver_group;
  out->cache_hit = e->tune_state == 2 ? 1 : 0;
  out->rate_bucket = e->rate_bucket;
  out->trial_steps = e->trial_steps;
  const int nc = ( int ) std::min< size_t >( e->tune_log.size(), NG_TUNE_MAX_CANDIDATES );
  out->n_candidates = nc;
  for ( int k = 0; k < nc; ++k )
  {
    const auto& c = e->tune_log[ ( size_t ) k ];
    out->cand_variant[ k ] = iaf ? c.variant : 4;
    out->cand_per_sm[ k ] = c.per_sm;
    out->cand_group[ k ] = c.group;
    out->cand_us_per_slice[ k ] = e->trial_steps > 0 ? c.us * e->cfg.min_delay / ( double ) e->trial_steps : 0.0;
  }
  return NG_OK;
}

int
ng_set_option( ng_engine* e, const char* name, double value )
{
  if ( !e || !name )
    return fail( NG_ERR_ARG, "null argument" );
  int rc = e->sync_pending();
  if ( rc )
    return rc;
  cudaSetDevice( e->cfg.device );
  const std::string nm( name );
  if ( nm == "late_delivery" )
  {
    e->late_env = value != 0.0;
    e->refresh_late();
    ++e->generation;
  }
  else if ( nm == "late_ctas_per_sm" )
  {
    if ( !( value >= 1 ) )
      return fail( NG_ERR_ARG, "late_ctas_per_sm must be >= 1" );
    e->late_per_sm = ( int ) value;
    e->refresh_late();
    ++e->generation;
  }
  else if ( nm == "aeif_binning" )
  {
    e->aeif_binning = value != 0.0;
    ++e->generation;
  }
  else if ( nm == "gather" || nm == "gather_frac" )
  {
    if ( !e->serving )
      return fail( NG_ERR_STATE, "the per-target gather belongs to serving engines in the FP32 form" );
    for ( const auto& nw : e->nets )
      if ( nw.used )
        return fail( NG_ERR_STATE, "the per-target gather is set before any network is admitted" );
    if ( nm == "gather" )
    {
      if ( value != 0.0 && !e->gather_on )
        return fail( NG_ERR_STATE, "this engine has no per-target gather (FP32 serving form, min_delay <= 16)" );
      e->gather_on = e->gather_on && value != 0.0;
    }
    else
    {
      if ( !( value >= 0 ) )
        return fail( NG_ERR_ARG, "gather_frac must be >= 0" );
      e->gather_frac = ( float ) value;
    }
    e->refresh_late();
    ++e->generation;
  }
  else
  {
    return fail( NG_ERR_UNKNOWN_NAME,
      "unknown option: " + nm + " (late_delivery, late_ctas_per_sm, aeif_binning, gather, gather_frac)" );
  }
  return NG_OK;
}

static int
net_check( ng_engine* e, int32_t id )
{
  if ( !e || !e->serving )
    return fail( NG_ERR_STATE, "not a serving engine (ng_config.serving = 0)" );
  if ( id < 0 || id >= ( int32_t ) e->nets.size() || !e->nets[ id ].used )
    return fail( NG_ERR_ARG, "unknown network id" );
  return NG_OK;
}

int
ng_net_add( ng_engine* e, const ng_net_desc* desc, int32_t* net_id )
{
  if ( !e || !desc || !net_id )
    return fail( NG_ERR_ARG, "ng_net_add: null argument" );
  if ( !e->serving )
    return fail( NG_ERR_STATE, "ng_net_add: not a serving engine (ng_config.serving = 0)" );
  if ( e->from != 0 )
    return fail( NG_ERR_STATE, "ng_net_add: networks are admitted at slice boundaries" );
  const int64_t n = desc->n;
  if ( n < 1 || n >= ( 1ll << LOG_ID_SHIFT ) || desc->steps < 0 || desc->n_vars < 0 || ( desc->n_vars > 0 && ( !desc->var_names || !desc->var_values ) ) )
    return fail( NG_ERR_ARG, "ng_net_add: bad network description" );
  const ng_fixed_indegree* fb = desc->build;
  const ng_pairwise_bernoulli* pb = desc->build_pb;
  if ( pb )
  {
    if ( fb || pb->n_pops < 1 || pb->n_pops > NG_MAX_POPS )
      return fail( NG_ERR_ARG, "ng_net_add: bad pairwise_bernoulli description" );
    int64_t tot = 0;
    for ( int j = 0; j < pb->n_pops; ++j )
    {
      if ( pb->pop_size[ j ] < 0 )
        return fail( NG_ERR_ARG, "ng_net_add: negative population size" );
      tot += pb->pop_size[ j ];
      for ( int i = 0; i < pb->n_pops; ++i )
        if ( !( pb->p[ i * NG_MAX_POPS + j ] >= 0.0 && pb->p[ i * NG_MAX_POPS + j ] <= 1.0 ) )
          return fail( NG_ERR_ARG, "ng_net_add: connection probability outside [0, 1]" );
    }
    if ( tot != n )
      return fail( NG_ERR_ARG, "ng_net_add: population sizes do not add up to n" );
  }
  if ( fb && ( fb->n_exc < 0 || fb->n_exc > n || fb->k_exc < 0 || fb->k_inh < 0 || ( fb->k_exc > 0 && fb->n_exc == 0 )
               || ( fb->k_inh > 0 && fb->n_exc == n ) ) )
    return fail( NG_ERR_ARG, "ng_net_add: bad fixed_indegree description" );
  if ( !fb && desc->nnz > 0 && ( !desc->source || !desc->target || !desc->weight || !desc->delay_steps ) )
    return fail( NG_ERR_ARG, "ng_net_add: edges without arrays" );
  cudaSetDevice( e->cfg.device );
  int32_t id = -1;
  for ( size_t k = 0; k < e->nets.size(); ++k )
    if ( !e->nets[ k ].used )
    {
      id = ( int32_t ) k;
      break;
    }
  if ( id < 0 )
    return fail( NG_ERR_CAPACITY, "ng_net_add: no free network slot" );
  // host side of explicit edges: rows padded to multiples of 4
  std::vector< int64_t > prow;
  std::vector< int32_t > rdeg;
  int64_t ne_need;
  if ( pb )
    ne_need = 0;  // known after the counting pass
  else if ( fb )
    ne_need = n * ( int64_t ) ( fb->k_exc + fb->k_inh ) + 3 * n;
  else
  {
    prow.assign( ( size_t ) n + 1, 0 );
    rdeg.assign( ( size_t ) n, 0 );
    for ( int64_t k = 0; k < desc->nnz; ++k )
    {
      if ( desc->source[ k ] < 0 || desc->source[ k ] >= n || desc->target[ k ] < 0 || desc->target[ k ] >= n )
        return fail( NG_ERR_ARG, "ng_net_add: edge endpoint outside the network" );
      ++rdeg[ desc->source[ k ] ];
    }
    for ( int64_t sidx = 0; sidx < n; ++sidx )
      prow[ sidx + 1 ] = prow[ sidx ] + ( ( rdeg[ sidx ] + 3 ) & ~3 );
    ne_need = prow[ n ];
  }
  // the region's preparation runs on the admission stream (every helper
  // below works on e->stream); the engine's stream is restored on every exit
  struct StreamSwap
  {
    ng_engine* e;
    cudaStream_t main;
    ~StreamSwap() { e->stream = main; }
  } swap { e, e->stream };
  e->stream = e->adm_stream;
  int64_t n0 = 0, e0 = 0;
  if ( !ng_engine::take_run( e->free_neurons, n, &n0 ) )
    return fail( NG_ERR_CAPACITY, "ng_net_add: not enough free neurons in the pool" );
  if ( !ng_engine::take_run( e->free_edges, ne_need, &e0 ) )
  {
    ng_engine::give_run( e->free_neurons, n0, n );
    return fail( NG_ERR_CAPACITY, "ng_net_add: not enough free edges in the pool" );
  }
  int64_t g0 = -1, gn = 0;  // gather table run, if any
  int64_t sg0 = -1, sgn = 0;  // segment table run, if any
  auto undo = [ & ]( int code ) {
    cudaStreamSynchronize( e->adm_stream );  // its copies read the pinned staging
    ng_engine::give_run( e->free_neurons, n0, n );
    ng_engine::give_run( e->free_edges, e0, ne_need );
    if ( g0 >= 0 )
      ng_engine::give_run( e->free_gin, g0, gn );
    if ( sg0 >= 0 )
      ng_engine::give_run( e->free_seg, sg0, sgn );
    return code;
  };
  auto& b = e->blk[ 0 ];
  const int model = b.model;
  // parameters (host copies) and state (device) of the region
  std::vector< double > defaults;
  default_params( model, defaults );
  for ( int p2 = 0; p2 < n_params( model ); ++p2 )
    std::fill( b.par[ p2 ].begin() + n0, b.par[ p2 ].begin() + n0 + n, defaults[ p2 ] );
  std::vector< const double* > state_src( MAX_STATE, nullptr );
  for ( int32_t v = 0; v < desc->n_vars; ++v )
  {
    const VarSpec* vs = desc->var_names[ v ] ? find_var( model, desc->var_names[ v ] ) : nullptr;
    if ( !vs || !desc->var_values[ v ] )
      return undo( fail( NG_ERR_UNKNOWN_NAME, std::string( "ng_net_add: unknown variable '" )
                                                + ( desc->var_names[ v ] ? desc->var_names[ v ] : "(null)" ) + "'" ) );
    if ( vs->kind == PARAM )
      std::copy( desc->var_values[ v ], desc->var_values[ v ] + n, b.par[ vs->slot ].begin() + n0 );
    else if ( vs->kind == STATE )
      state_src[ vs->slot ] = desc->var_values[ v ];
  }
  // the per-neuron uploads (state, RKF45 step, drive tables) are staged in
  // the engine's pinned buffer, which stays untouched until the function
  // returns (after its last synchronisation of the admission stream), so no
  // copy waits for the device here: an admission's host work overlaps slices
  // still running on the device
  const size_t n_st = ( size_t ) n_states( model );
  const auto al16 = []( size_t x ) { return ( x + 15 ) & ~( size_t ) 15; };
  const size_t st_bytes = al16( ( size_t ) n * e->rsz );
  const size_t hs_bytes = model == NG_AEIF_COND_ALPHA ? al16( ( size_t ) n * 8 ) : 0;
  const size_t drv_bytes = al16( ( size_t ) n * sizeof( double4 ) ) + al16( ( size_t ) n * 8 )
    + al16( ( size_t ) n * 8 ) + al16( ( size_t ) n * 4 );
  {
    const int rcp = e->grow_adm_pin( n_st * st_bytes + hs_bytes + drv_bytes );
    if ( rcp )
      return undo( rcp );
  }
  char* stage = e->adm_pin;
  {
    for ( size_t sl = 0; sl < n_st; ++sl )
    {
      char* tmp = stage;
      stage += st_bytes;
      for ( int64_t i = 0; i < n; ++i )
      {
        const double v = state_src[ sl ] ? state_src[ sl ][ i ] : default_state( model, ( int ) sl );
        if ( e->rsz == 8 )
          reinterpret_cast< double* >( tmp )[ i ] = v;
        else
          reinterpret_cast< float* >( tmp )[ i ] = ( float ) v;
      }
      CU( cudaMemcpyAsync( ( char* ) b.st[ sl ].p + n0 * e->rsz, tmp, ( size_t ) n * e->rsz, cudaMemcpyHostToDevice,
        e->stream ) );
    }
    CU( cudaMemsetAsync( ( int32_t* ) b.r.p + n0, 0, ( size_t ) n * 4, e->stream ) );
    if ( model == NG_AEIF_COND_ALPHA )
    {
      double* hs = reinterpret_cast< double* >( stage );
      stage += hs_bytes;
      std::fill( hs, hs + n, e->h );
      CU( cudaMemcpyAsync( ( double* ) b.istep.p + n0, hs, ( size_t ) n * 8, cudaMemcpyHostToDevice, e->stream ) );
    }
  }
  // coefficient classes, shared by all networks
  double row[ CT_STRIDE ];
  double log_rate = 0.0;
  const int ri = refr_index( model );
  const int64_t first_new = ( int64_t ) e->cls_ids.size();
  const int np_model = n_params( model );
  for ( int64_t i = n0; i < n0 + n; ++i )
  {
    // a neuron with its predecessor's parameters has its class
    if ( i > n0 )
    {
      bool same = true;
      for ( int p2 = 0; p2 < np_model && same; ++p2 )
        same = b.par[ p2 ][ ( size_t ) i ] == b.par[ p2 ][ ( size_t ) i - 1 ];
      if ( same )
      {
        b.host_cls[ ( size_t ) i ] = b.host_cls[ ( size_t ) i - 1 ];
        log_rate += 1.0 / ( row[ ri ] + 1.0 );
        continue;
      }
    }
    std::fill( row, row + CT_STRIDE, 0.0 );
    int rc = e->coef_row( b, i, row );
    if ( rc )
      return undo( rc );
    std::string key( reinterpret_cast< const char* >( row ), sizeof( row ) );
    auto it = e->cls_ids.find( key );
    int32_t cid;
    if ( it == e->cls_ids.end() )
    {
      cid = ( int32_t ) e->cls_ids.size();
      if ( cid >= e->cls_cap )
        return undo( fail( NG_ERR_CAPACITY, "ng_net_add: coefficient class table full" ) );
      e->cls_ids.emplace( std::move( key ), cid );
      b.host_ctab.insert( b.host_ctab.end(), row, row + CT_STRIDE );
    }
    else
      cid = it->second;
    b.host_cls[ ( size_t ) i ] = cid;
    log_rate += 1.0 / ( row[ ri ] + 1.0 );
  }
  const int64_t n_cls = ( int64_t ) e->cls_ids.size();
  if ( n_cls > first_new )
    CU( cudaMemcpyAsync( ( double* ) b.ctab.p + first_new * CT_STRIDE, b.host_ctab.data() + first_new * CT_STRIDE,
      ( size_t ) ( n_cls - first_new ) * CT_STRIDE * 8, cudaMemcpyHostToDevice, e->stream ) );
  CU( cudaMemcpyAsync( ( int32_t* ) b.cls.p + n0, b.host_cls.data() + n0, ( size_t ) n * 4, cudaMemcpyHostToDevice,
    e->stream ) );
  // edges of the region
  const bool fx = e->prec != NG_FP64;
  const size_t wsz = fx ? 4 : 8;
  if ( ne_need > 0 )
  {
    CU( cudaMemsetAsync( ( uint32_t* ) e->tdc.p + e0, 0, ( size_t ) ne_need * 4, e->stream ) );
    CU( cudaMemsetAsync( ( char* ) e->w.p + e0 * wsz, 0, ( size_t ) ne_need * wsz, e->stream ) );
  }
  auto to_fixed = [ & ]( double wv, int32_t* out ) {
    const double sc = std::ldexp( wv, e->fx_S );
    if ( !( std::fabs( sc ) < 2147483647.0 ) )
      return false;
    *out = ( int32_t ) std::llrint( sc );
    return true;
  };
  int64_t ne_used = ne_need;
  if ( pb )
  {
    PbSpec sp {};
    sp.n_pops = pb->n_pops;
    sp.pop_lo[ 0 ] = 0;
    int nb = 0;
    for ( int j = 0; j < pb->n_pops; ++j )
    {
      sp.pop_lo[ j + 1 ] = sp.pop_lo[ j ] + pb->pop_size[ j ];
      sp.pop_exc[ j ] = pb->pop_exc[ j ];
      nb += ( int ) ( ( pb->pop_size[ j ] + PB_BLOCK - 1 ) / PB_BLOCK );
    }
    for ( int i = 0; i < pb->n_pops; ++i )
      for ( int j = 0; j < pb->n_pops; ++j )
      {
        const double pp = pb->p[ i * NG_MAX_POPS + j ];
        sp.inv_log1mp[ i * PB_MAX_POPS + j ] = pp <= 0.0 ? NAN : pp >= 1.0 ? 0.0 : 1.0 / std::log1p( -pp );
      }
    for ( int k = 0; k < 2; ++k )
    {
      sp.w_mean[ k ] = pb->w_mean[ k ];
      sp.w_sd[ k ] = pb->w_sd[ k ];
      sp.d_mean[ k ] = pb->d_mean_ms[ k ];
      sp.d_sd[ k ] = pb->d_sd_ms[ k ];
    }
    sp.h = e->h;
    sp.min_steps = e->cfg.min_delay;
    sp.max_steps = e->cfg.max_delay;
    sp.d_max = std::min( pb->d_max_ms, e->cfg.max_delay * e->h );
    sp.allow_aut = pb->allow_autapses;
    sp.key0 = ( uint32_t ) pb->seed;
    sp.key1 = ( uint32_t ) ( pb->seed >> 32 );
    sp.nb = nb;
    const int64_t items = n * ( int64_t ) nb;
    int rc;
    if ( ( rc = e->grow_scratch( e->sc_sb, ( size_t ) std::max< int64_t >( items, 1 ) * 4 ) )
      || ( rc = e->grow_scratch( e->sc_cnt, ( size_t ) n * 4 ) ) || ( rc = e->grow_scratch( e->sc_beg, ( size_t ) n * 8 ) )
      || ( rc = e->grow_scratch( e->sc_plen, ( size_t ) n * 4 ) ) || ( rc = e->grow_scratch( e->sc_total, 8 ) ) )
      return undo( rc );
    const unsigned g = ( unsigned ) std::max< int64_t >( 1, ( items + 255 ) / 256 );
    const bool ex_m = sign_channels( model ), ae_m = model == NG_AEIF_COND_ALPHA;
    const double fxs = std::ldexp( 1.0, e->fx_S );
    k_pb_pass< double ><<< g, 256, 0, e->stream >>>( sp, n, false, ( int* ) e->sc_sb.p, nullptr, 0, 0, e->tbits, ex_m,
      ae_m, 1.0, nullptr, nullptr );
    k_pb_rowsum<<< ( unsigned ) ( ( n + 255 ) / 256 ), 256, 0, e->stream >>>( n, nb, ( const int* ) e->sc_sb.p,
      ( int32_t* ) e->sc_cnt.p );
    k_fi_scan<<< 1, 1024, 0, e->stream >>>( n, ( const int32_t* ) e->sc_cnt.p, ( int64_t* ) e->sc_beg.p,
      ( int32_t* ) e->sc_plen.p, ( long long* ) e->sc_total.p );
    long long total = 0;
    CU( cudaMemcpyAsync( &total, e->sc_total.p, 8, cudaMemcpyDeviceToHost, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
    if ( !ng_engine::take_run( e->free_edges, total, &e0 ) )
      return undo( fail( NG_ERR_CAPACITY, "ng_net_add: not enough free edges in the pool" ) );
    ne_need = total;
    ne_used = total;
    CU( cudaMemsetAsync( ( uint32_t* ) e->tdc.p + e0, 0, ( size_t ) total * 4, e->stream ) );
    CU( cudaMemsetAsync( ( char* ) e->w.p + e0 * wsz, 0, ( size_t ) total * wsz, e->stream ) );
    if ( fx )
      k_pb_pass< int32_t ><<< g, 256, 0, e->stream >>>( sp, n, true, ( int* ) e->sc_sb.p, ( const int64_t* ) e->sc_beg.p,
        n0, e0, e->tbits, ex_m, ae_m, fxs, ( uint32_t* ) e->tdc.p, ( int32_t* ) e->w.p );
    else
      k_pb_pass< double ><<< g, 256, 0, e->stream >>>( sp, n, true, ( int* ) e->sc_sb.p, ( const int64_t* ) e->sc_beg.p,
        n0, e0, e->tbits, ex_m, ae_m, 1.0, ( uint32_t* ) e->tdc.p, ( double* ) e->w.p );
    k_fi_rows<<< ( unsigned ) ( ( n + 255 ) / 256 ), 256, 0, e->stream >>>( n, n0, e0, ( const int64_t* ) e->sc_beg.p,
      ( const int32_t* ) e->sc_plen.p, ( const int32_t* ) e->sc_cnt.p, ( int64_t* ) e->row_beg.p,
      ( int32_t* ) e->row_len.p, ( int32_t* ) e->real_deg.p );
    // the rows are sorted by target: segment table of the target-tiled delivery
    if ( e->tiled_on )
    {
      // tiles: about a multiple of the SM count, at most tile_t targets each
      const int64_t rounds = ( n + ( int64_t ) e->tile_t * e->sms - 1 ) / ( ( int64_t ) e->tile_t * e->sms );
      int tt = ( int ) ( ( n + rounds * e->sms - 1 ) / ( rounds * e->sms ) );
      tt = std::min( e->tile_t, ( tt + 31 ) / 32 * 32 );
      const int nt = ( int ) ( ( n + tt - 1 ) / tt );
      const int64_t need = n * ( int64_t ) ( nt + 1 );
      if ( !ng_engine::take_run( e->free_seg, need, &sg0 ) )
        return undo( fail( NG_ERR_CAPACITY, "ng_net_add: not enough free segment-table space (tile_capacity)" ) );
      sgn = need;
      k_seg_build<<< ( unsigned ) ( ( need + 255 ) / 256 ), 256, 0, e->stream >>>( n, nt, tt, n0,
        ( const int64_t* ) e->row_beg.p, ( const int32_t* ) e->real_deg.p, ( const uint32_t* ) e->tdc.p, e->tmask,
        ( int32_t* ) e->seg.p + sg0 );
      TileNet tn {};
      tn.seg_base = sg0;
      tn.off = n0;
      tn.n = ( int ) n;
      tn.nt = nt;
      tn.tt = tt;
      e->host_t[ id ] = tn;
    }
    if ( e->late_possible() )
    {
      int rc3;
      if ( ( rc3 = e->split_rows( n, n0, e0, total ) ) )
        return undo( rc3 );
    }
    CU( cudaGetLastError() );
    CU( cudaStreamSynchronize( e->stream ) );
  }
  else if ( fb )
  {
    const int K = fb->k_exc + fb->k_inh;
    const int64_t nk = n * K;
    if ( fb->delay_steps < e->cfg.min_delay || fb->delay_steps > e->cfg.max_delay )
      return undo( fail( NG_ERR_ARG, "ng_net_add: delay outside [min_delay, max_delay]" ) );
    int rc;
    if ( ( rc = e->grow_scratch( e->sc_src, ( size_t ) std::max< int64_t >( nk, 1 ) * 4 ) )
      || ( rc = e->grow_scratch( e->sc_cnt, ( size_t ) n * 4 ) ) || ( rc = e->grow_scratch( e->sc_fill, ( size_t ) n * 4 ) )
      || ( rc = e->grow_scratch( e->sc_beg, ( size_t ) n * 8 ) ) || ( rc = e->grow_scratch( e->sc_plen, ( size_t ) n * 4 ) )
      || ( rc = e->grow_scratch( e->sc_total, 8 ) ) )
      return undo( rc );
    CU( cudaMemsetAsync( e->sc_cnt.p, 0, ( size_t ) n * 4, e->stream ) );
    CU( cudaMemsetAsync( e->sc_fill.p, 0, ( size_t ) n * 4, e->stream ) );
    const unsigned g = ( unsigned ) std::max< int64_t >( 1, ( nk + 255 ) / 256 );
    if ( nk > 0 )
      k_fi_draw<<< g, 256, 0, e->stream >>>( n, fb->n_exc, fb->k_exc, fb->k_inh, fb->allow_autapses,
        ( uint32_t ) fb->seed, ( uint32_t ) ( fb->seed >> 32 ), ( int32_t* ) e->sc_src.p, ( int32_t* ) e->sc_cnt.p );
    k_fi_scan<<< 1, 1024, 0, e->stream >>>( n, ( const int32_t* ) e->sc_cnt.p, ( int64_t* ) e->sc_beg.p,
      ( int32_t* ) e->sc_plen.p, ( long long* ) e->sc_total.p );
    uint32_t chx, chi;
    double wex, win;
    e->edge_word( fb->w_exc, &chx, &wex );
    e->edge_word( fb->w_inh, &chi, &win );
    const uint32_t dword = ( uint32_t ) fb->delay_steps << e->tbits;
    const uint32_t wordx = dword | ( chx << 31 ), wordi = dword | ( chi << 31 );
    if ( nk > 0 )
    {
      if ( fx )
      {
        int32_t fwx = 0, fwi = 0;
        if ( !to_fixed( wex, &fwx ) || !to_fixed( win, &fwi ) )
          return undo( fail( NG_ERR_ARG, "ng_net_add: weight above the engine's max_abs_weight" ) );
        k_fi_scatter< int32_t ><<< g, 256, 0, e->stream >>>( n, fb->k_exc, fb->k_inh, ( const int32_t* ) e->sc_src.p,
          ( const int64_t* ) e->sc_beg.p, ( int32_t* ) e->sc_fill.p, n0, e0, wordx, wordi, fwx, fwi,
          ( uint32_t* ) e->tdc.p, ( int32_t* ) e->w.p );
      }
      else
      {
        k_fi_scatter< double ><<< g, 256, 0, e->stream >>>( n, fb->k_exc, fb->k_inh, ( const int32_t* ) e->sc_src.p,
          ( const int64_t* ) e->sc_beg.p, ( int32_t* ) e->sc_fill.p, n0, e0, wordx, wordi, wex, win,
          ( uint32_t* ) e->tdc.p, ( double* ) e->w.p );
      }
    }
    k_fi_rows<<< ( unsigned ) ( ( n + 255 ) / 256 ), 256, 0, e->stream >>>( n, n0, e0, ( const int64_t* ) e->sc_beg.p,
      ( const int32_t* ) e->sc_plen.p, ( const int32_t* ) e->sc_cnt.p, ( int64_t* ) e->row_beg.p,
      ( int32_t* ) e->row_len.p, ( int32_t* ) e->real_deg.p );
    // one delay: every row is of one delay class
    k_row_uniform<<< ( unsigned ) ( ( n + 255 ) / 256 ), 256, 0, e->stream >>>( n, n0, ( const int32_t* ) e->row_len.p,
      fb->delay_steps < e->late_thr() ? 1 : 0, ( int32_t* ) e->row_ue.p, ( int32_t* ) e->row_ls.p );
    // the in-edge table of the per-target gather (16-bit local ids)
    const int64_t g_need = ( ( n + 31 ) / 32 * 32 ) * ( int64_t ) ( ( K + 7 ) / 8 * 8 );
    if ( e->gather_on && fx && nk > 0 && n <= G_MAX_N && K <= G_MAX_K
      && ng_engine::take_run( e->free_gin, g_need, &g0 ) )
    {
      gn = g_need;
      k_fill_u16<<< ( unsigned ) ( ( g_need + 255 ) / 256 ), 256, 0, e->stream >>>( ( uint16_t* ) e->gin.p + g0, g_need,
        ( uint16_t ) n );
      k_fi_gtab<<< g, 256, 0, e->stream >>>( n, K, ( const int32_t* ) e->sc_src.p, ( uint16_t* ) e->gin.p + g0 );
      GatherNet gt {};
      gt.base = g0;
      gt.off = n0;
      gt.n = ( int ) n;
      gt.ke = fb->k_exc;
      gt.ki = fb->k_inh;
      gt.d = fb->delay_steps;
      to_fixed( wex, &gt.we );
      to_fixed( win, &gt.wi );
      gt.ce = ( int ) chx;
      gt.ci = ( int ) chi;
      e->host_g[ id ] = gt;
    }
    CU( cudaGetLastError() );
    long long total = 0;
    CU( cudaMemcpyAsync( &total, e->sc_total.p, 8, cudaMemcpyDeviceToHost, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
    ne_used = total;
  }
  else
  {
    const int64_t np = prow[ n ];
    // each row: its edges of delay below the late-delivery threshold first
    const int32_t thr = e->late_thr();
    std::vector< int32_t > nu( ( size_t ) n, 0 );
    for ( int64_t k = 0; k < desc->nnz; ++k )
      if ( desc->delay_steps[ k ] < thr )
        ++nu[ desc->source[ k ] ];
    std::vector< int64_t > pos( prow.begin(), prow.end() - 1 ), pos_l( ( size_t ) n );
    std::vector< int32_t > ue( ( size_t ) n ), ls( ( size_t ) n );
    for ( int64_t sidx = 0; sidx < n; ++sidx )
    {
      pos_l[ sidx ] = prow[ sidx ] + nu[ sidx ];
      row_ranges( nu[ sidx ], rdeg[ sidx ], ( int ) ( prow[ sidx + 1 ] - prow[ sidx ] ), ue[ sidx ], ls[ sidx ] );
    }
    std::vector< uint32_t > tw( ( size_t ) std::max< int64_t >( np, 1 ), 0u );
    std::vector< double > wd( fx ? 0 : ( size_t ) std::max< int64_t >( np, 1 ), 0.0 );
    std::vector< int32_t > wi( fx ? ( size_t ) std::max< int64_t >( np, 1 ) : 0, 0 );
    for ( int64_t k = 0; k < desc->nnz; ++k )
    {
      const int32_t d = desc->delay_steps[ k ];
      if ( d < e->cfg.min_delay || d > e->cfg.max_delay )
        return undo( fail( NG_ERR_ARG, "ng_net_add: delay outside [min_delay, max_delay]" ) );
      uint32_t ch;
      double we;
      e->edge_word( desc->weight[ k ], &ch, &we );
      const int64_t j = d < thr ? pos[ desc->source[ k ] ]++ : pos_l[ desc->source[ k ] ]++;
      tw[ j ] = ( uint32_t ) ( n0 + desc->target[ k ] ) | ( ( uint32_t ) d << e->tbits ) | ( ch << 31 );
      if ( fx )
      {
        if ( !to_fixed( we, &wi[ j ] ) )
          return undo( fail( NG_ERR_ARG, "ng_net_add: weight above the engine's max_abs_weight" ) );
      }
      else
        wd[ j ] = we;
    }
    if ( np > 0 )
    {
      CU( cudaMemcpyAsync( ( uint32_t* ) e->tdc.p + e0, tw.data(), ( size_t ) np * 4, cudaMemcpyHostToDevice, e->stream ) );
      if ( fx )
        CU( cudaMemcpyAsync( ( int32_t* ) e->w.p + e0, wi.data(), ( size_t ) np * 4, cudaMemcpyHostToDevice, e->stream ) );
      else
        CU( cudaMemcpyAsync( ( double* ) e->w.p + e0, wd.data(), ( size_t ) np * 8, cudaMemcpyHostToDevice, e->stream ) );
    }
    std::vector< int64_t > beg( ( size_t ) n );
    std::vector< int32_t > plen( ( size_t ) n );
    for ( int64_t sidx = 0; sidx < n; ++sidx )
    {
      beg[ sidx ] = e0 + prow[ sidx ];
      plen[ sidx ] = ( int32_t ) ( prow[ sidx + 1 ] - prow[ sidx ] );
    }
    CU( cudaMemcpyAsync( ( int64_t* ) e->row_beg.p + n0, beg.data(), ( size_t ) n * 8, cudaMemcpyHostToDevice, e->stream ) );
    CU( cudaMemcpyAsync( ( int32_t* ) e->row_len.p + n0, plen.data(), ( size_t ) n * 4, cudaMemcpyHostToDevice, e->stream ) );
    CU( cudaMemcpyAsync( ( int32_t* ) e->real_deg.p + n0, rdeg.data(), ( size_t ) n * 4, cudaMemcpyHostToDevice,
      e->stream ) );
    CU( cudaMemcpyAsync( ( int32_t* ) e->row_ue.p + n0, ue.data(), ( size_t ) n * 4, cudaMemcpyHostToDevice, e->stream ) );
    CU( cudaMemcpyAsync( ( int32_t* ) e->row_ls.p + n0, ls.data(), ( size_t ) n * 4, cudaMemcpyHostToDevice, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
  }
  // 32-bit rings: no ring cell of this network may exceed 31 bits
  if ( e->ring_bytes == 4 && ne_used > 0 )
  {
    int rc2;
    if ( ( rc2 = e->grow_scratch( e->sc_bound, ( size_t ) n * 8 + 8 ) ) )
      return undo( rc2 );
    CU( cudaMemsetAsync( e->sc_bound.p, 0, ( size_t ) n * 8 + 8, e->stream ) );
    unsigned long long* sums = ( unsigned long long* ) e->sc_bound.p;
    const unsigned gg = ( unsigned ) std::min< int64_t >( ( ne_used + 255 ) / 256, ( int64_t ) e->sms * 16 );
    k_in_abs_sum<<< gg, 256, 0, e->stream >>>( e0, ne_used, ( const uint32_t* ) e->tdc.p, ( const int32_t* ) e->w.p,
      e->tmask, n0, sums );
    k_max_u64<<< ( unsigned ) std::min< int64_t >( ( n + 255 ) / 256, ( int64_t ) e->sms * 4 ), 256, 0, e->stream >>>(
      n, sums, sums + n );
    CU( cudaGetLastError() );
    unsigned long long mx = 0;
    CU( cudaMemcpyAsync( &mx, sums + n, 8, cudaMemcpyDeviceToHost, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
    if ( mx > 2147483647ull )
      return undo( fail( NG_ERR_ARG, "ng_net_add: the network's in-edge weight sum exceeds the engine's ring_bound "
                                     "(32-bit ring cells could overflow)" ) );
  }
  // give back the unused tail of the edge reservation
  if ( ne_used < ne_need )
    ng_engine::give_run( e->free_edges, e0 + ne_used, ne_need - ne_used );
  // drive: Poisson tables and CDF references of the region
  {
    double4* tab = reinterpret_cast< double4* >( stage );
    stage += al16( ( size_t ) n * sizeof( double4 ) );
    int2* ref = reinterpret_cast< int2* >( stage );
    stage += al16( ( size_t ) n * 8 );
    double* pw = reinterpret_cast< double* >( stage );
    stage += al16( ( size_t ) n * 8 );
    int32_t* pd = reinterpret_cast< int32_t* >( stage );
    std::fill( ref, ref + n, make_int2( 0, 0 ) );
    std::fill( pw, pw + n, 0.0 );
    std::fill( pd, pd + n, e->cfg.min_delay );
    const int64_t cdf_old = ( int64_t ) e->cdf_host.size();
    for ( int64_t i = 0; i < n; ++i )
    {
      const double rate = desc->poisson_rate ? desc->poisson_rate[ i ] : 0.0;
      // a neuron with its predecessor's drive has its entries
      if ( i > 0 && desc->poisson_rate && rate == desc->poisson_rate[ i - 1 ]
        && ( !desc->poisson_weight || desc->poisson_weight[ i ] == desc->poisson_weight[ i - 1 ] )
        && ( !desc->poisson_delay || desc->poisson_delay[ i ] == desc->poisson_delay[ i - 1 ] ) )
      {
        tab[ i ] = tab[ i - 1 ];
        ref[ i ] = ref[ i - 1 ];
        pw[ i ] = pw[ i - 1 ];
        pd[ i ] = pd[ i - 1 ];
        continue;
      }
      const double lam = rate > 0 ? e->h * rate * 1e-3 : 0.0;
      tab[ i ] = poisson_table( lam );
      if ( !( lam > 0 ) )
        continue;
      pw[ i ] = desc->poisson_weight ? desc->poisson_weight[ i ] : 0.0;
      pd[ i ] = desc->poisson_delay ? desc->poisson_delay[ i ] : e->cfg.min_delay;
      if ( pd[ i ] < e->cfg.min_delay || pd[ i ] > e->cfg.max_delay )
        return undo( fail( NG_ERR_ARG, "ng_net_add: Poisson delay outside [min_delay, max_delay]" ) );
      auto it = e->cdf_tables.find( lam );
      if ( it == e->cdf_tables.end() )
      {
        int2 r2 = make_int2( ( int ) e->cdf_host.size(), -1 );
        std::vector< uint64_t > t2;
        if ( poisson_cdf_table( lam, t2 ) )
        {
          if ( ( int64_t ) ( e->cdf_host.size() + t2.size() ) > e->cdf_cap )
            return undo( fail( NG_ERR_CAPACITY, "ng_net_add: Poisson table pool full" ) );
          r2.y = ( int ) t2.size();
          e->cdf_host.insert( e->cdf_host.end(), t2.begin(), t2.end() );
        }
        it = e->cdf_tables.emplace( lam, r2 ).first;
      }
      ref[ i ] = it->second;
    }
    const int64_t cdf_new = ( int64_t ) e->cdf_host.size();
    if ( cdf_new > cdf_old )
      CU( cudaMemcpyAsync( ( uint64_t* ) e->pois_cdf.p + cdf_old, e->cdf_host.data() + cdf_old,
        ( size_t ) ( cdf_new - cdf_old ) * 8, cudaMemcpyHostToDevice, e->stream ) );
    CU( cudaMemcpyAsync( ( double4* ) e->pois.p + n0, tab, ( size_t ) n * sizeof( double4 ), cudaMemcpyHostToDevice,
      e->stream ) );
    CU( cudaMemcpyAsync( ( int2* ) e->pois_ref.p + n0, ref, ( size_t ) n * 8, cudaMemcpyHostToDevice, e->stream ) );
    CU( cudaMemcpyAsync( ( double* ) e->pois_w.p + n0, pw, ( size_t ) n * 8, cudaMemcpyHostToDevice, e->stream ) );
    CU( cudaMemcpyAsync( ( int32_t* ) e->pois_d.p + n0, pd, ( size_t ) n * 4, cudaMemcpyHostToDevice, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
  }
  // activation, in the engine's stream order behind the prepared region and
  // the slices already enqueued: recording, network table, ids, a clean ring
  // region (no host memory is read by these, so nothing waits here)
  CU( cudaEventRecord( e->ev_adm, e->adm_stream ) );
  e->stream = swap.main;
  CU( cudaStreamWaitEvent( e->stream, e->ev_adm, 0 ) );
  CU( cudaMemsetAsync( ( uint8_t* ) e->rec.p + n0, desc->record ? 1 : 0, ( size_t ) n, e->stream ) );
  std::fill( e->rec_host.begin() + n0, e->rec_host.begin() + n0 + n, ( uint8_t ) ( desc->record ? 1 : 0 ) );
  const long long step0 = e->origin, until = e->origin + desc->steps, off = n0;
  const uint2 key = make_uint2( ( uint32_t ) desc->seed, ( uint32_t ) ( desc->seed >> 32 ) );
  if ( e->gather_on && g0 < 0 )
    e->host_g[ id ] = GatherNet {};
  if ( e->tiled_on && sg0 < 0 )
    e->host_t[ id ] = TileNet {};
  k_net_set<<< 1, 32, 0, e->stream >>>( id, 1, step0, until, off, key, ( long long* ) e->d_step0.p,
    ( long long* ) e->d_until.p, ( long long* ) e->d_off.p, ( uint2* ) e->d_key.p,
    e->gather_on ? e->host_g[ id ] : GatherNet {}, e->gather_on ? ( GatherNet* ) e->net_g.p : nullptr,
    ( int* ) e->net_mode.p, ( unsigned* ) e->net_spk.p, e->tiled_on ? e->host_t[ id ] : TileNet {},
    e->tiled_on ? ( TileNet* ) e->net_t.p : nullptr );
  k_fill_i32<<< ( unsigned ) ( ( n + 255 ) / 256 ), 256, 0, e->stream >>>( ( int32_t* ) e->d_nid.p + n0, n, id );
  CU( cudaMemset2DAsync( ( char* ) e->ring.p + n0 * e->ring_bytes, ( size_t ) e->N * e->ring_bytes, 0,
    ( size_t ) n * e->ring_bytes, ( size_t ) e->L * e->C,
    e->stream ) );
  CU( cudaGetLastError() );
  std::fill( e->nid_host.begin() + n0, e->nid_host.begin() + n0 + n, id );
  auto& nw = e->nets[ id ];
  nw = ng_engine::NetInfo();
  nw.used = true;
  nw.off = n0;
  nw.n = n;
  nw.e0 = e0;
  nw.ne = ne_used;
  nw.g0 = g0;
  nw.gn = gn;
  nw.s0 = sg0;
  nw.sn = sgn;
  nw.step0 = step0;
  nw.until = until;
  nw.rec = desc->record != 0;
  nw.log_rate = desc->record ? log_rate : 0.0;
  e->n_rec += desc->record ? n : 0;
  e->log_per_step = std::max( 1.0, e->log_per_step + nw.log_rate );
  e->refresh_late();
  *net_id = id;
  return NG_OK;
}

int
ng_net_poll( ng_engine* e, int32_t id, int64_t* steps_done, int32_t* finished )
{
  int rc = net_check( e, id );
  if ( rc )
    return rc;
  const auto& nw = e->nets[ id ];
  const int64_t clock = e->origin + e->from;
  if ( steps_done )
    *steps_done = std::min( clock, nw.until ) - nw.step0;
  if ( finished )
    *finished = clock >= nw.until ? 1 : 0;
  return NG_OK;
}

int
ng_net_spikes( ng_engine* e, int32_t id, int32_t* source, int64_t* stamp, int64_t cap, int64_t* n_out )
{
  int rc = net_check( e, id );
  if ( rc )
    return rc;
  if ( !n_out || cap < 0 || ( source && !stamp ) )
    return fail( NG_ERR_ARG, "ng_net_spikes: bad argument" );
  auto& nw = e->nets[ id ];
  if ( e->og_sel >= 0 || nw.until > e->pend_gi.clock )
    SETTLE( e );  // the running group may hold spikes of this network
  if ( !source )
  {
    *n_out = nw.held;  // count only
    return NG_OK;
  }
  const uint32_t lmask = ( 1u << LOG_ID_SHIFT ) - 1u;
  if ( cap >= nw.held && nw.held >= ( 1 << 18 ) )
  {
    // the whole store, large: decoded by several host threads, each a share
    // of every block (entries of multiplicity 1 land at their own index)
    bool unit = true;
    for ( size_t q = 0; q < nw.blocks.size() && unit; ++q )
      unit = nw.blocks[ q ].m == nw.blocks[ q ].n;
    if ( unit )
    {
      const int T = ( int ) std::max( 1u, std::min( 8u, std::thread::hardware_concurrency() ) );
      std::vector< int64_t > base( nw.blocks.size() + 1, 0 );
      for ( size_t q = 0; q < nw.blocks.size(); ++q )
        base[ q + 1 ] = base[ q ] + nw.blocks[ q ].n - ( q == 0 ? nw.first : 0 );
      auto work = [ & ]( int t ) {
        for ( size_t q = 0; q < nw.blocks.size(); ++q )
        {
          const ng_engine::RawBlock& rb = nw.blocks[ q ];
          const int64_t f = q == 0 ? nw.first : 0, cnt = rb.n - f;
          const int64_t lo = f + cnt * t / T, hi = f + cnt * ( t + 1 ) / T;
          const int64_t sh = rb.clock - nw.step0;
          int32_t* so = source + base[ q ] - f;
          int64_t* to = stamp + base[ q ] - f;
          for ( int64_t j = lo; j < hi; ++j )
          {
            const uint2 en = rb.e[ j ];
            so[ j ] = ( int32_t ) ( en.x & lmask );
            to[ j ] = sh + ( int64_t ) ( en.y & 0xFFFFFFu );
          }
        }
      };
      std::vector< std::thread > pool;
      int started = 1;
      try
      {
        for ( ; started < T; ++started )
          pool.emplace_back( work, started );
      }
      catch ( ... )
      {
        // no more threads: this one takes the remaining shares
      }
      work( 0 );
      for ( int t = started; t < T; ++t )
        work( t );
      for ( auto& th : pool )
        th.join();
      const int64_t k = base.back();
      ng_engine::free_blocks( nw.blocks );
      nw.first = 0;
      nw.held -= k;
      *n_out = k;
      return NG_OK;
    }
  }
  int64_t k = 0;
  size_t bi = 0;
  for ( ; bi < nw.blocks.size(); ++bi )
  {
    const ng_engine::RawBlock& rb = nw.blocks[ bi ];
    int64_t q = bi == 0 ? nw.first : 0;
    for ( ; q < rb.n; ++q )
    {
      const uint2 en = rb.e[ q ];
      const uint32_t m = en.y >> 24;
      if ( k + m > cap )
        break;
      const int32_t src = ( int32_t ) ( en.x & lmask );
      const int64_t st = rb.clock + ( int64_t ) ( en.y & 0xFFFFFFu ) - nw.step0;
      for ( uint32_t r = 0; r < m; ++r, ++k )
      {
        source[ k ] = src;
        stamp[ k ] = st;
      }
    }
    if ( q < rb.n )
    {
      // cap reached inside this block: it stays first
      nw.first = q;
      break;
    }
    nw.first = 0;
  }
  for ( size_t q = 0; q < bi; ++q )
    std::free( nw.blocks[ q ].e );
  nw.blocks.erase( nw.blocks.begin(), nw.blocks.begin() + ( std::ptrdiff_t ) bi );
  nw.held -= k;
  *n_out = k;
  return NG_OK;
}

int
ng_net_get_var( ng_engine* e, int32_t id, const char* name, double* out )
{
  int rc = net_check( e, id );
  if ( rc )
    return rc;
  const auto& nw = e->nets[ id ];
  return ng_get_var( e, 0, name, out, nw.off, nw.n );
}

int
ng_net_get_connections( ng_engine* e, int32_t id, int32_t* source, int32_t* target, double* weight,
  int32_t* delay_steps, int64_t cap, int64_t* n_out )
{
  SETTLE( e );
  int rc = net_check( e, id );
  if ( rc )
    return rc;
  if ( !n_out || cap < 0 || ( cap > 0 && ( !source || !target || !weight || !delay_steps ) ) )
    return fail( NG_ERR_ARG, "ng_net_get_connections: bad argument" );
  cudaSetDevice( e->cfg.device );
  const auto& nw = e->nets[ id ];
  std::vector< int64_t > beg( ( size_t ) nw.n );
  std::vector< int32_t > deg( ( size_t ) nw.n );
  CU( cudaMemcpyAsync( beg.data(), ( int64_t* ) e->row_beg.p + nw.off, ( size_t ) nw.n * 8, cudaMemcpyDeviceToHost,
    e->stream ) );
  CU( cudaMemcpyAsync( deg.data(), ( int32_t* ) e->real_deg.p + nw.off, ( size_t ) nw.n * 4, cudaMemcpyDeviceToHost,
    e->stream ) );
  CU( cudaStreamSynchronize( e->stream ) );
  int64_t total = 0;
  for ( int32_t d : deg )
    total += d;
  *n_out = total;
  if ( !source )
    return NG_OK;  // count only
  if ( cap < total )
    return fail( NG_ERR_ARG, "ng_net_get_connections: output smaller than the network's connection count" );
  const bool fx = e->prec != NG_FP64;
  std::vector< uint32_t > tw( ( size_t ) std::max< int64_t >( nw.ne, 1 ) );
  std::vector< char > wb( ( size_t ) std::max< int64_t >( nw.ne, 1 ) * ( fx ? 4 : 8 ) );
  if ( nw.ne > 0 )
  {
    CU( cudaMemcpyAsync( tw.data(), ( uint32_t* ) e->tdc.p + nw.e0, ( size_t ) nw.ne * 4, cudaMemcpyDeviceToHost,
      e->stream ) );
    CU( cudaMemcpyAsync( wb.data(), ( char* ) e->w.p + nw.e0 * ( fx ? 4 : 8 ), ( size_t ) nw.ne * ( fx ? 4 : 8 ),
      cudaMemcpyDeviceToHost, e->stream ) );
    CU( cudaStreamSynchronize( e->stream ) );
  }
  const bool aeif = e->blk[ 0 ].model == NG_AEIF_COND_ALPHA;
  const double inv_fx = std::ldexp( 1.0, -e->fx_S );
  int64_t k = 0;
  for ( int64_t s2 = 0; s2 < nw.n; ++s2 )
    for ( int32_t j = 0; j < deg[ s2 ]; ++j, ++k )
    {
      const int64_t q = beg[ s2 ] - nw.e0 + j;
      const uint32_t word = tw[ ( size_t ) q ];
      double wv = fx ? reinterpret_cast< const int32_t* >( wb.data() )[ q ] * inv_fx
                     : reinterpret_cast< const double* >( wb.data() )[ q ];
      if ( aeif && ( word >> 31 ) )
        wv = -wv;
      source[ k ] = ( int32_t ) s2;
      target[ k ] = ( int32_t ) ( ( int64_t ) ( word & e->tmask ) - nw.off );
      delay_steps[ k ] = ( int32_t ) ( ( word >> e->tbits ) & e->dmask );
      weight[ k ] = wv;
    }
  return NG_OK;
}

int
ng_net_remove( ng_engine* e, int32_t id )
{
  int rc = net_check( e, id );
  if ( rc )
    return rc;
  if ( e->og_sel >= 0 || e->nets[ id ].until > e->pend_gi.clock )
    SETTLE( e );  // the running group may hold spikes of this network
  cudaSetDevice( e->cfg.device );
  auto& nw = e->nets[ id ];
  // in stream order behind the slices already enqueued; nothing waits here.
  // The region's rows and state are left as they are (a free neuron never
  // spikes nor updates), so an admission may prepare the region again on
  // its own stream while these are still queued.
  k_fill_i32<<< ( unsigned ) ( ( nw.n + 255 ) / 256 ), 256, 0, e->stream >>>( ( int32_t* ) e->d_nid.p + nw.off, nw.n, -1 );
  CU( cudaMemsetAsync( ( uint8_t* ) e->rec.p + nw.off, 0, ( size_t ) nw.n, e->stream ) );
  k_net_set<<< 1, 32, 0, e->stream >>>( id, 0, 0, 0, 0, make_uint2( 0u, 0u ), nullptr, nullptr, nullptr, nullptr,
    GatherNet {}, e->gather_on ? ( GatherNet* ) e->net_g.p : nullptr, ( int* ) e->net_mode.p,
    ( unsigned* ) e->net_spk.p, TileNet {}, e->tiled_on ? ( TileNet* ) e->net_t.p : nullptr );
  CU( cudaGetLastError() );
  std::fill( e->nid_host.begin() + nw.off, e->nid_host.begin() + nw.off + nw.n, -1 );
  std::fill( e->rec_host.begin() + nw.off, e->rec_host.begin() + nw.off + nw.n, ( uint8_t ) 0 );
  ng_engine::give_run( e->free_neurons, nw.off, nw.n );
  ng_engine::give_run( e->free_edges, nw.e0, nw.ne );
  if ( e->tiled_on )
  {
    if ( nw.s0 >= 0 )
      ng_engine::give_run( e->free_seg, nw.s0, nw.sn );
    e->host_t[ id ] = TileNet {};
  }
  if ( e->gather_on )
  {
    if ( nw.g0 >= 0 )
      ng_engine::give_run( e->free_gin, nw.g0, nw.gn );
    e->host_g[ id ] = GatherNet {};
  }
  e->n_rec -= nw.rec ? nw.n : 0;
  e->log_per_step = std::max( 1.0, e->log_per_step - nw.log_rate );
  ng_engine::free_blocks( nw.blocks );
  nw = ng_engine::NetInfo();
  e->refresh_late();
  return NG_OK;
}

int
ng_net_capacity( ng_engine* e, int64_t* free_neurons, int64_t* free_edges )
{
  if ( !e || !e->serving || !free_neurons || !free_edges )
    return fail( NG_ERR_STATE, "ng_net_capacity: not a serving engine" );
  int64_t a = 0, b2 = 0;
  for ( auto& kv : e->free_neurons )
    a = std::max( a, kv.second );
  for ( auto& kv : e->free_edges )
    b2 = std::max( b2, kv.second );
  *free_neurons = a;
  *free_edges = b2;
  return NG_OK;
}

int
ng_debug_coefficients( ng_engine* e, int32_t block, int64_t index, double* out, int32_t cap, int32_t* n_out )
{
  SETTLE( e );
  int rc = check_range( e, block, index, 1 );
  if ( rc )
    return rc;
  auto& b = e->blk[ block ];
  if ( b.dirty && ( rc = e->build_classes( b ) ) )
    return rc;
  const double* row = b.host_ctab.data() + ( size_t ) b.host_cls[ ( size_t ) index ] * CT_STRIDE;
  std::vector< double > v;
  if ( b.model == NG_IAF_PSC_DELTA )
    v = { row[ 0 ], row[ 1 ], row[ 5 ] };
  else if ( b.model == NG_IAF_PSC_EXP )
    v = { row[ 4 ], row[ 5 ], row[ 0 ], row[ 1 ], row[ 2 ], row[ 3 ], row[ 8 ] };
  else if ( b.model == NG_IAF_PSC_ALPHA )
    v = { row[ 0 ], row[ 1 ], row[ 2 ], row[ 3 ], row[ 4 ], row[ 5 ], row[ 6 ], row[ 7 ], row[ 8 ], row[ 9 ], row[ 10 ],
      row[ 11 ], row[ 15 ] };
  else
    v = { row[ 15 ], row[ 16 ], row[ 17 ], row[ 18 ] };
  const int32_t k = std::min< int32_t >( cap, ( int32_t ) v.size() );
  std::copy( v.begin(), v.begin() + k, out );
  *n_out = k;
  return NG_OK;
}

}  // extern "C"
