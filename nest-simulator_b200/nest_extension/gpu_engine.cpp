/*
 * gpu_engine.cpp -- the engine node of the NEST extension module (see
 * gpu_engine.h for what it does and what it supports).
 */
#include "gpu_engine.h"

#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <stdexcept>

#include "connection_id.h"
#include "connection_manager.h"
#include "exceptions.h"
#include "kernel_manager.h"
#include "model_manager.h"
#include "mpi_manager.h"
#include "node_collection.h"
#include "node_manager.h"
#include "simulation_manager.h"
#include "vp_manager.h"

#include "ng_errors.h"

namespace nestgpu
{

namespace
{

// the engine's status code as the reference's exception
void
check( int status, const std::string& where, const std::string& model = "gpu_engine" )
{
  const ErrorKind k = error_kind( status );
  if ( k == ErrorKind::none )
    return;
  const std::string msg = where + ": " + ng_last_error();
  switch ( k )
  {
  case ErrorKind::bad_property:
    throw nest::BadProperty( msg );
  case ErrorKind::numerical_instability:
    throw nest::NumericalInstability( model );
  default:
    throw nest::KernelException( msg );
  }
}

double
get_d( const Dictionary& d, const std::string& key )
{
  return d.get< double >( key );
}

// the engine's variable names and how they come from a neuron's status
// (relative voltages: models/iaf_psc_delta.cpp:94-200, iaf_psc_exp.cpp keep
// V_m, V_th, V_reset, V_min relative to E_L)
struct Var
{
  const char* engine;
  const char* status;
  bool relative;  // status value minus E_L
};

const std::vector< Var >&
vars_of( int model )
{
  static const std::vector< Var > delta = { { "tau_m", "tau_m", false }, { "C_m", "C_m", false },
    { "t_ref", "t_ref", false }, { "I_e", "I_e", false }, { "V_th_rel", "V_th", true },
    { "V_reset_rel", "V_reset", true }, { "V_min_rel", "V_min", true }, { "V_m_rel", "V_m", true },
    { "tau_minus", "tau_minus", false } };
  // (the synaptic currents are not in the iaf models' status; the engine
  // takes the population over at time 0, where they are 0)
  static const std::vector< Var > exp = { { "tau_m", "tau_m", false }, { "C_m", "C_m", false },
    { "t_ref", "t_ref", false }, { "I_e", "I_e", false }, { "V_th_rel", "V_th", true },
    { "V_reset_rel", "V_reset", true }, { "tau_syn_ex", "tau_syn_ex", false },
    { "tau_syn_in", "tau_syn_in", false }, { "V_m_rel", "V_m", true }, { "tau_minus", "tau_minus", false } };
  static const std::vector< Var > alpha = { { "tau_m", "tau_m", false }, { "C_m", "C_m", false },
    { "t_ref", "t_ref", false }, { "I_e", "I_e", false }, { "V_th_rel", "V_th", true },
    { "V_reset_rel", "V_reset", true }, { "V_min_rel", "V_min", true }, { "tau_syn_ex", "tau_syn_ex", false },
    { "tau_syn_in", "tau_syn_in", false }, { "V_m_rel", "V_m", true }, { "tau_minus", "tau_minus", false } };
  static const std::vector< Var > aeif = { { "V_peak", "V_peak", false }, { "V_reset", "V_reset", false },
    { "t_ref", "t_ref", false }, { "g_L", "g_L", false }, { "C_m", "C_m", false }, { "E_ex", "E_ex", false },
    { "E_in", "E_in", false }, { "E_L", "E_L", false }, { "Delta_T", "Delta_T", false },
    { "tau_w", "tau_w", false }, { "a", "a", false }, { "b", "b", false }, { "V_th", "V_th", false },
    { "tau_syn_ex", "tau_syn_ex", false }, { "tau_syn_in", "tau_syn_in", false }, { "I_e", "I_e", false },
    { "gsl_error_tol", "gsl_error_tol", false }, { "V_m", "V_m", false }, { "g_ex", "g_ex", false },
    { "g_in", "g_in", false }, { "w", "w", false } };
  return model == NG_IAF_PSC_DELTA ? delta
    : model == NG_IAF_PSC_EXP       ? exp
    : model == NG_IAF_PSC_ALPHA     ? alpha
                                    : aeif;
}

// state variables written back to the neurons after a Run
const std::vector< Var >&
state_of( int model )
{
  static const std::vector< Var > delta = { { "V_m_rel", "V_m", true } };
  static const std::vector< Var > exp = { { "V_m_rel", "V_m", true } };
  static const std::vector< Var > aeif = { { "V_m", "V_m", false }, { "g_ex", "g_ex", false },
    { "g_in", "g_in", false }, { "w", "w", false } };
  if ( model == NG_IAF_PSC_ALPHA )
    return exp;
  return model == NG_IAF_PSC_DELTA ? delta : model == NG_IAF_PSC_EXP ? exp : aeif;
}

int
model_id( const std::string& name )
{
  if ( name == "iaf_psc_delta" )
    return NG_IAF_PSC_DELTA;
  if ( name == "iaf_psc_exp" )
    return NG_IAF_PSC_EXP;
  if ( name == "iaf_psc_alpha" )
    return NG_IAF_PSC_ALPHA;
  if ( name == "aeif_cond_alpha" )
    return NG_AEIF_COND_ALPHA;
  return -1;
}

// stdp_pl_synapse_hom (models/stdp_pl_synapse_hom.h) and its copies: a
// connection model whose defaults hold its common properties lambda, alpha,
// mu and tau_plus (STDPPLHomCommonProperties::get_status,
// models/stdp_pl_synapse_hom.cpp:55-63) and none of the other STDP rules' keys
bool
is_stdp_pl( const std::string& name, const Dictionary& defaults )
{
  if ( name == "stdp_pl_synapse_hom" || name == "stdp_pl_synapse_hom_hpc" )
    return true;
  return defaults.known( "lambda" ) and defaults.known( "alpha" ) and defaults.known( "mu" )
    and defaults.known( "tau_plus" ) and not defaults.known( "mu_plus" ) and not defaults.known( "Wmax" );
}

}  // namespace

gpu_engine::gpu_engine()
  : nest::Node()
{
}

gpu_engine::gpu_engine( const gpu_engine& n )
  : nest::Node( n )
  , P_( n.P_ )
{
}

gpu_engine::~gpu_engine()
{
  release_();
}

void
gpu_engine::release_()
{
  if ( eng_ )
  {
    ng_destroy( eng_ );
    eng_ = nullptr;
  }
}

void
gpu_engine::init_buffers_()
{
}

void
gpu_engine::get_status( Dictionary& d ) const
{
  d[ "first_node_id" ] = P_.first_node_id;
  d[ "n_nodes" ] = P_.n_nodes;
  d[ "device" ] = P_.device;
  d[ "precision" ] = P_.precision;
  d[ "seed" ] = P_.seed;
  d[ "sync_weights" ] = P_.sync_weights;
  d[ "spikes_routed" ] = static_cast< long >( routed_ );
  d[ "plastic_connections" ] = static_cast< long >( pl_conns_.size() );
  if ( eng_ )
  {
    ng_stats st {};
    if ( ng_get_stats( eng_, &st ) == NG_OK )
    {
      d[ "engine_steps" ] = static_cast< long >( st.clock_steps );
      d[ "engine_spikes" ] = static_cast< long >( st.spikes );
      d[ "engine_syn_events" ] = static_cast< long >( st.syn_events );
      d[ "engine_host_ms" ] = st.simulate_ms;
    }
  }
}

void
gpu_engine::set_status( const Dictionary& d )
{
  if ( eng_ )
    throw nest::KernelException( "gpu_engine: the population is fixed once it has run (ResetKernel to change it)" );
  Parameters_ p = P_;
  d.update_value( "first_node_id", p.first_node_id );
  d.update_value( "n_nodes", p.n_nodes );
  d.update_value( "device", p.device );
  d.update_value( "precision", p.precision );
  d.update_value( "seed", p.seed );
  d.update_value( "sync_weights", p.sync_weights );
  if ( p.n_nodes < 0 || p.first_node_id < 0 || p.device < 0 )
    throw nest::BadProperty( "gpu_engine: first_node_id, n_nodes and device must be >= 0" );
  if ( p.precision != "fp64" && p.precision != "fp32" )
    throw nest::BadProperty( "gpu_engine: precision is \"fp64\" or \"fp32\"" );
  P_ = p;
}

void
gpu_engine::pre_run_hook()
{
  if ( not eng_ && P_.n_nodes > 0 )
    build_();
}

void
gpu_engine::build_()
{
  using nest::kernel;
  if ( kernel().vp_manager.get_num_threads() != 1 || kernel().mpi_manager.get_num_processes() != 1 )
    throw nest::BadProperty( "gpu_engine: runs with local_num_threads = 1 in one process" );
  if ( kernel().simulation_manager.get_clock().get_steps() != 0 )
    throw nest::BadProperty( "gpu_engine: the engine takes the population over at time 0 (the synaptic "
                             "currents and pending spikes of a simulated network are not in its status)" );
  const size_t first = static_cast< size_t >( P_.first_node_id );
  const size_t n = static_cast< size_t >( P_.n_nodes );
  std::vector< nest::Node* > nodes( n );
  for ( size_t k = 0; k < n; ++k )
  {
    nest::Node* node = kernel().node_manager.get_node_or_proxy( first + k );
    const int m = node ? model_id( node->get_name() ) : -1;
    if ( m < 0 || ( k > 0 && m != model_ ) )
      throw nest::BadProperty( "gpu_engine: the population must be one of iaf_psc_delta, iaf_psc_exp, "
                               "iaf_psc_alpha, aeif_cond_alpha, all the same model" );
    model_ = m;
    nodes[ k ] = node;
  }
  // parameters and state, in the engine's representation
  const auto& vars = vars_of( model_ );
  std::vector< std::vector< double > > vals( vars.size(), std::vector< double >( n ) );
  E_L_per_node_.assign( n, 0.0 );
  for ( size_t k = 0; k < n; ++k )
  {
    const Dictionary d = nodes[ k ]->get_status_base();
    const double E_L = get_d( d, "E_L" );
    E_L_per_node_[ k ] = E_L;
    for ( size_t v = 0; v < vars.size(); ++v )
      vals[ v ][ k ] = get_d( d, vars[ v ].status ) - ( vars[ v ].relative ? E_L : 0.0 );
  }
  // connections into the population: static_synapse from its own neurons,
  // poisson_generator drive from outside
  Dictionary q;
  std::vector< size_t > ids( n );
  for ( size_t k = 0; k < n; ++k )
    ids[ k ] = first + k;
  q[ "target" ] = nest::NodeCollection::create( ids );
  const std::deque< nest::ConnectionID > conns = kernel().connection_manager.get_connections( q );
  std::vector< int32_t > src, tgt, dly;
  std::vector< double > w;
  std::vector< double > rate( n, 0.0 ), pw( n, 0.0 );
  std::vector< int32_t > pd( n, 1 );
  long long g_start = -1, g_stop = -1;
  // stdp_pl_synapse_hom connections among the population (one set of common properties)
  std::vector< int32_t > psrc, ptgt, pdly;
  std::vector< double > pwt;
  pl_conns_.clear();
  int pl_syn = -1;
  double pl_common[ 4 ] = { 0, 0, 0, 0 };  // lambda, alpha, mu, tau_plus
  for ( const auto& c : conns )
  {
    const size_t s = static_cast< size_t >( c.get_source_node_id() );
    const size_t t = static_cast< size_t >( c.get_target_node_id() );
    const auto syn = static_cast< nest::synindex >( c.get_synapse_model_id() );
    const std::string syn_name = kernel().model_manager.get_connection_model( syn, 0 ).get_name();
    bool plastic = false;
    if ( syn_name != "static_synapse" )
    {
      const Dictionary defaults = kernel().model_manager.get_connector_defaults( syn );
      if ( not is_stdp_pl( syn_name, defaults ) )
        throw nest::BadProperty( "gpu_engine: connections run on the engine as static_synapse or "
                                 "stdp_pl_synapse_hom, not " + syn_name );
      const double common[ 4 ] = { get_d( defaults, "lambda" ), get_d( defaults, "alpha" ), get_d( defaults, "mu" ),
        get_d( defaults, "tau_plus" ) };
      if ( pl_syn >= 0 and not std::equal( common, common + 4, pl_common ) )
        throw nest::BadProperty( "gpu_engine: stdp_pl_synapse_hom models with different common properties" );
      pl_syn = syn;
      std::copy( common, common + 4, pl_common );
      plastic = true;
    }
    const Dictionary sd = kernel().connection_manager.get_synapse_status(
      s, t, static_cast< size_t >( c.get_target_thread() ), syn, static_cast< size_t >( c.get_port() ) );
    const double weight = get_d( sd, "weight" );
    const long d_steps = nest::Time::delay_ms_to_steps( get_d( sd, "delay" ) );
    if ( plastic )
    {
      if ( s < first || s >= first + n )
        throw nest::BadProperty( "gpu_engine: stdp_pl_synapse_hom connections start at the population's neurons" );
      psrc.push_back( static_cast< int32_t >( s - first ) );
      ptgt.push_back( static_cast< int32_t >( t - first ) );
      pwt.push_back( weight );
      pdly.push_back( static_cast< int32_t >( d_steps ) );
      pl_conns_.push_back( c );
      continue;
    }
    if ( s >= first && s < first + n )
    {
      src.push_back( static_cast< int32_t >( s - first ) );
      tgt.push_back( static_cast< int32_t >( t - first ) );
      w.push_back( weight );
      dly.push_back( static_cast< int32_t >( d_steps ) );
      continue;
    }
    nest::Node* gen = kernel().node_manager.get_node_or_proxy( s );
    if ( not gen || gen->get_name() != "poisson_generator" )
      throw nest::BadProperty( "gpu_engine: input from outside the population must come from poisson_generator" );
    const Dictionary gd = gen->get_status_base();
    const size_t k = t - first;
    if ( rate[ k ] > 0.0 )
      throw nest::BadProperty( "gpu_engine: one poisson_generator per neuron" );
    rate[ k ] = get_d( gd, "rate" );
    pw[ k ] = weight;
    pd[ k ] = static_cast< int32_t >( d_steps );
    const double origin = get_d( gd, "origin" );
    const long long st = nest::Time( nest::Time::ms( origin + get_d( gd, "start" ) ) ).get_steps();
    const double stop_ms = get_d( gd, "stop" );
    const long long sp = std::isinf( stop_ms ) ? ( 1ll << 62 ) : nest::Time( nest::Time::ms( origin + stop_ms ) ).get_steps();
    if ( ( g_start >= 0 && ( st != g_start || sp != g_stop ) ) )
      throw nest::BadProperty( "gpu_engine: the poisson_generators share one start/stop window" );
    g_start = st;
    g_stop = sp;
  }
  // the engine
  ng_config cfg {};
  cfg.device = static_cast< int32_t >( P_.device );
  cfg.precision = P_.precision == "fp32" ? NG_FP32 : NG_FP64;
  cfg.h = nest::Time::get_resolution().get_ms();
  cfg.tics_per_ms = nest::Time::get_tics_per_ms();
  cfg.min_delay = static_cast< int32_t >( kernel().connection_manager.get_min_delay() );
  cfg.max_delay = static_cast< int32_t >( kernel().connection_manager.get_max_delay() );
  cfg.n_blocks = 1;
  cfg.block_model[ 0 ] = model_;
  cfg.block_size[ 0 ] = static_cast< int64_t >( n );
  cfg.start_step = kernel().simulation_manager.get_clock().get_steps();
  check( ng_create( &cfg, &eng_ ), "gpu_engine: ng_create" );
  for ( size_t v = 0; v < vars.size(); ++v )
    check( ng_set_var( eng_, 0, vars[ v ].engine, vals[ v ].data(), 0, static_cast< int64_t >( n ) ),
      std::string( "gpu_engine: " ) + vars[ v ].engine );
  check( ng_set_connections_coo( eng_, static_cast< int64_t >( n ), static_cast< int64_t >( src.size() ), src.data(),
           tgt.data(), w.data(), dly.data() ),
    "gpu_engine: connections" );
  if ( g_start >= 0 )
    check( ng_set_poisson( eng_, rate.data(), pw.data(), pd.data(), g_start, g_stop,
             static_cast< uint64_t >( P_.seed ) ),
      "gpu_engine: poisson_generator drive" );
  if ( not pl_conns_.empty() )
  {
    // a CSR over the population's neurons, stable in the order NEST listed them
    const size_t m = pl_conns_.size();
    std::vector< int64_t > row( n + 1, 0 );
    for ( size_t k = 0; k < m; ++k )
      ++row[ static_cast< size_t >( psrc[ k ] ) + 1 ];
    for ( size_t i = 0; i < n; ++i )
      row[ i + 1 ] += row[ i ];
    std::vector< int64_t > fill( row.begin(), row.end() - 1 );
    pl_pos_.assign( m, 0 );
    std::vector< int32_t > ct( m ), cd( m );
    std::vector< double > cw( m );
    for ( size_t k = 0; k < m; ++k )
    {
      const int64_t q = fill[ static_cast< size_t >( psrc[ k ] ) ]++;
      pl_pos_[ k ] = q;
      ct[ static_cast< size_t >( q ) ] = ptgt[ k ];
      cd[ static_cast< size_t >( q ) ] = pdly[ k ];
      cw[ static_cast< size_t >( q ) ] = pwt[ k ];
    }
    check( ng_set_plastic_connections( eng_, static_cast< int64_t >( n ), row.data(), ct.data(), cw.data(), cd.data(),
             pl_common[ 0 ], pl_common[ 1 ], pl_common[ 2 ], pl_common[ 3 ] ),
      "gpu_engine: stdp_pl_synapse_hom connections" );
  }
  std::vector< uint8_t > rec( n, 1 );
  check( ng_set_recording( eng_, rec.data() ), "gpu_engine: recording" );
  // the neurons stay in NEST for recorders, GetStatus and connections, but
  // are no longer updated by it
  Dictionary frozen;
  frozen[ "frozen" ] = true;
  for ( auto* node : nodes )
    node->set_status_base( frozen );
}

void
gpu_engine::update( nest::Time const& origin, const long from, const long to )
{
  if ( not eng_ )
    return;
  check( ng_update( eng_, origin.get_steps(), static_cast< int32_t >( from ), static_cast< int32_t >( to ) ),
    "gpu_engine: update", model_ == NG_AEIF_COND_ALPHA ? "aeif_cond_alpha" : "gpu_engine" );
}

void
gpu_engine::post_run_cleanup()
{
  if ( eng_ )
    drain_and_route_();
}

void
gpu_engine::drain_and_route_()
{
  using nest::kernel;
  check( ng_sync( eng_ ), "gpu_engine: sync", model_ == NG_AEIF_COND_ALPHA ? "aeif_cond_alpha" : "gpu_engine" );
  int64_t cnt = 0;
  check( ng_spike_count( eng_, &cnt ), "gpu_engine: spike count" );
  src_buf_.resize( static_cast< size_t >( cnt ) );
  stamp_buf_.resize( static_cast< size_t >( cnt ) );
  int64_t got = 0;
  check( ng_get_spikes( eng_, src_buf_.data(), stamp_buf_.data(), cnt, &got ), "gpu_engine: spikes" );
  const size_t first = static_cast< size_t >( P_.first_node_id );
  for ( int64_t k = 0; k < got; ++k )
  {
    const size_t node_id = first + static_cast< size_t >( src_buf_[ k ] );
    nest::Node* node = kernel().node_manager.get_node_or_proxy( node_id );
    nest::SpikeEvent se;
    se.set_sender_node_id( node_id );
    se.set_sender( *node );
    se.set_stamp( nest::Time( nest::Time::step( stamp_buf_[ k ] ) ) );
    kernel().connection_manager.send_to_devices( node->get_thread(), node_id, se );
  }
  routed_ += got;
  // the neurons' state as the engine left it
  const auto& sv = state_of( model_ );
  const size_t n = static_cast< size_t >( P_.n_nodes );
  std::vector< std::vector< double > > vals( sv.size(), std::vector< double >( n ) );
  for ( size_t v = 0; v < sv.size(); ++v )
    check( ng_get_var( eng_, 0, sv[ v ].engine, vals[ v ].data(), 0, static_cast< int64_t >( n ) ),
      std::string( "gpu_engine: read " ) + sv[ v ].engine );
  for ( size_t k = 0; k < n; ++k )
  {
    Dictionary d;
    for ( size_t v = 0; v < sv.size(); ++v )
      d[ sv[ v ].status ] = vals[ v ][ k ] + ( sv[ v ].relative ? E_L_per_node_[ k ] : 0.0 );
    kernel().node_manager.get_node_or_proxy( first + k )->set_status_base( d );
  }
  // the plastic weights, so that GetConnections reads the engine's values
  if ( P_.sync_weights and not pl_conns_.empty() )
  {
    std::vector< double > wv( pl_conns_.size() );
    check( ng_get_plastic_weights( eng_, wv.data(), static_cast< int64_t >( wv.size() ) ), "gpu_engine: weights" );
    for ( size_t k = 0; k < pl_conns_.size(); ++k )
    {
      const nest::ConnectionID& c = pl_conns_[ k ];
      Dictionary d;
      d[ "weight" ] = wv[ static_cast< size_t >( pl_pos_[ k ] ) ];
      kernel().connection_manager.set_synapse_status( static_cast< size_t >( c.get_source_node_id() ),
        static_cast< size_t >( c.get_target_node_id() ), static_cast< size_t >( c.get_target_thread() ),
        static_cast< nest::synindex >( c.get_synapse_model_id() ), static_cast< size_t >( c.get_port() ), d );
    }
  }
}

void
gpu_engine::finalize()
{
  release_();
}

}  // namespace nestgpu
