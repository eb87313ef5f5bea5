// ng_stdp.cuh -- stdp_pl_synapse_hom connections (models/stdp_pl_synapse_hom.h)
// and the spike history of their postsynaptic neurons
// (nestkernel/archiving_node.cpp).
//
// Plastic connections live in a CSR of their own (targets, delays in steps,
// FP64 weights that the delivery rewrites).  A connection's Kplus_ and
// t_lastspike_ are the same for every connection of one source -- all start
// at 0 and see the same presynaptic spikes -- so they are kept per source.
// At the close of a slice, after the node update has set each neuron's lag
// bits of the slice (gmask):
//   k_stdp_archive  records every postsynaptic spike of the slice in its
//                   neuron's history (time, Kminus trace), in time order
//                   (ArchivingNode::set_spiketime, archiving_node.cpp:182-220);
//   k_stdp_deliver  one warp per spiking source walks its plastic row for each
//                   of its spikes in time order: facilitation by the target's
//                   history entries in (t_last - d, t_spike - d], depression by
//                   the target's trace at t_spike - d, the new weight into the
//                   ring buffer (stdp_pl_synapse_hom::send, :255-298); then the
//                   source's Kplus and t_last.
// The lanes of a warp own distinct connections, and a source's spikes are
// processed by one warp in order, so no weight is updated concurrently.
// A neuron's history is a ring of STDP_HIST entries; a read that needs an
// entry already overwritten sets ERR_STDP_HISTORY.
#pragma once

#include "ng_kernels.cuh"

namespace ng
{

constexpr int STDP_HIST = 64;
constexpr int ERR_STDP_HISTORY = 32;
constexpr double STDP_EPS = 1.0e-6;  // ConnectionManager's stdp_eps default

struct StdpNet
{
  const int64_t* row;     // per source: plastic CSR row pointers (n_src + 1)
  const int32_t* tgt;
  const int32_t* dly;     // steps
  double* w;
  double* Kplus;          // per source
  double* tlast;          // per source [ms]
  int64_t n_src;
  const uint8_t* n_inc;   // per neuron: has incoming plastic connections
  const double* tau_minus_inv;  // per neuron
  double* Kminus;         // per neuron: trace after its last spike
  double* last_spike;     // per neuron [ms]
  double* hist_t;         // [neuron][STDP_HIST]
  double* hist_K;
  int64_t* hist_n;        // per neuron: spikes archived so far
  double lambda, alpha, mu, tau_plus_inv;
  double ms_per_tic;      // Time::get_ms = MS_PER_TIC * tics
  int64_t tics_per_step;
  int sign_channels;      // targets split input by sign (iaf_psc_exp, iaf_psc_alpha), else one channel
};

__device__ __forceinline__ double
stdp_stamp_ms( const StdpNet& p, long long stamp )
{
  return p.ms_per_tic * ( double ) ( stamp * p.tics_per_step );
}

__global__ void
k_stdp_archive( Net d, StdpNet p )
{
  const long long origin = cta_origin( d );
  for ( int64_t i = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x; i < d.N; i += ( int64_t ) gridDim.x * blockDim.x )
  {
    if ( !p.n_inc[ i ] )
      continue;
    unsigned m = d.gmask[ i ];
    if ( m == 0 )
      continue;
    double Km = p.Kminus[ i ], last = p.last_spike[ i ];
    int64_t hn = p.hist_n[ i ];
    const double inv = p.tau_minus_inv[ i ];
    while ( m )
    {
      const int k = __ffs( m ) - 1;
      m &= m - 1;
      const double t = stdp_stamp_ms( p, origin + k + 1 );
      Km = Km * exp( ( last - t ) * inv ) + 1.0;
      last = t;
      const int64_t slot = i * STDP_HIST + ( hn % STDP_HIST );
      p.hist_t[ slot ] = t;
      p.hist_K[ slot ] = Km;
      ++hn;
    }
    p.Kminus[ i ] = Km;
    p.last_spike[ i ] = last;
    p.hist_n[ i ] = hn;
  }
}

// weight of one connection after one presynaptic spike at t_spike
__device__ __forceinline__ double
stdp_pl_update( const StdpNet& p, int32_t tg, double w, double d_ms, double Kplus, double tlast, double t_spike,
  bool& overflow )
{
  const int64_t hn = p.hist_n[ tg ];
  const int64_t oldest = hn > STDP_HIST ? hn - STDP_HIST : 0;
  const double* ht = p.hist_t + ( int64_t ) tg * STDP_HIST;
  const double* hk = p.hist_K + ( int64_t ) tg * STDP_HIST;
  // get_history( t_last - d, t_spike - d ): entries t1 + eps <= t < t2 + eps
  const double t1_lim = tlast - d_ms + STDP_EPS;
  const double t2_lim = t_spike - d_ms + STDP_EPS;
  int64_t fin = hn;
  while ( fin > oldest && ht[ ( fin - 1 ) % STDP_HIST ] >= t2_lim )
    --fin;
  int64_t st = fin;
  while ( st > oldest && ht[ ( st - 1 ) % STDP_HIST ] >= t1_lim )
    --st;
  if ( st == oldest && oldest > 0 )
    overflow = true;  // entries before the ring's oldest might belong to the range
  // facilitation, in time order
  for ( int64_t k = st; k < fin; ++k )
  {
    const double minus_dt = tlast - ( ht[ k % STDP_HIST ] + d_ms );
    const double kplus = Kplus * exp( minus_dt * p.tau_plus_inv );
    w = w + ( p.lambda * pow( w, p.mu ) * kplus );
  }
  // depression by the trace at t_spike - d (get_K_value: the latest entry
  // strictly before, archiving_node.cpp:87-113)
  const double t = t_spike - d_ms;
  double kminus = 0.;
  for ( int64_t k = hn - 1; k >= oldest; --k )
  {
    const double te = ht[ k % STDP_HIST ];
    if ( t - te > STDP_EPS )
    {
      kminus = hk[ k % STDP_HIST ] * exp( ( te - t ) * p.tau_minus_inv[ tg ] );
      break;
    }
    if ( k == oldest && oldest > 0 )
      overflow = true;
  }
  const double new_w = w - ( p.lambda * p.alpha * w * kminus );
  return new_w > 0.0 ? new_w : 0.0;
}

template < bool FIX >
__global__ void __launch_bounds__( 256 )
k_stdp_deliver( Net d, StdpNet p )
{
  const long long origin = cta_origin( d );
  const int lane = threadIdx.x & 31;
  const int64_t nw = ( ( int64_t ) gridDim.x * blockDim.x ) >> 5;
  bool overflow = false;
  unsigned long long events = 0;
  for ( int64_t src = ( ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x ) >> 5; src < p.n_src; src += nw )
  {
    unsigned m = d.gmask[ src ];
    const int64_t e0 = p.row[ src ], e1 = p.row[ src + 1 ];
    if ( m == 0 || e1 == e0 )
      continue;
    double Kp = p.Kplus[ src ], tl = p.tlast[ src ];
    while ( m )
    {
      const int k = __ffs( m ) - 1;
      m &= m - 1;
      const long long te = origin + k;
      const double t_spike = stdp_stamp_ms( p, te + 1 );
      for ( int64_t e = e0 + lane; e < e1; e += 32 )
      {
        const int32_t tg = p.tgt[ e ];
        const int32_t dl = p.dly[ e ];
        const double d_ms = ( double ) dl * ( p.ms_per_tic * ( double ) p.tics_per_step );
        const double w = stdp_pl_update( p, tg, p.w[ e ], d_ms, Kp, tl, t_spike, overflow );
        p.w[ e ] = w;
        // handle(SpikeEvent&): weight x multiplicity into the channel of its sign
        int slot = ( int ) ( ( te + dl ) % d.L );
        const int ch = ( p.sign_channels && !( w > 0.0 ) ) ? 1 : 0;
        const int64_t idx = ( ( int64_t ) slot * d.C + ch ) * d.N + tg;
        if constexpr ( FIX )
          atomicAdd( ( unsigned long long* ) d.ring + idx,
            ( unsigned long long ) __double2ll_rn( w * ( 1.0 / d.fx_inv ) ) );
        else
          atomicAdd( ( double* ) d.ring + idx, w );
      }
      events += ( unsigned long long ) ( e1 - e0 );
      Kp = Kp * exp( ( tl - t_spike ) * p.tau_plus_inv ) + 1.0;
      tl = t_spike;
      __syncwarp();
    }
    if ( lane == 0 )
    {
      p.Kplus[ src ] = Kp;
      p.tlast[ src ] = tl;
    }
  }
  if ( lane == 0 && events )
    atomicAdd( &d.ctl->syn_events, events );
  if ( overflow )
    atomicOr( &d.ctl->err, ERR_STDP_HISTORY );
}

}  // namespace ng
