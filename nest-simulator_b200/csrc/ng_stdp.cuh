// ng_stdp.cuh -- stdp_pl_synapse_hom connections (models/stdp_pl_synapse_hom.h)
// and the spike history of their postsynaptic neurons
// (nestkernel/archiving_node.cpp).
//
// Plastic connections live in a CSR of their own (targets, delays in steps,
// FP64 weights that the delivery rewrites) with a target-major index of the
// same edges.  A connection's Kplus_ and t_lastspike_ are the same for every
// connection of one source -- all start at 0 and see the same presynaptic
// spikes -- so they are kept per source.  At the close of a slice, after the
// node update has set each neuron's lag bits of the slice (gmask):
//   k_stdp_deliver  one CTA per spiking source splits its plastic row; each
//                   thread applies the source's spikes of the slice to its
//                   connections in time order: facilitation by the target's
//                   history entries in (t_last - d, t_spike - d], depression by
//                   the target's trace at t_spike - d, the new weight into the
//                   ring buffer (stdp_pl_synapse_hom::send, :255-298); then the
//                   source's Kplus and t_last.  The slice's own postsynaptic
//                   spikes are never read here: t_spike - d <= the slice origin.
//   k_stdp_archive  appends every postsynaptic spike of the slice to its
//                   neuron's history (time, Kminus trace), in time order
//                   (ArchivingNode::set_spiketime, archiving_node.cpp:182-220),
//                   and marks a history that is filling up;
//   k_stdp_flush    for a marked neuron, applies its oldest entries'
//                   facilitation to every incoming connection whose window
//                   still holds them, then drops them.
// A neuron's history is a ring of STDP_HIST entries holding the live entries
// [lo, n).  The reference keeps an entry until every incoming connection has
// read it, which a long-silent presynaptic neuron can delay without bound;
// here an entry leaves the ring early with its effect applied: a connection's
// weight changes only at its own source's spikes and at these flushes, its
// facilitation terms are applied oldest first either way, and Kplus / t_last
// do not change before the source's next spike, which lies after the entry's
// arrival (entries are flushed only once t + max_delay has passed).  The
// flushed terms go into a running copy of the weight (w_run) that the next
// presynaptic spike continues from; the weight the reference would report
// between two presynaptic spikes (w) changes only at them.  The newest
// dropped entry is kept for the trace lookup of the depression.
// A connection is owned by one thread in each kernel, so no weight is
// updated concurrently.
#pragma once

#include "ng_kernels.cuh"

namespace ng
{

constexpr int STDP_HIST = 64;
constexpr int STDP_KEEP = 16;        // entries a flush leaves in the ring
constexpr int ERR_STDP_HISTORY = 32;
constexpr double STDP_EPS = 1.0e-6;  // ConnectionManager's stdp_eps default

struct StdpNet
{
  const int64_t* row;     // per source: plastic CSR row pointers (n_src + 1)
  const int32_t* tgt;
  const int32_t* dly;     // steps
  double* w;              // the weights as the reference holds them (after each presynaptic spike)
  double* w_run;          // ... with the facilitation of flushed history entries applied ahead
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
  int64_t* hist_lo;       // per neuron: first live entry
  double* drop_t;         // per neuron: newest dropped entry (time, Kminus)
  double* drop_K;
  int32_t* n_flush;       // per neuron: entries the next flush drops
  const int64_t* in_row;  // per neuron: its incoming plastic connections (N + 1)
  const uint32_t* in_edge;  // their indices in the CSR
  const int32_t* in_src;
  double dmax_ms;         // the largest plastic delay
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
    // a history that the next slice could overrun: drop all but the newest
    // STDP_KEEP entries whose arrival time (t + max_delay) has passed
    const int64_t lo = p.hist_lo[ i ];
    if ( hn - lo > STDP_HIST - 32 )
    {
      const double t_now = stdp_stamp_ms( p, origin + d.min_delay );
      int64_t k = lo;
      while ( k < hn - STDP_KEEP && p.hist_t[ i * STDP_HIST + ( k % STDP_HIST ) ] + p.dmax_ms <= t_now )
        ++k;
      if ( hn - k > STDP_HIST - 32 )
        atomicOr( &d.ctl->err, ERR_STDP_HISTORY );
      p.n_flush[ i ] = ( int32_t ) ( k - lo );
    }
  }
}

// weight of one connection after one presynaptic spike at t_spike
__device__ __forceinline__ double
stdp_pl_update( const StdpNet& p, int32_t tg, double w, double d_ms, double Kplus, double tlast, double t_spike,
  bool& overflow )
{
  const int64_t hn = p.hist_n[ tg ];
  const int64_t lo = p.hist_lo[ tg ];
  const double* ht = p.hist_t + ( int64_t ) tg * STDP_HIST;
  const double* hk = p.hist_K + ( int64_t ) tg * STDP_HIST;
  // get_history( t_last - d, t_spike - d ): entries t1 + eps <= t < t2 + eps
  // (entries before lo in the range were applied when they were dropped)
  const double t1_lim = tlast - d_ms + STDP_EPS;
  const double t2_lim = t_spike - d_ms + STDP_EPS;
  int64_t fin = hn;
  while ( fin > lo && ht[ ( fin - 1 ) % STDP_HIST ] >= t2_lim )
    --fin;
  int64_t st = fin;
  while ( st > lo && ht[ ( st - 1 ) % STDP_HIST ] >= t1_lim )
    --st;
  // facilitation, in time order
  for ( int64_t k = st; k < fin; ++k )
  {
    const double minus_dt = tlast - ( ht[ k % STDP_HIST ] + d_ms );
    const double kplus = Kplus * exp( minus_dt * p.tau_plus_inv );
    w = w + ( p.lambda * pow( w, p.mu ) * kplus );
  }
  // depression by the trace at t_spike - d (get_K_value: the latest entry
  // strictly before, archiving_node.cpp:87-113); the newest dropped entry
  // when every live one is later
  const double t = t_spike - d_ms;
  double kminus = 0.;
  int64_t k = fin - 1;
  while ( k >= lo && !( t - ht[ k % STDP_HIST ] > STDP_EPS ) )
    --k;
  if ( k >= lo )
    kminus = hk[ k % STDP_HIST ] * exp( ( ht[ k % STDP_HIST ] - t ) * p.tau_minus_inv[ tg ] );
  else if ( lo > 0 )
  {
    const double te = p.drop_t[ tg ];
    if ( t - te > STDP_EPS )
      kminus = p.drop_K[ tg ] * exp( ( te - t ) * p.tau_minus_inv[ tg ] );
    else
      overflow = true;  // cannot happen: dropped entries lie max_delay before the slice
  }
  const double new_w = w - ( p.lambda * p.alpha * w * kminus );
  return new_w > 0.0 ? new_w : 0.0;
}

// The oldest n_flush entries of a marked neuron: each incoming connection
// applies the facilitation of those in its current window (t >= t_last - d
// + eps; later bounds hold since the entries arrived before the slice's
// end), in time order, with its source's Kplus and t_last.
__global__ void __launch_bounds__( 256 )
k_stdp_flush( Net d, StdpNet p )
{
  for ( int64_t tg = blockIdx.x; tg < d.N; tg += gridDim.x )
  {
    const int nf = p.n_flush[ tg ];
    if ( nf == 0 )
      continue;  // uniform over the CTA
    const int64_t lo = p.hist_lo[ tg ];
    const double* ht = p.hist_t + tg * STDP_HIST;
    const int64_t i0 = p.in_row[ tg ], i1 = p.in_row[ tg + 1 ];
    for ( int64_t q = i0 + threadIdx.x; q < i1; q += blockDim.x )
    {
      const uint32_t e = p.in_edge[ q ];
      const int32_t src = p.in_src[ q ];
      const double d_ms = ( double ) p.dly[ e ] * ( p.ms_per_tic * ( double ) p.tics_per_step );
      const double tl = p.tlast[ src ], Kp = p.Kplus[ src ];
      const double t1_lim = tl - d_ms + STDP_EPS;
      double w = p.w_run[ e ];
      bool changed = false;
      for ( int64_t k = lo; k < lo + nf; ++k )
      {
        const double te = ht[ k % STDP_HIST ];
        if ( te >= t1_lim )
        {
          const double kplus = Kp * exp( ( tl - ( te + d_ms ) ) * p.tau_plus_inv );
          w = w + ( p.lambda * pow( w, p.mu ) * kplus );
          changed = true;
        }
      }
      if ( changed )
        p.w_run[ e ] = w;
    }
    __syncthreads();
    if ( threadIdx.x == 0 )
    {
      const int64_t last = ( lo + nf - 1 ) % STDP_HIST;
      p.drop_t[ tg ] = ht[ last ];
      p.drop_K[ tg ] = p.hist_K[ tg * STDP_HIST + last ];
      p.hist_lo[ tg ] = lo + nf;
      p.n_flush[ tg ] = 0;
    }
  }
}

// One CTA per spiking source at a time (grid-stride over sources): the
// CTA's threads split the source's plastic row, so a spike's thousands of
// connections -- each a chain of dependent history loads -- run on 256
// threads instead of 32.  Every thread reads the source's Kplus and t_last
// before the CTA's closing barrier; thread 0 writes them after it.
template < bool FIX >
__global__ void __launch_bounds__( 256 )
k_stdp_deliver( Net d, StdpNet p )
{
  const long long origin = cta_origin( d );
  bool overflow = false;
  unsigned long long events = 0;
  for ( int64_t src = blockIdx.x; src < p.n_src; src += gridDim.x )
  {
    const unsigned m0 = d.gmask[ src ];
    const int64_t e0 = p.row[ src ], e1 = p.row[ src + 1 ];
    if ( m0 == 0 || e1 == e0 )
      continue;  // uniform over the CTA
    const double Kp0 = p.Kplus[ src ], tl0 = p.tlast[ src ];
    for ( int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x )
    {
      const int32_t tg = p.tgt[ e ];
      const int32_t dl = p.dly[ e ];
      const double d_ms = ( double ) dl * ( p.ms_per_tic * ( double ) p.tics_per_step );
      double w = p.w_run[ e ];
      double Kp = Kp0, tl = tl0;
      unsigned m = m0;
      while ( m )
      {
        const int k = __ffs( m ) - 1;
        m &= m - 1;
        const long long te = origin + k;
        const double t_spike = stdp_stamp_ms( p, te + 1 );
        w = stdp_pl_update( p, tg, w, d_ms, Kp, tl, t_spike, overflow );
        // handle(SpikeEvent&): weight x multiplicity into the channel of its sign
        const int slot = ( int ) ( ( te + dl ) % d.L );
        const int ch = ( p.sign_channels && !( w > 0.0 ) ) ? 1 : 0;
        const int64_t idx = ( ( int64_t ) slot * d.C + ch ) * d.N + tg;
        if constexpr ( FIX )
          atomicAdd( ( unsigned long long* ) d.ring + idx,
            ( unsigned long long ) __double2ll_rn( w * ( 1.0 / d.fx_inv ) ) );
        else
          atomicAdd( ( double* ) d.ring + idx, w );
        Kp = Kp * exp( ( tl - t_spike ) * p.tau_plus_inv ) + 1.0;
        tl = t_spike;
      }
      p.w[ e ] = w;
      p.w_run[ e ] = w;
    }
    if ( threadIdx.x == 0 )
      events += ( unsigned long long ) ( e1 - e0 ) * ( unsigned long long ) __popc( m0 );
    __syncthreads();
    if ( threadIdx.x == 0 )
    {
      double Kp = Kp0, tl = tl0;
      unsigned m = m0;
      while ( m )
      {
        const int k = __ffs( m ) - 1;
        m &= m - 1;
        const double t_spike = stdp_stamp_ms( p, origin + k + 1 );
        Kp = Kp * exp( ( tl - t_spike ) * p.tau_plus_inv ) + 1.0;
        tl = t_spike;
      }
      p.Kplus[ src ] = Kp;
      p.tlast[ src ] = tl;
    }
  }
  if ( threadIdx.x == 0 && events )
    atomicAdd( &d.ctl->syn_events, events );
  if ( overflow )
    atomicOr( &d.ctl->err, ERR_STDP_HISTORY );
}

}  // namespace ng
