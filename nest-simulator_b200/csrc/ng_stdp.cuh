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
  int32_t dconst;         // the plastic delay in steps when all are equal, else -1
  int32_t* tab_fin;       // dconst >= 0: per (neuron, lag of the slice) the end of the
  double* tab_km;         //   facilitation range and the depression trace (k_stdp_arrivals)
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

// One facilitation term lambda w^mu Kplus exp(minus_dt / tau_plus) of
// stdp_pl_synapse_hom::facilitate_: for w > 0 as lambda Kplus
// exp(mu log w + minus_dt / tau_plus) -- one exponential for the power and
// the trace's decay (within a few ulp of the reference's pow and exp); the
// power law's value at w = 0 otherwise
__device__ __forceinline__ double
stdp_facilitation( const StdpNet& p, double w, double Kplus, double minus_dt )
{
  const double a = minus_dt * p.tau_plus_inv;
  if ( w > 0.0 )
    return p.lambda * Kplus * exp( p.mu * log( w ) + a );
  return p.lambda * pow( w, p.mu ) * ( Kplus * exp( a ) );
}

// end of the facilitation range of an arrival at t = t_spike - d: the live
// entries before t + eps (get_history's upper bound)
__device__ __forceinline__ int64_t
stdp_fin( const double* ht, int64_t lo, int64_t hn, double t )
{
  const double t2_lim = t + STDP_EPS;
  int64_t fin = hn;
  while ( fin > lo && ht[ ( fin - 1 ) & ( STDP_HIST - 1 ) ] >= t2_lim )
    --fin;
  return fin;
}

// the postsynaptic trace at t (get_K_value, archiving_node.cpp:87-113: the
// latest entry strictly before t); the newest dropped entry when every live
// one is later
__device__ __forceinline__ double
stdp_kminus( const StdpNet& p, int32_t tg, const double* ht, const double* hk, int64_t lo, int64_t fin, double t,
  bool& overflow )
{
  int64_t k = fin - 1;
  while ( k >= lo && !( t - ht[ k & ( STDP_HIST - 1 ) ] > STDP_EPS ) )
    --k;
  if ( k >= lo )
    return hk[ k & ( STDP_HIST - 1 ) ] * exp( ( ht[ k & ( STDP_HIST - 1 ) ] - t ) * p.tau_minus_inv[ tg ] );
  if ( lo > 0 )
  {
    const double te = p.drop_t[ tg ];
    if ( t - te > STDP_EPS )
      return p.drop_K[ tg ] * exp( ( te - t ) * p.tau_minus_inv[ tg ] );
    overflow = true;  // cannot happen: dropped entries lie max_delay before the slice
  }
  return 0.;
}

// weight of one connection after one presynaptic spike at t_spike, given
// the end of its facilitation range (fin) and the depression trace:
// facilitation by the live entries in [t_last - d + eps, t_spike - d + eps)
// in time order (entries before lo in the range were applied when they were
// dropped), then depression (stdp_pl_synapse_hom::send, :255-298)
__device__ __forceinline__ double
stdp_pl_apply( const StdpNet& p, const double* ht, int64_t lo, int64_t fin, double w, double d_ms, double Kplus,
  double tlast, double kminus )
{
  const double t1_lim = tlast - d_ms + STDP_EPS;
  int64_t st = fin;
  while ( st > lo && ht[ ( st - 1 ) & ( STDP_HIST - 1 ) ] >= t1_lim )
    --st;
  for ( int64_t k = st; k < fin; ++k )
  {
    const double minus_dt = tlast - ( ht[ k & ( STDP_HIST - 1 ) ] + d_ms );
    w = w + stdp_facilitation( p, w, Kplus, minus_dt );
  }
  const double new_w = w - ( p.lambda * p.alpha * w * kminus );
  return new_w > 0.0 ? new_w : 0.0;
}

// With one plastic delay for all connections, every arrival at a neuron in
// a slice happens at one of min_delay times (lag k: t = stamp(origin + k + 1)
// - d), so the end of its facilitation range and its depression trace are
// computed here once per (neuron, lag) instead of once per connection.
__global__ void
k_stdp_arrivals( Net d, StdpNet p )
{
  const long long origin = cta_origin( d );
  const double d_ms = ( double ) p.dconst * ( p.ms_per_tic * ( double ) p.tics_per_step );
  const int md = d.min_delay;
  bool overflow = false;
  for ( int64_t q = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x; q < d.N * md;
        q += ( int64_t ) gridDim.x * blockDim.x )
  {
    const int64_t tg = q / md;
    const int k = ( int ) ( q - tg * md );
    if ( !p.n_inc[ tg ] )
      continue;
    const int64_t hn = p.hist_n[ tg ], lo = p.hist_lo[ tg ];
    const double* ht = p.hist_t + tg * STDP_HIST;
    const double* hk = p.hist_K + tg * STDP_HIST;
    const double t = stdp_stamp_ms( p, origin + k + 1 ) - d_ms;
    const int64_t fin = stdp_fin( ht, lo, hn, t );
    p.tab_fin[ q ] = ( int32_t ) ( fin - lo );
    p.tab_km[ q ] = stdp_kminus( p, ( int32_t ) tg, ht, hk, lo, fin, t, overflow );
  }
  if ( overflow )
    atomicOr( &d.ctl->err, ERR_STDP_HISTORY );
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
          w = w + stdp_facilitation( p, w, Kp, tl - ( te + d_ms ) );
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
// threads instead of 32.  Thread 0 first lays out the source's spikes of
// the slice in shared memory (lag, time, ring slot, and Kplus / t_last
// before each spike) and advances the source's Kplus and t_last; each
// thread then applies the spikes to its connections in time order.
// (registers capped for four CTAs per SM: more resident warps hide the
// dependent history loads better than spill-free code -- measured RTF 0.407
// against 0.424 with 80 registers, 0.420 with 48 on the hpc_benchmark network)
template < bool FIX >
__global__ void __launch_bounds__( 256, 4 )
k_stdp_deliver( Net d, StdpNet p )
{
  __shared__ double s_t[ 32 ], s_Kp[ 32 ], s_tl[ 32 ];
  __shared__ int s_k[ 32 ], s_slot0[ 32 ];
  __shared__ int s_n;
  const long long origin = cta_origin( d );
  const double h_ms = p.ms_per_tic * ( double ) p.tics_per_step;
  const int md = d.min_delay;
  bool overflow = false;
  unsigned long long events = 0;
  for ( int64_t src = blockIdx.x; src < p.n_src; src += gridDim.x )
  {
    const unsigned m0 = d.gmask[ src ];
    const int64_t e0 = p.row[ src ], e1 = p.row[ src + 1 ];
    if ( m0 == 0 || e1 == e0 )
      continue;  // uniform over the CTA
    if ( threadIdx.x == 0 )
    {
      double Kp = p.Kplus[ src ], tl = p.tlast[ src ];
      int n = 0;
      unsigned m = m0;
      while ( m )
      {
        const int k = __ffs( m ) - 1;
        m &= m - 1;
        const double t_spike = stdp_stamp_ms( p, origin + k + 1 );
        s_k[ n ] = k;
        s_t[ n ] = t_spike;
        s_Kp[ n ] = Kp;
        s_tl[ n ] = tl;
        s_slot0[ n ] = ( int ) ( ( origin + k ) % d.L );
        Kp = Kp * exp( ( tl - t_spike ) * p.tau_plus_inv ) + 1.0;
        tl = t_spike;
        ++n;
      }
      s_n = n;
      p.Kplus[ src ] = Kp;
      p.tlast[ src ] = tl;
      events += ( unsigned long long ) ( e1 - e0 ) * ( unsigned long long ) n;
    }
    __syncthreads();
    const int ns = s_n;
    for ( int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x )
    {
      const int32_t tg = p.tgt[ e ];
      const int32_t dl = p.dconst >= 0 ? p.dconst : p.dly[ e ];
      const double d_ms = ( double ) dl * h_ms;
      double w = p.w_run[ e ];
      const int64_t lo = p.hist_lo[ tg ];
      const int64_t hn = p.dconst >= 0 ? lo : p.hist_n[ tg ];  // (the arrival tables hold the range end)
      const double* ht = p.hist_t + ( int64_t ) tg * STDP_HIST;
      for ( int j = 0; j < ns; ++j )
      {
        int64_t fin;
        double kminus;
        if ( p.dconst >= 0 )
        {
          const int64_t q = ( int64_t ) tg * md + s_k[ j ];
          fin = lo + p.tab_fin[ q ];
          kminus = p.tab_km[ q ];
        }
        else
        {
          const double t = s_t[ j ] - d_ms;
          fin = stdp_fin( ht, lo, hn, t );
          kminus = stdp_kminus( p, tg, ht, p.hist_K + ( int64_t ) tg * STDP_HIST, lo, fin, t, overflow );
        }
        w = stdp_pl_apply( p, ht, lo, fin, w, d_ms, s_Kp[ j ], s_tl[ j ], kminus );
        // handle(SpikeEvent&): weight x multiplicity into the channel of its sign
        int slot = s_slot0[ j ] + dl;
        if ( slot >= d.L )
          slot -= d.L;
        const int ch = ( p.sign_channels && !( w > 0.0 ) ) ? 1 : 0;
        const int64_t idx = ( ( int64_t ) slot * d.C + ch ) * d.N + tg;
        if constexpr ( FIX )
          atomicAdd( ( unsigned long long* ) d.ring + idx,
            ( unsigned long long ) __double2ll_rn( w * ( 1.0 / d.fx_inv ) ) );
        else
          atomicAdd( ( double* ) d.ring + idx, w );
      }
      p.w[ e ] = w;
      p.w_run[ e ] = w;
    }
    __syncthreads();  // the spike table is rewritten for the next source
  }
  if ( threadIdx.x == 0 && events )
    atomicAdd( &d.ctl->syn_events, events );
  if ( overflow )
    atomicOr( &d.ctl->err, ERR_STDP_HISTORY );
}

}  // namespace ng
