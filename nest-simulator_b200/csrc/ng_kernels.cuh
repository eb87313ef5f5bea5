// ng_kernels.cuh -- sm_100a kernels of one min_delay slice.
//
// Per slice: one node-update launch per model block (thread per neuron, the
// lags of the slice in registers, warp-ballot spike compaction, Philox drive
// fused), then one delivery launch (source-spike-driven scatter over the CSR
// with 128-bit edge loads and red.global adds into the ring buffers).  The
// delivery launch's last CTA closes the slice: it resets the spike list and
// advances the device clock, so a run of slices needs no host round trip and
// can be captured as one CUDA graph.
//
// Compiled with -fmad=false: every FP64 multiply and add rounds on its own as
// in the reference's x86-64 build, which makes the plain form bit-exact where
// the ring sums are order independent.
#pragma once

#include <type_traits>

#include "ng_device.cuh"

namespace ng
{

constexpr unsigned FULL = 0xffffffffu;
constexpr int NG_IAF_PSC_DELTA_ID = 0;
constexpr int NG_IAF_PSC_EXP_ID = 1;
constexpr int NG_IAF_PSC_ALPHA_ID = 3;

template < typename T >
__device__ __forceinline__ T
ld_volatile( const T* p )
{
  return *( const volatile T* ) p;
}

__device__ __forceinline__ long long
warp_sum_ll( long long v )
{
#pragma unroll
  for ( int o = 16; o > 0; o >>= 1 )
    v += __shfl_xor_sync( FULL, v, o );
  return v;
}

// The half of the spike log the running group writes, and the source
// field of a log entry (serving: network-local id | network id << 22).
__device__ __forceinline__ uint2*
log_half( const Net& d )
{
  return d.log + ( ld_volatile( &d.ctl->log_sel ) ? d.log_cap : 0 );
}

__device__ __forceinline__ uint32_t
log_source( const Net& d, int32_t src )
{
  if ( d.nid == nullptr )
    return ( uint32_t ) src;
  const int id = d.nid[ src ];
  return ( uint32_t ) ( src - d.net_off[ id ] ) | ( ( uint32_t ) id << LOG_ID_SHIFT );
}

// The out-edges of a spiking source as delivery work: chunks of <= 128
// edges of its padded CSR row.  With late delivery on, the slice-close
// chunks cover the row's edges [0, ue) and the late chunks [ls, pdeg);
// otherwise the slice-close chunks cover the whole row.
struct RowWork
{
  long long row;
  int pdeg, ue, ls;
  int nu, nl;  // chunks: slice close, late
};

__device__ __forceinline__ RowWork
row_work( const Net& d, int32_t src )
{
  RowWork w;
  w.row = d.row_beg[ src ];
  w.pdeg = d.row_len[ src ];
  w.ue = w.pdeg;
  w.ls = w.pdeg;
  if ( d.late_min != INT32_MAX )
  {
    w.ue = d.row_ue[ src ];
    w.ls = d.row_ls[ src ];
  }
  w.nu = ( w.ue + CHUNK_EDGES - 1 ) / CHUNK_EDGES;
  w.nl = ( w.pdeg - w.ls + CHUNK_EDGES - 1 ) / CHUNK_EDGES;
  return w;
}

// The late list the open slice appends to.
__device__ __forceinline__ int4*
late_list( const Net& d, int sel )
{
  return d.ent_late + ( sel ? d.ent_cap : 0 );
}

// Work item e of a list: chunk c of the edge range [lo, hi) of a row.
__device__ __forceinline__ void
put_chunk( const Net& d, int4* list, long long e, long long row, int lo, int hi, long long c, int slot, int mult )
{
  const long long r = row + lo + c * CHUNK_EDGES;
  const long long left = ( long long ) ( hi - lo ) - c * CHUNK_EDGES;
  const int ne = ( int ) ( left < CHUNK_EDGES ? left : CHUNK_EDGES );
  if ( e < d.ent_cap )
    list[ e ] = make_int4( ( int ) ( unsigned ) ( r & 0xffffffffll ), ( int ) ( r >> 32 ), ne, slot | ( mult << 16 ) );
  else
    atomicOr( &d.ctl->err, ERR_SPIKE_LIST );
}

// Inclusive warp prefix sums of two counters.
__device__ __forceinline__ void
warp_scan2( long long& a, long long& b )
{
  const int lane = threadIdx.x & 31;
#pragma unroll
  for ( int o = 1; o < 32; o <<= 1 )
  {
    const long long x = __shfl_up_sync( FULL, a, o );
    const long long y = __shfl_up_sync( FULL, b, o );
    if ( lane >= o )
    {
      a += x;
      b += y;
    }
  }
}

// Append this lane's spike (if any, with its multiplicity) to the slice's
// delivery work and the recorder log.  Must be called by all 32 lanes.
__device__ __forceinline__ void
warp_append( const Net& d, bool spk, int32_t src, int32_t tmod, int32_t mult, long long stamp )
{
  const unsigned m = __ballot_sync( FULL, spk );
  if ( m == 0 )
    return;
  const int lane = threadIdx.x & 31;
  const unsigned lt = ( 1u << lane ) - 1u;
  RowWork rw {};
  long long rdeg = 0;
  if ( spk )
  {
    rw = row_work( d, src );
    rdeg = ( long long ) d.real_deg[ src ] * mult;
  }
  long long inc_u = rw.nu, inc_l = rw.nl;
  warp_scan2( inc_u, inc_l );
  const long long tot_u = __shfl_sync( FULL, inc_u, 31 );
  const long long tot_l = __shfl_sync( FULL, inc_l, 31 );
  const long long rtot = warp_sum_ll( rdeg );
  const long long mtot = warp_sum_ll( spk ? ( long long ) mult : 0ll );
  const bool lg = spk && ( d.rec == nullptr || d.rec[ src ] );
  const unsigned lm = __ballot_sync( FULL, lg );
  unsigned long long base = 0, lb = 0, xb = 0;
  int sel = 0;
  if ( lane == 0 )
  {
    if ( tot_u > 0 )
      base = atomicAdd( &d.ctl->n_ent, ( unsigned long long ) tot_u );
    if ( tot_l > 0 )
    {
      sel = ld_volatile( &d.ctl->late_wr );
      xb = atomicAdd( &d.ctl->n_late[ sel ], ( unsigned long long ) tot_l );
    }
    if ( lm )
      lb = atomicAdd( &d.ctl->log_count, ( unsigned long long ) __popc( lm ) );
    atomicAdd( &d.ctl->syn_events, ( unsigned long long ) rtot );
    atomicAdd( &d.ctl->n_spikes, ( unsigned long long ) mtot );
  }
  base = __shfl_sync( FULL, base, 0 );
  xb = __shfl_sync( FULL, xb, 0 );
  lb = __shfl_sync( FULL, lb, 0 );
  sel = __shfl_sync( FULL, sel, 0 );
  if ( spk )
  {
    for ( int c = 0; c < rw.nu; ++c )
      put_chunk( d, d.ent, ( long long ) base + inc_u - rw.nu + c, rw.row, 0, rw.ue, c, tmod, mult );
    for ( int c = 0; c < rw.nl; ++c )
      put_chunk( d, late_list( d, sel ), ( long long ) xb + inc_l - rw.nl + c, rw.row, rw.ls, rw.pdeg, c, tmod, mult );
  }
  if ( lg )
  {
    const long long li = ( long long ) lb + __popc( lm & lt );
    if ( li < d.log_cap )
    {
      const uint32_t rel = ( uint32_t ) ( stamp - ld_volatile( &d.ctl->log_base ) );
      const uint32_t mu = ( uint32_t ) ( mult < 255 ? mult : 255 );
      log_half( d )[ li ] = make_uint2( log_source( d, src ), rel | ( mu << 24 ) );
    }
    else
    {
      atomicOr( &d.ctl->err, ERR_LOG );
    }
  }
}

// Append all spikes of a chunk of up to 32 lags at once: bit k of `mask` is
// a spike of this lane's neuron at lag k (emission step t0 + k, ring slot
// (slot0 + k) mod L).  One work and one log reservation per warp and chunk,
// issued together, instead of an atomic round trip per lag.  Must be called
// by all 32 lanes.
__device__ __forceinline__ void
warp_append_mask( const Net& d, unsigned mask, int32_t src, int slot0, long long t0 )
{
  const int cnt = __popc( mask );
  if ( __ballot_sync( FULL, cnt > 0 ) == 0 )
    return;
  const int lane = threadIdx.x & 31;
  RowWork rw {};
  long long rdeg = 0;
  const bool lg = cnt > 0 && ( d.rec == nullptr || d.rec[ src ] );
  if ( cnt > 0 )
  {
    rw = row_work( d, src );
    rdeg = d.real_deg[ src ];
  }
  long long inc_u = ( long long ) cnt * rw.nu, inc_l = ( long long ) cnt * rw.nl;
  warp_scan2( inc_u, inc_l );
  long long inc_g = lg ? cnt : 0, dummy = 0;
  warp_scan2( inc_g, dummy );
  const long long tot_u = __shfl_sync( FULL, inc_u, 31 );
  const long long tot_l = __shfl_sync( FULL, inc_l, 31 );
  const long long tot_g = __shfl_sync( FULL, inc_g, 31 );
  const long long rtot = warp_sum_ll( cnt * rdeg );
  const long long ctot = warp_sum_ll( cnt );
  unsigned long long base = 0, xb = 0, lbase = 0;
  int sel = 0;
  if ( lane == 0 )
  {
    if ( tot_u > 0 )
      base = atomicAdd( &d.ctl->n_ent, ( unsigned long long ) tot_u );
    if ( tot_l > 0 )
    {
      sel = ld_volatile( &d.ctl->late_wr );
      xb = atomicAdd( &d.ctl->n_late[ sel ], ( unsigned long long ) tot_l );
    }
    if ( tot_g > 0 )
      lbase = atomicAdd( &d.ctl->log_count, ( unsigned long long ) tot_g );
    atomicAdd( &d.ctl->syn_events, ( unsigned long long ) rtot );
    atomicAdd( &d.ctl->n_spikes, ( unsigned long long ) ctot );
  }
  base = __shfl_sync( FULL, base, 0 );
  xb = __shfl_sync( FULL, xb, 0 );
  lbase = __shfl_sync( FULL, lbase, 0 );
  sel = __shfl_sync( FULL, sel, 0 );
  if ( cnt == 0 )
    return;
  long long iu = ( long long ) base + inc_u - ( long long ) cnt * rw.nu;
  long long il = ( long long ) xb + inc_l - ( long long ) cnt * rw.nl;
  long long li = ( long long ) lbase + inc_g - ( lg ? cnt : 0 );
  const long long lb0 = lg ? ld_volatile( &d.ctl->log_base ) : 0;
  uint2* const lg_buf = lg ? log_half( d ) : nullptr;
  const uint32_t lsrc = lg ? log_source( d, src ) : 0u;
  unsigned m = mask;
  while ( m )
  {
    const int k = __ffs( m ) - 1;
    m &= m - 1;
    int slot = slot0 + k;
    if ( slot >= d.L )
      slot -= d.L;
    for ( int c = 0; c < rw.nu; ++c )
      put_chunk( d, d.ent, iu + c, rw.row, 0, rw.ue, c, slot, 1 );
    for ( int c = 0; c < rw.nl; ++c )
      put_chunk( d, late_list( d, sel ), il + c, rw.row, rw.ls, rw.pdeg, c, slot, 1 );
    iu += rw.nu;
    il += rw.nl;
    if ( lg )
    {
      if ( li < d.log_cap )
        lg_buf[ li ] = make_uint2( lsrc, ( uint32_t ) ( t0 + k + 1 - lb0 ) | ( 1u << 24 ) );
      else
        atomicOr( &d.ctl->err, ERR_LOG );
      ++li;
    }
  }
}

// The same as warp_append_mask, with the reservations of all warps of the
// CTA combined: one global atomic per counter and CTA (thousands of warps of
// a large network each reserving on the same control-block line serialise
// in L2).  A neuron of a network in gather mode queues no edge chunks (its
// targets gather); spikes are counted per network for the mode choice.  The
// whole warp writes each spike's chunk entries, consecutive lanes
// consecutive entries (a source with thousands of out-edges has dozens).
// Must be called by every thread of the CTA.
__device__ __forceinline__ void
cta_append_mask( const Net& d, unsigned mask, int32_t src, int slot0, long long t0, int netid, bool gath )
{
  const bool tiled = !gath && netid >= 0 && d.net_t != nullptr && d.net_t[ netid ].nt > 0;
  __shared__ unsigned long long s_e, s_x, s_l, s_r, s_c, g_e, g_x, g_l;
  __shared__ int s_any, s_sel;
  const int lane = threadIdx.x & 31;
  if ( threadIdx.x == 0 )
  {
    s_e = s_x = s_l = s_r = s_c = 0ull;
    s_any = 0;
  }
  __syncthreads();
  const int cnt = __popc( mask );
  const bool any = __ballot_sync( FULL, cnt > 0 ) != 0;
  RowWork rw {};
  long long rdeg = 0;
  const bool lg = cnt > 0 && ( d.rec == nullptr || d.rec[ src ] );
  long long inc_u = 0, inc_l = 0, inc_g = 0;
  unsigned long long w_e = 0, w_x = 0, w_l = 0;
  if ( any )
  {
    if ( cnt > 0 )
    {
      // a spike of a tiled network is one work entry (its source), of a
      // network in gather mode none, else its row's chunks
      if ( !gath )
      {
        if ( tiled )
        {
          rw.nu = 1;
          rw.row = d.row_beg[ src ];
        }
        else
          rw = row_work( d, src );
      }
      rdeg = d.real_deg[ src ];
      if ( d.net_spk && netid >= 0 )
      {
        // one atomic per network present in the warp
        const unsigned peers = __match_any_sync( __activemask(), netid );
        const unsigned tot = __reduce_add_sync( peers, ( unsigned ) cnt );
        if ( lane == __ffs( peers ) - 1 )
          atomicAdd( d.net_spk + netid, tot );
      }
    }
    inc_u = ( long long ) cnt * rw.nu;
    inc_l = ( long long ) cnt * rw.nl;
    warp_scan2( inc_u, inc_l );
    long long dummy = 0;
    inc_g = lg ? cnt : 0;
    warp_scan2( inc_g, dummy );
    const long long tot_u = __shfl_sync( FULL, inc_u, 31 );
    const long long tot_l = __shfl_sync( FULL, inc_l, 31 );
    const long long tot_g = __shfl_sync( FULL, inc_g, 31 );
    const long long rtot = warp_sum_ll( cnt * rdeg );
    const long long ctot = warp_sum_ll( cnt );
    if ( lane == 0 )
    {
      w_e = atomicAdd( &s_e, ( unsigned long long ) tot_u );
      w_x = atomicAdd( &s_x, ( unsigned long long ) tot_l );
      w_l = atomicAdd( &s_l, ( unsigned long long ) tot_g );
      atomicAdd( &s_r, ( unsigned long long ) rtot );
      atomicAdd( &s_c, ( unsigned long long ) ctot );
      s_any = 1;
    }
  }
  __syncthreads();
  if ( !s_any )
    return;  // uniform across the CTA
  if ( threadIdx.x == 0 )
  {
    g_e = s_e > 0 ? atomicAdd( &d.ctl->n_ent, s_e ) : 0ull;
    s_sel = 0;
    g_x = 0ull;
    if ( s_x > 0 )
    {
      s_sel = ld_volatile( &d.ctl->late_wr );
      g_x = atomicAdd( &d.ctl->n_late[ s_sel ], s_x );
    }
    g_l = s_l > 0 ? atomicAdd( &d.ctl->log_count, s_l ) : 0ull;
    atomicAdd( &d.ctl->syn_events, s_r );
    atomicAdd( &d.ctl->n_spikes, s_c );
  }
  __syncthreads();
  // every lane takes part in these shuffles (lanes without a spike leave below)
  const long long iu0 = ( long long ) ( g_e + __shfl_sync( FULL, w_e, 0 ) ) + inc_u - ( long long ) cnt * rw.nu;
  const long long il0 = ( long long ) ( g_x + __shfl_sync( FULL, w_x, 0 ) ) + inc_l - ( long long ) cnt * rw.nl;
  long long li = ( long long ) ( g_l + __shfl_sync( FULL, w_l, 0 ) ) + inc_g - ( lg ? cnt : 0 );
  int4* const xlist = late_list( d, s_sel );
  unsigned owners = __ballot_sync( FULL, cnt > 0 && !gath && !tiled && ( rw.nu + rw.nl ) > 0 );
  while ( owners )
  {
    const int ol = __ffs( owners ) - 1;
    owners &= owners - 1;
    const long long o_row = __shfl_sync( FULL, rw.row, ol );
    const int o_pdeg = __shfl_sync( FULL, rw.pdeg, ol );
    const int o_ue = __shfl_sync( FULL, rw.ue, ol );
    const int o_ls = __shfl_sync( FULL, rw.ls, ol );
    const int o_nu = __shfl_sync( FULL, rw.nu, ol );
    const int o_nl = __shfl_sync( FULL, rw.nl, ol );
    long long o_iu = __shfl_sync( FULL, iu0, ol );
    long long o_il = __shfl_sync( FULL, il0, ol );
    unsigned om = __shfl_sync( FULL, mask, ol );
    const int o_slot0 = __shfl_sync( FULL, slot0, ol );
    while ( om )
    {
      const int k = __ffs( om ) - 1;
      om &= om - 1;
      int slot = o_slot0 + k;
      if ( slot >= d.L )
        slot -= d.L;
      for ( int c = lane; c < o_nu; c += 32 )
        put_chunk( d, d.ent, o_iu + c, o_row, 0, o_ue, c, slot, 1 );
      for ( int c = lane; c < o_nl; c += 32 )
        put_chunk( d, xlist, o_il + c, o_row, o_ls, o_pdeg, c, slot, 1 );
      o_iu += o_nu;
      o_il += o_nl;
    }
  }
  if ( cnt == 0 )
    return;
  long long idx = iu0;
  const long long lb0 = lg ? ld_volatile( &d.ctl->log_base ) : 0;
  uint2* const lg_buf = lg ? log_half( d ) : nullptr;
  const uint32_t lsrc = lg ? log_source( d, src ) : 0u;
  unsigned m = mask;
  while ( m )
  {
    const int k = __ffs( m ) - 1;
    m &= m - 1;
    int slot = slot0 + k;
    if ( slot >= d.L )
      slot -= d.L;
    if ( tiled )
    {
      if ( idx < d.ent_cap )
        d.ent[ idx ] = make_int4( src, 0, -1, slot | ( 1 << 16 ) );  // edge count -1: no scatter chunk
      else
        atomicOr( &d.ctl->err, ERR_SPIKE_LIST );
      ++idx;
    }
    if ( lg )
    {
      if ( li < d.log_cap )
        lg_buf[ li ] = make_uint2( lsrc, ( uint32_t ) ( t0 + k + 1 - lb0 ) | ( 1u << 24 ) );
      else
        atomicOr( &d.ctl->err, ERR_LOG );
      ++li;
    }
  }
}

// Steps at which neuron i is simulated: [.., until); a free neuron of a
// serving engine never is.
__device__ __forceinline__ long long
active_until( const Net& d, int64_t i )
{
  if ( d.nid == nullptr )
    return 0x7fffffffffffffffll;
  const int id = d.nid[ i ];
  return id < 0 ? -1ll : d.net_until[ id ];
}

// Read the slice origin once per CTA (a load by every warp of a large grid
// queues thousands of requests on one L2 line).  Call from all threads.
__device__ __forceinline__ long long
cta_origin( const Net& d )
{
  __shared__ long long s_origin;
  if ( threadIdx.x == 0 )
    s_origin = ld_volatile( &d.ctl->origin );
  __syncthreads();
  return s_origin;
}

// Poisson drive of one neuron (generator step t - delay): inversion over
// the neuron's precomputed CDF table (cdf[k] = P(X <= k)), or, for tables
// too long to store, the walk from the mode.  The per-neuron constants are
// loaded once per launch (drive_ctx): inside the lag loop the ring stores
// would otherwise force every one of them to be re-read at every lag.
struct DriveCtx
{
  const uint64_t* cdf;
  uint64_t c[ 4 ];    // the first table thresholds (2^53 past the table's end: never exceeded)
  double w;
  long long t_off;    // global step -> network-local step
  int n;              // table length; 0: no drive; -1: walk from the mode
  int pd;             // delay [steps]
  uint32_t il, k0, k1;
  long long pair;     // generator-step pair of the cached draw (-1: none)
  uint32_t o[ 4 ];    // its Philox words: (o0, o1) even step, (o2, o3) odd step
};

__device__ __forceinline__ void
drive_ctx( const Net& d, int64_t i, DriveCtx& c )
{
  c.n = 0;
  c.pair = -1;
  if ( !d.has_pois )
    return;
  // counter = (neuron, generator step) in the network's local numbering,
  // key = the network's seed: a network draws the same drive wherever and
  // whenever it is placed
  c.t_off = 0;
  c.il = ( uint32_t ) i;
  c.k0 = d.key0;
  c.k1 = d.key1;
  int id = 0;
  if ( d.nid )
  {
    id = d.nid[ i ];
    if ( id < 0 )
      return;  // a free neuron of a serving engine
  }
  const int2 tb = __ldg( d.pois_cdf_ref + i );
  c.n = tb.y;
  if ( tb.y == 0 )
    return;
  if ( d.nid )
  {
    const uint2 kk = d.net_key[ id ];
    c.t_off = d.net_step0[ id ];
    c.il = ( uint32_t ) ( i - d.net_off[ id ] );
    c.k0 = kk.x;
    c.k1 = kk.y;
  }
  c.pd = __ldg( d.pois_d + i );
  c.w = __ldg( d.pois_w + i );
  c.cdf = d.pois_cdf + tb.x;
#pragma unroll
  for ( int q = 0; q < 4; ++q )
    c.c[ q ] = q < tb.y ? __ldg( c.cdf + q ) : ( 1ull << 53 );
}

// One Philox4x32-10 block serves two generator steps: counter (neuron,
// tg >> 1, DRIVE_STREAM), words (o0, o1) for the even step and (o2, o3) for
// the odd one, each turned into a 53-bit uniform.
template < typename Real >
__device__ __forceinline__ Real
drive_at( const Net& d, DriveCtx& c, int64_t i, long long t, long long& cnt )
{
  if ( c.n == 0 )
    return Real( 0 );
  const long long tg = t - c.t_off - c.pd;
  if ( !( d.pois_start < tg && tg <= d.pois_stop ) || tg < 0 )
    return Real( 0 );
  const long long tp = tg >> 1;
  if ( tp != c.pair )
  {
    philox4x32_10( c.il, ( uint32_t ) tp, ( uint32_t ) ( ( unsigned long long ) tp >> 32 ), DRIVE_STREAM, c.k0, c.k1,
      c.o );
    c.pair = tp;
  }
  const uint32_t ua = ( tg & 1 ) ? c.o[ 2 ] : c.o[ 0 ];
  const uint32_t ub = ( tg & 1 ) ? c.o[ 3 ] : c.o[ 1 ];
  long long k;
  if ( c.n > 0 )
  {
    // j = first index with u <= cdf[j] (or the last one), compared as the
    // 53-bit integers of u and of the thresholds (u53_bits)
    const uint64_t m = u53_bits( ua, ub );
    int j = 0;
#pragma unroll
    for ( int q = 0; q < 4; ++q )
      if ( j == q && q < c.n - 1 && m > c.c[ q ] )
        j = q + 1;
    while ( j >= 4 && j < c.n - 1 && m > __ldg( c.cdf + j ) )
      ++j;
    k = j;
  }
  else
  {
    k = poisson_from_mode( d.pois[ i ], u53( ua, ub ) );
  }
  cnt += k;
  if ( k <= 0 )
    return Real( 0 );
  // k < 2^32: a table index or a count walked from the mode
  return ( Real ) ( c.w * u32_to_f64( ( uint32_t ) k ) );
}

// Ring cell of (slot, channel, neuron): read it, then, separately and only
// after the value has been used, clear it.  A load followed at once by a
// store to the same address makes the store wait for the load, and the
// next lag's loads behind it: the reads of a slice's lags would run one
// round trip at a time.
template < bool FIX >
struct RingVal
{
  using type = typename std::conditional< FIX, long long, double >::type;
};

template < bool FIX >
__device__ __forceinline__ typename RingVal< FIX >::type
ring_ld( const Net& d, int slot, int ch, int64_t i )
{
  const int64_t idx = ( ( int64_t ) slot * d.C + ch ) * d.N + i;
  if constexpr ( FIX )
    if ( d.ring32 )
      return reinterpret_cast< const int32_t* >( d.ring )[ idx ];
  return reinterpret_cast< const typename RingVal< FIX >::type* >( d.ring )[ idx ];
}

template < typename Real, bool FIX >
__device__ __forceinline__ Real
ring_real( const Net& d, typename RingVal< FIX >::type v )
{
  // fx_inv is a power of two: rounding v to Real and then scaling gives the
  // same value as scaling in FP64 and then rounding, without the FP64 ops
  if constexpr ( FIX )
    return ( Real ) v * ( Real ) d.fx_inv;
  else
    return ( Real ) v;
}

template < bool FIX >
__device__ __forceinline__ void
ring_clear( const Net& d, int slot, int ch, int64_t i )
{
  const int64_t idx = ( ( int64_t ) slot * d.C + ch ) * d.N + i;
  if constexpr ( FIX )
    if ( d.ring32 )
    {
      reinterpret_cast< int32_t* >( d.ring )[ idx ] = 0;
      return;
    }
  reinterpret_cast< typename RingVal< FIX >::type* >( d.ring )[ idx ] = 0;
}

// vals[slot] holds the model's state variables in slot order.
__device__ __forceinline__ void
trace_put( const Net& d, int64_t i, long long stamp, const double* vals )
{
  if ( d.trace_col == nullptr || ( stamp % d.trace_interval ) != 0 )
    return;
  const int32_t col = d.trace_col[ i ];
  if ( col < 0 )
    return;
  const long long row = stamp / d.trace_interval - ld_volatile( &d.ctl->trace_row0 );
  if ( row >= 0 && row < d.trace_rows )
  {
    for ( int v = 0; v < d.n_trace_vars; ++v )
      d.trace[ ( row * d.n_trace_vars + v ) * d.n_trace_idx + col ] = vals[ d.trace_slot[ v ] ];
  }
  else
  {
    atomicOr( &d.ctl->err, ERR_TRACE );
  }
}

// Drive counts: warp sums, then one atomic per CTA (a same-address atomic
// per warp serialises thousands of L2 atomics at large grids).  Must be
// called by every thread of the CTA.
__device__ __forceinline__ void
flush_drive_count( const Net& d, long long cnt )
{
  __shared__ unsigned long long s_cnt;
  if ( threadIdx.x == 0 )
    s_cnt = 0ull;
  __syncthreads();
  const long long s = warp_sum_ll( cnt );
  if ( ( threadIdx.x & 31 ) == 0 && s > 0 )
    atomicAdd( &s_cnt, ( unsigned long long ) s );
  __syncthreads();
  if ( threadIdx.x == 0 && s_cnt > 0 )
    atomicAdd( &d.ctl->drive_events, s_cnt );
}

// Scheduled generator spikes with emission step in [origin+from, origin+to):
// one warp consumes them in order (CTA 0 of the first block's launch).
__device__ __forceinline__ void
append_scheduled( const Net& d, long long origin, int from, int to )
{
  if ( d.n_sched == 0 )
    return;
  long long pos = ld_volatile( &d.ctl->sched_pos );
  const int lane = threadIdx.x & 31;
  const long long lo = origin + from, hi = origin + to;
  for ( ;; )
  {
    const long long p = pos + lane;
    const bool in_range = p < d.n_sched;
    const long long st = in_range ? d.sched_step[ p ] : hi;
    const bool consumed = in_range && st < hi;
    const bool emit = consumed && st >= lo;
    const int32_t src = emit ? d.sched_src[ p ] : 0;
    warp_append( d, emit, src, emit ? ( int32_t ) ( st % d.L ) : 0, 1, st + 1 );
    const unsigned cm = __ballot_sync( FULL, consumed );
    pos += __popc( cm );
    if ( cm != FULL )
      break;
  }
  if ( lane == 0 )
    d.ctl->sched_pos = pos;
}

// ---------------------------------------------------------------------
// iaf_psc_alpha (models/iaf_psc_alpha.cpp, update): exact integration of
// alpha-shaped currents.  ctab: P11ex (= P22ex), P11in, P21ex, P21in, P30,
// P31ex, P32ex, P31in, P32in, expm1(-h/tau_m), EPSC and IPSC initial values
// (e / tau_syn), Theta, V_reset, LowerBound, RefractoryCounts; state in the
// slots of iaf_psc_exp's layout: V_m - E_L, I_syn_ex, I_syn_in, dI_syn_ex,
// dI_syn_in, I_e.  The operations and their order are the reference's
// (every product and sum rounds on its own: -fmad=false); the model's
// current input y0 is 0 on this path (no CurrentEvent sources).
// ---------------------------------------------------------------------
template < typename Real >
struct AlphaCoef
{
  Real P11e, P11i, P21e, P21i, P30, P31e, P32e, P31i, P32i, em1, Ee, Ei, Vth, Vreset, Vmin;
  int refr;
};

template < typename Real >
__device__ __forceinline__ void
alpha_coef( const double* ct, AlphaCoef< Real >& c )
{
  c.P11e = ( Real ) ct[ 0 ];
  c.P11i = ( Real ) ct[ 1 ];
  c.P21e = ( Real ) ct[ 2 ];
  c.P21i = ( Real ) ct[ 3 ];
  c.P30 = ( Real ) ct[ 4 ];
  c.P31e = ( Real ) ct[ 5 ];
  c.P32e = ( Real ) ct[ 6 ];
  c.P31i = ( Real ) ct[ 7 ];
  c.P32i = ( Real ) ct[ 8 ];
  c.em1 = ( Real ) ct[ 9 ];
  c.Ee = ( Real ) ct[ 10 ];
  c.Ei = ( Real ) ct[ 11 ];
  c.Vth = ( Real ) ct[ 12 ];
  c.Vreset = ( Real ) ct[ 13 ];
  c.Vmin = ( Real ) ct[ 14 ];
  c.refr = ( int ) ct[ 15 ];
}

// one step; ex / inh: this step's ring input per channel (SYN_EX, SYN_IN)
template < typename Real >
__device__ __forceinline__ bool
alpha_step( const AlphaCoef< Real >& c, Real& V, Real& Iex, Real& Iin, Real& dIex, Real& dIin, int& r, const Real Ie,
  const Real ex, const Real inh )
{
  const Real y0 = Real( 0 );
  if ( r == 0 )
  {
    V = c.P30 * ( y0 + Ie ) + c.P31e * dIex + c.P32e * Iex + c.P31i * dIin + c.P32i * Iin + c.em1 * V + V;
    V = ( V < c.Vmin ? c.Vmin : V );
  }
  else
  {
    --r;
  }
  Iex = c.P21e * dIex + c.P11e * Iex;
  dIex *= c.P11e;
  dIex += c.Ee * ex;
  Iin = c.P21i * dIin + c.P11i * Iin;
  dIin *= c.P11i;
  dIin += c.Ei * inh;
  if ( V >= c.Vth )
  {
    r = c.refr;
    V = c.Vreset;
    return true;
  }
  return false;
}

// ---------------------------------------------------------------------
// iaf_psc_delta (models/iaf_psc_delta.cpp:272-329) and iaf_psc_exp
// (models/iaf_psc_exp.cpp:288-348), one thread per neuron.
//
// Used for slices of one or two steps and for large networks, where one
// thread per neuron already gives enough warps to hide memory latency.  The
// lags run in order in registers; spikes are collected as a bit mask per
// chunk of up to 32 lags and appended once per chunk (warp_append_mask).
//
// iaf_psc_delta ctab: P33, P30, V_th, V_reset, V_min, RefractoryCounts
//               state: s0 = y3 (V_m - E_L), s1 = y0, s2 = I_e
// iaf_psc_exp   ctab: P22, P21ex, P21in, P20, P11ex, P11in, Theta, V_reset,
//                     RefractoryCounts, 1 - P11ex
//               state: s0 = V_m - E_L, s1 = i_syn_ex, s2 = i_syn_in,
//                      s3 = i_0, s4 = i_1, s5 = I_e
// ---------------------------------------------------------------------
// Launched with CTAs of 128 threads.  The FP32 form (fixed-point rings)
// caps its registers for five resident CTAs per SM (96 registers, a few
// spills outside the lag loop): on the serving workload, whose many small
// networks fill several waves, the extra resident warps hide more of the
// ring-load and drive latency (update time -6 %).
template < typename Real, bool FIX, int MODEL, int SUB >
__global__ void __launch_bounds__( 128, FIX ? 5 : 1 )
k_update_iaf( Net d, Block b, int from, int to, int sched )
{
  const long long origin = cta_origin( d );
  if ( sched && blockIdx.x == 0 && threadIdx.x < 32 )
    append_scheduled( d, origin, from, to );
  const int64_t li = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = li < b.n;
  const int64_t i = b.off + ( act ? li : 0 );
  const long long until = act ? active_until( d, i ) : -1ll;
  const int netid = ( act && d.nid ) ? d.nid[ i ] : -1;
  const bool gath = netid >= 0 && d.net_mode && d.net_mode[ netid ] != 0;
  // iaf_psc_alpha keeps iaf_psc_exp's two channels and state layout
  constexpr bool ALPHA = MODEL == NG_IAF_PSC_ALPHA_ID;
  constexpr bool EXP = MODEL == NG_IAF_PSC_EXP_ID || ALPHA;
  Real* s0 = ( Real* ) b.s[ 0 ];
  Real* s1 = ( Real* ) b.s[ 1 ];
  Real* s2 = ( Real* ) b.s[ 2 ];
  Real* s3 = ( Real* ) b.s[ 3 ];
  Real* s4 = ( Real* ) b.s[ 4 ];
  Real V = 0, x1 = 0, x2 = 0, i0 = 0, i1 = 0, Ie = 0;
  Real c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0, Vth = 0, Vreset = 0, c9 = 0;
  AlphaCoef< Real > ac {};
  int r = 0, refr = 0;
  if ( act )
  {
    const double* ct = b.ctab + ( int64_t ) b.cls[ li ] * CT_STRIDE;
    if constexpr ( ALPHA )
      alpha_coef< Real >( ct, ac );
    if constexpr ( EXP && !ALPHA )
    {
      c0 = ( Real ) ct[ 0 ];
      c1 = ( Real ) ct[ 1 ];
      c2 = ( Real ) ct[ 2 ];
      c3 = ( Real ) ct[ 3 ];
      c4 = ( Real ) ct[ 4 ];
      c5 = ( Real ) ct[ 5 ];
      Vth = ( Real ) ct[ 6 ];
      Vreset = ( Real ) ct[ 7 ];
      refr = ( int ) ct[ 8 ];
      c9 = ( Real ) ct[ 9 ];
    }
    if constexpr ( EXP )
    {
      V = s0[ li ];
      x1 = s1[ li ];
      x2 = s2[ li ];
      i0 = s3[ li ];
      i1 = s4[ li ];
      Ie = ( ( const Real* ) b.s[ 5 ] )[ li ];
    }
    else
    {
      c0 = ( Real ) ct[ 0 ];
      c1 = ( Real ) ct[ 1 ];
      Vth = ( Real ) ct[ 2 ];
      Vreset = ( Real ) ct[ 3 ];
      c2 = ( Real ) ct[ 4 ];
      refr = ( int ) ct[ 5 ];
      V = s0[ li ];
      x1 = s1[ li ];
      Ie = s2[ li ];
    }
    r = b.r[ li ];
  }
  DriveCtx dc;
  dc.n = 0;
  if ( act )
    drive_ctx( d, i, dc );
  long long dcnt = 0;
  // SUB: lags whose inputs are gathered before the recurrence runs over them
  // (8; 1 for slices of one step, where the unrolled code would only cost
  // instruction fetch)
  for ( int cb = from; cb < to; cb += 32 )
  {
    const int nl = min( 32, to - cb );
    const long long t0 = origin + cb;
    const int slot0 = ( int ) ( t0 % d.L );
    // lags of this chunk the neuron is simulated at: [0, nact)
    const int nact = act ? ( int ) max( 0ll, min( ( long long ) nl, until - t0 ) ) : 0;
    unsigned smask = 0;
    for ( int sb = 0; sb < nl; sb += SUB )
    {
      // inputs of up to SUB lags: the ring reads and drive draws of all of
      // them issued before any is used
      typename RingVal< FIX >::type raw_ex[ SUB ], raw_in[ SUB ];
      Real dvs[ SUB ];
#pragma unroll
      for ( int q = 0; q < SUB; ++q )
      {
        raw_ex[ q ] = 0;
        raw_in[ q ] = 0;
        dvs[ q ] = Real( 0 );
        const int k = sb + q;
        if ( k < nact )
        {
          int slot = slot0 + k;
          if ( slot >= d.L )
            slot -= d.L;
          raw_ex[ q ] = ring_ld< FIX >( d, slot, 0, i );
          if constexpr ( EXP )
            raw_in[ q ] = ring_ld< FIX >( d, slot, 1, i );
          dvs[ q ] = drive_at< Real >( d, dc, i, t0 + k, dcnt );
        }
      }
      // the recurrence over these lags, in order
#pragma unroll
      for ( int q = 0; q < SUB; ++q )
      {
        const int k = sb + q;
        if ( k >= nact )
          continue;
        Real ex = ring_real< Real, FIX >( d, raw_ex[ q ] );
        Real inh = EXP ? ring_real< Real, FIX >( d, raw_in[ q ] ) : Real( 0 );
        const Real dv = dvs[ q ];
        if ( dv != Real( 0 ) )
        {
          if constexpr ( EXP )
          {
            if ( dv > Real( 0 ) )
              ex = ex + dv;
            else
              inh = inh + dv;
          }
          else
          {
            ex = ex + dv;
          }
        }
        bool spk = false;
        if constexpr ( ALPHA )
        {
          spk = alpha_step< Real >( ac, V, x1, x2, i0, i1, r, Ie, ex, inh );
        }
        else if constexpr ( EXP )
        {
          if ( r == 0 )
            V = V * c0 + x1 * c1 + x2 * c2 + ( Ie + i0 ) * c3;
          else
            --r;
          x1 *= c4;
          x2 *= c5;
          x1 += c9 * i1;
          x1 += ex;
          x2 += inh;
          if ( V >= Vth )
          {
            r = refr;
            V = Vreset;
            spk = true;
          }
          i0 = Real( 0 );
          i1 = Real( 0 );
        }
        else
        {
          if ( r == 0 )
          {
            V = c1 * ( x1 + Ie ) + c0 * V + ex;
            V = ( V < c2 ? c2 : V );
          }
          else
          {
            --r;
          }
          if ( V >= Vth )
          {
            r = refr;
            V = Vreset;
            spk = true;
          }
          x1 = Real( 0 );
        }
        if ( spk )
          smask |= 1u << k;
        if ( d.trace_col )
        {
          if constexpr ( EXP )
          {
            const double vals[ 6 ] = { ( double ) V, ( double ) x1, ( double ) x2, ( double ) i0, ( double ) i1,
              ( double ) Ie };
            trace_put( d, i, t0 + k + 1, vals );
          }
          else
          {
            const double vals[ 3 ] = { ( double ) V, ( double ) x1, ( double ) Ie };
            trace_put( d, i, t0 + k + 1, vals );
          }
        }
      }
      // clear the cells read (their loads have completed)
#pragma unroll
      for ( int q = 0; q < SUB; ++q )
      {
        const int k = sb + q;
        if ( k < nact )
        {
          int slot = slot0 + k;
          if ( slot >= d.L )
            slot -= d.L;
          ring_clear< FIX >( d, slot, 0, i );
          if constexpr ( EXP )
            ring_clear< FIX >( d, slot, 1, i );
        }
      }
    }
    if ( d.gmask && act )
    {
      // lag bits of the slice for the gather (min_delay <= 32: one chunk)
      if ( cb == 0 )
        d.gmask[ i ] = smask;
      else
        d.gmask[ i ] |= smask << cb;
    }
    cta_append_mask( d, smask, ( int32_t ) i, slot0, t0, netid, gath );
  }
  flush_drive_count( d, dcnt );
  // only neurons simulated in this launch write their state back: a free
  // neuron's state may be in the middle of an admission's upload
  if ( act && until > origin + from )
  {
    s0[ li ] = V;
    s1[ li ] = x1;
    if constexpr ( EXP )
    {
      s2[ li ] = x2;
      s3[ li ] = i0;
      s4[ li ] = i1;
    }
    b.r[ li ] = r;
  }
}

// ---------------------------------------------------------------------
// Two-phase variant for slices of 3 or more lags.  A CTA serves 32 neurons.
// Phase 1: all 256 threads read and clear the ring slots and draw the
// Poisson drive of the CTA's (neuron, lag) pairs -- the state-independent,
// latency-heavy part -- into shared memory, coalesced across neurons.
// Phase 2: warp 0 runs the state recurrence, one lane per neuron, reading
// its inputs from shared memory, and appends each lag's spikes with one
// ballot.  Same arithmetic, in the same order, as k_update_iaf.
// ---------------------------------------------------------------------
constexpr int P2_NB = 32;  // neurons per CTA

// TPB threads per CTA, CH lags per chunk (the autotuner picks between
// 256 threads with chunks of 32 lags and 128 threads with chunks of 16:
// the same phase-1 items per thread, half the CTA -- more CTAs resident
// per SM where the registers of the 256-thread form allow only one)
template < typename Real, bool FIX, int MODEL, int TPB, int CH >
__global__ void __launch_bounds__( TPB )
k_update_iaf2( Net d, Block b, int from, int to, int sched )
{
  // iaf_psc_alpha keeps iaf_psc_exp's two channels and state layout
  constexpr bool ALPHA = MODEL == NG_IAF_PSC_ALPHA_ID;
  constexpr bool EXP = MODEL == NG_IAF_PSC_EXP_ID || ALPHA;
  constexpr int P2_CH = CH;
  static_assert( TPB % 32 == 0 && CH <= 32 && ( CH * P2_NB ) % TPB == 0, "two-phase update shape" );
  __shared__ Real s_ex[ P2_CH ][ P2_NB ];
  __shared__ Real s_in[ EXP ? P2_CH : 1 ][ P2_NB ];
  const long long origin = cta_origin( d );
  if ( sched && blockIdx.x == 0 && threadIdx.x < 32 )
    append_scheduled( d, origin, from, to );
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t nb0 = ( int64_t ) blockIdx.x * P2_NB;
  const int64_t li = nb0 + lane;
  const bool act = warp == 0 && li < b.n;
  const int64_t i = b.off + ( act ? li : 0 );
  const long long until = act ? active_until( d, i ) : -1ll;
  Real* s0 = ( Real* ) b.s[ 0 ];
  Real* s1 = ( Real* ) b.s[ 1 ];
  Real* s2 = ( Real* ) b.s[ 2 ];
  Real* s3 = ( Real* ) b.s[ 3 ];
  Real* s4 = ( Real* ) b.s[ 4 ];
  Real V = 0, x1 = 0, x2 = 0, i0 = 0, i1 = 0, Ie = 0;
  Real c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0, Vth = 0, Vreset = 0, c9 = 0;
  AlphaCoef< Real > ac {};
  int r = 0, refr = 0;
  if ( act )
  {
    const double* ct = b.ctab + ( int64_t ) b.cls[ li ] * CT_STRIDE;
    if constexpr ( ALPHA )
      alpha_coef< Real >( ct, ac );
    if constexpr ( EXP && !ALPHA )
    {
      c0 = ( Real ) ct[ 0 ];
      c1 = ( Real ) ct[ 1 ];
      c2 = ( Real ) ct[ 2 ];
      c3 = ( Real ) ct[ 3 ];
      c4 = ( Real ) ct[ 4 ];
      c5 = ( Real ) ct[ 5 ];
      Vth = ( Real ) ct[ 6 ];
      Vreset = ( Real ) ct[ 7 ];
      refr = ( int ) ct[ 8 ];
      c9 = ( Real ) ct[ 9 ];
    }
    if constexpr ( EXP )
    {
      V = s0[ li ];
      x1 = s1[ li ];
      x2 = s2[ li ];
      i0 = s3[ li ];
      i1 = s4[ li ];
      Ie = ( ( const Real* ) b.s[ 5 ] )[ li ];
    }
    else
    {
      c0 = ( Real ) ct[ 0 ];
      c1 = ( Real ) ct[ 1 ];
      Vth = ( Real ) ct[ 2 ];
      Vreset = ( Real ) ct[ 3 ];
      c2 = ( Real ) ct[ 4 ];
      refr = ( int ) ct[ 5 ];
      V = s0[ li ];
      x1 = s1[ li ];
      Ie = s2[ li ];
    }
    r = b.r[ li ];
  }
  // phase 1 items j = threadIdx.x + m * TPB all belong to neuron nb0 + (threadIdx.x & 31)
  DriveCtx dc;
  dc.n = 0;
  if ( nb0 + ( threadIdx.x & 31 ) < b.n )
    drive_ctx( d, b.off + nb0 + ( threadIdx.x & 31 ), dc );
  long long dcnt = 0;
  for ( int cb = from; cb < to; cb += P2_CH )
  {
    const int nl = min( P2_CH, to - cb );
    const long long t0 = origin + cb;
    const int slot0 = ( int ) ( t0 % d.L );
    // ---- phase 1: inputs of (neuron q, lag k), item j = k * 32 + q; a
    // thread's items j = threadIdx.x + m * TPB (m < P1_MAX): all ring reads
    // and draws first, then their use, then the clears
    constexpr int P1_MAX = P2_CH * P2_NB / TPB;
    typename RingVal< FIX >::type rex[ P1_MAX ], rin[ P1_MAX ];
    Real dvs[ P1_MAX ];
    int slots[ P1_MAX ];
#pragma unroll
    for ( int m = 0; m < P1_MAX; ++m )
    {
      const int j = threadIdx.x + m * TPB;
      rex[ m ] = 0;
      rin[ m ] = 0;
      dvs[ m ] = Real( 0 );
      slots[ m ] = -1;
      if ( j < nl * P2_NB )
      {
        const int k = j >> 5;
        const int64_t lq = nb0 + ( j & 31 );
        if ( lq < b.n && t0 + k < active_until( d, b.off + lq ) )
        {
          const int64_t iq = b.off + lq;
          int slot = slot0 + k;
          if ( slot >= d.L )
            slot -= d.L;
          slots[ m ] = slot;
          rex[ m ] = ring_ld< FIX >( d, slot, 0, iq );
          if constexpr ( EXP )
            rin[ m ] = ring_ld< FIX >( d, slot, 1, iq );
          dvs[ m ] = drive_at< Real >( d, dc, iq, t0 + k, dcnt );
        }
      }
    }
#pragma unroll
    for ( int m = 0; m < P1_MAX; ++m )
    {
      const int j = threadIdx.x + m * TPB;
      if ( j >= nl * P2_NB )
        continue;
      const int k = j >> 5;
      const int q = j & 31;
      Real ex = 0, inh = 0;
      if ( slots[ m ] >= 0 )
      {
        ex = ring_real< Real, FIX >( d, rex[ m ] );
        if constexpr ( EXP )
          inh = ring_real< Real, FIX >( d, rin[ m ] );
        const Real dv = dvs[ m ];
        if ( dv != Real( 0 ) )
        {
          if constexpr ( EXP )
          {
            if ( dv > Real( 0 ) )
              ex = ex + dv;
            else
              inh = inh + dv;
          }
          else
          {
            ex = ex + dv;
          }
        }
      }
      s_ex[ k ][ q ] = ex;
      if constexpr ( EXP )
        s_in[ k ][ q ] = inh;
    }
#pragma unroll
    for ( int m = 0; m < P1_MAX; ++m )
    {
      if ( slots[ m ] < 0 )
        continue;
      const int64_t iq = b.off + nb0 + ( ( threadIdx.x + m * TPB ) & 31 );
      ring_clear< FIX >( d, slots[ m ], 0, iq );
      if constexpr ( EXP )
        ring_clear< FIX >( d, slots[ m ], 1, iq );
    }
    __syncthreads();
    // ---- phase 2: the recurrence, one lane per neuron
    if ( warp == 0 )
    {
      int slot = slot0;
      unsigned smask = 0;
      for ( int k = 0; k < nl; ++k )
      {
        bool spk = false;
        if ( act && t0 + k < until )
        {
          const Real in_ex = s_ex[ k ][ lane ];
          if constexpr ( ALPHA )
          {
            spk = alpha_step< Real >( ac, V, x1, x2, i0, i1, r, Ie, in_ex, s_in[ k ][ lane ] );
          }
          else if constexpr ( EXP )
          {
            const Real in_in = s_in[ k ][ lane ];
            if ( r == 0 )
              V = V * c0 + x1 * c1 + x2 * c2 + ( Ie + i0 ) * c3;
            else
              --r;
            x1 *= c4;
            x2 *= c5;
            x1 += c9 * i1;
            x1 += in_ex;
            x2 += in_in;
            if ( V >= Vth )
            {
              r = refr;
              V = Vreset;
              spk = true;
            }
            i0 = Real( 0 );
            i1 = Real( 0 );
          }
          else
          {
            if ( r == 0 )
            {
              V = c1 * ( x1 + Ie ) + c0 * V + in_ex;
              V = ( V < c2 ? c2 : V );
            }
            else
            {
              --r;
            }
            if ( V >= Vth )
            {
              r = refr;
              V = Vreset;
              spk = true;
            }
            x1 = Real( 0 );
          }
        }
        if ( spk )
          smask |= 1u << k;
        if ( act && t0 + k < until && d.trace_col )
        {
          if constexpr ( EXP )
          {
            const double vals[ 6 ] = { ( double ) V, ( double ) x1, ( double ) x2, ( double ) i0, ( double ) i1,
              ( double ) Ie };
            trace_put( d, i, t0 + k + 1, vals );
          }
          else
          {
            const double vals[ 3 ] = { ( double ) V, ( double ) x1, ( double ) Ie };
            trace_put( d, i, t0 + k + 1, vals );
          }
        }
        if ( ++slot == d.L )
          slot = 0;
      }
      warp_append_mask( d, smask, ( int32_t ) i, slot0, t0 );
    }
    __syncthreads();
  }
  flush_drive_count( d, dcnt );
  // only neurons simulated in this launch write their state back: a free
  // neuron's state may be in the middle of an admission's upload
  if ( act && until > origin + from )
  {
    s0[ li ] = V;
    s1[ li ] = x1;
    if constexpr ( EXP )
    {
      s2[ li ] = x2;
      s3[ li ] = i0;
      s4[ li ] = i1;
    }
    b.r[ li ] = r;
  }
}

// ---------------------------------------------------------------------
// aeif_cond_alpha (models/aeif_cond_alpha.cpp:74-126, 450-533) with a
// per-neuron adaptive Runge-Kutta-Fehlberg 4(5) step in FP64.
// ctab: V_peak, V_reset, g_L, C_m, E_ex, E_in, E_L, Delta_T, tau_w, a, b, V_th,
//       tau_syn_ex, tau_syn_in, tol, g0_ex, g0_in, V_peak_eff, RefractoryCounts
// state: s0..s5 = V, dg_ex, g_ex, dg_in, g_in, w; s6 = I_e; istep (FP64)
// ---------------------------------------------------------------------
struct AeifPar
{
  double V_peak, V_reset, g_L, C_m, E_ex, E_in, E_L, Delta_T, tau_w, a, b, V_th, tau_ex, tau_in, I_e;
  // reciprocals of the divisors, set once per launch (aeif_reciprocals)
  double inv_Delta_T, inv_C_m, inv_tau_w, inv_tau_ex, inv_tau_in;
};

__device__ __forceinline__ void
aeif_reciprocals( AeifPar& p )
{
  p.inv_Delta_T = p.Delta_T == 0. ? 0. : 1.0 / p.Delta_T;
  p.inv_C_m = 1.0 / p.C_m;
  p.inv_tau_w = 1.0 / p.tau_w;
  p.inv_tau_ex = 1.0 / p.tau_ex;
  p.inv_tau_in = 1.0 / p.tau_in;
}

// The right-hand side of aeif_cond_alpha (aeif_cond_alpha.cpp:74-126), with
// each division by a parameter taken as a multiplication by its reciprocal
// (within an ulp per operation of the reference's quotients): seven FP64
// divisions per evaluation, seven evaluations per RKF45 attempt, were most
// of an attempt's instructions and two of them sat on the V chain.
__device__ __forceinline__ void
aeif_rhs( const AeifPar& p, bool refr, const double* y, double* f )
{
  const double V = refr ? p.V_reset : fmin( y[ 0 ], p.V_peak );
  const double I_syn_exc = y[ 2 ] * ( V - p.E_ex );
  const double I_syn_inh = y[ 4 ] * ( V - p.E_in );
  const double I_spike = p.Delta_T == 0. ? 0. : ( p.g_L * p.Delta_T * exp( ( V - p.V_th ) * p.inv_Delta_T ) );
  // the other currents are summed while the exponential is evaluated; the
  // spike current joins last (one add and one multiply after the exp)
  const double I_rest = -p.g_L * ( V - p.E_L ) - I_syn_exc - I_syn_inh - y[ 5 ] + p.I_e;
  f[ 0 ] = refr ? 0. : ( I_rest + I_spike ) * p.inv_C_m;
  f[ 1 ] = -y[ 1 ] * p.inv_tau_ex;
  f[ 2 ] = y[ 1 ] - y[ 2 ] * p.inv_tau_ex;
  f[ 3 ] = -y[ 3 ] * p.inv_tau_in;
  f[ 4 ] = y[ 3 ] - y[ 4 ] * p.inv_tau_in;
  f[ 5 ] = ( p.a * ( V - p.E_L ) - y[ 5 ] ) * p.inv_tau_w;
}

// Fehlberg 4(5): advance with the fifth-order weights; error = 5th - 4th.
__device__ __forceinline__ void
rkf45( const AeifPar& p, bool refr, const double* y, const double* k1, double hs, double* yn, double* err, double* fout )
{
  // Each stage's weighted sum as a chain of fused multiply-adds with the
  // newest slope last, so that only two dependent operations follow the
  // previous stage's right-hand side.
  double k2[ 6 ], k3[ 6 ], k4[ 6 ], k5[ 6 ], k6[ 6 ], yt[ 6 ];
#pragma unroll
  for ( int i = 0; i < 6; ++i )
    yt[ i ] = fma( hs, ( 1.0 / 4.0 ) * k1[ i ], y[ i ] );
  aeif_rhs( p, refr, yt, k2 );
#pragma unroll
  for ( int i = 0; i < 6; ++i )
    yt[ i ] = fma( hs, fma( 9.0 / 32.0, k2[ i ], ( 3.0 / 32.0 ) * k1[ i ] ), y[ i ] );
  aeif_rhs( p, refr, yt, k3 );
#pragma unroll
  for ( int i = 0; i < 6; ++i )
    yt[ i ] = fma( hs, fma( 7296.0 / 2197.0, k3[ i ], fma( -7200.0 / 2197.0, k2[ i ], ( 1932.0 / 2197.0 ) * k1[ i ] ) ),
      y[ i ] );
  aeif_rhs( p, refr, yt, k4 );
#pragma unroll
  for ( int i = 0; i < 6; ++i )
    yt[ i ] = fma( hs,
      fma( -845.0 / 4104.0, k4[ i ], fma( 3680.0 / 513.0, k3[ i ], fma( -8.0, k2[ i ], ( 439.0 / 216.0 ) * k1[ i ] ) ) ),
      y[ i ] );
  aeif_rhs( p, refr, yt, k5 );
#pragma unroll
  for ( int i = 0; i < 6; ++i )
    yt[ i ] = fma( hs,
      fma( -11.0 / 40.0, k5[ i ],
        fma( 1859.0 / 4104.0, k4[ i ], fma( -3544.0 / 2565.0, k3[ i ], fma( 2.0, k2[ i ], ( -8.0 / 27.0 ) * k1[ i ] ) ) ) ),
      y[ i ] );
  aeif_rhs( p, refr, yt, k6 );
#pragma unroll
  for ( int i = 0; i < 6; ++i )
  {
    const double d5 = fma( 2.0 / 55.0, k6[ i ],
      fma( -9.0 / 50.0, k5[ i ],
        fma( 28561.0 / 56430.0, k4[ i ], fma( 6656.0 / 12825.0, k3[ i ], ( 16.0 / 135.0 ) * k1[ i ] ) ) ) );
    yn[ i ] = fma( hs, d5, y[ i ] );
    err[ i ] = hs
      * fma( 2.0 / 55.0, k6[ i ],
        fma( 1.0 / 50.0, k5[ i ],
          fma( -2197.0 / 75240.0, k4[ i ], fma( -128.0 / 4275.0, k3[ i ], ( 1.0 / 360.0 ) * k1[ i ] ) ) ) );
  }
  aeif_rhs( p, refr, yn, fout );
}

// Step-size control with D_i = tol + tol * h |y'_i|; q = 5 (stepper order).
__device__ __forceinline__ int
control_yp( double tol, const double* err, const double* f, double& hs )
{
  const double h_old = hs;
  // the largest |err_i| / D_i, found by cross-multiplied comparisons (the
  // D_i are positive) with one division for the winner
  double en = 0.0, ed = 1.0;
#pragma unroll
  for ( int i = 0; i < 6; ++i )
  {
    const double D0 = fabs( tol * fabs( h_old * f[ i ] ) + tol );
    const double e = fabs( err[ i ] );
    if ( e * ed > en * D0 )
    {
      en = e;
      ed = D0;
    }
  }
  double rmax = en / ed;
  rmax = rmax > 2.2250738585072014e-308 ? rmax : 2.2250738585072014e-308;
  if ( rmax > 1.1 )
  {
    // (rmax^(1/5) as exp(log(rmax) / 5): rmax > 1.1 is finite and positive)
    double r = 0.9 / exp( log( rmax ) * ( 1.0 / 5.0 ) );
    if ( r < 0.2 )
      r = 0.2;
    hs = r * h_old;
    return -1;
  }
  if ( rmax < 0.5 )
  {
    // 0.9 / rmax^(1/6) >= 5 below (0.9 / 5)^6: the growth is capped there
    double r = rmax <= 3.4012224e-05 ? 5.0 : 0.9 / exp( log( rmax ) * ( 1.0 / 6.0 ) );
    if ( r > 5.0 )
      r = 5.0;
    if ( r < 1.0 )
      r = 1.0;
    hs = r * h_old;
    return 1;
  }
  return 0;
}

// Substep binning of aeif_cond_alpha: a neuron near a spike takes many
// adaptive RKF45 sub-steps per step, a quiet one a single step, and a warp
// runs as long as its slowest lane.  Before each slice the neurons are
// ordered by their last step size (bucket k: h / 2^k > hs >= h / 2^(k+1),
// a counting sort), and the update kernel's thread j simulates neuron
// perm[j], so the neurons of a warp need similar numbers of sub-steps.  The
// order changes only which thread computes a neuron, not any arithmetic.
constexpr int AEIF_BINS = 16;

__device__ __forceinline__ int
aeif_bin( double hs, double h )
{
  if ( !( hs < h ) )
    return 0;
  const int k = 1 + ( int ) floor( log2( h / hs ) );
  return k < AEIF_BINS - 1 ? k : AEIF_BINS - 1;
}

// counts[0..BINS) histogram, counts[BINS..2 BINS) fill positions (zeroed here)
__global__ void
k_aeif_bin_count( const double* istep, int64_t n, double h, unsigned* counts )
{
  __shared__ unsigned s_h[ AEIF_BINS ];
  if ( threadIdx.x < AEIF_BINS )
    s_h[ threadIdx.x ] = 0u;
  __syncthreads();
  for ( int64_t i = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += ( int64_t ) gridDim.x * blockDim.x )
    atomicAdd( &s_h[ aeif_bin( istep[ i ], h ) ], 1u );
  __syncthreads();
  if ( threadIdx.x < AEIF_BINS && s_h[ threadIdx.x ] )
    atomicAdd( &counts[ threadIdx.x ], s_h[ threadIdx.x ] );
}

__global__ void
k_aeif_bin_scatter( const double* istep, int64_t n, double h, unsigned* counts, int32_t* perm )
{
  __shared__ unsigned s_off[ AEIF_BINS ];
  if ( threadIdx.x == 0 )
  {
    unsigned acc = 0;
    for ( int k = 0; k < AEIF_BINS; ++k )
    {
      s_off[ k ] = acc;
      acc += counts[ k ];
    }
  }
  __syncthreads();
  for ( int64_t i = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += ( int64_t ) gridDim.x * blockDim.x )
  {
    const int k = aeif_bin( istep[ i ], h );
    const unsigned pos = s_off[ k ] + atomicAdd( &counts[ AEIF_BINS + k ], 1u );
    perm[ pos ] = ( int32_t ) i;
  }
}

template < typename Real, bool FIX >
__global__ void __launch_bounds__( 64, 6 )
k_update_aeif( Net d, Block b, int from, int to, int sched, double h )
{
  const long long origin = cta_origin( d );
  if ( sched && blockIdx.x == 0 && threadIdx.x < 32 )
    append_scheduled( d, origin, from, to );
  const int64_t gj = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = gj < b.n;
  const int64_t li = ( act && b.perm ) ? ( int64_t ) b.perm[ gj ] : gj;
  const int64_t i = b.off + ( act ? li : 0 );
  const long long until = act ? active_until( d, i ) : -1ll;
  Real* sy[ 6 ];
#pragma unroll
  for ( int k = 0; k < 6; ++k )
    sy[ k ] = ( Real* ) b.s[ k ];
  AeifPar p {};
  double y[ 6 ] = { 0, 0, 0, 0, 0, 0 };
  double tol = 0, g0ex = 0, g0in = 0, Vpk = 0, hs = h;
  int r = 0, refr = 0;
  if ( act )
  {
    const double* ct = b.ctab + ( int64_t ) b.cls[ li ] * CT_STRIDE;
    p.V_peak = ct[ 0 ];
    p.V_reset = ct[ 1 ];
    p.g_L = ct[ 2 ];
    p.C_m = ct[ 3 ];
    p.E_ex = ct[ 4 ];
    p.E_in = ct[ 5 ];
    p.E_L = ct[ 6 ];
    p.Delta_T = ct[ 7 ];
    p.tau_w = ct[ 8 ];
    p.a = ct[ 9 ];
    p.b = ct[ 10 ];
    p.V_th = ct[ 11 ];
    p.tau_ex = ct[ 12 ];
    p.tau_in = ct[ 13 ];
    tol = ct[ 14 ];
    g0ex = ct[ 15 ];
    g0in = ct[ 16 ];
    Vpk = ct[ 17 ];
    refr = ( int ) ct[ 18 ];
    p.I_e = ( double ) ( ( const Real* ) b.s[ 6 ] )[ li ];
    aeif_reciprocals( p );
#pragma unroll
    for ( int k = 0; k < 6; ++k )
      y[ k ] = ( double ) sy[ k ][ li ];
    r = b.r[ li ];
    hs = b.istep[ li ];
  }
  DriveCtx dc;
  dc.n = 0;
  if ( act )
    drive_ctx( d, i, dc );
  long long t = origin + from;
  int slot = ( int ) ( t % d.L );
  long long dcnt = 0;
  bool unstable = false;
  for ( int lag = from; lag < to; ++lag, ++t )
  {
    int mult = 0;
    const bool live = act && t < until;
    // this lag's ring cells, read before the integration so the loads overlap it
    typename RingVal< FIX >::type rex = 0, rin = 0;
    if ( live && !unstable )
    {
      rex = ring_ld< FIX >( d, slot, 0, i );
      rin = ring_ld< FIX >( d, slot, 1, i );
    }
    if ( live && !unstable )
    {
      double tt = 0.0;
      int guard = 0;
      // k1 = f(y) at the start of a sub-step: the previous accepted
      // attempt's f(y_new) when y was not reset after it (the same function
      // of the same values), else evaluated
      double k1[ 6 ];
      bool k1_ok = false;
      while ( tt < h )
      {
        // one accepted sub-step (evolve_apply), retried on rejection
        const double t0 = tt;
        const double dt = h - t0;
        double h0 = hs;
        double yn[ 6 ], err[ 6 ], fo[ 6 ];
        if ( !k1_ok )
          aeif_rhs( p, r > 0, y, k1 );
        for ( ;; )
        {
          bool final_step = false;
          if ( h0 > dt )
          {
            h0 = dt;
            final_step = true;
          }
          rkf45( p, r > 0, y, k1, h0, yn, err, fo );
          tt = final_step ? h : t0 + h0;
          const double h_old = h0;
          const int adj = control_yp( tol, err, fo, h0 );
          if ( adj < 0 )
          {
            const double t_next = tt + h0;
            if ( fabs( h0 ) < fabs( h_old ) && t_next != tt && ++guard < 100000 )
              continue;
            h0 = h_old;
          }
          break;
        }
#pragma unroll
        for ( int k = 0; k < 6; ++k )
          y[ k ] = yn[ k ];
        hs = h0;
        if ( y[ 0 ] < -1e3 || y[ 5 ] < -1e6 || y[ 5 ] > 1e6 || ++guard >= 100000 )
        {
          unstable = true;
          break;
        }
        k1_ok = false;
        if ( r > 0 )
        {
          y[ 0 ] = p.V_reset;
        }
        else if ( y[ 0 ] >= Vpk )
        {
          y[ 0 ] = p.V_reset;
          y[ 5 ] += p.b;
          r = refr > 0 ? refr + 1 : 0;
          ++mult;
        }
        else
        {
#pragma unroll
          for ( int k = 0; k < 6; ++k )
            k1[ k ] = fo[ k ];
          k1_ok = true;
        }
      }
      if ( r > 0 )
        --r;
      Real ex = ring_real< Real, FIX >( d, rex );
      Real inh = ring_real< Real, FIX >( d, rin );
      ring_clear< FIX >( d, slot, 0, i );
      ring_clear< FIX >( d, slot, 1, i );
      const Real dv = drive_at< Real >( d, dc, i, t, dcnt );
      if ( dv != Real( 0 ) )
      {
        if ( dv > Real( 0 ) )
          ex = ex + dv;
        else
          inh = inh - dv;
      }
      y[ 1 ] += ( double ) ex * g0ex;
      y[ 3 ] += ( double ) inh * g0in;
      if constexpr ( sizeof( Real ) == 4 )
      {
#pragma unroll
        for ( int k = 0; k < 6; ++k )
          y[ k ] = ( double ) ( float ) y[ k ];
      }
    }
    warp_append( d, mult > 0, ( int32_t ) i, slot, mult, t + 1 );
    if ( live && d.trace_col )
    {
      const double vals[ 7 ] = { y[ 0 ], y[ 1 ], y[ 2 ], y[ 3 ], y[ 4 ], y[ 5 ], p.I_e };
      trace_put( d, i, t + 1, vals );
    }
    if ( ++slot == d.L )
      slot = 0;
  }
  flush_drive_count( d, dcnt );
  if ( unstable )
    atomicOr( &d.ctl->err, ERR_NUMERIC );
  if ( act && until > origin + from )
  {
#pragma unroll
    for ( int k = 0; k < 6; ++k )
      sy[ k ][ li ] = ( Real ) y[ k ];
    b.r[ li ] = r;
    b.istep[ li ] = hs;
  }
}

// One lane's share of an edge chunk: 4 edge words and 4 weights.
template < bool FIX >
struct ChunkLane
{
  uint32_t t[ 4 ];
  typename std::conditional< FIX, int32_t, double >::type w[ 4 ];
  int slot0, mult;
};

template < bool FIX >
__device__ __forceinline__ void
load_chunk( const Net& d, const int4 en, const int lane, ChunkLane< FIX >& c )
{
  const int j = lane << 2;
  c.slot0 = en.w & 0xffff;
  c.mult = en.w >> 16;
  if ( j < en.z )
  {
    const long long edge = ( ( ( long long ) en.y << 32 ) | ( unsigned ) en.x ) + j;
    const uint4 tdc = __ldg( reinterpret_cast< const uint4* >( d.edge_tdc + edge ) );
    c.t[ 0 ] = tdc.x;
    c.t[ 1 ] = tdc.y;
    c.t[ 2 ] = tdc.z;
    c.t[ 3 ] = tdc.w;
    if constexpr ( FIX )
    {
      const int4 w4 = __ldg( reinterpret_cast< const int4* >( ( const int32_t* ) d.edge_w + edge ) );
      c.w[ 0 ] = w4.x;
      c.w[ 1 ] = w4.y;
      c.w[ 2 ] = w4.z;
      c.w[ 3 ] = w4.w;
    }
    else
    {
      const double2* wp = reinterpret_cast< const double2* >( ( const double* ) d.edge_w + edge );
      const double2 wa = __ldg( wp ), wb = __ldg( wp + 1 );
      c.w[ 0 ] = wa.x;
      c.w[ 1 ] = wa.y;
      c.w[ 2 ] = wb.x;
      c.w[ 3 ] = wb.y;
    }
  }
  else
  {
#pragma unroll
    for ( int k = 0; k < 4; ++k )
    {
      c.t[ k ] = 0u;
      c.w[ k ] = 0;
    }
  }
}

template < bool FIX, bool LATE >
__device__ __forceinline__ void
apply_chunk( const Net& d, const ChunkLane< FIX >& c )
{
#pragma unroll
  for ( int k = 0; k < 4; ++k )
  {
    const int dl = ( int ) ( ( c.t[ k ] >> d.tbits ) & d.dmask );
    // each delivery applies the delays of its own class
    if ( c.w[ k ] == 0 || ( dl >= d.late_min ) != LATE )
      continue;
    const uint32_t tgt = c.t[ k ] & d.tmask;
    int slot = c.slot0 + dl;
    if ( slot >= d.L )
      slot -= d.L;
    const int64_t idx = ( ( int64_t ) slot * d.C + ( c.t[ k ] >> 31 ) ) * d.N + tgt;
    if constexpr ( FIX )
    {
      if ( d.ring32 )  // the admission bound keeps every cell inside 32 bits
        atomicAdd( ( int* ) d.ring + idx, c.w[ k ] * c.mult );
      else
        atomicAdd( ( unsigned long long* ) d.ring + idx,
          ( unsigned long long ) ( ( long long ) c.w[ k ] * ( long long ) c.mult ) );
    }
    else
      atomicAdd( ( double* ) d.ring + idx, c.mult == 1 ? c.w[ k ] : c.w[ k ] * ( double ) c.mult );
  }
}

__device__ __forceinline__ int4
shfl_int4( const int4 v, const int src )
{
  return make_int4( __shfl_sync( FULL, v.x, src ), __shfl_sync( FULL, v.y, src ), __shfl_sync( FULL, v.z, src ),
    __shfl_sync( FULL, v.w, src ) );
}

// ---------------------------------------------------------------------
// Delivery: every spike of the closing slice, every out-edge, one red.global
// add into ring[(t_emit + d) mod L][channel][target]
// (EventDeliveryManager::deliver_events_ -> Connector::send -> handle,
// event_delivery_manager.cpp:599-700, connector_base.h:398-434).
// Work item = one edge chunk (<= 128 edges of one padded CSR row) queued by
// the update kernel when the spike was emitted.  A warp takes a group of up
// to 4 consecutive chunks (one load of their descriptors), and walks them
// with the next chunk's edges already in flight while the adds of the
// current one issue: each lane loads 4 edges (one 16-byte edge-word
// load, 16 or 32 bytes of weights) and issues their red.global adds.
// ---------------------------------------------------------------------
template < bool FIX, bool LATE >
__global__ void __launch_bounds__( 256 )
k_deliver( Net d )
{
  __shared__ unsigned long long s_nent;
  __shared__ int s_err;
  __shared__ int s_last;
  __shared__ int s_q;
  if ( threadIdx.x == 0 )
  {
    if constexpr ( LATE )
    {
      s_q = ld_volatile( &d.ctl->late_rd );
      s_nent = ld_volatile( &d.ctl->n_late[ s_q ] );
    }
    else
      s_nent = ld_volatile( &d.ctl->n_ent );
    s_err = ld_volatile( &d.ctl->err );
  }
  __syncthreads();
  const int4* const list = LATE ? late_list( d, s_q ) : d.ent;
  const bool ok = ( long long ) s_nent <= d.ent_cap && ( s_err & ERR_SPIKE_LIST ) == 0;
  const long long nent = ok ? ( long long ) s_nent : 0;
  const int lane = threadIdx.x & 31;
  const long long nwarps = ( ( long long ) gridDim.x * blockDim.x ) >> 5;
  const long long gw = ( ( long long ) blockIdx.x * blockDim.x + threadIdx.x ) >> 5;
  // chunks per group: at most deliver_group (autotuned, 1 to 8), so the
  // warps sweep the list together (the chunks of one network, queued
  // together, are delivered together)
  const long long G = max( 1ll, min( ( long long ) d.deliver_group, nent / nwarps ) );
  for ( long long base = gw * G; base < nent; base += nwarps * G )
  {
    const int cnt = ( int ) min( G, nent - base );
    const int4 my = lane < cnt ? list[ base + lane ] : make_int4( 0, 0, 0, 0 );
    ChunkLane< FIX > cur, nxt;
    load_chunk< FIX >( d, shfl_int4( my, 0 ), lane, cur );
    for ( int k = 0; k < cnt; ++k )
    {
      const int4 en = shfl_int4( my, min( k + 1, 31 ) );
      if ( k + 1 < cnt )
        load_chunk< FIX >( d, en, lane, nxt );
      apply_chunk< FIX, LATE >( d, cur );
      cur = nxt;
    }
  }
  // the last CTA to finish closes the slice (a late delivery: its list)
  __syncthreads();
  if ( threadIdx.x == 0 )
  {
    __threadfence();
    s_last = atomicAdd( LATE ? &d.ctl->late_done : &d.ctl->deliver_done, 1 ) == ( int ) gridDim.x - 1;
  }
  __syncthreads();
  if constexpr ( LATE )
  {
    if ( s_last && threadIdx.x == 0 )
    {
      d.ctl->n_late[ s_q ] = 0ull;
      d.ctl->late_done = 0;
      d.ctl->late_rd = s_q ^ 1;
      __threadfence();
    }
    return;
  }
  if ( s_last && d.net_mode )
  {
    // delivery mode of every network for the next slice: gather when this
    // slice's spikes reached gather_frac of its neurons (the gather reads
    // every in-edge once, the scatter one edge per spike and out-edge)
    for ( int id = threadIdx.x; id < d.n_nets; id += blockDim.x )
    {
      const unsigned sp = d.net_spk[ id ];
      d.net_spk[ id ] = 0u;
      const GatherNet g = d.net_g[ id ];
      if ( d.net_mode[ id ] )
        atomicAdd( &d.ctl->gathered, 1ull );
      d.net_mode[ id ] = ( g.ke + g.ki > 0 && ( float ) sp >= d.gather_frac * ( float ) g.n ) ? 1 : 0;
    }
  }
  if ( s_last && threadIdx.x == 0 )
  {
    d.ctl->n_ent = 0ull;
    d.ctl->deliver_done = 0;
    d.ctl->origin = d.ctl->origin + d.min_delay;
    if ( d.late_min != INT32_MAX )
      d.ctl->late_wr ^= 1;
    __threadfence();
  }
}

// ---------------------------------------------------------------------
// Graph upload (ng_set_connections): the caller's CSR (row pointers,
// targets, weights, delays) is copied as it is and packed on the device
// into padded rows of edge words and stored weights -- the channel by the
// target model's sign rule (iaf_psc_exp.cpp:351-362, aeif_cond_alpha.cpp:
// 536-550), the aeif inhibitory weight stored as -w, the precision form's
// weights in int32 fixed point.
// ---------------------------------------------------------------------
struct PackSpec
{
  int n_blocks;
  long long bend[ 8 ];  // end of each block's neuron range
  int model[ 8 ];
  long long N;
  int min_d, max_d, tbits;
};

__device__ __forceinline__ void
edge_channel( const PackSpec& ps, int32_t t, double wv, uint32_t& ch, double& we )
{
  int bk = 0;
  while ( bk + 1 < ps.n_blocks && t >= ps.bend[ bk ] )
    ++bk;
  ch = 0u;
  we = wv;
  if ( ps.model[ bk ] == NG_IAF_PSC_EXP_ID || ps.model[ bk ] == NG_IAF_PSC_ALPHA_ID )
    ch = wv > 0 ? 0u : 1u;
  else if ( ps.model[ bk ] == 2 && !( wv > 0.0 ) )
  {
    ch = 1u;
    we = -wv;
  }
}

// validation (error bits: 1 target, 2 delay, 4 weight) and the largest |stored weight|
__global__ void
k_edge_check( long long nnz, const int32_t* tgt, const double* w, const int32_t* dl, PackSpec ps,
  unsigned long long* absmax, int* err )
{
  unsigned long long m = 0ull;
  int e = 0;
  for ( long long j = ( long long ) blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += ( long long ) gridDim.x * blockDim.x )
  {
    const int32_t t = tgt[ j ];
    const int32_t d = dl[ j ];
    const double wv = w[ j ];
    if ( t < 0 || t >= ps.N )
    {
      e |= 1;
      continue;
    }
    if ( d < ps.min_d || d > ps.max_d )
      e |= 2;
    if ( !isfinite( wv ) )
    {
      e |= 4;
      continue;
    }
    uint32_t ch;
    double we;
    edge_channel( ps, t, wv, ch, we );
    const unsigned long long b = ( unsigned long long ) __double_as_longlong( fabs( we ) );
    m = b > m ? b : m;  // the bit patterns of non-negative doubles order like their values
  }
#pragma unroll
  for ( int o = 16; o > 0; o >>= 1 )
  {
    const unsigned long long v = __shfl_xor_sync( FULL, m, o );
    m = v > m ? v : m;
    e |= __shfl_xor_sync( FULL, e, o );
  }
  if ( ( threadIdx.x & 31 ) == 0 )
  {
    if ( m )
      atomicMax( absmax, m );
    if ( e )
      atomicOr( err, e );
  }
}

// Slice-close and late edge ranges of a row whose real edges [0, deg) hold
// its nu edges of delay < late_min first (padded length pdeg): the
// slice-close chunks cover [0, ue), the late ones [ls, pdeg).
__host__ __device__ __forceinline__ void
row_ranges( int nu, int deg, int pdeg, int32_t& ue, int32_t& ls )
{
  if ( nu >= deg )
  {
    ue = pdeg;
    ls = pdeg;
  }
  else if ( nu == 0 )
  {
    ue = 0;
    ls = 0;
  }
  else
  {
    ue = ( nu + 3 ) & ~3;
    ls = nu & ~3;
  }
}

// Position of an edge in its row after a stable partition by delay class
// (delay < thr first), for one 32-edge window of the row: cu / cl count the
// slice-close / late edges of the earlier windows, nu the row's total of
// slice-close edges.  All 32 lanes call it.
__device__ __forceinline__ int
split_pos( bool in, bool early, int nu, int& cu, int& cl )
{
  const unsigned lt = ( 1u << ( threadIdx.x & 31 ) ) - 1u;
  const unsigned bu = __ballot_sync( FULL, in && early ), bl = __ballot_sync( FULL, in && !early );
  const int pos = early ? cu + __popc( bu & lt ) : nu + cl + __popc( bl & lt );
  cu += __popc( bu );
  cl += __popc( bl );
  return pos;
}

__device__ __forceinline__ int
warp_sum_i( int v )
{
#pragma unroll
  for ( int o = 16; o > 0; o >>= 1 )
    v += __shfl_xor_sync( FULL, v, o );
  return v;
}

// one warp per source row: the row's edges go to its padded positions from
// prow[s] on, those of delay < late_min first (late_min == INT32_MAX: in
// the caller's order)
__global__ void
k_pack_edges( long long n_src, const long long* row_ptr, const long long* prow, const int32_t* tgt, const double* w,
  const int32_t* dl, PackSpec ps, int fx, double scale, uint32_t* tdc, void* wout, int32_t late_min, int32_t* row_ue,
  int32_t* row_ls )
{
  const long long s = ( ( long long ) blockIdx.x * blockDim.x + threadIdx.x ) >> 5;
  const int lane = threadIdx.x & 31;
  if ( s >= n_src )
    return;
  const long long r0 = row_ptr[ s ], r1 = row_ptr[ s + 1 ], p0 = prow[ s ];
  const int deg = ( int ) ( r1 - r0 );
  int nu = deg;
  if ( late_min != INT32_MAX )
  {
    int c = 0;
    for ( long long j = r0 + lane; j < r1; j += 32 )
      c += dl[ j ] < late_min ? 1 : 0;
    nu = warp_sum_i( c );
  }
  int cu = 0, cl = 0;
  for ( long long j0 = r0; j0 < r1; j0 += 32 )
  {
    const long long j = j0 + lane;
    const bool in = j < r1;
    const int32_t dj = in ? dl[ j ] : 0;
    const int pos = split_pos( in, dj < late_min, nu, cu, cl );
    if ( !in )
      continue;
    const int32_t t = tgt[ j ];
    uint32_t ch;
    double we;
    edge_channel( ps, t, w[ j ], ch, we );
    const long long k = p0 + pos;
    tdc[ k ] = ( uint32_t ) t | ( ( uint32_t ) dj << ps.tbits ) | ( ch << 31 );
    if ( fx )
      reinterpret_cast< int32_t* >( wout )[ k ] = ( int32_t ) llrint( we * scale );
    else
      reinterpret_cast< double* >( wout )[ k ] = we;
  }
  if ( lane == 0 )
  {
    int32_t ue, ls;
    row_ranges( nu, deg, ( deg + 3 ) & ~3, ue, ls );
    row_ue[ s ] = ue;
    row_ls[ s ] = ls;
  }
}

// Rows [n0, n0 + n) of a network built on the device, edges [e0, e0 + ne):
// the same stable partition by delay class, out of place into (stdc, sw),
// padding entries kept at their positions.  One warp per row.
template < typename W >
__global__ void
k_row_split( long long n, long long n0, long long e0, const int64_t* row_beg, const int32_t* row_len,
  const int32_t* real_deg, const uint32_t* tdc, const W* w, uint32_t* stdc, W* sw, int32_t late_min, int tbits,
  uint32_t dmask, int32_t* row_ue, int32_t* row_ls )
{
  const long long s = ( ( long long ) blockIdx.x * blockDim.x + threadIdx.x ) >> 5;
  const int lane = threadIdx.x & 31;
  if ( s >= n )
    return;
  const long long r0 = row_beg[ n0 + s ];
  const int pdeg = row_len[ n0 + s ], deg = real_deg[ n0 + s ];
  int c = 0;
  for ( int j = lane; j < deg; j += 32 )
    c += ( int ) ( ( tdc[ r0 + j ] >> tbits ) & dmask ) < late_min ? 1 : 0;
  const int nu = warp_sum_i( c );
  int cu = 0, cl = 0;
  const long long o = r0 - e0;
  for ( int j0 = 0; j0 < deg; j0 += 32 )
  {
    const int j = j0 + lane;
    const bool in = j < deg;
    const uint32_t t = in ? tdc[ r0 + j ] : 0u;
    const int pos = split_pos( in, ( int ) ( ( t >> tbits ) & dmask ) < late_min, nu, cu, cl );
    if ( in )
    {
      stdc[ o + pos ] = t;
      sw[ o + pos ] = w[ r0 + j ];
    }
  }
  for ( int j = deg + lane; j < pdeg; j += 32 )
  {
    stdc[ o + j ] = tdc[ r0 + j ];
    sw[ o + j ] = w[ r0 + j ];
  }
  if ( lane == 0 )
  {
    int32_t ue, ls;
    row_ranges( nu, deg, pdeg, ue, ls );
    row_ue[ n0 + s ] = ue;
    row_ls[ n0 + s ] = ls;
  }
}

// Row ranges without a partition: mode 1, every edge of the row is of the
// shorter delay class (fixed_indegree networks, one delay); 0, every edge is
// late; 2, mixed rows in any order (both deliveries walk the whole row).
__global__ void
k_row_uniform( long long n, long long n0, const int32_t* row_len, int mode, int32_t* row_ue, int32_t* row_ls )
{
  const long long s = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( s >= n )
    return;
  const int32_t p = row_len[ n0 + s ];
  row_ue[ n0 + s ] = mode != 0 ? p : 0;
  row_ls[ n0 + s ] = mode == 1 ? p : 0;
}

// A serving network's per-network entries, written in stream order behind
// the slices already enqueued (kernel arguments: no host memory that must
// outlive the call).  on == 0: the network's slot is cleared.
__global__ void
k_net_set( int id, int on, long long step0, long long until, long long off, uint2 key, long long* d_step0,
  long long* d_until, long long* d_off, uint2* d_key, GatherNet g, GatherNet* net_g, int* net_mode,
  unsigned* net_spk, TileNet tn, TileNet* net_t )
{
  if ( threadIdx.x != 0 || blockIdx.x != 0 )
    return;
  if ( on )
  {
    d_step0[ id ] = step0;
    d_until[ id ] = until;
    d_off[ id ] = off;
    d_key[ id ] = key;
  }
  if ( net_g )
  {
    net_g[ id ] = g;
    net_mode[ id ] = 0;
    net_spk[ id ] = 0u;
  }
  if ( net_t )
    net_t[ id ] = tn;
}

// Host-side ctl edits between groups (log drain, trace window).
__global__ void
k_set_ctl( Ctl* ctl, long long log_base, long long trace_row0, int reset_log, int log_sel )
{
  if ( reset_log )
    ctl->log_count = 0ull;
  ctl->log_sel = log_sel;
  ctl->log_base = log_base;
  ctl->trace_row0 = trace_row0;
}

}  // namespace ng
