// ng_persistent.cuh -- the whole min_delay-slice cycle of a network that
// fits one resident wave, run by one cooperative launch over many slices.
//
// The per-slice path of the graph form is two launches (node update, then
// delivery), each re-reading the neurons' state, coefficients, drive tables
// and CSR rows and paying a launch gap; for a network of ten thousand
// neurons those fixed costs are most of a slice.  Here a CTA's warp 0 keeps
// 32 neurons' state and coefficients in registers for the whole launch (and
// every thread the drive context of its neuron); each slice is the update of
// its lags in k_update_iaf2's two-phase layout (the reference's operations in
// the reference's order), a grid barrier, the delivery of the slice's spikes
// by every warp of the grid (the chunk loop of k_deliver), and a second
// barrier before the next slice reads the ring.  Results equal the graph
// form's bit for bit wherever the ring sums are order independent.
//
// Delivery work of consecutive slices goes to one list used as a ring
// (entry index = running count mod capacity): slice s reads the entries
// [end of slice s-1, end of slice s), so the count is never reset inside
// the launch and no extra barrier is needed.  The barriers spin with a
// bounded number of polls and set an error bit instead of waiting for ever;
// the launch is cooperative (every CTA resident), so they cannot wait on a
// CTA that is not running.
#pragma once

#include "ng_kernels.cuh"

namespace ng
{

constexpr int PK_THREADS = 128;
constexpr int ERR_BARRIER = 16;
constexpr unsigned PK_POLL_LIMIT = 1u << 21;  // polls of ~0.5 us: a barrier gives up within about a second

struct PkCtl
{
  unsigned count;  // arrivals at the launch's barriers so far
  unsigned gen;    // barriers completed before the launch (0: the counter is zeroed per launch)
  int err;         // a barrier gave up (every CTA then leaves its slice loop)
};

// Grid-wide barrier over a monotonic arrival counter: barrier b of a launch
// (the counter is zeroed before each launch) completes when the counter
// reaches (b + 1) * grid.  A CTA arrives with a fire-and-forget release add
// (after __syncthreads, so its threads' writes are ordered before it) and
// polls the counter with acquire loads -- one L2 round trip fewer than an
// arrival atomic that waits for its result followed by a release flag
// (measured: 1.97 us against 3.0 us per barrier on 391 CTAs).  Returns false
// if the polls gave up or another CTA's did; all threads of the CTA get the
// same answer.
// The other threads of the CTA may work between the arrival and the final
// __syncthreads (`while_waiting`, run by every thread but thread 0): work
// that depends on nothing the barrier orders.
template < typename F >
__device__ __forceinline__ bool
pk_grid_sync( PkCtl* pk, unsigned& gen, F&& while_waiting )
{
  __shared__ int s_ok;
  __syncthreads();
  if ( threadIdx.x != 0 )
    while_waiting();
  else
  {
    int ok = 1;
    const unsigned target = ( gen + 1u ) * gridDim.x;
    asm volatile( "red.release.gpu.global.add.u32 [%0], 1;" ::"l"( &pk->count ) : "memory" );
    unsigned polls = 0, cur;
    for ( ;; )
    {
      asm volatile( "ld.acquire.gpu.global.u32 %0, [%1];" : "=r"( cur ) : "l"( &pk->count ) : "memory" );
      if ( ( int ) ( cur - target ) >= 0 )
        break;
      if ( ++polls > PK_POLL_LIMIT || ld_volatile( &pk->err ) )
      {
        atomicOr( &pk->err, 1 );
        ok = 0;
        break;
      }
      if ( polls > 16 )
        __nanosleep( 20 );
    }
    if ( ld_volatile( &pk->err ) )
      ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  ++gen;
  return s_ok != 0;
}

__device__ __forceinline__ bool
pk_grid_sync( PkCtl* pk, unsigned& gen )
{
  return pk_grid_sync( pk, gen, [] {} );
}

// A ring cell read through L2 only: the cell was written by other SMs'
// atomics during this launch, and a line an SM's L1 kept from an earlier
// slice would be stale (a kernel boundary would have dropped it).
template < bool FIX >
__device__ __forceinline__ typename RingVal< FIX >::type
ring_ld_l2( const Net& d, int slot, int ch, int64_t i )
{
  const int64_t idx = ( ( int64_t ) slot * d.C + ch ) * d.N + i;
  if constexpr ( FIX )
    if ( d.ring32 )
      return __ldcg( reinterpret_cast< const int32_t* >( d.ring ) + idx );
  return __ldcg( reinterpret_cast< const typename RingVal< FIX >::type* >( d.ring ) + idx );
}

// Warp 0's spikes of a chunk of lags as delivery work (entries at running
// indices of the ring list) and recorder log entries, one reservation per
// counter and warp; lane 0 adds the events and spikes to ev_acc / spk_acc.  The row data (start, chunks, real degree) and the
// recorder flag of the lane's neuron are passed in registers: they do not
// change during the launch.  Must be called by all 32 lanes of warp 0.
__device__ __forceinline__ void
pk_append( const Net& d, unsigned mask, int32_t src, int slot0, long long t0, long long row, int ue, int nu, int rdeg,
  bool rec, long long lb0, unsigned long long& ev_acc, unsigned long long& spk_acc )
{
  const int cnt = __popc( mask );
  if ( __ballot_sync( FULL, cnt > 0 ) == 0 )
    return;
  const int lane = threadIdx.x & 31;
  const bool lg = cnt > 0 && rec;
  long long inc_u = ( long long ) cnt * nu, inc_g = lg ? cnt : 0;
  warp_scan2( inc_u, inc_g );
  const long long tot_u = __shfl_sync( FULL, inc_u, 31 );
  const long long tot_g = __shfl_sync( FULL, inc_g, 31 );
  const long long rtot = warp_sum_ll( ( long long ) cnt * rdeg );
  const long long ctot = warp_sum_ll( cnt );
  unsigned long long base = 0, lbase = 0;
  if ( lane == 0 )
  {
    if ( tot_u > 0 )
      base = atomicAdd( &d.ctl->n_ent, ( unsigned long long ) tot_u );
    if ( tot_g > 0 )
      lbase = atomicAdd( &d.ctl->log_count, ( unsigned long long ) tot_g );
    // the statistics: once per launch (same-address atomics of every CTA
    // in every slice would queue at one L2 line)
    ev_acc += ( unsigned long long ) rtot;
    spk_acc += ( unsigned long long ) ctot;
  }
  base = __shfl_sync( FULL, base, 0 );
  lbase = __shfl_sync( FULL, lbase, 0 );
  const long long iu0 = ( long long ) base + inc_u - ( long long ) cnt * nu;
  long long li = ( long long ) lbase + inc_g - ( lg ? cnt : 0 );
  // the whole warp writes each spike's chunk entries
  unsigned owners = __ballot_sync( FULL, cnt > 0 && nu > 0 );
  while ( owners )
  {
    const int ol = __ffs( owners ) - 1;
    owners &= owners - 1;
    const long long o_row = __shfl_sync( FULL, row, ol );
    const int o_ue = __shfl_sync( FULL, ue, ol );
    const int o_nu = __shfl_sync( FULL, nu, ol );
    long long o_iu = __shfl_sync( FULL, iu0, ol );
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
      {
        const long long r = o_row + ( long long ) c * CHUNK_EDGES;
        const long long left = ( long long ) o_ue - ( long long ) c * CHUNK_EDGES;
        const int ne = ( int ) ( left < CHUNK_EDGES ? left : CHUNK_EDGES );
        const long long e = ( o_iu + c ) % d.ent_cap;
        d.ent[ e ] = make_int4( ( int ) ( unsigned ) ( r & 0xffffffffll ), ( int ) ( r >> 32 ), ne, slot | ( 1 << 16 ) );
      }
      o_iu += o_nu;
    }
  }
  if ( !lg )
    return;
  uint2* const lg_buf = log_half( d );
  unsigned m = mask;
  while ( m )
  {
    const int k = __ffs( m ) - 1;
    m &= m - 1;
    if ( li < d.log_cap )
      lg_buf[ li ] = make_uint2( ( uint32_t ) src, ( uint32_t ) ( t0 + k + 1 - lb0 ) | ( 1u << 24 ) );
    else
      atomicOr( &d.ctl->err, ERR_LOG );
    ++li;
  }
}

// n_slices full slices of a single-block iaf network (static engine, every
// edge delivered at its slice's close, no scheduled generator spikes, no
// traces), in the two-phase layout of k_update_iaf2: a CTA of 128 threads
// serves 32 neurons, all its threads read the ring cells and draw the drive
// of the (neuron, lag) pairs of up to 16 lags at a time into shared memory,
// warp 0 runs the recurrence -- its lanes keep their neuron's state and
// coefficients in registers for the whole launch -- and appends the spikes;
// then every warp of the grid delivers.
constexpr int PK_NB = 32;  // neurons per CTA
constexpr int PK_CH = 16;  // lags per phase-1 chunk

template < typename Real, bool FIX, int MODEL >
__global__ void __launch_bounds__( PK_THREADS, 3 )
k_run_slices( Net d, Block b, int n_slices, PkCtl* pk )
{
  constexpr bool ALPHA = MODEL == NG_IAF_PSC_ALPHA_ID;
  constexpr bool EXP = MODEL == NG_IAF_PSC_EXP_ID || ALPHA;
  constexpr int P1 = PK_CH * PK_NB / PK_THREADS;  // phase-1 items per thread
  __shared__ Real s_ex[ PK_CH ][ PK_NB ];
  __shared__ Real s_in[ EXP ? PK_CH : 1 ][ PK_NB ];
  __shared__ Real s_dv[ 2 ][ PK_CH ][ PK_NB ];  // drive of (lag, neuron) of the current and the next chunk
  __shared__ unsigned s_gen;
  if ( threadIdx.x == 0 )
    s_gen = ld_volatile( &pk->gen );
  const long long origin0 = ld_volatile( &d.ctl->origin );
  const long long lb0 = ld_volatile( &d.ctl->log_base );
  unsigned long long ent_start = ld_volatile( &d.ctl->n_ent );
  __syncthreads();
  unsigned gen = s_gen;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t nb0 = ( int64_t ) blockIdx.x * PK_NB;
  const int64_t li = nb0 + lane;
  const bool act = warp == 0 && li < b.n;
  const int64_t i = b.off + ( act ? li : 0 );
  Real* s0 = ( Real* ) b.s[ 0 ];
  Real* s1 = ( Real* ) b.s[ 1 ];
  Real* s2 = ( Real* ) b.s[ 2 ];
  Real* s3 = ( Real* ) b.s[ 3 ];
  Real* s4 = ( Real* ) b.s[ 4 ];
  Real V = 0, x1 = 0, x2 = 0, i0 = 0, i1 = 0, Ie = 0;
  Real c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0, Vth = 0, Vreset = 0, c9 = 0;
  AlphaCoef< Real > ac {};
  int r = 0, refr = 0;
  // the neuron's CSR row as delivery work (whole row at the slice close)
  long long row = 0;
  int ue = 0, nu = 0, rdeg = 0;
  bool rec = false;
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
    const RowWork rw = row_work( d, ( int32_t ) i );
    row = rw.row;
    ue = rw.ue;
    nu = rw.nu;
    rdeg = d.real_deg[ i ];
    rec = d.rec == nullptr || d.rec[ i ] != 0;
  }
  // the drive of the neuron this thread's phase-1 items belong to
  const int64_t lq = nb0 + lane;
  const bool qact = lq < b.n;
  const int64_t iq = b.off + ( qact ? lq : 0 );
  DriveCtx dc;
  dc.n = 0;
  if ( qact )
    drive_ctx( d, iq, dc );
  long long dcnt = 0;
  unsigned long long ev_acc = 0, spk_acc = 0;
  const int md = d.min_delay;
  const long long nwarps = ( ( long long ) gridDim.x * blockDim.x ) >> 5;
  const long long gw = ( ( long long ) blockIdx.x * blockDim.x + threadIdx.x ) >> 5;
  // The drive of a chunk's (lag, neuron) pairs: it depends on no spike, so
  // warps 1-3 draw the next chunk's while warp 0 runs the current recurrence.
  // Lane q draws for neuron q; warp w takes the lag pairs p = w - 1, w + 2, ...
  // (one Philox block serves the two steps of a pair).
  auto draw_chunk = [ & ]( int buf, long long t0c, int nlc, int w0, int nw ) {
    for ( int pr = warp - w0; 2 * pr < nlc; pr += nw )
#pragma unroll
      for ( int h2 = 0; h2 < 2; ++h2 )
      {
        const int k = 2 * pr + h2;
        if ( k < nlc )
          s_dv[ buf ][ k ][ lane ] = qact ? drive_at< Real >( d, dc, iq, t0c + k, dcnt ) : Real( 0 );
      }
  };
  int buf = 0;
  draw_chunk( 0, origin0, min( PK_CH, md ), 0, PK_THREADS / 32 );
  __syncthreads();
  int sl = 0;
  for ( ; sl < n_slices; ++sl )
  {
    const long long origin = origin0 + ( long long ) sl * md;
    for ( int cb = 0; cb < md; cb += PK_CH )
    {
      const int nl = min( PK_CH, md - cb );
      const long long t0 = origin + cb;
      const int slot0 = ( int ) ( t0 % d.L );
      // ---- phase 1: ring cells of (neuron q, lag k), item j = k * 32 + q
      typename RingVal< FIX >::type rex[ P1 ], rin[ P1 ];
      int slots[ P1 ];
#pragma unroll
      for ( int m = 0; m < P1; ++m )
      {
        const int j = threadIdx.x + m * PK_THREADS;
        rex[ m ] = 0;
        rin[ m ] = 0;
        slots[ m ] = -1;
        if ( j < nl * PK_NB && qact )
        {
          const int k = j >> 5;
          int slot = slot0 + k;
          if ( slot >= d.L )
            slot -= d.L;
          slots[ m ] = slot;
          rex[ m ] = ring_ld_l2< FIX >( d, slot, 0, iq );
          if constexpr ( EXP )
            rin[ m ] = ring_ld_l2< FIX >( d, slot, 1, iq );
        }
      }
#pragma unroll
      for ( int m = 0; m < P1; ++m )
      {
        const int j = threadIdx.x + m * PK_THREADS;
        if ( j >= nl * PK_NB )
          continue;
        Real ex = 0, inh = 0;
        if ( slots[ m ] >= 0 )
        {
          ex = ring_real< Real, FIX >( d, rex[ m ] );
          if constexpr ( EXP )
            inh = ring_real< Real, FIX >( d, rin[ m ] );
          const Real dv = s_dv[ buf ][ j >> 5 ][ j & 31 ];
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
        s_ex[ j >> 5 ][ j & 31 ] = ex;
        if constexpr ( EXP )
          s_in[ j >> 5 ][ j & 31 ] = inh;
      }
#pragma unroll
      for ( int m = 0; m < P1; ++m )
      {
        if ( slots[ m ] < 0 )
          continue;
        ring_clear< FIX >( d, slots[ m ], 0, iq );
        if constexpr ( EXP )
          ring_clear< FIX >( d, slots[ m ], 1, iq );
      }
      __syncthreads();
      // ---- phase 2: the recurrence, one lane per neuron (iaf_psc_delta:272-329,
      // iaf_psc_exp:288-348, iaf_psc_alpha update)
      if ( warp == 0 )
      {
        unsigned smask = 0;
        if ( act )
        {
          for ( int k = 0; k < nl; ++k )
          {
            bool spk = false;
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
            if ( spk )
              smask |= 1u << k;
          }
        }
        pk_append( d, smask, ( int32_t ) i, slot0, t0, row, ue, nu, rdeg, rec, lb0, ev_acc, spk_acc );
      }
      else if ( cb + PK_CH < md )
      {
        // the next chunk's drive (same slice), beside the recurrence
        draw_chunk( buf ^ 1, t0 + PK_CH, min( PK_CH, md - cb - PK_CH ), 1, PK_THREADS / 32 - 1 );
      }
      buf ^= 1;
      __syncthreads();  // s_ex / s_in are refilled by the next chunk
    }
    if ( !pk_grid_sync( pk, gen ) )
      break;
    // ---- delivery of the slice's spikes (k_deliver's chunk loop)
    const unsigned long long ent_end = ld_volatile( &d.ctl->n_ent );
    const long long nent = ( long long ) ( ent_end - ent_start );
    if ( nent > d.ent_cap )
    {
      if ( threadIdx.x == 0 )
        atomicOr( &d.ctl->err, ERR_SPIKE_LIST );
    }
    else
    {
      // whole groups of consecutive chunks per warp (rounded up: a warp walks
      // its group with the next chunk's loads in flight, where a second
      // round of single chunks would wait a full round trip)
      const long long G = max( 1ll, min( ( long long ) d.deliver_group, ( nent + nwarps - 1 ) / nwarps ) );
      for ( long long base = gw * G; base < nent; base += nwarps * G )
      {
        const int cnt = ( int ) min( G, nent - base );
        // entries written by other SMs in this launch: read through L2
        const int4 my = lane < cnt ? __ldcg( d.ent + ( long long ) ( ( ent_start + base + lane ) % d.ent_cap ) )
                                   : make_int4( 0, 0, 0, 0 );
        ChunkLane< FIX > cur, nxt;
        load_chunk< FIX >( d, shfl_int4( my, 0 ), lane, cur );
        for ( int k = 0; k < cnt; ++k )
        {
          const int4 en = shfl_int4( my, min( k + 1, 31 ) );
          if ( k + 1 < cnt )
            load_chunk< FIX >( d, en, lane, nxt );
          apply_chunk< FIX, false >( d, cur );
          cur = nxt;
        }
      }
    }
    ent_start = ent_end;
    // the next slice's first chunk of drive, while thread 0 waits at the barrier
    // (buf already names the buffer after the slice's last chunk; the other
    // one was last read by a chunk before it)
    const bool next = sl + 1 < n_slices;
    if ( !pk_grid_sync( pk, gen, [ & ] {
           if ( next && warp > 0 )
             draw_chunk( buf, origin + md, min( PK_CH, md ), 1, PK_THREADS / 32 - 1 );
         } ) )
      break;
  }
  flush_drive_count( d, dcnt );
  if ( threadIdx.x == 0 && ( ev_acc | spk_acc ) )
  {
    atomicAdd( &d.ctl->syn_events, ev_acc );
    atomicAdd( &d.ctl->n_spikes, spk_acc );
  }
  if ( blockIdx.x == 0 && threadIdx.x == 0 )
  {
    // the graph form's state at a slice boundary: empty work list, clock advanced
    d.ctl->n_ent = 0ull;
    d.ctl->origin = origin0 + ( long long ) sl * md;
    if ( ld_volatile( &pk->err ) )
      atomicOr( &d.ctl->err, ERR_BARRIER );
    __threadfence();
  }
  if ( act )
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

// The same cycle for a network larger than one resident wave (many
// networks of a batch concatenated into one block, or one large network):
// each CTA walks its 32-neuron groups g = block, block + grid, ... in every
// slice.  A group's state, coefficients, row data and drive context are
// loaded at the start of its turn and the state written back at its end --
// from L2, where the state of a network of this size stays (about 130 bytes
// per neuron) -- instead of living in registers for the launch; the ring,
// the delivery and the barriers are k_run_slices'.  All four warps read the
// ring cells and draw the drive of the group's (neuron, lag) pairs, then
// warp 0 runs the recurrence.
#ifndef PK_MG_MIN_CTAS
#define PK_MG_MIN_CTAS 3
#endif
template < typename Real, bool FIX, int MODEL >
__global__ void __launch_bounds__( PK_THREADS, PK_MG_MIN_CTAS )
k_run_slices_mg( Net d, Block b, int n_slices, PkCtl* pk )
{
  constexpr bool ALPHA = MODEL == NG_IAF_PSC_ALPHA_ID;
  constexpr bool EXP = MODEL == NG_IAF_PSC_EXP_ID || ALPHA;
  constexpr int P1 = PK_CH * PK_NB / PK_THREADS;  // phase-1 items per thread
  __shared__ Real s_ex[ PK_CH ][ PK_NB ];
  __shared__ Real s_in[ EXP ? PK_CH : 1 ][ PK_NB ];
  __shared__ unsigned s_gen;
  if ( threadIdx.x == 0 )
    s_gen = ld_volatile( &pk->gen );
  const long long origin0 = ld_volatile( &d.ctl->origin );
  const long long lb0 = ld_volatile( &d.ctl->log_base );
  unsigned long long ent_start = ld_volatile( &d.ctl->n_ent );
  __syncthreads();
  unsigned gen = s_gen;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  Real* s0 = ( Real* ) b.s[ 0 ];
  Real* s1 = ( Real* ) b.s[ 1 ];
  Real* s2 = ( Real* ) b.s[ 2 ];
  Real* s3 = ( Real* ) b.s[ 3 ];
  Real* s4 = ( Real* ) b.s[ 4 ];
  const int64_t n_groups = ( b.n + PK_NB - 1 ) / PK_NB;
  long long dcnt = 0;
  unsigned long long ev_acc = 0, spk_acc = 0;
  const int md = d.min_delay;
  const long long nwarps = ( ( long long ) gridDim.x * blockDim.x ) >> 5;
  const long long gw = ( ( long long ) blockIdx.x * blockDim.x + threadIdx.x ) >> 5;
  int sl = 0;
  for ( ; sl < n_slices; ++sl )
  {
    const long long origin = origin0 + ( long long ) sl * md;
    for ( int64_t g = blockIdx.x; g < n_groups; g += gridDim.x )
    {
      const int64_t nb0 = g * PK_NB;
      const int64_t li = nb0 + lane;
      const bool qact = li < b.n;                // this lane's neuron (every warp)
      const bool act = warp == 0 && qact;        // ... whose recurrence this lane runs
      const int64_t i = b.off + ( qact ? li : 0 );
      DriveCtx dc;
      dc.n = 0;
      if ( qact )
        drive_ctx( d, i, dc );
      Real V = 0, x1 = 0, x2 = 0, i0 = 0, i1 = 0, Ie = 0;
      Real c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0, Vth = 0, Vreset = 0, c9 = 0;
      AlphaCoef< Real > ac {};
      int r = 0, refr = 0;
      long long row = 0;
      int ue = 0, nu = 0, rdeg = 0;
      bool rec = false;
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
        const RowWork rw = row_work( d, ( int32_t ) i );
        row = rw.row;
        ue = rw.ue;
        nu = rw.nu;
        rdeg = d.real_deg[ i ];
        rec = d.rec == nullptr || d.rec[ i ] != 0;
      }
      for ( int cb = 0; cb < md; cb += PK_CH )
      {
        const int nl = min( PK_CH, md - cb );
        const long long t0 = origin + cb;
        const int slot0 = ( int ) ( t0 % d.L );
        // ---- phase 1: ring cells and drive of (neuron q, lag k), item j = k * 32 + q
        typename RingVal< FIX >::type rex[ P1 ], rin[ P1 ];
        Real dvs[ P1 ];
        int slots[ P1 ];
#pragma unroll
        for ( int m = 0; m < P1; ++m )
        {
          const int j = threadIdx.x + m * PK_THREADS;
          rex[ m ] = 0;
          rin[ m ] = 0;
          dvs[ m ] = Real( 0 );
          slots[ m ] = -1;
          if ( j < nl * PK_NB && qact )
          {
            const int k = j >> 5;
            int slot = slot0 + k;
            if ( slot >= d.L )
              slot -= d.L;
            slots[ m ] = slot;
            rex[ m ] = ring_ld_l2< FIX >( d, slot, 0, i );
            if constexpr ( EXP )
              rin[ m ] = ring_ld_l2< FIX >( d, slot, 1, i );
            dvs[ m ] = drive_at< Real >( d, dc, i, t0 + k, dcnt );
          }
        }
#pragma unroll
        for ( int m = 0; m < P1; ++m )
        {
          const int j = threadIdx.x + m * PK_THREADS;
          if ( j >= nl * PK_NB )
            continue;
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
          s_ex[ j >> 5 ][ j & 31 ] = ex;
          if constexpr ( EXP )
            s_in[ j >> 5 ][ j & 31 ] = inh;
        }
#pragma unroll
        for ( int m = 0; m < P1; ++m )
        {
          if ( slots[ m ] < 0 )
            continue;
          ring_clear< FIX >( d, slots[ m ], 0, i );
          if constexpr ( EXP )
            ring_clear< FIX >( d, slots[ m ], 1, i );
        }
        __syncthreads();
        // ---- phase 2: the recurrence, one lane per neuron (iaf_psc_delta:272-329,
        // iaf_psc_exp:288-348, iaf_psc_alpha update)
        if ( warp == 0 )
        {
          unsigned smask = 0;
          if ( act )
          {
            for ( int k = 0; k < nl; ++k )
            {
              bool spk = false;
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
              if ( spk )
                smask |= 1u << k;
            }
          }
          pk_append( d, smask, ( int32_t ) i, slot0, t0, row, ue, nu, rdeg, rec, lb0, ev_acc, spk_acc );
        }
        __syncthreads();  // s_ex / s_in are refilled by the next chunk
      }
      if ( act )
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
    if ( !pk_grid_sync( pk, gen ) )
      break;
    // ---- delivery of the slice's spikes (k_deliver's chunk loop)
    const unsigned long long ent_end = ld_volatile( &d.ctl->n_ent );
    const long long nent = ( long long ) ( ent_end - ent_start );
    if ( nent > d.ent_cap )
    {
      if ( threadIdx.x == 0 )
        atomicOr( &d.ctl->err, ERR_SPIKE_LIST );
    }
    else
    {
      const long long G = max( 1ll, min( ( long long ) d.deliver_group, ( nent + nwarps - 1 ) / nwarps ) );
      for ( long long base = gw * G; base < nent; base += nwarps * G )
      {
        const int cnt = ( int ) min( G, nent - base );
        const int4 my = lane < cnt ? __ldcg( d.ent + ( long long ) ( ( ent_start + base + lane ) % d.ent_cap ) )
                                   : make_int4( 0, 0, 0, 0 );
        ChunkLane< FIX > cur, nxt;
        load_chunk< FIX >( d, shfl_int4( my, 0 ), lane, cur );
        for ( int k = 0; k < cnt; ++k )
        {
          const int4 en = shfl_int4( my, min( k + 1, 31 ) );
          if ( k + 1 < cnt )
            load_chunk< FIX >( d, en, lane, nxt );
          apply_chunk< FIX, false >( d, cur );
          cur = nxt;
        }
      }
    }
    ent_start = ent_end;
    if ( !pk_grid_sync( pk, gen ) )
      break;
  }
  flush_drive_count( d, dcnt );
  if ( threadIdx.x == 0 && ( ev_acc | spk_acc ) )
  {
    atomicAdd( &d.ctl->syn_events, ev_acc );
    atomicAdd( &d.ctl->n_spikes, spk_acc );
  }
  if ( blockIdx.x == 0 && threadIdx.x == 0 )
  {
    d.ctl->n_ent = 0ull;
    d.ctl->origin = origin0 + ( long long ) sl * md;
    if ( ld_volatile( &pk->err ) )
      atomicOr( &d.ctl->err, ERR_BARRIER );
    __threadfence();
  }
}

}  // namespace ng
