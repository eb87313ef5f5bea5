// ng_serving.cuh -- device kernels of the serving engine: fixed_indegree
// connectivity drawn on the GPU into a network's region of the edge pool,
// and the per-region bookkeeping (network ids, rows).
//
// Graph construction follows the reference's FixedInDegreeBuilder
// (nestkernel/conn_builder.cpp:1508-...): every target draws k_exc sources
// uniformly from the excitatory range and k_inh from the inhibitory range,
// multapses allowed, autapses redrawn unless allowed.  The draws come from a
// Philox4x32-10 stream keyed by the network's graph seed, counter (target,
// draw index, attempt), so a network's graph depends on its seed only.  The
// edges are then grouped by source with a counting sort (histogram, scan of
// the padded row lengths, scatter).
#pragma once

#include "ng_kernels.cuh"

namespace ng
{

constexpr uint32_t CONN_STREAM = 0x434F4E4Eu;

// uniform integer in [0, size) from a 32-bit draw (multiply-high)
__device__ __forceinline__ int64_t
uniform_below( uint32_t u, int64_t size )
{
  return ( int64_t ) ( ( ( unsigned long long ) u * ( unsigned long long ) size ) >> 32 );
}

__global__ void
k_fi_draw( int64_t n, int64_t n_exc, int k_exc, int k_inh, int allow_aut, uint32_t key0, uint32_t key1,
  int32_t* tmp_src, int32_t* cnt )
{
  const int K = k_exc + k_inh;
  const int64_t idx = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( idx >= n * K )
    return;
  const int64_t t = idx / K;
  const int j = ( int ) ( idx - t * K );
  const bool ex = j < k_exc;
  const int64_t base = ex ? 0 : n_exc;
  const int64_t size = ex ? n_exc : n - n_exc;
  int64_t src = base;
  for ( int attempt = 0; attempt < 64; ++attempt )
  {
    uint32_t o[ 4 ];
    philox4x32_10( ( uint32_t ) t, ( uint32_t ) j, ( uint32_t ) attempt, CONN_STREAM, key0, key1, o );
    src = base + uniform_below( o[ 0 ], size );
    if ( allow_aut || src != t )
      break;
  }
  tmp_src[ idx ] = ( int32_t ) src;
  atomicAdd( &cnt[ src ], 1 );
}

// Exclusive scan of the padded row lengths (one CTA of 1024 threads; each
// thread sums a contiguous run of sources, then a block scan of the runs).
__global__ void __launch_bounds__( 1024 )
k_fi_scan( int64_t n, const int32_t* cnt, int64_t* beg, int32_t* plen, long long* total )
{
  __shared__ long long s_part[ 1024 ];
  const int t = threadIdx.x;
  const int64_t per = ( n + 1023 ) / 1024;
  const int64_t lo = t * per, hi = min( n, lo + per );
  long long sum = 0;
  for ( int64_t s = lo; s < hi; ++s )
    sum += ( cnt[ s ] + 3 ) & ~3;
  s_part[ t ] = sum;
  __syncthreads();
  for ( int o = 1; o < 1024; o <<= 1 )
  {
    const long long v = t >= o ? s_part[ t - o ] : 0;
    __syncthreads();
    s_part[ t ] += v;
    __syncthreads();
  }
  long long run = s_part[ t ] - sum;
  for ( int64_t s = lo; s < hi; ++s )
  {
    const int p = ( cnt[ s ] + 3 ) & ~3;
    beg[ s ] = run;
    plen[ s ] = p;
    run += p;
  }
  if ( t == 1023 )
    *total = s_part[ 1023 ];
}

// Place every drawn edge into its source's row of the network's region.
template < typename W >
__global__ void
k_fi_scatter( int64_t n, int k_exc, int k_inh, const int32_t* tmp_src, const int64_t* beg, int32_t* fill,
  int64_t n0, int64_t e0, uint32_t word_exc, uint32_t word_inh, W w_exc, W w_inh, uint32_t* tdc, W* w )
{
  const int K = k_exc + k_inh;
  const int64_t idx = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( idx >= n * K )
    return;
  const int64_t t = idx / K;
  const int j = ( int ) ( idx - t * K );
  const int32_t src = tmp_src[ idx ];
  const int64_t e = e0 + beg[ src ] + atomicAdd( &fill[ src ], 1 );
  const bool ex = j < k_exc;
  tdc[ e ] = ( uint32_t ) ( n0 + t ) | ( ex ? word_exc : word_inh );
  w[ e ] = ex ? w_exc : w_inh;
}

// In-edge table of the per-target gather (layout at k_gather): draw j of
// target t, from the drawn sources tmp_src[t * K + j]; the table was
// filled with the padding id n beforehand.
__global__ void
k_fi_gtab( int64_t n, int K, const int32_t* tmp_src, uint16_t* gin )
{
  const int64_t idx = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( idx >= n * K )
    return;
  const int64_t t = idx / K;
  const int j = ( int ) ( idx - t * K );
  const int nb = ( K + 7 ) >> 3;
  gin[ ( ( ( t >> 5 ) * nb + ( j >> 3 ) ) * 32 + ( t & 31 ) ) * 8 + ( j & 7 ) ] = ( uint16_t ) tmp_src[ idx ];
}

__global__ void
k_fill_u16( uint16_t* p, int64_t n, uint16_t v )
{
  const int64_t k = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( k < n )
    p[ k ] = v;
}

// Rows of the region's sources: begin, padded length, real degree.
__global__ void
k_fi_rows( int64_t n, int64_t n0, int64_t e0, const int64_t* beg, const int32_t* plen, const int32_t* cnt,
  int64_t* row_beg, int32_t* row_len, int32_t* real_deg )
{
  const int64_t s = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( s >= n )
    return;
  row_beg[ n0 + s ] = e0 + beg[ s ];
  row_len[ n0 + s ] = plen[ s ];
  real_deg[ n0 + s ] = cnt[ s ];
}

__global__ void
k_fill_i32( int32_t* p, int64_t n, int32_t v )
{
  const int64_t k = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( k < n )
    p[ k ] = v;
}

}  // namespace ng

namespace ng
{

// ---------------------------------------------------------------------
// pairwise_bernoulli connectivity drawn on the device (the reference's
// BernoulliBuilder, nestkernel/conn_builder.h:716, with Philox streams):
// every (source, target) pair of source population i and target population
// j is connected with probability p[i][j].  Targets are walked in blocks of
// PB_BLOCK; inside a block the next connected target is found by geometric
// skipping, gap = floor(log(u) / log(1 - p)).  Weights and delays are
// normal per source type (excitatory / inhibitory), delays clipped to
// [h, d_max] and rounded to steps as Time::delay_ms_to_steps does (then
// raised to the engine's min_delay where that is longer than one step).
// Pass 1 counts the edges of every (source, block); pass 2 regenerates the
// same draws and writes them into the source's row.
// ---------------------------------------------------------------------
constexpr int PB_BLOCK = 1024;
constexpr uint32_t PB_STREAM = 0x50425244u;  // target draws
constexpr uint32_t WD_STREAM = 0x57444C59u;  // weight / delay draws
constexpr int PB_MAX_POPS = 16;

struct PbSpec
{
  int n_pops;
  long long pop_lo[ PB_MAX_POPS + 1 ];
  int pop_exc[ PB_MAX_POPS ];
  double inv_log1mp[ PB_MAX_POPS * PB_MAX_POPS ];  // 1 / log(1 - p), 0: p = 1, NaN: p = 0
  double w_mean[ 2 ], w_sd[ 2 ];                  // [inhibitory, excitatory] source
  double d_mean[ 2 ], d_sd[ 2 ];                  // ms
  double h, d_max;                                // ms
  int min_steps, max_steps;                       // delay bounds of the engine
  int allow_aut;
  uint32_t key0, key1;
  int nb;                                         // target blocks in the network
};

__device__ __forceinline__ int
pop_of( const PbSpec& sp, long long i )
{
  int j = 0;
  while ( j + 1 < sp.n_pops && i >= sp.pop_lo[ j + 1 ] )
    ++j;
  return j;
}

// block b covers targets [lo, hi) of one target population
__device__ __forceinline__ void
block_range( const PbSpec& sp, int b, long long& lo, long long& hi, int& pj )
{
  int acc = 0;
  for ( int j = 0; j < sp.n_pops; ++j )
  {
    const long long sz = sp.pop_lo[ j + 1 ] - sp.pop_lo[ j ];
    const int nbj = ( int ) ( ( sz + PB_BLOCK - 1 ) / PB_BLOCK );
    if ( b < acc + nbj )
    {
      lo = sp.pop_lo[ j ] + ( long long ) ( b - acc ) * PB_BLOCK;
      hi = min( lo + PB_BLOCK, sp.pop_lo[ j + 1 ] );
      pj = j;
      return;
    }
    acc += nbj;
  }
  lo = hi = 0;
  pj = 0;
}

__device__ __forceinline__ double
unit_open( uint32_t x )
{
  return ( ( double ) x + 0.5 ) * ( 1.0 / 4294967296.0 );
}

// pass 1 (write == false): count into cnt_sb; pass 2: write the edges
template < typename W >
__global__ void
k_pb_pass( PbSpec sp, long long n, bool write, int* cnt_sb, const int64_t* beg, long long n0, long long e0, int tbits,
  bool exp_model, bool aeif_model, double fx_scale, uint32_t* tdc, W* w )
{
  const long long idx = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( idx >= n * sp.nb )
    return;
  const long long s = idx / sp.nb;
  const int b = ( int ) ( idx - s * sp.nb );
  long long lo, hi;
  int pj;
  block_range( sp, b, lo, hi, pj );
  const int pi = pop_of( sp, s );
  const double inv = sp.inv_log1mp[ pi * PB_MAX_POPS + pj ];
  if ( isnan( inv ) )
  {
    if ( !write )
      cnt_sb[ idx ] = 0;
    return;
  }
  long long off = 0;
  int c_max = 0x7fffffff;
  if ( write )
  {
    off = beg[ s ];
    for ( int bb = 0; bb < b; ++bb )
      off += cnt_sb[ s * sp.nb + bb ];
    c_max = cnt_sb[ idx ];  // pass 2 never writes past what pass 1 counted
  }
  const int ex = sp.pop_exc[ pi ] ? 1 : 0;
  long long pos = lo - 1;
  int c = 0;
  uint32_t o[ 4 ];
  int q = 4;
  uint32_t k = 0;
  for ( ;; )
  {
    if ( q == 4 )
    {
      philox4x32_10( ( uint32_t ) s, ( uint32_t ) b, k++, PB_STREAM, sp.key0, sp.key1, o );
      q = 0;
    }
    const double u = unit_open( o[ q++ ] );
    const double gap = inv == 0.0 ? 0.0 : floor( log( u ) * inv );
    if ( !( gap < ( double ) ( hi - 1 - pos ) ) )  // the next target lies past the block (or gap is inf)
      break;
    pos += ( long long ) gap + 1;
    if ( !sp.allow_aut && pos == s )
      continue;
    if ( c >= c_max )
      break;
    if ( write )
    {
      uint32_t r[ 4 ];
      philox4x32_10( ( uint32_t ) s, ( uint32_t ) b, ( uint32_t ) c, WD_STREAM, sp.key0, sp.key1, r );
      // Box-Muller: two normals from two uniforms
      const double rr = sqrt( -2.0 * log( unit_open( r[ 0 ] ) ) );
      const double th = 6.283185307179586 * unit_open( r[ 1 ] );
      const double z0 = rr * cos( th ), z1 = rr * sin( th );
      double wv = sp.w_mean[ ex ] + sp.w_sd[ ex ] * z0;
      double dms = sp.d_mean[ ex ] + sp.d_sd[ ex ] * z1;
      dms = fmin( fmax( dms, sp.h ), sp.d_max );
      int dst = ( int ) floor( dms / sp.h + 0.5 );
      dst = max( sp.min_steps, min( dst, sp.max_steps ) );
      uint32_t ch = 0;
      if ( exp_model )
        ch = wv > 0 ? 0u : 1u;
      else if ( aeif_model && !( wv > 0.0 ) )
      {
        ch = 1u;
        wv = -wv;
      }
      const long long e = e0 + off + c;
      tdc[ e ] = ( uint32_t ) ( n0 + pos ) | ( ( uint32_t ) dst << tbits ) | ( ch << 31 );
      if constexpr ( sizeof( W ) == 4 )
        w[ e ] = ( W ) llrint( fmin( fmax( wv * fx_scale, -2147483647.0 ), 2147483647.0 ) );
      else
        w[ e ] = ( W ) wv;
    }
    ++c;
  }
  if ( !write )
    cnt_sb[ idx ] = c;
}

// per-source totals of pass 1
__global__ void
k_pb_rowsum( long long n, int nb, const int* cnt_sb, int32_t* cnt )
{
  const long long s = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( s >= n )
    return;
  long long t = 0;
  for ( int b = 0; b < nb; ++b )
    t += cnt_sb[ s * nb + b ];
  cnt[ s ] = ( int32_t ) t;
}

}  // namespace ng

namespace ng
{

// ---------------------------------------------------------------------
// Per-target gather (precision form of a serving engine): for the networks
// in gather mode this slice, every target walks its in-edge table and
// counts, per lag and draw type (excitatory / inhibitory), the in-edges
// whose source spiked at that lag; the ring then gets count * weight at
// slot (origin + lag + d) mod L.  The targets' ring cells have no other
// writer in this slice (their sources queue no edge chunks), so the adds
// are plain read-modify-writes, and the integer result equals the
// scatter's whatever the order.
//
// One CTA per SM walks a contiguous range of the slice's target tiles
// (GT targets of one network each).  The network's lag bits (16-bit, one
// per source, written by the update kernel) are staged in shared memory
// once per network, so the random source lookups never leave the SM; the
// in-edge table streams from HBM in 16-byte loads, coalesced per warp
// (layout below).  Counts are kept as 12 bit planes per thread (bit c of
// plane p = binary digit p of the count of lag/type c): 8 sources' lag
// bits at a time go through a Harley-Seal carry-save adder tree (two
// three-input logic ops per adder), so no counter is indexed dynamically
// and no lane branches on the data.
// GP threads share a target (runs of its in-edges); their planes are added
// in shared memory.
//
// In-edge table of a network (16-bit local source ids, Kp = K rounded up
// to 8, padding = n, whose lag bits are 0): entry (target tl, draw j) at
// ((tl / 32 * Kp / 8 + j / 8) * 32 + tl % 32) * 8 + j % 8.
// ---------------------------------------------------------------------
constexpr int GT = 256;                  // targets per tile
constexpr int GP = 4;                    // threads per target
constexpr int G_THREADS = GT * GP;
constexpr int G_PLANES = 12;             // in-degrees below 4096
constexpr int G_MAX_N = 65535;           // 16-bit local ids, n itself is the padding id
constexpr int G_MAX_K = ( 1 << G_PLANES ) - 1;
constexpr size_t G_SMEM = ( size_t ) ( GP - 1 ) * G_PLANES * GT * 4 + ( size_t ) ( G_MAX_N + 1 ) * 2;

// carry-save adder: (acc, a, b) -> acc = acc ^ a ^ b, hi = majority(acc, a, b)
__device__ __forceinline__ void
csa( uint32_t& hi, uint32_t& acc, uint32_t a, uint32_t b )
{
  const uint32_t u = acc ^ a;
  hi = ( acc & a ) | ( u & b );
  acc = u ^ b;
}

__device__ __forceinline__ unsigned
plane_count( const uint32_t* P, int bit )
{
  unsigned c = 0;
#pragma unroll
  for ( int b = 0; b < G_PLANES; ++b )
    c |= ( ( P[ b ] >> bit ) & 1u ) << b;
  return c;
}

__global__ void __launch_bounds__( G_THREADS, 1 )
k_gather( Net d )
{
  extern __shared__ __align__( 16 ) unsigned char g_smem[];
  uint32_t* s_pl = reinterpret_cast< uint32_t* >( g_smem );  // [GP - 1][G_PLANES][GT]
  uint16_t* s_mask = reinterpret_cast< uint16_t* >( g_smem + ( size_t ) ( GP - 1 ) * G_PLANES * GT * 4 );  // [n + 1]
  __shared__ int s_pref[ 1025 ];
  const long long origin = cta_origin( d );  // synchronises the CTA
  const int tid = threadIdx.x;
  // tiles per network in gather mode, prefix sums (n_nets <= 1024)
  for ( int id = tid; id < d.n_nets; id += blockDim.x )
  {
    int c = 0;
    if ( d.net_mode[ id ] )
    {
      const GatherNet g = d.net_g[ id ];
      if ( g.ke + g.ki > 0 )
        c = ( g.n + GT - 1 ) / GT;
    }
    s_pref[ id + 1 ] = c;
  }
  if ( tid == 0 )
    s_pref[ 0 ] = 0;
  __syncthreads();
  if ( tid == 0 )
    for ( int id = 0; id < d.n_nets; ++id )
      s_pref[ id + 1 ] += s_pref[ id ];
  __syncthreads();
  const int total = s_pref[ d.n_nets ];
  const int w0 = ( int ) ( ( long long ) total * blockIdx.x / gridDim.x );
  const int w1 = ( int ) ( ( long long ) total * ( blockIdx.x + 1 ) / gridDim.x );
  const int ti = tid % GT;
  const int part = tid / GT;
  long long* ring = ( long long* ) d.ring;
  int staged = -1;
  for ( int w = w0; w < w1; ++w )
  {
    // the tile's network: last id with s_pref[id] <= w
    int lo = 0, hi = d.n_nets;
    while ( hi - lo > 1 )
    {
      const int mid = ( lo + hi ) >> 1;
      if ( s_pref[ mid ] <= w )
        lo = mid;
      else
        hi = mid;
    }
    const int id = lo;
    const GatherNet g = d.net_g[ id ];
    if ( id != staged )
    {
      __syncthreads();
      // 8 independent loads per thread in flight (a load-store loop waits
      // one round trip per element)
      const uint32_t* gm = d.gmask + g.off;
      for ( int q0 = tid; q0 <= g.n; q0 += 8 * blockDim.x )
      {
        uint32_t v[ 8 ];
#pragma unroll
        for ( int u = 0; u < 8; ++u )
        {
          const int q = q0 + u * blockDim.x;
          v[ u ] = q < g.n ? gm[ q ] : 0u;
        }
#pragma unroll
        for ( int u = 0; u < 8; ++u )
        {
          const int q = q0 + u * blockDim.x;
          if ( q <= g.n )
            s_mask[ q ] = ( uint16_t ) v[ u ];
        }
      }
      __syncthreads();
      staged = id;
    }
    const int64_t tl = ( int64_t ) ( w - s_pref[ id ] ) * GT + ti;
    const int K = g.ke + g.ki;
    const int nb = ( K + 7 ) >> 3;
    // bit-parallel counters: bit c of (ones, twos, fours, hi[0..]) holds the
    // binary digits 1, 2, 4, 8, 16, ... of the count of lag/type c
    uint32_t P[ G_PLANES ];
#pragma unroll
    for ( int b = 0; b < G_PLANES; ++b )
      P[ b ] = 0u;
    if ( tl < g.n )
    {
      const uint4* col = reinterpret_cast< const uint4* >( d.gin + g.base ) + ( ( tl >> 5 ) * nb ) * 32 + ( tl & 31 );
      const int b0 = nb * part / GP, b1 = nb * ( part + 1 ) / GP;
      // one 16-byte word (8 draws) into the planes
      auto eat = [ & ]( const uint4 q, const int jw ) {
        const uint32_t wv[ 4 ] = { q.x, q.y, q.z, q.w };
        uint32_t x[ 8 ];
#pragma unroll
        for ( int r = 0; r < 8; ++r )
          x[ r ] = s_mask[ ( wv[ r >> 1 ] >> ( ( r & 1 ) * 16 ) ) & 0xffffu ];
        // inhibitory draws count in the upper half (uniform across the warp)
        const int j0 = jw * 8;
        if ( j0 >= g.ke )
        {
#pragma unroll
          for ( int r = 0; r < 8; ++r )
            x[ r ] <<= 16;
        }
        else if ( j0 + 8 > g.ke )
        {
#pragma unroll
          for ( int r = 0; r < 8; ++r )
            if ( j0 + r >= g.ke )
              x[ r ] <<= 16;
        }
        // Harley-Seal: 8 inputs through carry-save adders into P[0..2],
        // the weight-8 carries rippled into P[3..]
        uint32_t tA, tB, fA, fB, e;
        csa( tA, P[ 0 ], x[ 0 ], x[ 1 ] );
        csa( tB, P[ 0 ], x[ 2 ], x[ 3 ] );
        csa( fA, P[ 1 ], tA, tB );
        csa( tA, P[ 0 ], x[ 4 ], x[ 5 ] );
        csa( tB, P[ 0 ], x[ 6 ], x[ 7 ] );
        csa( fB, P[ 1 ], tA, tB );
        csa( e, P[ 2 ], fA, fB );
#pragma unroll
        for ( int b2 = 3; b2 < G_PLANES; ++b2 )
        {
          const uint32_t t = P[ b2 ] & e;
          P[ b2 ] ^= e;
          e = t;
          if ( e == 0u )
            break;
        }
      };
      // two words per step, the next step's two loaded before this step's
      // are counted (four 16-byte loads in flight per thread)
      const uint4 z4 = make_uint4( 0, 0, 0, 0 );
      uint4 c0 = b0 < b1 ? __ldg( col + ( int64_t ) b0 * 32 ) : z4;
      uint4 c1 = b0 + 1 < b1 ? __ldg( col + ( int64_t ) ( b0 + 1 ) * 32 ) : z4;
      for ( int jb = b0; jb < b1; jb += 2 )
      {
        const uint4 n0 = jb + 2 < b1 ? __ldg( col + ( int64_t ) ( jb + 2 ) * 32 ) : z4;
        const uint4 n1 = jb + 3 < b1 ? __ldg( col + ( int64_t ) ( jb + 3 ) * 32 ) : z4;
        eat( c0, jb );
        if ( jb + 1 < b1 )
          eat( c1, jb + 1 );
        c0 = n0;
        c1 = n1;
      }
    }
    // parts 1.. hand their planes to part 0, which adds them bit-parallel
    // (a ripple-carry adder over the 12 planes) and hands the sum back; then
    // every part adds count * weight into the ring for its share of the
    // (lag, type) pairs, all its ring loads issued before any store
    if ( part > 0 )
    {
#pragma unroll
      for ( int b = 0; b < G_PLANES; ++b )
        s_pl[ ( ( part - 1 ) * G_PLANES + b ) * GT + ti ] = P[ b ];
    }
    __syncthreads();
    if ( part == 0 )
    {
      for ( int q = 0; q < GP - 1; ++q )
      {
        uint32_t c = 0u;
#pragma unroll
        for ( int b = 0; b < G_PLANES; ++b )
        {
          const uint32_t y = s_pl[ ( q * G_PLANES + b ) * GT + ti ];
          const uint32_t u = P[ b ] ^ y;
          const uint32_t c2 = ( P[ b ] & y ) | ( u & c );
          P[ b ] = u ^ c;
          c = c2;
        }
      }
    }
    __syncthreads();
    if ( part == 0 )
    {
#pragma unroll
      for ( int b = 0; b < G_PLANES; ++b )
        s_pl[ b * GT + ti ] = P[ b ];
    }
    __syncthreads();
    if ( tl < g.n )
    {
      uint32_t S[ G_PLANES ];
#pragma unroll
      for ( int b = 0; b < G_PLANES; ++b )
        S[ b ] = s_pl[ b * GT + ti ];
      const int64_t t = g.off + tl;
      // this part owns lags k = part, part + GP, ... (< min_delay <= 16), both
      // types; with one channel (ce == ci) the two types share a ring cell
      // and are summed first
      constexpr int NLAG = 16 / GP;
      const int64_t dci = ( int64_t ) ( g.ci - g.ce ) * d.N;
      int64_t idx[ NLAG ];  // ring cell of the excitatory channel; inhibitory at + dci
      long long v[ 2 * NLAG ];
      unsigned act = 0u;
#pragma unroll
      for ( int j = 0; j < NLAG; ++j )
      {
        const int k = part + j * GP;
        long long ae = 0, ai = 0;
        if ( k < d.min_delay )
        {
          ae = ( long long ) plane_count( S, k ) * ( long long ) g.we;
          ai = ( long long ) plane_count( S, 16 + k ) * ( long long ) g.wi;
        }
        if ( dci == 0 )
        {
          ae += ai;
          ai = 0;
        }
        idx[ j ] = ( ( int64_t ) ( ( origin + k + g.d ) % d.L ) * d.C + g.ce ) * d.N + t;
        act |= ( ae ? 1u : 0u ) << ( 2 * j );
        act |= ( ai ? 1u : 0u ) << ( 2 * j + 1 );
        v[ 2 * j ] = ae;
        v[ 2 * j + 1 ] = ai;
      }
#pragma unroll
      for ( int u = 0; u < 2 * NLAG; ++u )
        if ( act >> u & 1u )
        {
          const int64_t i = idx[ u >> 1 ] + ( u & 1 ? dci : 0 );
          v[ u ] += d.ring32 ? ( long long ) reinterpret_cast< const int32_t* >( ring )[ i ] : ring[ i ];
        }
#pragma unroll
      for ( int u = 0; u < 2 * NLAG; ++u )
        if ( act >> u & 1u )
        {
          const int64_t i = idx[ u >> 1 ] + ( u & 1 ? dci : 0 );
          if ( d.ring32 )
            reinterpret_cast< int32_t* >( ring )[ i ] = ( int32_t ) v[ u ];
          else
            ring[ i ] = v[ u ];
        }
    }
    __syncthreads();
  }
}

}  // namespace ng

namespace ng
{

// ---------------------------------------------------------------------
// Spike log of a serving engine grouped by network at the end of a group
// (counting sort on the network id of each entry), so the host appends
// each network's spikes with one copy instead of routing them one by one.
// ---------------------------------------------------------------------
__global__ void
k_log_count( const Ctl* ctl, const uint2* half, int64_t cap, int n_nets, unsigned* cnt )
{
  __shared__ unsigned s_cnt[ 1024 ];
  for ( int k = threadIdx.x; k < n_nets; k += blockDim.x )
    s_cnt[ k ] = 0u;
  __syncthreads();
  const int64_t nl = min( ( int64_t ) ctl->log_count, cap );
  for ( int64_t k = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x; k < nl; k += ( int64_t ) gridDim.x * blockDim.x )
  {
    const unsigned id = half[ k ].x >> LOG_ID_SHIFT;
    if ( id < ( unsigned ) n_nets )
      atomicAdd( &s_cnt[ id ], 1u );
  }
  __syncthreads();
  for ( int k = threadIdx.x; k < n_nets; k += blockDim.x )
    if ( s_cnt[ k ] )
      atomicAdd( &cnt[ k ], s_cnt[ k ] );
}

// exclusive offsets per network (off[n_nets] = total); the counters are
// reset here and count again as the scatter's fill positions
__global__ void __launch_bounds__( 1024 )
k_log_offsets( unsigned* cnt, long long* off, int n_nets )
{
  __shared__ long long s[ 1024 ];
  const int t = threadIdx.x;
  const long long v = t < n_nets ? ( long long ) cnt[ t ] : 0ll;
  s[ t ] = v;
  __syncthreads();
  for ( int o = 1; o < 1024; o <<= 1 )
  {
    const long long a = t >= o ? s[ t - o ] : 0ll;
    __syncthreads();
    s[ t ] += a;
    __syncthreads();
  }
  if ( t < n_nets )
  {
    off[ t ] = s[ t ] - v;
    cnt[ t ] = 0u;
  }
  if ( t == 1023 )
    off[ n_nets ] = s[ 1023 ];
}

__global__ void
k_log_scatter( const Ctl* ctl, const uint2* half, int64_t cap, int n_nets, const long long* off, unsigned* fill,
  uint2* out )
{
  const int64_t nl = min( ( int64_t ) ctl->log_count, cap );
  for ( int64_t k = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x; k < nl; k += ( int64_t ) gridDim.x * blockDim.x )
  {
    const uint2 e = half[ k ];
    const unsigned id = e.x >> LOG_ID_SHIFT;
    if ( id < ( unsigned ) n_nets )
      out[ off[ id ] + atomicAdd( &fill[ id ], 1u ) ] = e;
  }
}

}  // namespace ng

namespace ng
{

// Largest sum of |stored weight| over one target's in-edges in a region of
// the edge pool (the ring-cell bound of a 32-bit ring).
__global__ void
k_in_abs_sum( long long e0, long long ne, const uint32_t* tdc, const int32_t* w, uint32_t tmask, long long n0,
  unsigned long long* sum )
{
  for ( long long k = ( long long ) blockIdx.x * blockDim.x + threadIdx.x; k < ne; k += ( long long ) gridDim.x * blockDim.x )
  {
    const int32_t wv = w[ e0 + k ];
    if ( wv != 0 )
      atomicAdd( sum + ( ( long long ) ( tdc[ e0 + k ] & tmask ) - n0 ),
        ( unsigned long long ) ( wv < 0 ? -( long long ) wv : ( long long ) wv ) );
  }
}

__global__ void
k_max_u64( long long n, const unsigned long long* v, unsigned long long* out )
{
  unsigned long long m = 0ull;
  for ( long long k = ( long long ) blockIdx.x * blockDim.x + threadIdx.x; k < n; k += ( long long ) gridDim.x * blockDim.x )
    m = v[ k ] > m ? v[ k ] : m;
#pragma unroll
  for ( int o = 16; o > 0; o >>= 1 )
  {
    const unsigned long long x = __shfl_xor_sync( FULL, m, o );
    m = x > m ? x : m;
  }
  if ( ( threadIdx.x & 31 ) == 0 && m )
    atomicMax( out, m );
}

}  // namespace ng

namespace ng
{

// ---------------------------------------------------------------------
// Target-tiled delivery (owner computes).  For a network whose rows are
// sorted by target, a CTA owns a tile of tile_t targets at a time: it walks
// the slice's spikes of the network, takes from each spike's row only the
// segment that falls into its tile, accumulates the weights in shared
// memory, and adds the non-zero cells to the ring with plain, coalesced
// read-modify-writes (the tile has no other writer).  The global atomics of
// the scatter -- one per synaptic event, which bound it on the L2 atomic
// units -- become shared-memory atomics.  Shared memory holds a window of
// TILE_W ring slots from the first slot the slice can reach; the rare events
// with longer delays go to the ring with global atomics.
// Work per warp: 8 spikes at a time -- their metadata (network, segment
// bounds, row) loaded by one lane each, in one round trip -- then their 8
// segments together, all lanes on consecutive edges of each, the loads of
// the 8 issued before any is used.  A network's tiles number about a
// multiple of the SM count (tt at admission), one CTA per SM.
// A spike of a tiled network is queued as one work entry (source, 0, -1,
// slot | multiplicity << 16); the scatter kernel skips it.
// A: accumulator type (int32: 32-bit rings, int64: fixed point, double: FP64).
// ---------------------------------------------------------------------
constexpr int TILE_W = 32;

template < typename A, bool FIX >
__device__ __forceinline__ void
tile_add( const Net& d, A* acc, int TT, int wbase, int slot, int ch, long long tl, long long gidx, A v )
{
  int ws = slot - wbase;
  if ( ws < 0 )
    ws += d.L;
  if ( ws < TILE_W && ws < d.L )
  {
    const int q = ( ws * d.C + ch ) * TT + ( int ) tl;
    if constexpr ( sizeof( A ) == 4 )
      atomicAdd( reinterpret_cast< int* >( acc ) + q, ( int ) v );
    else if constexpr ( FIX )
      atomicAdd( reinterpret_cast< unsigned long long* >( acc ) + q, ( unsigned long long ) v );
    else
      atomicAdd( reinterpret_cast< double* >( acc ) + q, ( double ) v );
  }
  else
  {
    const int64_t idx = ( ( int64_t ) slot * d.C + ch ) * d.N + gidx;
    if constexpr ( sizeof( A ) == 4 )
      atomicAdd( reinterpret_cast< int* >( d.ring ) + idx, ( int ) v );
    else if constexpr ( FIX )
      atomicAdd( reinterpret_cast< unsigned long long* >( d.ring ) + idx, ( unsigned long long ) v );
    else
      atomicAdd( reinterpret_cast< double* >( d.ring ) + idx, ( double ) v );
  }
}

template < typename A, bool FIX >
__global__ void __launch_bounds__( 1024, 1 )
k_deliver_tiled( Net d )
{
  extern __shared__ __align__( 16 ) unsigned char t_smem[];
  A* acc = reinterpret_cast< A* >( t_smem );  // [TILE_W][C][tile_t]
  __shared__ int s_pref[ 1025 ];
  __shared__ unsigned long long s_nent;
  __shared__ int s_err;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  if ( tid == 0 )
  {
    s_nent = ld_volatile( &d.ctl->n_ent );
    s_err = ld_volatile( &d.ctl->err );
  }
  const long long origin = cta_origin( d );  // synchronises the CTA
  for ( int id = tid; id < d.n_nets; id += blockDim.x )
    s_pref[ id + 1 ] = d.net_t[ id ].nt;
  if ( tid == 0 )
    s_pref[ 0 ] = 0;
  __syncthreads();
  if ( tid == 0 )
    for ( int id = 0; id < d.n_nets; ++id )
      s_pref[ id + 1 ] += s_pref[ id ];
  __syncthreads();
  const bool ok = ( long long ) s_nent <= d.ent_cap && ( s_err & ERR_SPIKE_LIST ) == 0;
  const long long nent = ok ? ( long long ) s_nent : 0;
  const int total = s_pref[ d.n_nets ];
  const int w0 = ( int ) ( ( long long ) total * blockIdx.x / gridDim.x );
  const int w1 = ( int ) ( ( long long ) total * ( blockIdx.x + 1 ) / gridDim.x );
  const int W = min( TILE_W, d.L );
  // first slot this slice's spikes can reach: origin + min_delay
  const int wbase = ( int ) ( ( origin + d.min_delay ) % d.L );
  for ( int w = w0; w < w1; ++w )
  {
    int lo = 0, hi = d.n_nets;
    while ( hi - lo > 1 )
    {
      const int mid = ( lo + hi ) >> 1;
      if ( s_pref[ mid ] <= w )
        lo = mid;
      else
        hi = mid;
    }
    const int id = lo;
    const TileNet g = d.net_t[ id ];
    const int TT = g.tt;
    const int cells = W * d.C * TT;
    const int tile = w - s_pref[ id ];
    const long long tb = ( long long ) tile * TT;
    const int tn = ( int ) min( ( long long ) TT, ( long long ) g.n - tb );
    for ( int q = tid; q < cells; q += blockDim.x )
      acc[ q ] = A( 0 );
    __syncthreads();
    for ( long long e0 = ( long long ) warp * 8; e0 < nent; e0 += ( long long ) nwarps * 8 )
    {
      // one spike per lane (lanes 0-7): its segment of this tile
      long long row = 0;
      int a = 0, b = 0, sw = 0;
      const long long e = e0 + lane;
      if ( lane < 8 && e < nent )
      {
        const int4 en = d.ent[ e ];
        if ( en.z == -1 && d.nid[ en.x ] == id )
        {
          const int32_t* sg = d.seg + g.seg_base + ( en.x - g.off ) * ( long long ) ( g.nt + 1 );
          a = sg[ tile ];
          b = sg[ tile + 1 ];
          row = d.row_beg[ en.x ];
          sw = en.w;
        }
      }
      // up to 8 spikes' segments at a time, their edge loads issued together
      unsigned live = __ballot_sync( FULL, b > a );
      while ( live )
      {
        long long ru[ 8 ];
        int au[ 8 ], bu[ 8 ], su[ 8 ];
        int span = 0;
#pragma unroll
        for ( int u = 0; u < 8; ++u )
        {
          const int j = live ? __ffs( live ) - 1 : 0;
          const bool has = live != 0;
          live &= live - 1;
          ru[ u ] = __shfl_sync( FULL, row, j );
          au[ u ] = __shfl_sync( FULL, a, j );
          bu[ u ] = has ? __shfl_sync( FULL, b, j ) : au[ u ];
          su[ u ] = __shfl_sync( FULL, sw, j );
          span = max( span, bu[ u ] - au[ u ] );
        }
        for ( int r = 0; r < span; r += 32 )
        {
          uint32_t tw[ 8 ];
          typename std::conditional< FIX, int32_t, double >::type wv[ 8 ];
#pragma unroll
          for ( int u = 0; u < 8; ++u )
          {
            const int k = au[ u ] + r + lane;
            tw[ u ] = 0u;
            wv[ u ] = 0;
            if ( k < bu[ u ] )
            {
              tw[ u ] = __ldg( d.edge_tdc + ru[ u ] + k );
              if constexpr ( FIX )
                wv[ u ] = __ldg( ( const int32_t* ) d.edge_w + ru[ u ] + k );
              else
                wv[ u ] = __ldg( ( const double* ) d.edge_w + ru[ u ] + k );
            }
          }
#pragma unroll
          for ( int u = 0; u < 8; ++u )
          {
            if ( au[ u ] + r + lane >= bu[ u ] )
              continue;
            const long long tl = ( long long ) ( tw[ u ] & d.tmask ) - g.off - tb;
            if ( tl < 0 || tl >= TT )
              continue;  // outside the tile: cannot happen for a correct segment table
            int slot = ( su[ u ] & 0xffff ) + ( int ) ( ( tw[ u ] >> d.tbits ) & d.dmask );
            if ( slot >= d.L )
              slot -= d.L;
            const int mult = su[ u ] >> 16;
            const int ch = ( int ) ( tw[ u ] >> 31 );
            if constexpr ( FIX )
              tile_add< A, FIX >( d, acc, TT, wbase, slot, ch, tl, g.off + tb + tl,
                ( A ) ( ( long long ) wv[ u ] * mult ) );
            else
              tile_add< A, FIX >( d, acc, TT, wbase, slot, ch, tl, g.off + tb + tl,
                ( A ) ( mult == 1 ? wv[ u ] : wv[ u ] * ( double ) mult ) );
          }
        }
      }
    }
    __syncthreads();
    for ( int q = tid; q < cells; q += blockDim.x )
    {
      const int t = q % TT;
      if ( t >= tn )
        continue;
      const A v = acc[ q ];
      if ( v == A( 0 ) )
        continue;
      const int sc = q / TT;  // window slot * C + channel
      int slot = wbase + sc / d.C;
      if ( slot >= d.L )
        slot -= d.L;
      const int64_t idx = ( ( int64_t ) slot * d.C + sc % d.C ) * d.N + g.off + tb + t;
      reinterpret_cast< A* >( d.ring )[ idx ] += v;
    }
    __syncthreads();
  }
}

// Segment table of one network (rows sorted by target): entry (s, b) is
// the first position in row s whose local target is >= b * tile_t.
__global__ void
k_seg_build( long long n, int nt, int tile_t, long long n0, const int64_t* row_beg, const int32_t* real_deg,
  const uint32_t* tdc, uint32_t tmask, int32_t* seg )
{
  const long long idx = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( idx >= n * ( nt + 1 ) )
    return;
  const long long s = idx / ( nt + 1 );
  const int b = ( int ) ( idx - s * ( nt + 1 ) );
  const int len = real_deg[ n0 + s ];
  if ( b == nt )
  {
    seg[ idx ] = len;
    return;
  }
  const long long row = row_beg[ n0 + s ];
  const long long bound = n0 + ( long long ) b * tile_t;
  int lo = 0, hi = len;  // first k with target >= bound
  while ( lo < hi )
  {
    const int mid = ( lo + hi ) >> 1;
    if ( ( long long ) ( tdc[ row + mid ] & tmask ) < bound )
      lo = mid + 1;
    else
      hi = mid;
  }
  seg[ idx ] = lo;
}

}  // namespace ng
