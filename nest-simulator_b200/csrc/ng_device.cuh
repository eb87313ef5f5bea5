// ng_device.cuh -- device-side data layout and helpers of the slice engine.
//
// HBM layout (one engine = one network, N neurons, ring length L = max_delay:
// a slice's update reads its min_delay slots before the slice's delivery
// writes arrivals t_emit + d <= t_end - 1 + max_delay, so max_delay slots
// hold every pending arrival -- the reference's rings hold min_delay +
// max_delay because it delivers before it updates):
//   state     SoA arrays per model block, FP64 (plain) or FP32 (precision form)
//   classes   per-neuron class id -> row of FP64 coefficients (propagators,
//             thresholds, refractory counts) computed on the host
//   ring      [L][C][N] FP64 (plain) or int64 fixed point (precision form),
//             C = 2 input channels (excitatory / inhibitory)
//   CSR       row_beg[n_src] (int64) and row_len[n_src] (int32): a source's
//             row, padded to a multiple of 4 edges (rows of the networks of a
//             serving engine live anywhere in the edge pool),
//             packed edge word tgt | delay << tbits | channel << 31 (u32),
//             weight FP64 (plain) or int32 fixed point (precision form)
//   edge work per-slice list of edge chunks of the spikes to deliver: (row
//             start, up to 128 edges, emission slot, multiplicity)
//   log       (source, stamp - log_base | multiplicity << 24) for recorders
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ng
{

constexpr int CT_STRIDE = 20;  // doubles per coefficient-class row
constexpr int MAX_STATE = 8;
constexpr uint32_t DRIVE_STREAM = 0x504F4953u;
constexpr int ERR_NUMERIC = 1;
constexpr int ERR_SPIKE_LIST = 2;
constexpr int ERR_LOG = 4;
constexpr int ERR_TRACE = 8;
constexpr int CHUNK_EDGES = 128;  // edges per delivery work item: 32 lanes x 4 edges

// Control block in device memory, shared by all kernels of an engine.
struct Ctl
{
  unsigned long long n_ent;       // edge chunks queued for delivery in the open slice
  unsigned long long log_count;
  unsigned long long syn_events;
  unsigned long long drive_events;
  unsigned long long n_spikes;
  long long origin;     // slice origin [steps]
  long long log_base;   // stamp offset of the log entries
  long long trace_row0; // first trace row index held in the buffer
  long long sched_pos;  // next unconsumed scheduled generator spike
  unsigned long long gathered;  // (network, slice) pairs delivered by the per-target gather
  int deliver_done;     // finished CTAs of the running delivery launch
  int err;
  int log_sel;          // half of the spike log the running group writes
  // late delivery (edges of delay >= 2 min_delay, delivered while the next
  // slice updates): two chunk lists used by alternate slices
  unsigned long long n_late[ 2 ];
  int late_wr;    // list the open slice's update appends to (flipped when the slice closes)
  int late_rd;    // list the next late delivery reads (flipped by that delivery)
  int late_done;  // finished CTAs of the running late delivery
};

// Spike-log entry of a serving engine: network-local source | network id << 22.
constexpr int LOG_ID_SHIFT = 22;

struct Block
{
  int64_t off, n;
  int model;
  const int32_t* cls;
  const double* ctab;
  void* s[ MAX_STATE ];
  int32_t* r;
  double* istep;
  const int32_t* perm;  // aeif: thread -> neuron order grouping equal RKF45 step sizes (nullptr: identity)
};

// Per-target gather of one fixed_indegree network of a serving engine
// (precision form): in-edge table gin[base + j * n + t] (16-bit local source
// ids, excitatory draws j < ke first, then ki inhibitory ones), uniform
// weights we / wi (fixed point) into ring channels ce / ci, delay d.
// ke + ki == 0: no table.
struct GatherNet
{
  long long base, off;
  int n, ke, ki, d;
  int we, wi, ce, ci;
};

// Target-tiled delivery of one network of a serving engine: its rows are
// sorted by target; seg[seg_base + s * (nt + 1) + b] = first position in
// source s's row whose target lies in tile b,
// seg[..+ nt] = the row's real length; tiles of tt targets (at most the
// engine's tile_t).  nt == 0: not tiled.
struct TileNet
{
  long long seg_base, off;
  int n, nt, tt;  // neurons, tiles, targets per tile
  int pad;
};

struct Net
{
  int64_t N, n_src;
  int32_t L, C, min_delay;
  int32_t tbits;
  uint32_t tmask, dmask;
  void* ring;
  double fx_inv;  // precision form: 2^-S of the fixed-point weights
  const int64_t* row_beg;
  const int32_t* row_len;
  const int32_t* real_deg;
  const uint32_t* edge_tdc;
  const void* edge_w;
  int4* ent;  // edge chunks: row start (lo, hi), edge count, slot | multiplicity << 16
  int64_t ent_cap;
  // late delivery; late_min == INT32_MAX: off (every edge is delivered when
  // its slice closes).  A row holds its edges of delay < late_min first:
  // edges [0, row_ue) are covered by the slice-close chunks and [row_ls,
  // padded length) by the late ones (row_ls <= row_ue: the ranges may share
  // a 4-edge group; each delivery applies only its own delays)
  int32_t late_min;
  const int32_t* row_ue;
  const int32_t* row_ls;
  int4* ent_late;  // two lists of ent_cap entries
  uint2* log;           // two halves of log_cap entries (groups alternate)
  int64_t log_cap;
  const uint8_t* rec;
  const double4* pois;  // lambda, p_m, F_m, m (walk from the mode, long tables)
  const int2* pois_cdf_ref;  // per neuron: (offset, length) into pois_cdf; length 0 = no drive, -1 = walk
  const uint64_t* pois_cdf;  // concatenated CDF tables, one per distinct rate, as 53-bit thresholds
  const double* pois_w;
  const int32_t* pois_d;
  int64_t pois_start, pois_stop;
  uint32_t key0, key1;
  int has_pois;
  int ring32;  // precision form with 32-bit ring cells
  const int32_t* trace_col;
  double* trace;
  int32_t n_trace_idx, trace_interval, n_trace_vars;
  int8_t trace_slot[ MAX_STATE ];
  int64_t trace_rows;
  // networks of a serving engine (nid == nullptr: one network, always on)
  const int32_t* nid;            // per neuron: network id, -1 = free
  const long long* net_step0;    // per network: admission step (its local time 0)
  const long long* net_until;    // per network: first step it no longer simulates
  const long long* net_off;      // per network: first neuron
  const uint2* net_key;          // per network: Philox key of its drive
  // per-target gather (serving, precision form); gmask == nullptr: off
  uint32_t* gmask;               // per neuron: bit k = spike at lag k of the open slice
  const uint16_t* gin;           // in-edge tables of the gather networks
  const GatherNet* net_g;        // per network
  int* net_mode;                 // per network: 1 = gather this slice, 0 = scatter
  unsigned* net_spk;             // per network: spikes in the open slice
  int n_nets;
  float gather_frac;             // gather the next slice when spikes >= gather_frac * n
  // target-tiled delivery; net_t == nullptr: off
  const TileNet* net_t;
  const int32_t* seg;
  int tile_t;
  const int64_t* sched_step;
  const int32_t* sched_src;
  int64_t n_sched;
  int32_t deliver_group;  // most edge chunks one delivery warp takes per descriptor load (autotuned)
  Ctl* ctl;
};

// ---------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11), u53 and Poisson inversion from the
// mode.  Identical arithmetic on host and device: only integer ops, exact
// int->double conversions, and IEEE multiplies/divides/adds (no contraction).
// ---------------------------------------------------------------------
__host__ __device__ inline void
philox4x32_10( uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t out[ 4 ] )
{
#pragma unroll
  for ( int r = 0; r < 10; ++r )
  {
    if ( r > 0 )
    {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = ( uint64_t ) 0xD2511F53u * c0;
    const uint64_t p1 = ( uint64_t ) 0xCD9E8D57u * c2;
    const uint32_t n0 = ( uint32_t ) ( p1 >> 32 ) ^ c1 ^ k0;
    const uint32_t n1 = ( uint32_t ) p1;
    const uint32_t n2 = ( uint32_t ) ( p0 >> 32 ) ^ c3 ^ k1;
    const uint32_t n3 = ( uint32_t ) p0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
  }
  out[ 0 ] = c0;
  out[ 1 ] = c1;
  out[ 2 ] = c2;
  out[ 3 ] = c3;
}

__host__ __device__ inline double
u53( uint32_t a, uint32_t b )
{
  return ( ( double ) ( a >> 5 ) * 67108864.0 + ( double ) ( b >> 6 ) ) * ( 1.0 / 9007199254740992.0 );
}

// The 53-bit integer m of u53(a, b) = m * 2^-53.  For a CDF value F in
// [0, 1], u > F holds exactly when m > floor(F * 2^53) (F * 2^53 is exact),
// so the inversion compares integers: no int->double conversion and no FP64
// compare per draw.
__host__ __device__ inline uint64_t
u53_bits( uint32_t a, uint32_t b )
{
  return ( ( uint64_t ) ( a >> 5 ) << 26 ) | ( uint64_t ) ( b >> 6 );
}

// (double) x, exactly, without a conversion instruction: 2^52 + x has x in
// the low mantissa bits.
__device__ __forceinline__ double
u32_to_f64( uint32_t x )
{
  return __hiloint2double( 0x43300000, ( int ) x ) - 4503599627370496.0;
}

// tab = (lambda, p_m, F_m, m): walk from the mode m up while u > F or down
// while u <= F - p.
__host__ __device__ inline long long
poisson_from_mode( double4 tab, double u )
{
  const double lam = tab.x;
  long long k = ( long long ) tab.w;
  double p = tab.y, F = tab.z;
  if ( u > F )
  {
    const long long kmax = k + 100000;
    while ( u > F && k < kmax )
    {
      k += 1;
      p = p * lam / ( double ) k;
      F += p;
      if ( p == 0.0 )
        break;
    }
    return k;
  }
  while ( k > 0 && u <= F - p )
  {
    F -= p;
    p = p * ( double ) k / lam;
    k -= 1;
  }
  return k;
}

}  // namespace ng
