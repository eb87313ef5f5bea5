// noalloc.cu -- ng_simulate_noalloc: the slice cycle of a small iaf_psc_delta
// network (plain FP64 form) that allocates no memory at all.
//
// Who needs it: callers that may not allocate device memory on the path
// that steps the network -- e.g. a host framework that owns all device
// memory through its own allocator or memory pool and forbids foreign
// cudaMalloc calls, or a closed-loop controller that steps a small network
// every control tick, where an allocation's implicit device synchronisation
// and latency jitter are not acceptable.  The caller passes every input and
// output as device memory it owns; the ring buffer, the per-slice spike list
// and the control counters live in one file-scope device array
// (g_noalloc_scratch, NG_NOALLOC_SCRATCH_BYTES = 16 MiB) that every GPU
// which loads the library holds until the process exits.
//
// The kernels are variants of the engine's node-update and delivery kernels
// (ng_kernels.cuh) for unpadded CSR input: same arithmetic in the same order,
// so a run matches ng_simulate on the same network.  A controller that steps
// the network a few steps per tick sets continue_run: the ring buffer and
// the open slice's spikes stay in the scratch array between its calls, and
// a chain of calls equals one call over the same steps.  The edges come from
// caller memory and are range-checked on the device before they index the
// ring.
#include <cstddef>
#include <cstdint>
#include <algorithm>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/nestgpu.h"

namespace
{

constexpr int NA_MAX_DEVICES = 64;

__device__ __align__( 256 ) unsigned char g_noalloc_scratch[ NG_NOALLOC_SCRATCH_BYTES ];

// counters at the start of the scratch array
struct NaCtl
{
  unsigned long long n_spk;   // spikes of the open slice
  unsigned long long n_out;   // spikes of this call (written to the caller's output up to out_cap)
  unsigned long long n_skip;  // edges of this call skipped for an out-of-range target or delay
};

// Where the previous call on a device stopped, for continue_run: the
// scratch array holds that run's ring and open-slice spike list.
struct NaRun
{
  bool valid = false;
  int64_t n = 0;
  int32_t min_delay = 0, max_delay = 0;
  int64_t next_step = 0;
};

struct NaNet
{
  int64_t n;
  int32_t L, min_delay, max_delay;
  const double *P33, *P30, *V_th, *V_reset, *V_min, *I_e;
  const int32_t* refr_counts;
  double* V;
  int32_t* r;
  const int64_t* row_ptr;
  const int32_t* target;
  const double* weight;
  const int32_t* delay;
  int32_t* out_src;
  int64_t* out_stamp;
  int64_t out_cap;
  unsigned long long* out_count;
  unsigned long long* out_skipped;
  // scratch
  NaCtl* ctl;
  double* ring;     // [L][n]
  int2* spk;       // (source, emission slot)
  int64_t spk_cap;
};

// iaf_psc_delta::update (models/iaf_psc_delta.cpp:272-329), one thread per
// neuron over the lags [from, to) of the slice at `origin`.
__global__ void
k_na_update( NaNet d, long long origin, int from, int to )
{
  const int64_t i = ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x;
  if ( i >= d.n )
    return;
  double V = d.V[ i ];
  int r = d.r[ i ];
  const double P33 = d.P33[ i ], P30 = d.P30[ i ], Vth = d.V_th[ i ], Vreset = d.V_reset[ i ], Vmin = d.V_min[ i ];
  const double Ie = d.I_e[ i ];
  const int refr = d.refr_counts[ i ];
  const double y0 = 0.0;
  for ( int lag = from; lag < to; ++lag )
  {
    const long long t = origin + lag;
    const int slot = ( int ) ( t % d.L );
    const double in = d.ring[ ( int64_t ) slot * d.n + i ];
    d.ring[ ( int64_t ) slot * d.n + i ] = 0.0;
    if ( r == 0 )
    {
      V = P30 * ( y0 + Ie ) + P33 * V + in;
      V = ( V < Vmin ? Vmin : V );
    }
    else
    {
      --r;
    }
    if ( V >= Vth )
    {
      r = refr;
      V = Vreset;
      const unsigned long long k = atomicAdd( &d.ctl->n_spk, 1ull );
      if ( ( int64_t ) k < d.spk_cap )
        d.spk[ k ] = make_int2( ( int ) i, slot );
      const unsigned long long o = atomicAdd( &d.ctl->n_out, 1ull );
      if ( ( int64_t ) o < d.out_cap )
      {
        d.out_src[ o ] = ( int32_t ) i;
        d.out_stamp[ o ] = t + 1;
      }
    }
  }
  d.V[ i ] = V;
  d.r[ i ] = r;
}

// Delivery of the closing slice: one warp per spike walks its CSR row and
// adds the weights into ring[(t_emit + d) mod L][target].  The edges come
// from caller memory: one whose target or delay is out of range would index
// outside the ring, so it is skipped and counted instead.
__global__ void
k_na_deliver( NaNet d )
{
  const unsigned long long nspk = *( volatile unsigned long long* ) &d.ctl->n_spk;
  const int64_t warp = ( ( int64_t ) blockIdx.x * blockDim.x + threadIdx.x ) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t nw = ( ( int64_t ) gridDim.x * blockDim.x ) >> 5;
  const int64_t ns = ( int64_t ) nspk < d.spk_cap ? ( int64_t ) nspk : d.spk_cap;
  for ( int64_t s = warp; s < ns; s += nw )
  {
    const int2 sp = d.spk[ s ];
    const int64_t e0 = d.row_ptr[ sp.x ], e1 = d.row_ptr[ sp.x + 1 ];
    for ( int64_t e = e0 + lane; e < e1; e += 32 )
    {
      const int32_t tg = d.target[ e ];
      const int32_t dl = d.delay[ e ];
      if ( tg < 0 || ( int64_t ) tg >= d.n || dl < d.min_delay || dl > d.max_delay )
      {
        atomicAdd( &d.ctl->n_skip, 1ull );
        continue;
      }
      int slot = sp.y + dl;  // sp.y < L and dl <= max_delay < L
      if ( slot >= d.L )
        slot -= d.L;
      atomicAdd( d.ring + ( int64_t ) slot * d.n + tg, d.weight[ e ] );
    }
  }
}

__global__ void
k_na_close_slice( NaNet d )
{
  d.ctl->n_spk = 0ull;
}

// A continued run keeps the ring and the open slice's spikes; only the
// per-call counters start from zero.
__global__ void
k_na_begin_call( NaNet d )
{
  d.ctl->n_out = 0ull;
  d.ctl->n_skip = 0ull;
}

__global__ void
k_na_finish( NaNet d )
{
  *d.out_count = d.ctl->n_out;
  if ( d.out_skipped )
    *d.out_skipped = d.ctl->n_skip;
}

std::mutex g_na_mutex;
void* g_na_addr[ NA_MAX_DEVICES ] = {};
NaRun g_na_run[ NA_MAX_DEVICES ];

}  // namespace

void ng_internal_set_error( const char* msg );

extern "C" {

int
ng_simulate_noalloc( const ng_noalloc_net* net, int64_t n_steps, void* cuda_stream )
{
  if ( !net || n_steps < 0 )
  {
    ng_internal_set_error( "ng_simulate_noalloc: null network or negative step count" );
    return NG_ERR_ARG;
  }
  if ( net->n < 1 || net->n > INT32_MAX || net->min_delay < 1 || net->max_delay < net->min_delay
    || net->start_step < 0 || net->out_cap < 0 || ( net->continue_run != 0 && net->continue_run != 1 )
    || net->reserved != 0 )
  {
    ng_internal_set_error( "ng_simulate_noalloc: need 1 <= n < 2^31, 1 <= min_delay <= max_delay, start_step >= 0, "
                           "out_cap >= 0, continue_run 0 or 1, reserved 0" );
    return NG_ERR_ARG;
  }
  if ( !net->continue_run && net->start_step % net->min_delay != 0 )
  {
    ng_internal_set_error( "ng_simulate_noalloc: a fresh run starts at a slice boundary (start_step a multiple of "
                           "min_delay)" );
    return NG_ERR_ARG;
  }
  if ( !net->P33 || !net->P30 || !net->V_th_rel || !net->V_reset_rel || !net->V_min_rel || !net->I_e
    || !net->refr_counts || !net->V_m_rel || !net->r || !net->row_ptr || !net->target || !net->weight || !net->delay
    || !net->out_src || !net->out_stamp || !net->out_count )
  {
    ng_internal_set_error( "ng_simulate_noalloc: a required device pointer is null" );
    return NG_ERR_ARG;
  }
  int dev = 0;
  if ( cudaGetDevice( &dev ) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES )
  {
    ng_internal_set_error( "ng_simulate_noalloc: no current CUDA device" );
    return NG_ERR_CUDA;
  }
  const int64_t L = ( int64_t ) net->min_delay + net->max_delay;
  // scratch layout: [NaCtl | pad to 256][ring L*n doubles][spike list n*min_delay int2]
  const size_t ctl_bytes = 256;
  const size_t ring_bytes = ( size_t ) L * ( size_t ) net->n * sizeof( double );
  const size_t spk_cap = ( size_t ) net->n * ( size_t ) net->min_delay;
  const size_t need = ctl_bytes + ( ( ring_bytes + 255 ) & ~( size_t ) 255 ) + spk_cap * sizeof( int2 );
  if ( L > INT32_MAX / 2 || need > NG_NOALLOC_SCRATCH_BYTES )
  {
    ng_internal_set_error( "ng_simulate_noalloc: the network's ring buffer and spike list need more than the "
                           "16 MiB static scratch array (NG_NOALLOC_SCRATCH_BYTES)" );
    return NG_ERR_CAPACITY;
  }
  std::lock_guard< std::mutex > lock( g_na_mutex );
  // once per device, with that device current: the scratch array's device
  // address (the symbol itself names a host-side stand-in)
  if ( !g_na_addr[ dev ] )
  {
    if ( cudaGetSymbolAddress( &g_na_addr[ dev ], g_noalloc_scratch ) != cudaSuccess )
    {
      g_na_addr[ dev ] = nullptr;
      ng_internal_set_error( "ng_simulate_noalloc: cudaGetSymbolAddress of the scratch array failed" );
      return NG_ERR_CUDA;
    }
  }
  void* const base = g_na_addr[ dev ];
  NaRun& run = g_na_run[ dev ];
  if ( net->continue_run
    && !( run.valid && run.n == net->n && run.min_delay == net->min_delay && run.max_delay == net->max_delay
      && run.next_step == net->start_step ) )
  {
    ng_internal_set_error( "ng_simulate_noalloc: continue_run needs the previous call on this device to have run the "
                           "same network (n, min_delay, max_delay) up to start_step" );
    return NG_ERR_STATE;
  }
  cudaStream_t st = ( cudaStream_t ) cuda_stream;
  NaNet d {};
  d.n = net->n;
  d.L = ( int32_t ) L;
  d.min_delay = net->min_delay;
  d.max_delay = net->max_delay;
  d.P33 = net->P33;
  d.P30 = net->P30;
  d.V_th = net->V_th_rel;
  d.V_reset = net->V_reset_rel;
  d.V_min = net->V_min_rel;
  d.I_e = net->I_e;
  d.refr_counts = net->refr_counts;
  d.V = net->V_m_rel;
  d.r = net->r;
  d.row_ptr = net->row_ptr;
  d.target = net->target;
  d.weight = net->weight;
  d.delay = net->delay;
  d.out_src = net->out_src;
  d.out_stamp = net->out_stamp;
  d.out_cap = net->out_cap;
  d.out_count = net->out_count;
  d.out_skipped = net->out_skipped;
  d.ctl = ( NaCtl* ) base;
  d.ring = ( double* ) ( ( unsigned char* ) base + ctl_bytes );
  d.spk = ( int2* ) ( ( unsigned char* ) base + ctl_bytes + ( ( ring_bytes + 255 ) & ~( size_t ) 255 ) );
  d.spk_cap = ( int64_t ) spk_cap;
  // until this call has been enqueued, no later call may continue its run
  run.valid = false;
  cudaError_t ce;
  if ( net->continue_run )
  {
    k_na_begin_call<<< 1, 1, 0, st >>>( d );
    ce = cudaGetLastError();
  }
  else
  {
    // a fresh run: counters and ring buffer to zero
    ce = cudaMemsetAsync( base, 0, ctl_bytes + ring_bytes, st );
  }
  if ( ce != cudaSuccess )
  {
    ng_internal_set_error( "ng_simulate_noalloc: clearing the scratch array failed" );
    return NG_ERR_CUDA;
  }
  const unsigned ugrid = ( unsigned ) ( ( net->n + 255 ) / 256 );
  const unsigned dgrid = 64;
  // slice origin and the lag the run stands at (a continued run may stop
  // and resume inside a slice; fresh runs start at a slice boundary)
  const int64_t lag0 = net->start_step % net->min_delay;
  long long origin = net->start_step - lag0;
  int from = ( int ) lag0;
  int64_t left = n_steps;
  while ( left > 0 )
  {
    const int to = ( int ) std::min< int64_t >( ( int64_t ) from + left, net->min_delay );
    k_na_update<<< ugrid, 256, 0, st >>>( d, origin, from, to );
    left -= to - from;
    if ( to == net->min_delay )
    {
      k_na_deliver<<< dgrid, 256, 0, st >>>( d );
      k_na_close_slice<<< 1, 1, 0, st >>>( d );
      origin += net->min_delay;
      from = 0;
    }
    else
    {
      from = to;
    }
  }
  k_na_finish<<< 1, 1, 0, st >>>( d );
  if ( cudaGetLastError() != cudaSuccess )
  {
    ng_internal_set_error( "ng_simulate_noalloc: kernel launch failed" );
    return NG_ERR_CUDA;
  }
  run.valid = true;
  run.n = net->n;
  run.min_delay = net->min_delay;
  run.max_delay = net->max_delay;
  run.next_step = net->start_step + n_steps;
  return NG_OK;
}

}  // extern "C"
