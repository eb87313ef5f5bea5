/*
 * nest_oracle.c -- CPU restatement of NEST's per-min_delay simulation cycle.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see nest_oracle.h).  Compiled with
 * -O2 -ffp-contract=off so that every multiply and add rounds separately, as
 * the reference's x86-64 build does (its baseline ISA has no FMA).
 *
 * Internal representations follow the reference's State_/Parameters_
 * structs: the iaf models keep V_m, V_th, V_reset and V_min relative to E_L
 * (models/iaf_psc_delta.cpp:94-150, models/iaf_psc_exp.cpp:100-190), aeif
 * keeps absolute values (models/aeif_cond_alpha.cpp:130-300).
 */
#include "nest_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static char g_err[ 256 ];
static void
set_err( const char* m )
{
  snprintf( g_err, sizeof( g_err ), "%s", m );
}
const char*
orc_error( void )
{
  return g_err;
}

/* ---------------------------------------------------------------------
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11).  Round: two 32x32->64 multiplies by the Philox
 * multipliers, a key xor, a lane permutation; the key is bumped by the Weyl
 * constants between rounds.
 * ------------------------------------------------------------------- */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void
orc_philox4x32( const uint32_t ctr[ 4 ], const uint32_t key[ 2 ], int rounds, uint32_t out[ 4 ] )
{
  uint32_t c0 = ctr[ 0 ], c1 = ctr[ 1 ], c2 = ctr[ 2 ], c3 = ctr[ 3 ];
  uint32_t k0 = key[ 0 ], k1 = key[ 1 ];
  for ( int r = 0; r < rounds; ++r )
  {
    if ( r > 0 )
    {
      k0 += PHILOX_W0;
      k1 += PHILOX_W1;
    }
    const uint64_t p0 = ( uint64_t ) PHILOX_M0 * c0;
    const uint64_t p1 = ( uint64_t ) PHILOX_M1 * c2;
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

/* Stream tag of the Poisson drive in the Philox counter's last word. */
#define DRIVE_STREAM 0x504F4953u

/* Uniform double in [0,1) with 53 random bits from two 32-bit words. */
static inline double
u53( uint32_t a, uint32_t b )
{
  return ( ( double ) ( a >> 5 ) * 67108864.0 + ( double ) ( b >> 6 ) ) * ( 1.0 / 9007199254740992.0 );
}

/* Poisson(lambda) by inversion: the smallest k with u <= F(k), read from a
 * precomputed CDF table, or for long tables by walking from the mode
 * (Kemp & Kemp 1991): start at m = floor(lambda) with p_m and F_m = P(X <= m)
 * precomputed, walk down while u <= F - p, else up while u > F. */
typedef struct
{
  double lambda, pm, Fm;
  int64_t m;
  double* cdf; /* cdf[k] = P(X <= k), last entry 1; NULL: walk from the mode */
  int len;
} pois_tab;

/* CDF table, summed upward in FP64 until 1 - F < 1e-17 (k > lambda) or 256
 * entries; the last entry is set to 1.  No table for lambda > 100 or when the
 * tail is not reached. */
static void
pois_cdf_table( pois_tab* t )
{
  t->cdf = NULL;
  t->len = 0;
  const double lambda = t->lambda;
  if ( !( lambda > 0.0 ) || lambda > 100.0 )
    return;
  double* c = malloc( sizeof( double ) * 256 );
  double p = exp( -lambda ), F = p;
  int n = 0;
  c[ n++ ] = F;
  for ( int k = 1; k < 256; ++k )
  {
    p = p * lambda / ( double ) k;
    F += p;
    c[ n++ ] = F;
    if ( 1.0 - F < 1e-17 && ( double ) k > lambda )
      break;
  }
  if ( 1.0 - F > 1e-15 )
  {
    free( c );
    return;
  }
  c[ n - 1 ] = 1.0;
  t->cdf = c;
  t->len = n;
}

static pois_tab
pois_prepare( double lambda )
{
  pois_tab t;
  t.lambda = lambda;
  t.m = ( int64_t ) floor( lambda );
  t.cdf = NULL;
  t.len = 0;
  if ( lambda <= 0.0 )
  {
    t.m = 0;
    t.pm = 1.0;
    t.Fm = 1.0;
    return t;
  }
  t.pm = exp( -lambda + ( double ) t.m * log( lambda ) - lgamma( ( double ) t.m + 1.0 ) );
  /* F_m by summing the pmf upward from 0 (exact enough in FP64 for m < 1e6) */
  double p = exp( -lambda ), F = p;
  for ( int64_t k = 1; k <= t.m; ++k )
  {
    p = p * lambda / ( double ) k;
    F += p;
  }
  t.Fm = F;
  pois_cdf_table( &t );
  return t;
}

static inline int64_t
pois_draw( const pois_tab* t, double u )
{
  if ( t->cdf )
  {
    int j = 0;
    while ( j < t->len - 1 && u > t->cdf[ j ] )
      ++j;
    return j;
  }
  int64_t k = t->m;
  double p = t->pm, F = t->Fm;
  if ( u > F )
  {
    while ( u > F && k < t->m + 100000 )
    {
      k += 1;
      p = p * t->lambda / ( double ) k;
      F += p;
      if ( p == 0.0 )
        break;
    }
    return k;
  }
  while ( k > 0 && u <= F - p )
  {
    F -= p;
    p = p * ( double ) k / t->lambda;
    k -= 1;
  }
  return k;
}

int64_t
orc_poisson_draw( double lambda, double u )
{
  pois_tab t = pois_prepare( lambda );
  const int64_t k = pois_draw( &t, u );
  free( t.cdf );
  return k;
}

/* ---------------------------------------------------------------------
 * Propagators (libnestutil/iaf_propagator.cpp:42-75)
 * ------------------------------------------------------------------- */
double
orc_iaf_propagator_exp( double tau_syn, double tau_m, double c_m, double h )
{
  const double beta = tau_syn * tau_m / ( tau_m - tau_syn );
  const double gamma = beta / c_m;
  const double inv_tau_syn = 1 / tau_syn;
  const double inv_tau_m = 1 / tau_m;
  const double inv_c_m = 1 / c_m;
  const double inv_beta = ( tau_m - tau_syn ) / ( tau_syn * tau_m );
  const double exp_h_tau_syn = exp( -h * inv_tau_syn );
  const double expm1_h_tau = expm1( h * inv_beta );
  const double P32 = gamma * exp_h_tau_syn * expm1_h_tau;
  if ( isnormal( P32 ) && P32 > 0 )
  {
    return P32;
  }
  const double exp_h_tau = exp( -h * inv_tau_m );
  return h * inv_c_m * exp_h_tau;
}

/* IAFPropagatorAlpha::evaluate (libnestutil/iaf_propagator.cpp:95-118) with
 * the base class's P32 (:56-75) and h_min_regular from
 * NUMERICAL_STABILITY_FACTOR_ = 1e-7 (iaf_propagator.h:66). */
void
orc_iaf_propagator_alpha( double tau_syn, double tau_m, double c_m, double h, double* out )
{
  const double h_min_regular = 1e-7 * tau_m * tau_m / fabs( tau_m - tau_syn );
  const double beta = tau_syn * tau_m / ( tau_m - tau_syn );
  const double gamma = beta / c_m;
  const double inv_tau_syn = 1 / tau_syn;
  const double inv_tau_m = 1 / tau_m;
  const double inv_c_m = 1 / c_m;
  const double inv_beta = ( tau_m - tau_syn ) / ( tau_syn * tau_m );
  const double exp_h_tau_syn = exp( -h * inv_tau_syn );
  const double expm1_h_tau = expm1( h * inv_beta );
  double P32 = gamma * exp_h_tau_syn * expm1_h_tau;
  double exp_h_tau = NAN;
  if ( !( isnormal( P32 ) && P32 > 0 ) )
  {
    exp_h_tau = exp( -h * inv_tau_m );
    P32 = h * inv_c_m * exp_h_tau;
  }
  out[ 1 ] = P32;
  if ( h > h_min_regular )
  {
    out[ 0 ] = gamma * exp_h_tau_syn * ( beta * expm1_h_tau - h );
    return;
  }
  if ( isnan( exp_h_tau ) )
    exp_h_tau = exp( -h * inv_tau_m );
  out[ 0 ] = 0.5 * h * h * inv_c_m * exp_h_tau;
}

/* Time(ms(t)).get_steps() with the default 1000 tics/ms
 * (nestkernel/nest_time.h:306-311, 508-521). */
static int64_t
ms_to_steps_roundup( double ms, double tics_per_ms, int64_t tics_per_step )
{
  const int64_t tics = ( int64_t ) ( ms * tics_per_ms + 0.5 );
  return ( int64_t ) ( ( double ) ( tics + tics_per_step - 1 ) * ( 1. / ( double ) tics_per_step ) );
}

/* ---------------------------------------------------------------------
 * Network state
 * ------------------------------------------------------------------- */
#define MAXV 24

typedef struct
{
  const char* name;
  int idx;
} var_name;

/* variable slots per model (param and state arrays, by name) */
static const var_name DELTA_VARS[] = { { "tau_m", 0 }, { "C_m", 1 }, { "t_ref", 2 }, { "I_e", 3 }, { "V_th_rel", 4 },
  { "V_reset_rel", 5 }, { "V_min_rel", 6 }, { "V_m_rel", 7 }, { "y0", 8 }, { "r", 9 }, { NULL, 0 } };
static const var_name EXP_VARS[] = { { "tau_m", 0 }, { "C_m", 1 }, { "t_ref", 2 }, { "I_e", 3 }, { "V_th_rel", 4 },
  { "V_reset_rel", 5 }, { "tau_syn_ex", 6 }, { "tau_syn_in", 7 }, { "V_m_rel", 8 }, { "I_syn_ex", 9 },
  { "I_syn_in", 10 }, { "i_0", 11 }, { "i_1", 12 }, { "r", 13 }, { NULL, 0 } };
/* iaf_psc_alpha: y3 = V_m_rel, I_ex, I_in, dI_ex, dI_in (models/iaf_psc_alpha.h State_) */
static const var_name ALPHA_VARS[] = { { "tau_m", 0 }, { "C_m", 1 }, { "t_ref", 2 }, { "I_e", 3 }, { "V_th_rel", 4 },
  { "V_reset_rel", 5 }, { "tau_syn_ex", 6 }, { "tau_syn_in", 7 }, { "V_min_rel", 8 }, { "V_m_rel", 9 },
  { "I_syn_ex", 10 }, { "I_syn_in", 11 }, { "dI_syn_ex", 12 }, { "dI_syn_in", 13 }, { "r", 14 }, { NULL, 0 } };
static const var_name AEIF_VARS[] = { { "V_peak", 0 }, { "V_reset", 1 }, { "t_ref", 2 }, { "g_L", 3 }, { "C_m", 4 },
  { "E_ex", 5 }, { "E_in", 6 }, { "E_L", 7 }, { "Delta_T", 8 }, { "tau_w", 9 }, { "a", 10 }, { "b", 11 },
  { "V_th", 12 }, { "tau_syn_ex", 13 }, { "tau_syn_in", 14 }, { "I_e", 15 }, { "gsl_error_tol", 16 },
  { "V_m", 17 }, { "dg_ex", 18 }, { "g_ex", 19 }, { "dg_in", 20 }, { "g_in", 21 }, { "w", 22 }, { "r", 23 },
  { NULL, 0 } };

struct orc_net
{
  int model;
  int64_t n;
  double h;
  int32_t min_delay, max_delay, L;
  double* v[ MAXV ];   /* per-neuron arrays by slot */
  double* istep;       /* aeif: per-neuron integration step (B_.IntegrationStep_) */
  double* I_stim;      /* aeif: B_.I_stim_ (currents are not used: stays 0) */
  double* ring;        /* [L][2][n] */
  /* connectivity */
  int64_t n_src;
  int nparts;
  int64_t** part_row;  /* per partition: row pointers over sources */
  int32_t** part_tgt;
  double** part_w;
  int32_t** part_d;
  /* generator sources */
  int64_t n_sched, sched_pos;
  int64_t* sched_step;
  int32_t* sched_src;
  /* Poisson drive */
  pois_tab* pois;
  double* pois_w;
  int32_t* pois_d;
  int64_t pois_start, pois_stop;
  uint32_t key[ 2 ];
  /* recording */
  uint8_t* rec;
  int64_t n_trace_idx;
  int32_t* trace_idx;
  int64_t* trace_col; /* per neuron: column in the trace row, or -1 */
  int trace_slot;
  double* trace;
  int64_t trace_len, trace_cap;
  int32_t* log_src;
  int64_t* log_stamp;
  int64_t log_len, log_cap;
  /* slice bookkeeping */
  int64_t clock;   /* slice origin, steps */
  int32_t from;    /* position inside the current slice */
  int32_t* sp_src; /* spikes of the current slice (source, emission step, multiplicity) */
  int64_t* sp_t;
  int32_t* sp_mult;
  int64_t sp_len, sp_cap;
  int64_t syn_events;
  int prepared;
  /* stdp_pl_synapse_hom connections (models/stdp_pl_synapse_hom.h) in a CSR
   * of their own: per-edge weight_, Kplus_ and t_lastspike_ as the
   * reference's Connection holds them, and the common properties */
  int64_t pl_nsrc, pl_nnz;
  int64_t* pl_row;
  int32_t *pl_tgt, *pl_d;
  double *pl_w, *pl_Kplus, *pl_tlast;
  double pl_lambda, pl_alpha, pl_mu, pl_tau_plus_inv;
  /* ArchivingNode (nestkernel/archiving_node.cpp) of each neuron: tau_minus,
   * the Kminus trace at the last spike, the spike history (t, Kminus) and
   * whether it has incoming STDP connections */
  double *tau_minus, *Kminus, *last_spike;
  int32_t* n_incoming;
  double **hist_t, **hist_K;
  int64_t *hist_len, *hist_cap;
  /* derived coefficients */
  double *P33, *P30, *P22, *P11ex, *P11in, *P21ex, *P21in, *P20, *g0ex, *g0in;
  double *P31ex, *P32ex, *P31in, *P32in, *em1; /* iaf_psc_alpha (P11, P21, P30, g0 above too) */
  int32_t* refr;
};

static inline double stamp_ms( const orc_net* net, int64_t stamp );
static void archive_spike( orc_net* net, int64_t i, double t_ms );

static const var_name*
vars_of( int model )
{
  return model == ORC_IAF_PSC_DELTA ? DELTA_VARS
    : model == ORC_IAF_PSC_EXP      ? EXP_VARS
    : model == ORC_IAF_PSC_ALPHA    ? ALPHA_VARS
                                    : AEIF_VARS;
}

static int
slot_of( int model, const char* name )
{
  for ( const var_name* v = vars_of( model ); v->name; ++v )
  {
    if ( strcmp( v->name, name ) == 0 )
      return v->idx;
  }
  return -1;
}

static int
nvars( int model )
{
  int k = 0;
  for ( const var_name* v = vars_of( model ); v->name; ++v )
    ++k;
  return k;
}

orc_net*
orc_create( int model, int64_t n, double h, int32_t min_delay, int32_t max_delay )
{
  if ( model < 0 || model > 3 || n < 0 || min_delay < 1 || max_delay < min_delay || !( h > 0 ) )
  {
    set_err( "orc_create: bad arguments" );
    return NULL;
  }
  orc_net* net = calloc( 1, sizeof( orc_net ) );
  net->model = model;
  net->n = n;
  net->h = h;
  net->min_delay = min_delay;
  net->max_delay = max_delay;
  net->L = min_delay + max_delay;
  const int nv = nvars( model );
  for ( int i = 0; i < nv; ++i )
    net->v[ i ] = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( double ) );
  /* reference defaults (Parameters_::Parameters_ and State_::State_ of each model) */
  for ( int64_t i = 0; i < n; ++i )
  {
    if ( model == ORC_IAF_PSC_DELTA )
    {
      double* const* v = net->v;
      v[ 0 ][ i ] = 10.0;
      v[ 1 ][ i ] = 250.0;
      v[ 2 ][ i ] = 2.0;
      v[ 3 ][ i ] = 0.0;
      v[ 4 ][ i ] = -55.0 - ( -70.0 );
      v[ 5 ][ i ] = -70.0 - ( -70.0 );
      v[ 6 ][ i ] = -DBL_MAX;
    }
    else if ( model == ORC_IAF_PSC_ALPHA )
    {
      double* const* v = net->v;
      v[ 0 ][ i ] = 10.0;
      v[ 1 ][ i ] = 250.0;
      v[ 2 ][ i ] = 2.0;
      v[ 3 ][ i ] = 0.0;
      v[ 4 ][ i ] = -55.0 - ( -70.0 );
      v[ 5 ][ i ] = -70.0 - ( -70.0 );
      v[ 6 ][ i ] = 2.0;
      v[ 7 ][ i ] = 2.0;
      v[ 8 ][ i ] = -INFINITY;
    }
    else if ( model == ORC_IAF_PSC_EXP )
    {
      double* const* v = net->v;
      v[ 0 ][ i ] = 10.0;
      v[ 1 ][ i ] = 250.0;
      v[ 2 ][ i ] = 2.0;
      v[ 3 ][ i ] = 0.0;
      v[ 4 ][ i ] = -55.0 - ( -70.0 );
      v[ 5 ][ i ] = -70.0 - ( -70.0 );
      v[ 6 ][ i ] = 2.0;
      v[ 7 ][ i ] = 2.0;
    }
    else
    {
      static const double d[ 17 ] = { 0.0, -60.0, 0.0, 30.0, 281.0, 0.0, -85.0, -70.6, 2.0, 144.0, 4.0, 80.5,
        -50.4, 0.2, 2.0, 0.0, 1e-6 };
      for ( int k = 0; k < 17; ++k )
        net->v[ k ][ i ] = d[ k ];
      net->v[ 17 ][ i ] = -70.6;
    }
  }
  net->istep = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( double ) );
  net->I_stim = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( double ) );
  net->tau_minus = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( double ) );
  net->Kminus = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( double ) );
  net->last_spike = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( double ) );
  net->n_incoming = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( int32_t ) );
  net->hist_t = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( double* ) );
  net->hist_K = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( double* ) );
  net->hist_len = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( int64_t ) );
  net->hist_cap = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( int64_t ) );
  for ( int64_t i = 0; i < n; ++i )
    net->tau_minus[ i ] = 20.0; /* ArchivingNode default */
  for ( int64_t i = 0; i < n; ++i )
    net->istep[ i ] = h;
  net->ring = calloc( ( size_t ) net->L * 2 * ( size_t ) ( n > 0 ? n : 1 ), sizeof( double ) );
  net->n_src = n;
  net->key[ 0 ] = 0;
  net->key[ 1 ] = 0;
  net->pois_stop = INT64_MAX;
  return net;
}

void
orc_destroy( orc_net* net )
{
  if ( !net )
    return;
  for ( int i = 0; i < MAXV; ++i )
    free( net->v[ i ] );
  free( net->istep );
  free( net->I_stim );
  for ( int64_t i = 0; i < net->n; ++i )
  {
    free( net->hist_t[ i ] );
    free( net->hist_K[ i ] );
  }
  free( net->hist_t );
  free( net->hist_K );
  free( net->hist_len );
  free( net->hist_cap );
  free( net->tau_minus );
  free( net->Kminus );
  free( net->last_spike );
  free( net->n_incoming );
  free( net->pl_row );
  free( net->pl_tgt );
  free( net->pl_d );
  free( net->pl_w );
  free( net->pl_Kplus );
  free( net->pl_tlast );
  free( net->ring );
  for ( int p = 0; p < net->nparts; ++p )
  {
    free( net->part_row[ p ] );
    free( net->part_tgt[ p ] );
    free( net->part_w[ p ] );
    free( net->part_d[ p ] );
  }
  free( net->part_row );
  free( net->part_tgt );
  free( net->part_w );
  free( net->part_d );
  free( net->sched_step );
  free( net->sched_src );
  if ( net->pois )
    for ( int64_t i = 0; i < net->n; ++i )
      free( net->pois[ i ].cdf );
  free( net->pois );
  free( net->pois_w );
  free( net->pois_d );
  free( net->rec );
  free( net->trace_idx );
  free( net->trace_col );
  free( net->trace );
  free( net->log_src );
  free( net->log_stamp );
  free( net->sp_src );
  free( net->sp_t );
  free( net->sp_mult );
  free( net->P33 );
  free( net->P30 );
  free( net->P22 );
  free( net->P11ex );
  free( net->P11in );
  free( net->P21ex );
  free( net->P21in );
  free( net->P20 );
  free( net->P31ex );
  free( net->P32ex );
  free( net->P31in );
  free( net->P32in );
  free( net->em1 );
  free( net->g0ex );
  free( net->g0in );
  free( net->refr );
  free( net );
}

int
orc_set( orc_net* net, const char* name, const double* values )
{
  if ( strcmp( name, "integration_step" ) == 0 )
  {
    memcpy( net->istep, values, sizeof( double ) * ( size_t ) net->n );
    return 0;
  }
  if ( strcmp( name, "tau_minus" ) == 0 )
  {
    memcpy( net->tau_minus, values, sizeof( double ) * ( size_t ) net->n );
    return 0;
  }
  const int s = slot_of( net->model, name );
  if ( s < 0 )
  {
    set_err( "orc_set: unknown variable" );
    return -1;
  }
  memcpy( net->v[ s ], values, sizeof( double ) * ( size_t ) net->n );
  net->prepared = 0;
  return 0;
}

int
orc_get( orc_net* net, const char* name, double* out )
{
  if ( strcmp( name, "integration_step" ) == 0 )
  {
    memcpy( out, net->istep, sizeof( double ) * ( size_t ) net->n );
    return 0;
  }
  const int s = slot_of( net->model, name );
  if ( s < 0 )
  {
    set_err( "orc_get: unknown variable" );
    return -1;
  }
  memcpy( out, net->v[ s ], sizeof( double ) * ( size_t ) net->n );
  return 0;
}

int
orc_set_csr( orc_net* net, int64_t n_src, const int64_t* row_ptr, const int32_t* tgt, const double* w,
  const int32_t* d, int nthreads )
{
  if ( n_src < net->n )
  {
    set_err( "orc_set_csr: n_src < n" );
    return -1;
  }
  int P = nthreads;
#ifdef _OPENMP
  if ( P <= 0 )
    P = omp_get_max_threads();
#endif
  if ( P <= 0 )
    P = 1;
  for ( int p = 0; p < net->nparts; ++p )
  {
    free( net->part_row[ p ] );
    free( net->part_tgt[ p ] );
    free( net->part_w[ p ] );
    free( net->part_d[ p ] );
  }
  free( net->part_row );
  free( net->part_tgt );
  free( net->part_w );
  free( net->part_d );
  net->n_src = n_src;
  net->nparts = P;
  net->part_row = calloc( P, sizeof( int64_t* ) );
  net->part_tgt = calloc( P, sizeof( int32_t* ) );
  net->part_w = calloc( P, sizeof( double* ) );
  net->part_d = calloc( P, sizeof( int32_t* ) );
  /* partition p owns targets [p*n/P, (p+1)*n/P), like NEST's per-thread
   * postsynaptic connection storage; edge order inside a row is kept */
  for ( int p = 0; p < P; ++p )
  {
    const int64_t lo = net->n * p / P, hi = net->n * ( p + 1 ) / P;
    int64_t cnt = 0;
    for ( int64_t e = 0; e < row_ptr[ n_src ]; ++e )
    {
      if ( tgt[ e ] >= lo && tgt[ e ] < hi )
        ++cnt;
      if ( d[ e ] < net->min_delay || d[ e ] > net->max_delay || tgt[ e ] < 0 || tgt[ e ] >= net->n )
      {
        set_err( "orc_set_csr: delay outside [min_delay, max_delay] or bad target" );
        return -1;
      }
    }
    int64_t* rp = calloc( ( size_t ) n_src + 1, sizeof( int64_t ) );
    int32_t* tg = malloc( sizeof( int32_t ) * ( size_t ) ( cnt > 0 ? cnt : 1 ) );
    double* ww = malloc( sizeof( double ) * ( size_t ) ( cnt > 0 ? cnt : 1 ) );
    int32_t* dd = malloc( sizeof( int32_t ) * ( size_t ) ( cnt > 0 ? cnt : 1 ) );
    int64_t k = 0;
    for ( int64_t s = 0; s < n_src; ++s )
    {
      rp[ s ] = k;
      for ( int64_t e = row_ptr[ s ]; e < row_ptr[ s + 1 ]; ++e )
      {
        if ( tgt[ e ] >= lo && tgt[ e ] < hi )
        {
          tg[ k ] = tgt[ e ];
          ww[ k ] = w[ e ];
          dd[ k ] = d[ e ];
          ++k;
        }
      }
    }
    rp[ n_src ] = k;
    net->part_row[ p ] = rp;
    net->part_tgt[ p ] = tg;
    net->part_w[ p ] = ww;
    net->part_d[ p ] = dd;
  }
  free( net->rec );
  net->rec = NULL;
  return 0;
}

int
orc_set_sched( orc_net* net, int64_t n, const int64_t* step, const int32_t* src )
{
  free( net->sched_step );
  free( net->sched_src );
  net->sched_step = malloc( sizeof( int64_t ) * ( size_t ) ( n > 0 ? n : 1 ) );
  net->sched_src = malloc( sizeof( int32_t ) * ( size_t ) ( n > 0 ? n : 1 ) );
  for ( int64_t i = 0; i < n; ++i )
  {
    if ( i > 0 && step[ i ] < step[ i - 1 ] )
    {
      set_err( "orc_set_sched: steps must be sorted" );
      return -1;
    }
    net->sched_step[ i ] = step[ i ];
    net->sched_src[ i ] = src[ i ];
  }
  net->n_sched = n;
  net->sched_pos = 0;
  while ( net->sched_pos < n && net->sched_step[ net->sched_pos ] < net->clock + net->from )
    ++net->sched_pos;
  return 0;
}

int
orc_set_poisson( orc_net* net, const double* rate_hz, const double* w, const int32_t* d, int64_t start_step,
  int64_t stop_step, uint64_t seed )
{
  if ( net->pois )
    for ( int64_t i = 0; i < net->n; ++i )
      free( net->pois[ i ].cdf );
  free( net->pois );
  free( net->pois_w );
  free( net->pois_d );
  const int64_t n = net->n;
  net->pois = malloc( sizeof( pois_tab ) * ( size_t ) ( n > 0 ? n : 1 ) );
  net->pois_w = malloc( sizeof( double ) * ( size_t ) ( n > 0 ? n : 1 ) );
  net->pois_d = malloc( sizeof( int32_t ) * ( size_t ) ( n > 0 ? n : 1 ) );
  for ( int64_t i = 0; i < n; ++i )
  {
    /* lambda = h * rate * 1e-3 (models/poisson_generator.cpp:114) */
    const double lam = rate_hz[ i ] > 0 ? net->h * rate_hz[ i ] * 1e-3 : 0.0;
    net->pois[ i ] = pois_prepare( lam );
    net->pois_w[ i ] = w[ i ];
    net->pois_d[ i ] = d[ i ];
  }
  net->pois_start = start_step;
  net->pois_stop = stop_step;
  net->key[ 0 ] = ( uint32_t ) seed;
  net->key[ 1 ] = ( uint32_t ) ( seed >> 32 );
  return 0;
}

int
orc_set_record( orc_net* net, const uint8_t* flags )
{
  free( net->rec );
  net->rec = NULL;
  if ( flags )
  {
    net->rec = malloc( ( size_t ) net->n_src );
    memcpy( net->rec, flags, ( size_t ) net->n_src );
  }
  return 0;
}

int
orc_set_trace( orc_net* net, int64_t n_idx, const int32_t* idx, const char* var )
{
  const int s = slot_of( net->model, var );
  if ( s < 0 )
  {
    set_err( "orc_set_trace: unknown variable" );
    return -1;
  }
  free( net->trace_idx );
  net->trace_idx = malloc( sizeof( int32_t ) * ( size_t ) ( n_idx > 0 ? n_idx : 1 ) );
  memcpy( net->trace_idx, idx, sizeof( int32_t ) * ( size_t ) n_idx );
  free( net->trace_col );
  net->trace_col = malloc( sizeof( int64_t ) * ( size_t ) ( net->n > 0 ? net->n : 1 ) );
  for ( int64_t i = 0; i < net->n; ++i )
    net->trace_col[ i ] = -1;
  for ( int64_t k = 0; k < n_idx; ++k )
  {
    if ( idx[ k ] < 0 || idx[ k ] >= net->n || net->trace_col[ idx[ k ] ] >= 0 )
    {
      set_err( "orc_set_trace: bad or repeated index" );
      net->n_trace_idx = 0;
      return -1;
    }
    net->trace_col[ idx[ k ] ] = k;
  }
  net->n_trace_idx = n_idx;
  net->trace_slot = s;
  net->trace_len = 0;
  return 0;
}

/* pre_run_hook restatements */
static void
prepare( orc_net* net )
{
  const int64_t n = net->n;
  const double h = net->h;
  double** pa[] = { &net->P33, &net->P30, &net->P22, &net->P11ex, &net->P11in, &net->P21ex, &net->P21in, &net->P20,
    &net->g0ex, &net->g0in, &net->P31ex, &net->P32ex, &net->P31in, &net->P32in, &net->em1 };
  for ( size_t k = 0; k < sizeof( pa ) / sizeof( pa[ 0 ] ); ++k )
  {
    free( *pa[ k ] );
    *pa[ k ] = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( double ) );
  }
  free( net->refr );
  net->refr = calloc( ( size_t ) ( n > 0 ? n : 1 ), sizeof( int32_t ) );
  /* h as Time::get_resolution().get_ms() = MS_PER_TIC * tics */
  const double tics_per_ms = 1000.0;
  const int64_t tps = ( int64_t ) floor( tics_per_ms * h + 0.5 );
  for ( int64_t i = 0; i < n; ++i )
  {
    if ( net->model == ORC_IAF_PSC_DELTA )
    {
      const double tau_m = net->v[ 0 ][ i ], c_m = net->v[ 1 ][ i ];
      net->P33[ i ] = exp( -h / tau_m );
      net->P30[ i ] = 1 / c_m * ( 1 - net->P33[ i ] ) * tau_m;
      net->refr[ i ] = ( int32_t ) ms_to_steps_roundup( net->v[ 2 ][ i ], tics_per_ms, tps );
    }
    else if ( net->model == ORC_IAF_PSC_ALPHA )
    {
      /* iaf_psc_alpha::pre_run_hook (models/iaf_psc_alpha.cpp), same order */
      const double tau_m = net->v[ 0 ][ i ], c_m = net->v[ 1 ][ i ];
      const double tex = net->v[ 6 ][ i ], tin = net->v[ 7 ][ i ];
      double pp[ 2 ];
      net->P11ex[ i ] = exp( -h / tex );
      net->P11in[ i ] = exp( -h / tin );
      net->em1[ i ] = expm1( -h / tau_m );
      net->P30[ i ] = -tau_m / c_m * expm1( -h / tau_m );
      net->P21ex[ i ] = h * net->P11ex[ i ];
      net->P21in[ i ] = h * net->P11in[ i ];
      orc_iaf_propagator_alpha( tex, tau_m, c_m, h, pp );
      net->P31ex[ i ] = pp[ 0 ];
      net->P32ex[ i ] = pp[ 1 ];
      orc_iaf_propagator_alpha( tin, tau_m, c_m, h, pp );
      net->P31in[ i ] = pp[ 0 ];
      net->P32in[ i ] = pp[ 1 ];
      net->g0ex[ i ] = 1.0 * M_E / tex;
      net->g0in[ i ] = 1.0 * M_E / tin;
      net->refr[ i ] = ( int32_t ) ms_to_steps_roundup( net->v[ 2 ][ i ], tics_per_ms, tps );
    }
    else if ( net->model == ORC_IAF_PSC_EXP )
    {
      const double tau_m = net->v[ 0 ][ i ], c_m = net->v[ 1 ][ i ];
      const double tex = net->v[ 6 ][ i ], tin = net->v[ 7 ][ i ];
      net->P11ex[ i ] = exp( -h / tex );
      net->P11in[ i ] = exp( -h / tin );
      net->P22[ i ] = exp( -h / tau_m );
      net->P21ex[ i ] = orc_iaf_propagator_exp( tex, tau_m, c_m, h );
      net->P21in[ i ] = orc_iaf_propagator_exp( tin, tau_m, c_m, h );
      net->P20[ i ] = tau_m / c_m * ( 1.0 - net->P22[ i ] );
      net->refr[ i ] = ( int32_t ) ms_to_steps_roundup( net->v[ 2 ][ i ], tics_per_ms, tps );
    }
    else
    {
      /* V_.V_peak = Delta_T > 0 ? V_peak : V_th  (models/aeif_cond_alpha.cpp:429-436) */
      net->g0ex[ i ] = 1.0 * M_E / net->v[ 13 ][ i ];
      net->g0in[ i ] = 1.0 * M_E / net->v[ 14 ][ i ];
      net->refr[ i ] = ( int32_t ) ms_to_steps_roundup( net->v[ 2 ][ i ], tics_per_ms, tps );
    }
  }
  net->prepared = 1;
}

/* ---------------------------------------------------------------------
 * aeif_cond_alpha: right-hand side and one adaptive RKF45 sub-step
 * ------------------------------------------------------------------- */
typedef struct
{
  double V_peak, V_reset, g_L, C_m, E_ex, E_in, E_L, Delta_T, tau_w, a, b, V_th, tau_syn_ex, tau_syn_in, I_e;
} aeif_par;

/* models/aeif_cond_alpha.cpp:74-126 (y = V, dg_ex, g_ex, dg_in, g_in, w) */
static void
aeif_rhs( const aeif_par* p, int refractory, double I_stim, const double* y, double* f )
{
  const double V = refractory ? p->V_reset : fmin( y[ 0 ], p->V_peak );
  const double dg_ex = y[ 1 ], g_ex = y[ 2 ], dg_in = y[ 3 ], g_in = y[ 4 ], w = y[ 5 ];
  const double I_syn_exc = g_ex * ( V - p->E_ex );
  const double I_syn_inh = g_in * ( V - p->E_in );
  const double I_spike = p->Delta_T == 0. ? 0. : ( p->g_L * p->Delta_T * exp( ( V - p->V_th ) / p->Delta_T ) );
  f[ 0 ] = refractory ? 0. : ( -p->g_L * ( V - p->E_L ) + I_spike - I_syn_exc - I_syn_inh - w + p->I_e + I_stim ) / p->C_m;
  f[ 1 ] = -dg_ex / p->tau_syn_ex;
  f[ 2 ] = dg_ex - g_ex / p->tau_syn_ex;
  f[ 3 ] = -dg_in / p->tau_syn_in;
  f[ 4 ] = dg_in - g_in / p->tau_syn_in;
  f[ 5 ] = ( p->a * ( V - p->E_L ) - w ) / p->tau_w;
}

/* Fehlberg 4(5) tableau (E. Fehlberg, NASA TR R-315, 1969); the step advances
 * with the fifth-order weights, the error is fifth minus fourth order. */
static const double RK_A2 = 1.0 / 4.0;
static const double RK_B3[ 2 ] = { 3.0 / 32.0, 9.0 / 32.0 };
static const double RK_B4[ 3 ] = { 1932.0 / 2197.0, -7200.0 / 2197.0, 7296.0 / 2197.0 };
static const double RK_B5[ 4 ] = { 439.0 / 216.0, -8.0, 3680.0 / 513.0, -845.0 / 4104.0 };
static const double RK_B6[ 5 ] = { -8.0 / 27.0, 2.0, -3544.0 / 2565.0, 1859.0 / 4104.0, -11.0 / 40.0 };
static const double RK_C[ 6 ] = { 16.0 / 135.0, 0.0, 6656.0 / 12825.0, 28561.0 / 56430.0, -9.0 / 50.0, 2.0 / 55.0 };
static const double RK_E[ 6 ] = { 1.0 / 360.0, 0.0, -128.0 / 4275.0, -2197.0 / 75240.0, 1.0 / 50.0, 2.0 / 55.0 };

/* one RKF45 step of size hs from y (k1 given), writes y5, err, dydt_out */
static void
rkf45_step( const aeif_par* p, int refr, double I_stim, const double* y, const double* k1, double hs, double* ynew,
  double* yerr, double* dydt_out )
{
  double k2[ 6 ], k3[ 6 ], k4[ 6 ], k5[ 6 ], k6[ 6 ], yt[ 6 ];
  for ( int i = 0; i < 6; ++i )
    yt[ i ] = y[ i ] + RK_A2 * hs * k1[ i ];
  aeif_rhs( p, refr, I_stim, yt, k2 );
  for ( int i = 0; i < 6; ++i )
    yt[ i ] = y[ i ] + hs * ( RK_B3[ 0 ] * k1[ i ] + RK_B3[ 1 ] * k2[ i ] );
  aeif_rhs( p, refr, I_stim, yt, k3 );
  for ( int i = 0; i < 6; ++i )
    yt[ i ] = y[ i ] + hs * ( RK_B4[ 0 ] * k1[ i ] + RK_B4[ 1 ] * k2[ i ] + RK_B4[ 2 ] * k3[ i ] );
  aeif_rhs( p, refr, I_stim, yt, k4 );
  for ( int i = 0; i < 6; ++i )
    yt[ i ] = y[ i ] + hs * ( RK_B5[ 0 ] * k1[ i ] + RK_B5[ 1 ] * k2[ i ] + RK_B5[ 2 ] * k3[ i ] + RK_B5[ 3 ] * k4[ i ] );
  aeif_rhs( p, refr, I_stim, yt, k5 );
  for ( int i = 0; i < 6; ++i )
    yt[ i ] = y[ i ]
      + hs * ( RK_B6[ 0 ] * k1[ i ] + RK_B6[ 1 ] * k2[ i ] + RK_B6[ 2 ] * k3[ i ] + RK_B6[ 3 ] * k4[ i ] + RK_B6[ 4 ] * k5[ i ] );
  aeif_rhs( p, refr, I_stim, yt, k6 );
  for ( int i = 0; i < 6; ++i )
  {
    const double d5 = RK_C[ 0 ] * k1[ i ] + RK_C[ 2 ] * k3[ i ] + RK_C[ 3 ] * k4[ i ] + RK_C[ 4 ] * k5[ i ] + RK_C[ 5 ] * k6[ i ];
    ynew[ i ] = y[ i ] + hs * d5;
    yerr[ i ] = hs * ( RK_E[ 0 ] * k1[ i ] + RK_E[ 2 ] * k3[ i ] + RK_E[ 3 ] * k4[ i ] + RK_E[ 4 ] * k5[ i ] + RK_E[ 5 ] * k6[ i ] );
  }
  aeif_rhs( p, refr, I_stim, ynew, dydt_out );
}

/* Standard step-size control with a_y = 0, a_dydt = 1 ("yp" control):
 * D_i = eps_abs + eps_rel * h |y'_i|; r = max_i |err_i| / D_i.
 * r > 1.1: shrink by max(0.2, 0.9 r^(-1/q)); r < 0.5: grow by
 * min(5, max(1, 0.9 r^(-1/(q+1)))); q = 5, the order of the rkf45 stepper.
 * Returns -1 (decrease), +1 (increase), 0 (keep). */
static int
control_yp( double tol, const double* yerr, const double* dydt, double* hs )
{
  const double h_old = *hs;
  double rmax = DBL_MIN;
  for ( int i = 0; i < 6; ++i )
  {
    const double D0 = tol * fabs( h_old * dydt[ i ] ) + tol;
    const double r = fabs( yerr[ i ] ) / fabs( D0 );
    rmax = r > rmax ? r : rmax;
  }
  if ( rmax > 1.1 )
  {
    double r = 0.9 / pow( rmax, 1.0 / 5.0 );
    if ( r < 0.2 )
      r = 0.2;
    *hs = r * h_old;
    return -1;
  }
  if ( rmax < 0.5 )
  {
    double r = 0.9 / pow( rmax, 1.0 / 6.0 );
    if ( r > 5.0 )
      r = 5.0;
    if ( r < 1.0 )
      r = 1.0;
    *hs = r * h_old;
    return 1;
  }
  return 0;
}

/* One call of the adaptive driver: advance y from *t towards t1 by one
 * accepted sub-step (never past t1; a step that reaches t1 sets *t = t1
 * exactly), retrying with a smaller step while the control rejects it and
 * the smaller step still moves t by at least one ulp.  *hs returns the
 * suggested next step. */
static void
evolve_apply( const aeif_par* p, int refr, double I_stim, double tol, double* t, double t1, double* hs, double* y )
{
  const double t0 = *t;
  double h0 = *hs;
  const double dt = t1 - t0;
  double y0[ 6 ], k1[ 6 ], yerr[ 6 ], dout[ 6 ], yn[ 6 ];
  memcpy( y0, y, sizeof( y0 ) );
  aeif_rhs( p, refr, I_stim, y0, k1 );
  for ( ;; )
  {
    int final_step = 0;
    if ( h0 > dt )
    {
      h0 = dt;
      final_step = 1;
    }
    rkf45_step( p, refr, I_stim, y0, k1, h0, yn, yerr, dout );
    *t = final_step ? t1 : t0 + h0;
    const double h_old = h0;
    const int adj = control_yp( tol, yerr, dout, &h0 );
    if ( adj < 0 )
    {
      const double t_curr = *t;
      const double t_next = ( *t ) + h0;
      if ( fabs( h0 ) < fabs( h_old ) && t_next != t_curr )
      {
        continue; /* reject: retry from y0 with the smaller step */
      }
      h0 = h_old;
    }
    memcpy( y, yn, sizeof( yn ) );
    *hs = h0;
    return;
  }
}

/* ---------------------------------------------------------------------
 * The slice cycle
 * ------------------------------------------------------------------- */
static inline int64_t
imod( int64_t a, int64_t m )
{
  int64_t r = a % m;
  return r < 0 ? r + m : r;
}

/* drive value for neuron i at step t (generator step tg = t - d): one
 * Philox4x32-10 block per pair of generator steps, counter (i, tg >> 1,
 * DRIVE_STREAM); words 0-1 serve the even step, words 2-3 the odd one */
static inline double
drive( const orc_net* net, int64_t i, int64_t t )
{
  if ( !net->pois || net->pois[ i ].lambda <= 0.0 )
    return 0.0;
  const int64_t tg = t - net->pois_d[ i ];
  if ( !( net->pois_start < tg && tg <= net->pois_stop ) || tg < 0 )
    return 0.0;
  const int64_t tp = tg >> 1;
  const uint32_t ctr[ 4 ] = { ( uint32_t ) i, ( uint32_t ) tp, ( uint32_t ) ( ( uint64_t ) tp >> 32 ), DRIVE_STREAM };
  uint32_t o[ 4 ];
  orc_philox4x32( ctr, net->key, 10, o );
  const double u = ( tg & 1 ) ? u53( o[ 2 ], o[ 3 ] ) : u53( o[ 0 ], o[ 1 ] );
  const int64_t k = pois_draw( &net->pois[ i ], u );
  return k > 0 ? net->pois_w[ i ] * ( double ) k : 0.0;
}

static void
push_spike( orc_net* net, int32_t src, int64_t t_emit, int32_t mult )
{
  if ( net->sp_len == net->sp_cap )
  {
    net->sp_cap = net->sp_cap ? 2 * net->sp_cap : 1024;
    net->sp_src = realloc( net->sp_src, sizeof( int32_t ) * ( size_t ) net->sp_cap );
    net->sp_t = realloc( net->sp_t, sizeof( int64_t ) * ( size_t ) net->sp_cap );
    net->sp_mult = realloc( net->sp_mult, sizeof( int32_t ) * ( size_t ) net->sp_cap );
  }
  net->sp_src[ net->sp_len ] = src;
  net->sp_t[ net->sp_len ] = t_emit;
  net->sp_mult[ net->sp_len ] = mult;
  ++net->sp_len;
  if ( !net->rec || net->rec[ src ] )
  {
    for ( int32_t m = 0; m < mult; ++m )
    {
      if ( net->log_len == net->log_cap )
      {
        net->log_cap = net->log_cap ? 2 * net->log_cap : 4096;
        net->log_src = realloc( net->log_src, sizeof( int32_t ) * ( size_t ) net->log_cap );
        net->log_stamp = realloc( net->log_stamp, sizeof( int64_t ) * ( size_t ) net->log_cap );
      }
      net->log_src[ net->log_len ] = src;
      net->log_stamp[ net->log_len ] = t_emit + 1;
      ++net->log_len;
    }
  }
}

/* per-thread spike buffers of one update pass */
typedef struct
{
  int32_t* src;
  int64_t* t;
  int32_t* mult;
  int64_t len, cap;
} tbuf;

static void
tb_push( tbuf* b, int32_t src, int64_t t, int32_t mult )
{
  if ( b->len == b->cap )
  {
    b->cap = b->cap ? 2 * b->cap : 256;
    b->src = realloc( b->src, sizeof( int32_t ) * ( size_t ) b->cap );
    b->t = realloc( b->t, sizeof( int64_t ) * ( size_t ) b->cap );
    b->mult = realloc( b->mult, sizeof( int32_t ) * ( size_t ) b->cap );
  }
  b->src[ b->len ] = src;
  b->t[ b->len ] = t;
  b->mult[ b->len ] = mult;
  ++b->len;
}

static int g_instability;

/* update neuron i over lags [from, to) of the slice at origin */
static void
update_neuron( orc_net* net, int64_t i, int64_t origin, int32_t from, int32_t to, tbuf* tb, double* trace_row,
  int64_t trace_col )
{
  const int64_t L = net->L, n = net->n;
  double* const* v = net->v;
  for ( int32_t lag = from; lag < to; ++lag )
  {
    const int64_t t = origin + lag;
    const int64_t slot = imod( t, L );
    double* r0 = net->ring + ( slot * 2 + 0 ) * n + i;
    double* r1 = net->ring + ( slot * 2 + 1 ) * n + i;
    int32_t mult = 0;
    if ( net->model == ORC_IAF_PSC_DELTA )
    {
      /* models/iaf_psc_delta.cpp:272-329 */
      double in = *r0;
      const double dv = drive( net, i, t );
      if ( dv != 0.0 )
        in = in + dv;
      *r0 = 0.0;
      double r = v[ 9 ][ i ];
      if ( r == 0 )
      {
        v[ 7 ][ i ] = net->P30[ i ] * ( v[ 8 ][ i ] + v[ 3 ][ i ] ) + net->P33[ i ] * v[ 7 ][ i ] + in;
        v[ 7 ][ i ] = ( v[ 7 ][ i ] < v[ 6 ][ i ] ? v[ 6 ][ i ] : v[ 7 ][ i ] );
      }
      else
      {
        v[ 9 ][ i ] = r - 1;
      }
      if ( v[ 7 ][ i ] >= v[ 4 ][ i ] )
      {
        v[ 9 ][ i ] = net->refr[ i ];
        v[ 7 ][ i ] = v[ 5 ][ i ];
        mult = 1;
      }
      v[ 8 ][ i ] = 0.0; /* currents ring: no current inputs on this path */
    }
    else if ( net->model == ORC_IAF_PSC_ALPHA )
    {
      /* iaf_psc_alpha::update (models/iaf_psc_alpha.cpp): y0 = 0 (no
       * current input on this path) */
      double ex = *r0, inh = *r1;
      const double dv = drive( net, i, t );
      if ( dv != 0.0 )
      {
        if ( dv > 0 )
          ex = ex + dv;
        else
          inh = inh + dv;
      }
      *r0 = 0.0;
      *r1 = 0.0;
      const double y0 = 0.0;
      if ( v[ 14 ][ i ] == 0 )
      {
        v[ 9 ][ i ] = net->P30[ i ] * ( y0 + v[ 3 ][ i ] ) + net->P31ex[ i ] * v[ 12 ][ i ] + net->P32ex[ i ] * v[ 10 ][ i ]
          + net->P31in[ i ] * v[ 13 ][ i ] + net->P32in[ i ] * v[ 11 ][ i ] + net->em1[ i ] * v[ 9 ][ i ] + v[ 9 ][ i ];
        v[ 9 ][ i ] = ( v[ 9 ][ i ] < v[ 8 ][ i ] ? v[ 8 ][ i ] : v[ 9 ][ i ] );
      }
      else
      {
        v[ 14 ][ i ] = v[ 14 ][ i ] - 1;
      }
      v[ 10 ][ i ] = net->P21ex[ i ] * v[ 12 ][ i ] + net->P11ex[ i ] * v[ 10 ][ i ];
      v[ 12 ][ i ] *= net->P11ex[ i ];
      v[ 12 ][ i ] += net->g0ex[ i ] * ex;
      v[ 11 ][ i ] = net->P21in[ i ] * v[ 13 ][ i ] + net->P11in[ i ] * v[ 11 ][ i ];
      v[ 13 ][ i ] *= net->P11in[ i ];
      v[ 13 ][ i ] += net->g0in[ i ] * inh;
      if ( v[ 9 ][ i ] >= v[ 4 ][ i ] )
      {
        v[ 14 ][ i ] = net->refr[ i ];
        v[ 9 ][ i ] = v[ 5 ][ i ];
        mult = 1;
      }
    }
    else if ( net->model == ORC_IAF_PSC_EXP )
    {
      /* models/iaf_psc_exp.cpp:288-348 */
      double ex = *r0, inh = *r1;
      const double dv = drive( net, i, t );
      if ( dv != 0.0 )
      {
        if ( dv > 0 )
          ex = ex + dv;
        else
          inh = inh + dv;
      }
      *r0 = 0.0;
      *r1 = 0.0;
      if ( v[ 13 ][ i ] == 0 )
      {
        v[ 8 ][ i ] = v[ 8 ][ i ] * net->P22[ i ] + v[ 9 ][ i ] * net->P21ex[ i ] + v[ 10 ][ i ] * net->P21in[ i ]
          + ( v[ 3 ][ i ] + v[ 11 ][ i ] ) * net->P20[ i ];
      }
      else
      {
        v[ 13 ][ i ] = v[ 13 ][ i ] - 1;
      }
      v[ 9 ][ i ] *= net->P11ex[ i ];
      v[ 10 ][ i ] *= net->P11in[ i ];
      v[ 9 ][ i ] += ( 1. - net->P11ex[ i ] ) * v[ 12 ][ i ];
      v[ 9 ][ i ] += ex;
      v[ 10 ][ i ] += inh;
      if ( v[ 8 ][ i ] >= v[ 4 ][ i ] )
      {
        v[ 13 ][ i ] = net->refr[ i ];
        v[ 8 ][ i ] = v[ 5 ][ i ];
        mult = 1;
      }
      v[ 11 ][ i ] = 0.0;
      v[ 12 ][ i ] = 0.0;
    }
    else
    {
      /* models/aeif_cond_alpha.cpp:450-533 */
      aeif_par p = { v[ 0 ][ i ], v[ 1 ][ i ], v[ 3 ][ i ], v[ 4 ][ i ], v[ 5 ][ i ], v[ 6 ][ i ], v[ 7 ][ i ],
        v[ 8 ][ i ], v[ 9 ][ i ], v[ 10 ][ i ], v[ 11 ][ i ], v[ 12 ][ i ], v[ 13 ][ i ], v[ 14 ][ i ],
        v[ 15 ][ i ] };
      const double V_peak_eff = p.Delta_T > 0. ? p.V_peak : p.V_th;
      double y[ 6 ] = { v[ 17 ][ i ], v[ 18 ][ i ], v[ 19 ][ i ], v[ 20 ][ i ], v[ 21 ][ i ], v[ 22 ][ i ] };
      int64_t r = ( int64_t ) v[ 23 ][ i ];
      double tt = 0.0;
      const double hstep = net->h;
      int guard = 0;
      while ( tt < hstep )
      {
        evolve_apply( &p, r > 0, net->I_stim[ i ], v[ 16 ][ i ], &tt, hstep, &net->istep[ i ], y );
        if ( y[ 0 ] < -1e3 || y[ 5 ] < -1e6 || y[ 5 ] > 1e6 )
        {
          g_instability = 1;
          break;
        }
        if ( r > 0 )
        {
          y[ 0 ] = p.V_reset;
        }
        else if ( y[ 0 ] >= V_peak_eff )
        {
          y[ 0 ] = p.V_reset;
          y[ 5 ] += p.b;
          r = net->refr[ i ] > 0 ? net->refr[ i ] + 1 : 0;
          ++mult;
        }
        if ( ++guard > 100000000 )
        {
          g_instability = 1;
          break;
        }
      }
      if ( r > 0 )
        --r;
      double ex = *r0, inh = *r1;
      const double dv = drive( net, i, t );
      if ( dv != 0.0 )
      {
        if ( dv > 0 )
          ex = ex + dv;
        else
          inh = inh - dv;
      }
      *r0 = 0.0;
      *r1 = 0.0;
      y[ 1 ] += ex * net->g0ex[ i ];
      y[ 3 ] += inh * net->g0in[ i ];
      net->I_stim[ i ] = 0.0;
      v[ 17 ][ i ] = y[ 0 ];
      v[ 18 ][ i ] = y[ 1 ];
      v[ 19 ][ i ] = y[ 2 ];
      v[ 20 ][ i ] = y[ 3 ];
      v[ 21 ][ i ] = y[ 4 ];
      v[ 22 ][ i ] = y[ 5 ];
      v[ 23 ][ i ] = ( double ) r;
    }
    if ( mult > 0 )
    {
      tb_push( tb, ( int32_t ) i, t, mult );
      archive_spike( net, i, stamp_ms( net, t + 1 ) );
    }
    if ( trace_row )
      trace_row[ ( int64_t ) lag * net->n_trace_idx + trace_col ] = v[ net->trace_slot ][ i ];
  }
}

/* ---------------------------------------------------------------------
 * stdp_pl_synapse_hom (models/stdp_pl_synapse_hom.h) and the spike history
 * of ArchivingNode (nestkernel/archiving_node.cpp)
 * ------------------------------------------------------------------- */
static const double STDP_EPS = 1.0e-6; /* ConnectionManager stdp_eps default */

int
orc_set_plastic( orc_net* net, int64_t n_src, const int64_t* row_ptr, const int32_t* tgt, const double* w,
  const int32_t* d, double lambda, double alpha, double mu, double tau_plus )
{
  if ( n_src < 0 || n_src > net->n || !( tau_plus > 0 ) )
  {
    set_err( "orc_set_plastic: plastic sources are neurons; tau_plus > 0" );
    return -1;
  }
  const int64_t nnz = row_ptr[ n_src ];
  free( net->pl_row );
  free( net->pl_tgt );
  free( net->pl_d );
  free( net->pl_w );
  free( net->pl_Kplus );
  free( net->pl_tlast );
  net->pl_nsrc = n_src;
  net->pl_nnz = nnz;
  net->pl_row = malloc( sizeof( int64_t ) * ( size_t ) ( n_src + 1 ) );
  memcpy( net->pl_row, row_ptr, sizeof( int64_t ) * ( size_t ) ( n_src + 1 ) );
  net->pl_tgt = malloc( sizeof( int32_t ) * ( size_t ) ( nnz > 0 ? nnz : 1 ) );
  net->pl_d = malloc( sizeof( int32_t ) * ( size_t ) ( nnz > 0 ? nnz : 1 ) );
  net->pl_w = malloc( sizeof( double ) * ( size_t ) ( nnz > 0 ? nnz : 1 ) );
  net->pl_Kplus = calloc( ( size_t ) ( nnz > 0 ? nnz : 1 ), sizeof( double ) );
  net->pl_tlast = calloc( ( size_t ) ( nnz > 0 ? nnz : 1 ), sizeof( double ) );
  memcpy( net->pl_tgt, tgt, sizeof( int32_t ) * ( size_t ) nnz );
  memcpy( net->pl_d, d, sizeof( int32_t ) * ( size_t ) nnz );
  memcpy( net->pl_w, w, sizeof( double ) * ( size_t ) nnz );
  for ( int64_t e = 0; e < nnz; ++e )
  {
    if ( tgt[ e ] < 0 || tgt[ e ] >= net->n || d[ e ] < net->min_delay || d[ e ] > net->max_delay )
    {
      set_err( "orc_set_plastic: target or delay out of range" );
      return -1;
    }
    net->n_incoming[ tgt[ e ] ] += 1;
  }
  net->pl_lambda = lambda;
  net->pl_alpha = alpha;
  net->pl_mu = mu;
  net->pl_tau_plus_inv = 1. / tau_plus;
  return 0;
}

int
orc_get_plastic( orc_net* net, double* w )
{
  memcpy( w, net->pl_w, sizeof( double ) * ( size_t ) net->pl_nnz );
  return 0;
}

/* Time::get_ms of a stamp and Time::delay_steps_to_ms of a delay: MS_PER_TIC
 * times the tics, with 1000 tics per ms (nestkernel/nest_time.h) */
static inline double
stamp_ms( const orc_net* net, int64_t stamp )
{
  const int64_t tps = ( int64_t ) floor( 1000.0 * net->h + 0.5 );
  return ( 1.0 / 1000.0 ) * ( double ) ( stamp * tps );
}

static inline double
delay_ms( const orc_net* net, int32_t d )
{
  const int64_t tps = ( int64_t ) floor( 1000.0 * net->h + 0.5 );
  return ( double ) d * ( ( double ) tps * ( 1.0 / 1000.0 ) );
}

/* ArchivingNode::set_spiketime (archiving_node.cpp:182-220): the Kminus
 * trace and the history entry of a neuron with incoming STDP connections
 * (pruning only frees memory and is left out) */
static void
archive_spike( orc_net* net, int64_t i, double t_ms )
{
  if ( !net->n_incoming[ i ] )
  {
    net->last_spike[ i ] = t_ms;
    return;
  }
  net->Kminus[ i ] = net->Kminus[ i ] * exp( ( net->last_spike[ i ] - t_ms ) * ( 1. / net->tau_minus[ i ] ) ) + 1.0;
  net->last_spike[ i ] = t_ms;
  if ( net->hist_len[ i ] == net->hist_cap[ i ] )
  {
    net->hist_cap[ i ] = net->hist_cap[ i ] ? 2 * net->hist_cap[ i ] : 16;
    net->hist_t[ i ] = realloc( net->hist_t[ i ], sizeof( double ) * ( size_t ) net->hist_cap[ i ] );
    net->hist_K[ i ] = realloc( net->hist_K[ i ], sizeof( double ) * ( size_t ) net->hist_cap[ i ] );
  }
  net->hist_t[ i ][ net->hist_len[ i ] ] = t_ms;
  net->hist_K[ i ][ net->hist_len[ i ] ] = net->Kminus[ i ];
  ++net->hist_len[ i ];
}

/* ArchivingNode::get_K_value (archiving_node.cpp:87-113) */
static double
k_value( const orc_net* net, int64_t i, double t )
{
  for ( int64_t k = net->hist_len[ i ] - 1; k >= 0; --k )
    if ( t - net->hist_t[ i ][ k ] > STDP_EPS )
      return net->hist_K[ i ][ k ] * exp( ( net->hist_t[ i ][ k ] - t ) * ( 1. / net->tau_minus[ i ] ) );
  return 0.;
}

/* stdp_pl_synapse_hom::send for every plastic out-edge of one spike, then
 * handle(SpikeEvent&) into the ring (stdp_pl_synapse_hom.h:255-298) */
static void
deliver_plastic_spike( orc_net* net, int32_t src, int64_t te, double mult )
{
  if ( src >= net->pl_nsrc )
    return;
  const int64_t L = net->L, n = net->n;
  const double t_spike = stamp_ms( net, te + 1 );
  for ( int64_t e = net->pl_row[ src ]; e < net->pl_row[ src + 1 ]; ++e )
  {
    const int32_t tg = net->pl_tgt[ e ];
    const double dd = delay_ms( net, net->pl_d[ e ] );
    double w = net->pl_w[ e ];
    /* get_history( t_lastspike - d, t_spike - d ): entries with
     * t1 + eps <= t < t2 + eps (archiving_node.cpp:154-180), in order */
    const double t1_lim = net->pl_tlast[ e ] - dd + STDP_EPS;
    const double t2_lim = t_spike - dd + STDP_EPS;
    int64_t fin = net->hist_len[ tg ];
    while ( fin > 0 && net->hist_t[ tg ][ fin - 1 ] >= t2_lim )
      --fin;
    int64_t st = fin;
    while ( st > 0 && net->hist_t[ tg ][ st - 1 ] >= t1_lim )
      --st;
    for ( int64_t k = st; k < fin; ++k )
    {
      const double minus_dt = net->pl_tlast[ e ] - ( net->hist_t[ tg ][ k ] + dd );
      const double kplus = net->pl_Kplus[ e ] * exp( minus_dt * net->pl_tau_plus_inv );
      w = w + ( net->pl_lambda * pow( w, net->pl_mu ) * kplus );
    }
    /* depression by the postsynaptic trace at the arrival */
    {
      const double kminus = k_value( net, tg, t_spike - dd );
      const double new_w = w - ( net->pl_lambda * net->pl_alpha * w * kminus );
      w = new_w > 0.0 ? new_w : 0.0;
    }
    net->pl_w[ e ] = w;
    const int64_t slot = imod( te + net->pl_d[ e ], L );
    const double wv = w * mult;
    if ( net->model == ORC_IAF_PSC_DELTA )
      net->ring[ ( slot * 2 + 0 ) * n + tg ] += wv;
    else
      net->ring[ ( slot * 2 + ( wv > 0 ? 0 : 1 ) ) * n + tg ] += wv;
    net->pl_Kplus[ e ] = net->pl_Kplus[ e ] * exp( ( net->pl_tlast[ e ] - t_spike ) * net->pl_tau_plus_inv ) + 1.0;
    net->pl_tlast[ e ] = t_spike;
  }
  net->syn_events += ( net->pl_row[ src + 1 ] - net->pl_row[ src ] ) * ( int64_t ) mult;
}

static void
deliver( orc_net* net, int nthreads )
{
  const int64_t L = net->L, n = net->n;
  const int P = net->nparts;  /* 0: no static connections */
  int64_t ev = 0;
  for ( int64_t s = 0; s < net->sp_len; ++s )
  {
    const int32_t src = net->sp_src[ s ];
    for ( int p = 0; p < P; ++p )
      ev += ( net->part_row[ p ][ src + 1 ] - net->part_row[ p ][ src ] ) * net->sp_mult[ s ];
  }
  net->syn_events += ev;
#pragma omp parallel for schedule( static, 1 ) num_threads( nthreads )
  for ( int p = 0; p < P; ++p )
  {
    const int64_t* rp = net->part_row[ p ];
    const int32_t* tg = net->part_tgt[ p ];
    const double* ww = net->part_w[ p ];
    const int32_t* dd = net->part_d[ p ];
    for ( int64_t s = 0; s < net->sp_len; ++s )
    {
      const int32_t src = net->sp_src[ s ];
      const int64_t te = net->sp_t[ s ];
      const double m = ( double ) net->sp_mult[ s ];
      for ( int64_t e = rp[ src ]; e < rp[ src + 1 ]; ++e )
      {
        const int64_t slot = imod( te + dd[ e ], L );
        /* handle(SpikeEvent&): weight * multiplicity; channel by sign
         * (iaf_psc_exp.cpp:351-362, aeif_cond_alpha.cpp:536-550) */
        const double wv = ww[ e ] * m;
        if ( net->model == ORC_IAF_PSC_DELTA )
          net->ring[ ( slot * 2 + 0 ) * n + tg[ e ] ] += wv;
        else if ( net->model == ORC_IAF_PSC_EXP || net->model == ORC_IAF_PSC_ALPHA )
          net->ring[ ( slot * 2 + ( wv > 0 ? 0 : 1 ) ) * n + tg[ e ] ] += wv;
        else if ( ww[ e ] > 0.0 )
          net->ring[ ( slot * 2 + 0 ) * n + tg[ e ] ] += wv;
        else
          net->ring[ ( slot * 2 + 1 ) * n + tg[ e ] ] += -ww[ e ] * m;
      }
    }
  }
  /* plastic connections: the slice's spikes in emission order per source */
  if ( net->pl_nnz > 0 )
    for ( int64_t s = 0; s < net->sp_len; ++s )
      deliver_plastic_spike( net, net->sp_src[ s ], net->sp_t[ s ], ( double ) net->sp_mult[ s ] );
  net->sp_len = 0;
}

int
orc_run( orc_net* net, int64_t n_steps, int nthreads )
{
#ifdef _OPENMP
  if ( nthreads <= 0 )
    nthreads = omp_get_max_threads();
#else
  nthreads = 1;
#endif
  if ( nthreads <= 0 )
    nthreads = 1;
  if ( !net->prepared )
    prepare( net );
  g_instability = 0;
  tbuf* tbs = calloc( ( size_t ) nthreads, sizeof( tbuf ) );
  int64_t remaining = n_steps;
  while ( remaining > 0 )
  {
    const int32_t from = net->from;
    const int32_t to = ( int32_t ) ( remaining < net->min_delay - from ? from + remaining : net->min_delay );
    const int64_t origin = net->clock;
    double* trace_rows = NULL;
    if ( net->n_trace_idx > 0 )
    {
      const int64_t need = ( net->trace_len + ( to - from ) ) * net->n_trace_idx;
      if ( need > net->trace_cap )
      {
        net->trace_cap = need * 2;
        net->trace = realloc( net->trace, sizeof( double ) * ( size_t ) net->trace_cap );
      }
      trace_rows = net->trace + ( net->trace_len - from ) * net->n_trace_idx;
    }
    /* generator sources emitting in this window */
    while ( net->sched_pos < net->n_sched && net->sched_step[ net->sched_pos ] < origin + to )
    {
      const int64_t te = net->sched_step[ net->sched_pos ];
      if ( te >= origin + from )
        push_spike( net, net->sched_src[ net->sched_pos ], te, 1 );
      ++net->sched_pos;
    }
    const int64_t n = net->n;
#pragma omp parallel num_threads( nthreads )
    {
#ifdef _OPENMP
      const int tid = omp_get_thread_num();
      const int nt = omp_get_num_threads();
#else
      const int tid = 0, nt = 1;
#endif
      const int64_t lo = n * tid / nt, hi = n * ( tid + 1 ) / nt;
      tbuf* tb = &tbs[ tid ];
      tb->len = 0;
      for ( int64_t i = lo; i < hi; ++i )
      {
        const int64_t col = trace_rows ? net->trace_col[ i ] : -1;
        update_neuron( net, i, origin, from, to, tb, col >= 0 ? trace_rows : NULL, col );
      }
    }
    for ( int k = 0; k < nthreads; ++k )
      for ( int64_t j = 0; j < tbs[ k ].len; ++j )
        push_spike( net, tbs[ k ].src[ j ], tbs[ k ].t[ j ], tbs[ k ].mult[ j ] );
    if ( net->n_trace_idx > 0 )
      net->trace_len += to - from;
    remaining -= to - from;
    if ( to == net->min_delay )
    {
      deliver( net, nthreads );
      net->clock += net->min_delay;
      net->from = 0;
    }
    else
    {
      net->from = to;
    }
    if ( g_instability )
      break;
  }
  for ( int k = 0; k < nthreads; ++k )
  {
    free( tbs[ k ].src );
    free( tbs[ k ].t );
    free( tbs[ k ].mult );
  }
  free( tbs );
  if ( g_instability )
  {
    set_err( "NumericalInstability" );
    return -2;
  }
  return 0;
}

int64_t
orc_n_spikes( orc_net* net )
{
  return net->log_len;
}

int64_t
orc_get_spikes( orc_net* net, int32_t* src, int64_t* stamp, int64_t cap )
{
  const int64_t k = net->log_len < cap ? net->log_len : cap;
  memcpy( src, net->log_src, sizeof( int32_t ) * ( size_t ) k );
  memcpy( stamp, net->log_stamp, sizeof( int64_t ) * ( size_t ) k );
  return k;
}

int64_t
orc_n_trace( orc_net* net )
{
  return net->trace_len * net->n_trace_idx;
}

int64_t
orc_get_trace( orc_net* net, double* out, int64_t cap )
{
  const int64_t tot = net->trace_len * net->n_trace_idx;
  const int64_t k = tot < cap ? tot : cap;
  memcpy( out, net->trace, sizeof( double ) * ( size_t ) k );
  return k;
}

int64_t
orc_clock( orc_net* net )
{
  return net->clock + net->from;
}

int64_t
orc_syn_events( orc_net* net )
{
  return net->syn_events;
}
