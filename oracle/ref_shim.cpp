// ref_shim.cpp -- extern "C" entry into the reference's own propagator code
// (libnestutil/iaf_propagator.cpp, compiled from the reference sources by
// oracle/build_ref.sh).  TEST INFRASTRUCTURE ONLY.
#include <tuple>

#include "iaf_propagator.h"

extern "C" double
ref_iaf_propagator_exp( double tau_syn, double tau_m, double c_m, double h )
{
  return IAFPropagatorExp( tau_syn, tau_m, c_m ).evaluate( h );
}

extern "C" void
ref_iaf_propagator_alpha( double tau_syn, double tau_m, double c_m, double h, double* out )
{
  std::tie( out[ 0 ], out[ 1 ] ) = IAFPropagatorAlpha( tau_syn, tau_m, c_m ).evaluate( h );
}
