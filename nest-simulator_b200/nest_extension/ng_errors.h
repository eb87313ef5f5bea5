/*
 * ng_errors.h -- how the engine's C ABI status codes (include/nestgpu.h)
 * become the reference's exceptions inside a NEST extension module.
 *
 * Kept free of NEST headers so that the mapping compiles and is tested on
 * its own; gpu_engine.cpp throws the nest:: exception each kind names
 * (nestkernel/exceptions.h: BadProperty :679, KernelException :64,
 * NumericalInstability :1062).
 */
#ifndef NESTGPU_NG_ERRORS_H
#define NESTGPU_NG_ERRORS_H

#include "../../include/nestgpu.h"

namespace nestgpu
{

enum class ErrorKind
{
  none,                 // NG_OK
  bad_property,         // nest::BadProperty: a parameter or state value the engine refuses
  kernel_exception,     // nest::KernelException: wrong call order, device or capacity failures
  numerical_instability // nest::NumericalInstability (aeif_cond_alpha.cpp:481-490)
};

inline ErrorKind
error_kind( int status )
{
  switch ( status )
  {
  case NG_OK:
    return ErrorKind::none;
  case NG_ERR_ARG:
  case NG_ERR_UNKNOWN_NAME:
    return ErrorKind::bad_property;
  case NG_ERR_NUMERIC:
    return ErrorKind::numerical_instability;
  case NG_ERR_CUDA:
  case NG_ERR_STATE:
  case NG_ERR_MEMORY:
  case NG_ERR_CAPACITY:
  default:
    return ErrorKind::kernel_exception;
  }
}

inline const char*
error_kind_name( ErrorKind k )
{
  switch ( k )
  {
  case ErrorKind::none:
    return "none";
  case ErrorKind::bad_property:
    return "BadProperty";
  case ErrorKind::numerical_instability:
    return "NumericalInstability";
  default:
    return "KernelException";
  }
}

}  // namespace nestgpu

#endif
