/* Oracle, Fortran-faithful type map (real = float).  TEST INFRASTRUCTURE. */
#define ORACLE_TYPEMAP_MIXED 1
#include "oracle_impl.h"
#include "oracle_driver.h"
