/* Oracle, all-double type map.  TEST INFRASTRUCTURE. */
#define ORACLE_TYPEMAP_MIXED 0
#include "oracle_impl.h"
#include "oracle_driver.h"
