/* Hand-written noarch build configuration used to compile the CPS reference
   (test oracle only). It stands in for the header that CPS's configure script
   would generate from precision.h.in: TARGET=NOARCH, double precision, namespace cps. */
#include <stdint.h>
#ifndef _PRECISION_H_
#define _PRECISION_H_
typedef double Float;
typedef double IFloat;
typedef uint64_t Pointer;
#endif
