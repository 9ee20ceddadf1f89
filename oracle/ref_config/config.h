/* Hand-written noarch build configuration used to compile the CPS reference
   (test oracle only). It stands in for the header that CPS's configure script
   would generate from config.h.in: TARGET=NOARCH, double precision, namespace cps. */
#ifndef INCLUDED_CONFIG_H_
#define INCLUDED_CONFIG_H_
#include <conf.h>
#define NOARCH 0
#define QCDOC  1
#define QCDSP  2
#define BGL    3
#define BGP    4
#define BGQ    5
#define VERSION_MAJOR 5
#define VERSION_MINOR 3
#define VERSION_SUB 1
#define VERSION_STR "CPS_V5.3.1"
#define TARGET NOARCH
#define CPS_FLOAT_ALIGN
#define CWDPREFIX(A) A
#define CAST_AWAY_CONST(x) ( const_cast<char*>(x) )
#define GLOBALSUM_TYPE double
#define CPS_END_NAMESPACE    }
#define CPS_START_NAMESPACE  namespace cps {
#define USING_NAMESPACE_CPS  using namespace cps;
#define CPS_NAMESPACE        cps
#define COMMS_DATASIZE (sizeof(double))
#undef UNIFORM_SEED_TESTING
#undef UNIFORM_SEED_NO_COMMS
#endif
