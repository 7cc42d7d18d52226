/*
 * Minimal stand-in for <papi.h>, test infrastructure only.
 *
 * The reference's merge/SpTRSV.cpp includes profile/include/papiProfiling.hpp, which
 * includes <papi.h> for six cache-event macros and PAPI_NULL. Every call into PAPI is
 * commented out in the reference (test/FusionDemo.cpp:117, merge/SpTRSV.cpp:453), and
 * profile/papiProfiling.cpp is not compiled by oracle/Makefile, so the header only has to
 * supply these constants for the reference sources to compile. PAPI is not installed here.
 */
#ifndef BAAS_ORACLE_PAPI_STUB_H
#define BAAS_ORACLE_PAPI_STUB_H

#define PAPI_NULL (-1)
#define PAPI_L1_DCA 0x80000040
#define PAPI_L1_DCM 0x80000000
#define PAPI_L2_DCA 0x80000041
#define PAPI_L2_DCM 0x80000002
#define PAPI_L3_DCA 0x80000042
#define PAPI_L3_DCM 0x80000004

#endif
