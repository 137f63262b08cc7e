/* helper_functions.h -- empty stand-in for the CUDA samples header the
 * reference includes; the step modules use nothing from it.  TEST
 * INFRASTRUCTURE ONLY. */
#ifndef REF_HARNESS_HELPER_FUNCTIONS_H
#define REF_HARNESS_HELPER_FUNCTIONS_H
#endif
