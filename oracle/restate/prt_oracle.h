/* Test infrastructure: see prt_oracle.c. */
#ifndef PRT_ORACLE_H
#define PRT_ORACLE_H
#include <stdint.h>
void prto_sobol(uint32_t seed, int64_t n, const uint32_t* sample_index, const uint32_t* pixel_id,
                const uint32_t* dim_set, int dims, float* out);
#endif
