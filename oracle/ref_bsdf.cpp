// Test infrastructure (oracle only): batched BSDF queries through the reference's own
// BsdfSimd classes. Filled in with the BSDF parity tuples.
#include "bsdf/albedo_tables.h"
