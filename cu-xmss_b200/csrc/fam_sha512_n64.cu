// Kernel instantiation of the Sha512N64 hash family (see families.cuh).
#include "../../include/params.h"
#include "family_ops.cuh"

namespace xb {
const FamilyOps kOpsSha512N64 = Launch<Sha512N64>::table("Sha512N64", XMSS_SHA2);
}  // namespace xb
