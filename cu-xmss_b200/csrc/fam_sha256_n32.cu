// Kernel instantiation of the Sha256N32 hash family (see families.cuh).
#include "../../include/params.h"
#include "family_ops.cuh"

namespace xb {
// Chain kernels keep many warps busy and use the FMA-pipe SHA-256 form
// (XB_CHAINS_MIX); the serial kernels use the plain form.
#ifndef XB_CHAINS_MIX
#define XB_CHAINS_MIX 1
#endif
const FamilyOps kOpsSha256N32 = Launch<Sha256N32, Sha256N32T<XB_CHAINS_MIX>>::table("Sha256N32", XMSS_SHA2);
}  // namespace xb
