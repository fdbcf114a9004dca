// ref_stub.cpp -- TEST INFRASTRUCTURE ONLY (part of the oracle build).
//
// The reference declares `mul_ntt_cuda` and `cuda_available` in
// include/bignum.h:200-205 and names a CPU stub for GPU-less builds at
// include/bignum.h:198-199, but that stub file is not in its tree. This file is
// that stub, written for the oracle build only: the oracle library is the
// reference's CPU code, so the "GPU" entry point forwards to the reference's CPU
// NTT and reports that no GPU is present. It is never linked into the product.
#include "bignum.h"

namespace pidigits {

std::vector<uint32_t> mul_ntt_cuda(const std::vector<uint32_t>& a,
                                   const std::vector<uint32_t>& b) {
    return mul_ntt_cpu(a, b);
}

bool cuda_available() { return false; }

}  // namespace pidigits
