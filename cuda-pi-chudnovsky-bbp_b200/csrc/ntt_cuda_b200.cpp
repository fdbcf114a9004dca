// ntt_cuda_b200.cpp -- drop-in definitions of the reference's GPU multiply
// backend (include/bignum.h:197-205) on top of the B200 C ABI.
//
// Link this file (with libb2m.so) in place of the reference's src/ntt_cuda.cu.
// The reference's mul_dispatch (src/bignum.cpp:204-232), `--backend ntt-cuda`
// (src/main.cpp:70-78), chudnovsky_bs and the self-test then run on the B200
// kernels without source changes.
//
// Behavioural differences from src/ntt_cuda.cu, both deliberate:
//  * no silent CPU fallback (src/ntt_cuda.cu:182,239-241): a failure throws
//    std::runtime_error carrying the library's status text;
//  * cuda_available() reports whether the B200 backend initialised on device
//    0, not merely whether some CUDA device exists (src/ntt_cuda.cu:165-173).
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "b2m.h"

namespace pidigits {

bool cuda_available() { return b2m_cuda_available() != 0; }

std::vector<uint32_t> mul_ntt_cuda(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {
    if (a.empty() || b.empty()) return {};
    if (!cuda_available())
        throw std::runtime_error(std::string("mul_ntt_cuda: B200 backend unavailable: ") + b2m_last_error());
    std::vector<uint32_t> out(a.size() + b.size());
    uint64_t len = 0;
    const b2m_status s = b2m_mul_host(a.data(), a.size(), b.data(), b.size(), out.data(), out.size(), &len);
    if (s != B2M_OK)
        throw std::runtime_error(std::string("mul_ntt_cuda: ") + b2m_strerror(s) + " (" + b2m_last_error() + ")");
    out.resize(len);
    return out;
}

}  // namespace pidigits

// Vector forms of the sub-quadratic division, square root and decimal
// conversion, for the seams the reference leaves for them: the body of
// div_fast (src/bignum_div.cpp:170-178), of isqrt (:189-204) and of
// BigInt::to_decimal (:239-267) can forward the magnitudes here (signs stay
// with the caller; all three take non-negative values). They throw on failure
// like mul_ntt_cuda.
namespace pidigits_b200 {

static void check(b2m_status s, const char* what) {
    if (s != B2M_OK)
        throw std::runtime_error(std::string(what) + ": " + b2m_strerror(s) + " (" + b2m_last_error() + ")");
}

std::vector<uint32_t> div_floor(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b,
                                std::vector<uint32_t>* rem) {
    std::vector<uint32_t> q(a.size() >= b.size() ? a.size() - b.size() + 1 : 1), r(b.size());
    uint64_t ql = 0, rl = 0;
    check(b2m_divmod_host(a.data(), a.size(), b.data(), b.size(), q.data(), q.size(), &ql, r.data(), r.size(), &rl),
          "div_floor");
    q.resize(ql);
    r.resize(rl);
    if (rem) *rem = std::move(r);
    return q;
}

std::vector<uint32_t> isqrt(const std::vector<uint32_t>& a) {
    std::vector<uint32_t> s((a.size() + 1) / 2 + 1);
    uint64_t n = 0;
    check(b2m_isqrt_host(a.data(), a.size(), s.data(), s.size(), &n), "isqrt");
    s.resize(n);
    return s;
}

std::string to_decimal(const std::vector<uint32_t>& a) {
    std::string out((size_t)(a.size() * 9.64) + 16, '\0');  // 32 log10(2) < 9.64 digits per limb
    uint64_t n = 0;
    check(b2m_to_decimal_host(a.data(), a.size(), &out[0], out.size(), &n), "to_decimal");
    out.resize(n);
    return out;
}

}  // namespace pidigits_b200
