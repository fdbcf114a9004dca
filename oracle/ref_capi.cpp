// ref_capi.cpp -- TEST INFRASTRUCTURE ONLY (part of the oracle build).
//
// A plain C ABI over the reference's own CPU code so that Python tests, the
// golden-fixture generator and the CPU-baseline leg of bench.py can call it via
// ctypes. Every function here forwards to an unmodified reference function:
//   ref_mul(0..3)      -> mul_schoolbook / mul_karatsuba / mul_ntt_cpu / mul_dispatch
//                         (src/bignum.cpp:125-232, src/ntt_cpu.cpp:111-129)
//   ref_gl_*           -> include/goldilocks.h:90-189
//   ref_ntt_length     -> include/ntt.h:37-50
//   ref_bs_*           -> chudnovsky_bs (src/chudnovsky.cpp:64-102)
//   ref_compute_pi     -> compute_pi_chudnovsky (src/chudnovsky.cpp:107-164)
// Nothing in the product links against this file.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "bignum.h"
#include "chudnovsky.h"
#include "goldilocks.h"
#include "ntt.h"

using namespace pidigits;

extern "C" {

// backend: 0 schoolbook, 1 karatsuba, 2 ntt-cpu, 3 mul_dispatch (Auto, CPU only).
// Returns 0 on success, 1 when out_cap is too small. *out_len = trimmed length.
int ref_mul(int backend, const uint32_t* a, size_t na, const uint32_t* b, size_t nb,
            uint32_t* out, size_t out_cap, size_t* out_len) {
    std::vector<uint32_t> va(a, a + na), vb(b, b + nb), r;
    switch (backend) {
        case 0: r = mul_schoolbook(va, vb); break;
        case 1: r = mul_karatsuba(va, vb); break;
        case 2: r = mul_ntt_cpu(va, vb); break;
        default: {
            MulBackend saved = g_mul.backend;
            bool saved_pc = g_mul.prefer_cuda;
            g_mul.backend = MulBackend::Auto;
            g_mul.prefer_cuda = false;
            r = mul_dispatch(va, vb);
            g_mul.backend = saved;
            g_mul.prefer_cuda = saved_pc;
        }
    }
    *out_len = r.size();
    if (r.size() > out_cap) return 1;
    if (!r.empty()) std::memcpy(out, r.data(), r.size() * sizeof(uint32_t));
    return 0;
}

uint64_t ref_gl_add(uint64_t a, uint64_t b) { return gl_add(a, b); }
uint64_t ref_gl_sub(uint64_t a, uint64_t b) { return gl_sub(a, b); }
uint64_t ref_gl_mul(uint64_t a, uint64_t b) { return gl_mul(a, b); }
uint64_t ref_gl_reduce128(uint64_t lo, uint64_t hi) { return gl_reduce128(lo, hi); }
uint64_t ref_gl_pow(uint64_t a, uint64_t e) { return gl_pow(a, e); }
uint64_t ref_gl_inv(uint64_t a) { return gl_inv(a); }
uint64_t ref_gl_root_of_unity(uint64_t n) { return gl_root_of_unity(n); }
uint64_t ref_ntt_length(uint64_t na, uint64_t nb) { return ntt_length(na, nb); }

// Binary splitting with the backend forced (0 schoolbook .. 3 auto-cpu), as
// the reference's tree would run it. The result lives in a heap handle.
struct RefPQT { PQT r; };

void* ref_bs_run(uint64_t a, uint64_t b, int backend) {
    MulBackend saved = g_mul.backend;
    bool saved_pc = g_mul.prefer_cuda;
    static const MulBackend map[] = {MulBackend::Schoolbook, MulBackend::Karatsuba,
                                     MulBackend::NttCpu, MulBackend::Auto};
    g_mul.backend = map[(backend < 0 || backend > 3) ? 3 : backend];
    g_mul.prefer_cuda = false;
    RefPQT* h = new RefPQT;
    h->r = chudnovsky_bs(a, b);
    g_mul.backend = saved;
    g_mul.prefer_cuda = saved_pc;
    return h;
}

static const BigInt& pick(void* h, int which) {
    RefPQT* p = static_cast<RefPQT*>(h);
    return which == 0 ? p->r.P : which == 1 ? p->r.Q : p->r.T;
}
size_t ref_bs_len(void* h, int which) { return pick(h, which).mag.size(); }
int ref_bs_sign(void* h, int which) { return pick(h, which).sign; }
void ref_bs_copy(void* h, int which, uint32_t* out) {
    const BigInt& v = pick(h, which);
    if (!v.mag.empty()) std::memcpy(out, v.mag.data(), v.mag.size() * 4);
}
void ref_bs_free(void* h) { delete static_cast<RefPQT*>(h); }

// pi to `digits` digits ("3.1415..."), Auto backend on the CPU. Returns the
// string length, or 0 when cap is too small.
size_t ref_compute_pi(uint64_t digits, char* out, size_t cap, uint64_t* terms) {
    g_mul.backend = MulBackend::Auto;
    g_mul.prefer_cuda = false;
    ChudnovskyResult r = compute_pi_chudnovsky(digits, false);
    if (terms) *terms = r.terms;
    if (r.pi.size() + 1 > cap) return 0;
    std::memcpy(out, r.pi.c_str(), r.pi.size() + 1);
    return r.pi.size();
}

uint64_t ref_chudnovsky_terms_for_digits(uint64_t digits) {
    return chudnovsky_terms_for_digits(digits);
}

}  // extern "C"
