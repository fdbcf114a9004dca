/*
 * gl_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle for the Goldilocks
 * NTT big-integer multiply path.
 *
 * This is a plain-C restatement of the reference's CPU algorithm. Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it, and only as
 * the checker; the product never links, loads or calls it.
 *
 * Each function cites the reference code it restates (paths are relative to
 * the reference project root). Parity of this restatement is pinned by the
 * tests against the reference's own compiled code (oracle/_ref, built by
 * oracle/Makefile) and against the golden fixtures in tests/golden/.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

#define ORC_P 0xFFFFFFFF00000001ULL   /* include/goldilocks.h:83 */
#define ORC_EPS 0xFFFFFFFFULL         /* include/goldilocks.h:84 */
#define ORC_G 7ULL                    /* include/goldilocks.h:85 */

/* ---- field: include/goldilocks.h:104-189 ---------------------------------- */

/* goldilocks.h:104-109: a+b folding a 2^64 carry as EPS, then one conditional
 * subtract of p. */
uint64_t orc_gl_add(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    if (s < a) s += ORC_EPS;
    if (s >= ORC_P) s -= ORC_P;
    return s;
}

/* goldilocks.h:114-118: a-b, a borrow is corrected by subtracting EPS. */
uint64_t orc_gl_sub(uint64_t a, uint64_t b) {
    uint64_t d = a - b;
    if (a < b) d -= ORC_EPS;
    return d;
}

/* goldilocks.h:130-154: Solinas fold of hi:lo using 2^64 = EPS, 2^96 = -1. */
uint64_t orc_gl_reduce128(uint64_t lo, uint64_t hi) {
    uint64_t hh = hi >> 32, hl = hi & 0xFFFFFFFFULL;
    uint64_t t0 = lo - hh;
    if (lo < hh) t0 -= ORC_EPS;
    uint64_t t1 = hl * ORC_EPS;
    uint64_t t2 = t0 + t1;
    if (t2 < t0) {
        uint64_t before = t2;
        t2 += ORC_EPS;
        if (t2 < before) t2 += ORC_EPS;
    }
    while (t2 >= ORC_P) t2 -= ORC_P;
    return t2;
}

/* goldilocks.h:158-162 */
uint64_t orc_gl_mul(uint64_t a, uint64_t b) {
    u128 p = (u128)a * b;
    return orc_gl_reduce128((uint64_t)p, (uint64_t)(p >> 64));
}

/* The definition itself, used by the tests as an independent check of the
 * Solinas restatement: (a*b) mod p through 128-bit division. */
uint64_t orc_gl_mul_def(uint64_t a, uint64_t b) {
    return (uint64_t)(((u128)a * b) % ORC_P);
}

/* goldilocks.h:165-173 */
uint64_t orc_gl_pow(uint64_t base, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = orc_gl_mul(r, base);
        base = orc_gl_mul(base, base);
        e >>= 1;
    }
    return r;
}

/* goldilocks.h:178-180 (Fermat) */
uint64_t orc_gl_inv(uint64_t a) { return orc_gl_pow(a, ORC_P - 2); }

/* goldilocks.h:187-189 */
uint64_t orc_gl_root_of_unity(uint64_t n) { return orc_gl_pow(ORC_G, (ORC_P - 1) / n); }

/* ---- NTT helpers: include/ntt.h:37-109 ----------------------------------- */

/* ntt.h:37-50: N = next power of two >= 2na + 2nb. */
uint64_t orc_ntt_length(uint64_t na, uint64_t nb) {
    uint64_t x = 2 * na + 2 * nb, n = 1;
    while (n < x) n <<= 1;
    return n;
}

static uint32_t bitrev(uint32_t i, int logn) {
    uint32_t r = 0;
    for (int b = 0; b < logn; ++b) { r = (r << 1) | (i & 1); i >>= 1; }
    return r;
}

/* src/ntt_cpu.cpp:64-104: in-place iterative radix-2 NTT, bit-reversal first,
 * per-stage root advanced multiplicatively, 1/N applied for the inverse. */
void orc_ntt_transform(uint64_t* a, uint64_t n, int inverse) {
    if (n <= 1) return;
    int logn = 0;
    while ((1ULL << logn) < n) ++logn;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t j = bitrev(i, logn);
        if (i < j) { uint64_t t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    for (uint64_t len = 2; len <= n; len <<= 1) {
        uint64_t wl = orc_gl_root_of_unity(len);
        if (inverse) wl = orc_gl_inv(wl);
        uint64_t half = len >> 1;
        for (uint64_t i = 0; i < n; i += len) {
            uint64_t w = 1;
            for (uint64_t j = 0; j < half; ++j) {
                uint64_t u = a[i + j];
                uint64_t v = orc_gl_mul(a[i + j + half], w);
                a[i + j] = orc_gl_add(u, v);
                a[i + j + half] = orc_gl_sub(u, v);
                w = orc_gl_mul(w, wl);
            }
        }
    }
    if (inverse) {
        uint64_t ninv = orc_gl_inv(n);
        for (uint64_t i = 0; i < n; ++i) a[i] = orc_gl_mul(a[i], ninv);
    }
}

/* ntt.h:56-64: limb i -> digits (lo16, hi16) at 2i, 2i+1, zero padded. */
static void repack16(const uint32_t* a, uint64_t na, uint64_t* out, uint64_t n) {
    memset(out, 0, n * sizeof(uint64_t));
    for (uint64_t i = 0; i < na; ++i) {
        out[2 * i] = a[i] & 0xFFFFu;
        out[2 * i + 1] = (a[i] >> 16) & 0xFFFFu;
    }
}

/* ntt.h:70-91: running 64-bit carry over base-2^16 coefficients, digits paired
 * into u32 limbs, trailing zero limbs trimmed. Writes at most cap limbs and
 * returns the trimmed length (or (uint64_t)-1 when cap is too small). */
uint64_t orc_carry_propagate(const uint64_t* conv, uint64_t n, uint32_t* out, uint64_t cap) {
    uint64_t carry = 0, i = 0, k = 0;
    while (i < n || carry) {
        uint64_t cur = carry + (i < n ? conv[i] : 0);
        uint32_t lo16 = (uint32_t)(cur & 0xFFFFu);
        carry = cur >> 16;
        ++i;
        uint64_t cur2 = carry + (i < n ? conv[i] : 0);
        uint32_t hi16 = (uint32_t)(cur2 & 0xFFFFu);
        carry = cur2 >> 16;
        ++i;
        uint32_t limb = lo16 | (hi16 << 16);
        if (k >= cap) {
            if (limb != 0) return (uint64_t)-1;
        } else {
            out[k] = limb;
        }
        ++k;
    }
    if (k > cap) k = cap;
    while (k > 0 && out[k - 1] == 0) --k;
    return k;
}

/* src/ntt_cpu.cpp:111-129: repack, forward x2, pointwise, inverse, carry.
 * out must hold na+nb limbs. Returns the trimmed length, 0 for an empty input. */
uint64_t orc_mul_ntt(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb,
                     uint32_t* out) {
    if (na == 0 || nb == 0) return 0;
    uint64_t n = orc_ntt_length(na, nb);
    uint64_t* fa = (uint64_t*)malloc(n * sizeof(uint64_t));
    uint64_t* fb = (uint64_t*)malloc(n * sizeof(uint64_t));
    if (!fa || !fb) { free(fa); free(fb); return (uint64_t)-1; }
    repack16(a, na, fa, n);
    repack16(b, nb, fb, n);
    orc_ntt_transform(fa, n, 0);
    orc_ntt_transform(fb, n, 0);
    for (uint64_t i = 0; i < n; ++i) fa[i] = orc_gl_mul(fa[i], fb[i]);
    orc_ntt_transform(fa, n, 1);
    uint64_t len = orc_carry_propagate(fa, n, out, na + nb);
    free(fa);
    free(fb);
    return len;
}

/* src/bignum.cpp:125-143: O(n*m) long multiplication, trimmed. */
uint64_t orc_mul_schoolbook(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb,
                            uint32_t* out) {
    if (na == 0 || nb == 0) return 0;
    memset(out, 0, (na + nb) * sizeof(uint32_t));
    for (uint64_t i = 0; i < na; ++i) {
        uint64_t carry = 0, ai = a[i];
        for (uint64_t j = 0; j < nb; ++j) {
            uint64_t cur = (uint64_t)out[i + j] + ai * (uint64_t)b[j] + carry;
            out[i + j] = (uint32_t)cur;
            carry = cur >> 32;
        }
        out[i + nb] += (uint32_t)carry;
    }
    uint64_t k = na + nb;
    while (k > 0 && out[k - 1] == 0) --k;
    return k;
}

/* ---- seeded operands --------------------------------------------------------
 * limb i of operand (seed, n) = high 32 bits of splitmix64's output function
 * applied to seed + (i+1)*0x9E3779B97F4A7C15; the top limb is forced non-zero.
 * kind 0 = random, 1 = all 0xFFFFFFFF. The product has the same generator on
 * the device and in numpy; this copy exists so the tests can cross-check them. */
static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
void orc_gen_operand(uint64_t seed, uint64_t n, int kind, uint32_t* out) {
    for (uint64_t i = 0; i < n; ++i)
        out[i] = kind == 1 ? 0xFFFFFFFFu
                           : (uint32_t)(mix64(seed + (i + 1) * 0x9E3779B97F4A7C15ULL) >> 32);
    if (n > 0 && out[n - 1] == 0) out[n - 1] = 1;
}

/* ---- Chudnovsky binary splitting: src/chudnovsky.cpp:64-102 ----------------
 * A restatement with a minimal sign-magnitude integer (little-endian u32
 * limbs) whose multiply is orc_mul_schoolbook below 64 limbs and orc_mul_ntt
 * above. Used for small trees only; large trees are checked against the
 * reference's own compiled code. */
typedef struct { uint32_t* m; uint64_t n; int s; } orc_big;

static void big_trim(orc_big* x) {
    while (x->n > 0 && x->m[x->n - 1] == 0) --x->n;
    if (x->n == 0) x->s = 0;
}
static orc_big big_from_u64(uint64_t v) {
    orc_big r;
    r.m = (uint32_t*)malloc(2 * sizeof(uint32_t));
    r.m[0] = (uint32_t)v; r.m[1] = (uint32_t)(v >> 32);
    r.n = 2; r.s = 1;
    big_trim(&r);
    return r;
}
static orc_big big_mul(const orc_big* a, const orc_big* b) {
    orc_big r;
    r.s = a->s * b->s;
    r.m = (uint32_t*)calloc(a->n + b->n + 1, sizeof(uint32_t));
    if (a->n == 0 || b->n == 0) { r.n = 0; r.s = 0; return r; }
    if (a->n < 64 || b->n < 64) r.n = orc_mul_schoolbook(a->m, a->n, b->m, b->n, r.m);
    else r.n = orc_mul_ntt(a->m, a->n, b->m, b->n, r.m);
    big_trim(&r);
    return r;
}
static int cmp_mag(const orc_big* a, const orc_big* b) {
    if (a->n != b->n) return a->n < b->n ? -1 : 1;
    for (uint64_t i = a->n; i-- > 0;)
        if (a->m[i] != b->m[i]) return a->m[i] < b->m[i] ? -1 : 1;
    return 0;
}
/* src/bignum.cpp:310-325: signed addition by sign-magnitude cases. */
static orc_big big_add(const orc_big* a, const orc_big* b) {
    orc_big r;
    uint64_t n = (a->n > b->n ? a->n : b->n) + 1;
    r.m = (uint32_t*)calloc(n, sizeof(uint32_t));
    r.n = n;
    if (a->s == 0 || b->s == 0) {
        const orc_big* x = a->s ? a : b;
        memcpy(r.m, x->m, x->n * 4); r.n = x->n; r.s = x->s;
        big_trim(&r);
        return r;
    }
    if (a->s == b->s) {
        uint64_t c = 0;
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t s = c + (i < a->n ? a->m[i] : 0) + (i < b->n ? b->m[i] : 0);
            r.m[i] = (uint32_t)s; c = s >> 32;
        }
        r.s = a->s;
    } else {
        int c = cmp_mag(a, b);
        const orc_big* big = c >= 0 ? a : b;
        const orc_big* sml = c >= 0 ? b : a;
        int64_t br = 0;
        for (uint64_t i = 0; i < n; ++i) {
            int64_t d = (int64_t)(i < big->n ? big->m[i] : 0) - (i < sml->n ? sml->m[i] : 0) - br;
            br = d < 0;
            r.m[i] = (uint32_t)(d + (br ? ((int64_t)1 << 32) : 0));
        }
        r.s = c == 0 ? 0 : big->s;
    }
    big_trim(&r);
    return r;
}
static void big_free(orc_big* x) { free(x->m); x->m = NULL; x->n = 0; }

typedef struct { orc_big P, Q, T; } orc_pqt;

/* src/chudnovsky.cpp:64-102 (leaves at :68-90, merge at :98-100). */
static orc_pqt orc_bs(uint64_t a, uint64_t b) {
    orc_pqt r;
    if (b - a == 1) {
        if (a == 0) {
            r.P = big_from_u64(1); r.Q = big_from_u64(1); r.T = big_from_u64(13591409ULL);
        } else {
            orc_big f1 = big_from_u64(6 * a - 5), f2 = big_from_u64(2 * a - 1), f3 = big_from_u64(6 * a - 1);
            orc_big t = big_mul(&f1, &f2);
            r.P = big_mul(&t, &f3);
            big_free(&t);
            orc_big A = big_from_u64(a), C = big_from_u64(10939058860032000ULL);
            orc_big aa = big_mul(&A, &A), aaa = big_mul(&aa, &A);
            r.Q = big_mul(&aaa, &C);
            orc_big k0 = big_from_u64(13591409ULL), k1 = big_from_u64(545140134ULL);
            orc_big ak = big_mul(&A, &k1);
            orc_big lin = big_add(&k0, &ak);
            r.T = big_mul(&r.P, &lin);
            if (a & 1) r.T.s = -r.T.s;
            big_free(&f1); big_free(&f2); big_free(&f3); big_free(&A); big_free(&C);
            big_free(&aa); big_free(&aaa); big_free(&k0); big_free(&k1); big_free(&ak); big_free(&lin);
        }
        return r;
    }
    uint64_t m = (a + b) / 2;
    orc_pqt L = orc_bs(a, m), R = orc_bs(m, b);
    r.P = big_mul(&L.P, &R.P);
    r.Q = big_mul(&L.Q, &R.Q);
    orc_big x = big_mul(&L.T, &R.Q), y = big_mul(&L.P, &R.T);
    r.T = big_add(&x, &y);
    big_free(&x); big_free(&y);
    big_free(&L.P); big_free(&L.Q); big_free(&L.T);
    big_free(&R.P); big_free(&R.Q); big_free(&R.T);
    return r;
}

void* orc_bs_run(uint64_t a, uint64_t b) {
    orc_pqt* h = (orc_pqt*)malloc(sizeof(orc_pqt));
    *h = orc_bs(a, b);
    return h;
}
static orc_big* orc_pick(void* h, int w) {
    orc_pqt* p = (orc_pqt*)h;
    return w == 0 ? &p->P : w == 1 ? &p->Q : &p->T;
}
uint64_t orc_bs_len(void* h, int w) { return orc_pick(h, w)->n; }
int orc_bs_sign(void* h, int w) { return orc_pick(h, w)->s; }
void orc_bs_copy(void* h, int w, uint32_t* out) {
    orc_big* x = orc_pick(h, w);
    memcpy(out, x->m, x->n * 4);
}
void orc_bs_free(void* h) {
    orc_pqt* p = (orc_pqt*)h;
    big_free(&p->P); big_free(&p->Q); big_free(&p->T);
    free(p);
}
