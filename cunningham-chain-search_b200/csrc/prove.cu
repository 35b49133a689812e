// Prove / chain-walk kernels for sm_100a.
//
// Reference behaviour replaced:
//   * cc18_prove_kernel (v13:1462-1538) and its u128 shift-and-add arithmetic
//     (v13:1265-1452): here Montgomery multiplication on 32-bit limbs (CIOS,
//     IMAD / IMAD.HI), limb count chosen per number (2..6 limbs, <= 192 bits),
//     so chain walks never wrap at 2^128;
//   * the CPU GMP prover pool (v13:1716-2068): the same per-survivor semantics
//     (62-prime trial division, primality, backward walk to the true root,
//     forward walk, MAX_CHAIN = 64) run on the device.
// Primality: CCS_PRIME_MR = strong-PRP for each witness after trial division
// by {3..71} (v13 gpu_is_prime, v13:1428-1452); CCS_PRIME_BPSW = Baillie-PSW
// (strong PRP base 2 + strong Lucas, Selfridge method A), the semantics of
// GMP 6.3 mpz_probab_prime_p(n, 1) used by the reference CPU prover;
// CCS_PRIME_V33 = the reference CPU engine's own per-role tests (strong PRP
// to 2, 3, 5 for n; Baillie-PSW for predecessors; screened Fermat base 2 for
// forward links, v33:1290-1339, 1512-1577).
#include "ccs_kernels.cuh"
#include "../../include/ccs.h"

namespace ccs {

__constant__ ProveConst c_prove[kMaxProfiles];

// Montgomery products executed by walk launches (one atomic per number)
__device__ unsigned long long g_modmul_count = 0;
// 32 x 32-bit word products of those (2 NL^2 + NL per CIOS product)
__device__ unsigned long long g_wordmul_count = 0;

cudaError_t upload_prove_const(int slot, const ProveConst& pc, cudaStream_t st) {
    return cudaMemcpyToSymbolAsync(c_prove, &pc, sizeof(ProveConst), slot * sizeof(ProveConst),
                                   cudaMemcpyHostToDevice, st);
}

// ---------------------------------------------------------------------------
// multi-limb helpers (little-endian 32-bit limbs, kMaxLimbs storage)
// ---------------------------------------------------------------------------
struct Big {
    uint32_t w[kMaxLimbs];
};

__device__ __forceinline__ int big_bits(const Big& a) {
#pragma unroll
    for (int i = kMaxLimbs - 1; i >= 0; i--)
        if (a.w[i]) return 32 * i + 32 - __clz(a.w[i]);
    return 0;
}

// x mod q for x < 2^32, magic = floor((2^32 - 1) / q)
__device__ __forceinline__ uint32_t mod_m32(uint32_t x, uint32_t q, uint32_t magic) {
    const uint32_t t = x - __umulhi(x, magic) * q;
    return t >= q ? t - q : t;
}

// a mod q for q < 2^16: 16-bit digits, one reciprocal
__device__ __forceinline__ uint32_t big_mod_small(const Big& a, uint32_t q) {
    const uint32_t magic = 0xFFFFFFFFu / q;
    uint32_t r = 0;
#pragma unroll
    for (int i = kMaxLimbs - 1; i >= 0; i--) {
        r = mod_m32((r << 16) | (a.w[i] >> 16), q, magic);
        r = mod_m32((r << 16) | (a.w[i] & 0xFFFFu), q, magic);
    }
    return r;
}

// a mod m for m < 2^32 with magic64 = floor((2^64 - 1) / m)
__device__ __forceinline__ uint32_t big_mod_u32(const Big& a, uint32_t m, uint64_t magic64) {
    uint64_t r = 0;
#pragma unroll
    for (int i = kMaxLimbs - 1; i >= 0; i--) {
        const uint64_t x = (r << 32) | a.w[i];
        uint64_t t = x - __umul64hi(x, magic64) * m;
        while (t >= m) t -= m;
        r = t;
    }
    return (uint32_t)r;
}

// a = 2a + 1 (returns carry-out)
__device__ __forceinline__ uint32_t big_shl1_inc(Big& a) {
    uint32_t carry = 1;
#pragma unroll
    for (int i = 0; i < kMaxLimbs; i++) {
        uint32_t nc = a.w[i] >> 31;
        a.w[i] = (a.w[i] << 1) | carry;
        carry = nc;
    }
    return carry;
}

// next chain member: 2a + 1 (first kind) or 2a - 1 (second kind, a >= 1)
__device__ __forceinline__ void big_next(Big& a, uint32_t kind) {
    if (kind != 2) { big_shl1_inc(a); return; }
    uint32_t carry = 0;
#pragma unroll
    for (int i = 0; i < kMaxLimbs; i++) {
        const uint32_t nc = a.w[i] >> 31;
        a.w[i] = (a.w[i] << 1) | carry;
        carry = nc;
    }
    uint32_t br = 1;
#pragma unroll
    for (int i = 0; i < kMaxLimbs; i++) {
        const uint32_t v = a.w[i];
        a.w[i] = v - br;
        br = (br && v == 0) ? 1u : 0u;
    }
}

// predecessor of an odd chain member: (a - 1) / 2 (first kind) or
// (a + 1) / 2 (second kind, v13b:1522)
__device__ __forceinline__ void big_prev(Big& a, uint32_t kind) {
    uint32_t top = 0;
    if (kind == 2) {
        uint32_t c = 1;
#pragma unroll
        for (int i = 0; i < kMaxLimbs; i++) {
            const uint64_t v = (uint64_t)a.w[i] + c;
            a.w[i] = (uint32_t)v;
            c = (uint32_t)(v >> 32);
        }
        top = c;
    }
#pragma unroll
    for (int i = 0; i < kMaxLimbs; i++) {
        const uint32_t hi = (i + 1 < kMaxLimbs) ? a.w[i + 1] : top;
        a.w[i] = (a.w[i] >> 1) | (hi << 31);
    }
}

__device__ __forceinline__ bool big_lt_u32(const Big& a, uint32_t v) {
#pragma unroll
    for (int i = 1; i < kMaxLimbs; i++)
        if (a.w[i]) return false;
    return a.w[0] < v;
}

// ---------------------------------------------------------------------------
// Montgomery arithmetic modulo n with NL limbs (R = 2^(32 NL))
// ---------------------------------------------------------------------------
template <int NL>
struct Mont {
    uint32_t n[NL];
    uint32_t ninv;        // -n^{-1} mod 2^32
    uint32_t one[NL];     // R mod n
    uint32_t mone[NL];    // n - (R mod n)  (Montgomery form of -1)
    uint32_t count;       // Montgomery products executed with this context
    uint32_t sq;          // of them squares (montsqr)
};

// word products of one Montgomery product (CIOS: NL rows of NL + 1 + NL) and
// of one square (montsqr: NL (NL - 1)/2 cross + NL diagonal + NL^2 + NL
// reduction, for the specialised 3 and 4 limbs)
__host__ __device__ constexpr uint32_t mul_words(int NL) { return 2 * NL * NL + NL; }
__host__ __device__ constexpr uint32_t sqr_words(int NL) {
    return (NL == 3 || NL == 4) ? NL * (NL - 1) / 2 + NL + NL * NL + NL : mul_words(NL);
}

template <int NL>
__device__ __forceinline__ bool ge(const uint32_t (&a)[NL], const uint32_t (&b)[NL]) {
#pragma unroll
    for (int i = NL - 1; i >= 0; i--)
        if (a[i] != b[i]) return a[i] > b[i];
    return true;
}

template <int NL>
__device__ __forceinline__ bool eq(const uint32_t (&a)[NL], const uint32_t (&b)[NL]) {
    bool e = true;
#pragma unroll
    for (int i = 0; i < NL; i++) e &= (a[i] == b[i]);
    return e;
}

template <int NL>
__device__ __forceinline__ bool is_zero(const uint32_t (&a)[NL]) {
    uint32_t o = 0;
#pragma unroll
    for (int i = 0; i < NL; i++) o |= a[i];
    return o == 0;
}

// r = a - b, returns borrow
template <int NL>
__device__ __forceinline__ uint32_t sub_n(uint32_t (&r)[NL], const uint32_t (&a)[NL],
                                          const uint32_t (&b)[NL]) {
    uint32_t br = 0;
#pragma unroll
    for (int i = 0; i < NL; i++) {
        uint64_t d = (uint64_t)a[i] - b[i] - br;
        r[i] = (uint32_t)d;
        br = (uint32_t)(d >> 32) & 1u;
    }
    return br;
}

template <int NL>
__device__ __forceinline__ uint32_t add_n(uint32_t (&r)[NL], const uint32_t (&a)[NL],
                                          const uint32_t (&b)[NL]) {
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < NL; i++) {
        uint64_t s = (uint64_t)a[i] + b[i] + c;
        r[i] = (uint32_t)s;
        c = (uint32_t)(s >> 32);
    }
    return c;
}

template <int NL>
__device__ __forceinline__ void addmod(uint32_t (&r)[NL], const uint32_t (&a)[NL],
                                       const uint32_t (&b)[NL], const uint32_t (&n)[NL]) {
    uint32_t t[NL];
    uint32_t c = add_n<NL>(t, a, b);
    if (c || ge<NL>(t, n)) sub_n<NL>(t, t, n);
#pragma unroll
    for (int i = 0; i < NL; i++) r[i] = t[i];
}

template <int NL>
__device__ __forceinline__ void submod(uint32_t (&r)[NL], const uint32_t (&a)[NL],
                                       const uint32_t (&b)[NL], const uint32_t (&n)[NL]) {
    uint32_t t[NL];
    if (sub_n<NL>(t, a, b)) add_n<NL>(t, t, n);
#pragma unroll
    for (int i = 0; i < NL; i++) r[i] = t[i];
}

template <int NL>
__device__ __forceinline__ void dblmod(uint32_t (&r)[NL], const uint32_t (&a)[NL],
                                       const uint32_t (&n)[NL]) {
    addmod<NL>(r, a, a, n);
}

// x / 2 mod n (n odd)
template <int NL>
__device__ __forceinline__ void halfmod(uint32_t (&x)[NL], const uint32_t (&n)[NL]) {
    uint32_t top = 0;
    if (x[0] & 1u) top = add_n<NL>(x, x, n);
#pragma unroll
    for (int i = 0; i < NL; i++) {
        uint32_t hi = (i + 1 < NL) ? x[i + 1] : top;
        x[i] = (x[i] >> 1) | (hi << 31);
    }
}

// CIOS Montgomery product r = a b R^{-1} mod n (a, b < n); the portable
// definition, specialised below for every limb count the prover uses
template <int NL>
__device__ __forceinline__ void montmul(uint32_t (&r)[NL], const uint32_t (&a)[NL],
                                        const uint32_t (&b)[NL], const uint32_t (&n)[NL],
                                        uint32_t ninv) {
    uint32_t t[NL + 2];
#pragma unroll
    for (int i = 0; i < NL + 2; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < NL; i++) {
        uint64_t carry = 0;
#pragma unroll
        for (int j = 0; j < NL; j++) {
            uint64_t p = (uint64_t)a[i] * b[j] + t[j] + carry;
            t[j] = (uint32_t)p;
            carry = p >> 32;
        }
        uint64_t s = (uint64_t)t[NL] + carry;
        t[NL] = (uint32_t)s;
        t[NL + 1] = (uint32_t)(s >> 32);
        uint32_t m = t[0] * ninv;
        carry = ((uint64_t)m * n[0] + t[0]) >> 32;
#pragma unroll
        for (int j = 1; j < NL; j++) {
            uint64_t p = (uint64_t)m * n[j] + t[j] + carry;
            t[j - 1] = (uint32_t)p;
            carry = p >> 32;
        }
        s = (uint64_t)t[NL] + carry;
        t[NL - 1] = (uint32_t)s;
        t[NL] = t[NL + 1] + (uint32_t)(s >> 32);
    }
    uint32_t res[NL];
#pragma unroll
    for (int i = 0; i < NL; i++) res[i] = t[i];
    if (t[NL] || ge<NL>(res, n)) sub_n<NL>(res, res, n);
#pragma unroll
    for (int i = 0; i < NL; i++) r[i] = res[i];
}

// The products actually used: CIOS with the carry chains written out in PTX
// (mad.lo/hi.cc, madc), one row of a_i * b and one of m * n per limb: 4 NL + 5
// instructions a row instead of the 64-bit sums above.  Generated for the
// limb counts 2..6 from one pattern: t (NL + 2 words) += x * v for x a word
// and v an NL-word vector, low halves then high halves, each a single carry
// chain.
template <>
__device__ __forceinline__ void montmul<2>(uint32_t (&r)[2], const uint32_t (&a)[2],
                                           const uint32_t (&b)[2], const uint32_t (&n)[2],
                                           uint32_t ninv) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const uint32_t ai = a[i];
        asm(
            "mad.lo.cc.u32 %0, %4, %5, %0;\n\t"
            "madc.lo.cc.u32 %1, %4, %6, %1;\n\t"
            "addc.cc.u32 %2, %2, 0;\n\t"
            "addc.u32 %3, %3, 0;\n\t"
            "mad.hi.cc.u32 %1, %4, %5, %1;\n\t"
            "madc.hi.cc.u32 %2, %4, %6, %2;\n\t"
            "addc.u32 %3, %3, 0;\n\t"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3)
            : "r"(ai), "r"(b[0]), "r"(b[1]));
        const uint32_t m = t0 * ninv;
        asm(
            "mad.lo.cc.u32 %0, %4, %5, %0;\n\t"
            "madc.lo.cc.u32 %1, %4, %6, %1;\n\t"
            "addc.cc.u32 %2, %2, 0;\n\t"
            "addc.u32 %3, %3, 0;\n\t"
            "mad.hi.cc.u32 %1, %4, %5, %1;\n\t"
            "madc.hi.cc.u32 %2, %4, %6, %2;\n\t"
            "addc.u32 %3, %3, 0;\n\t"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3)
            : "r"(m), "r"(n[0]), "r"(n[1]));
        t0 = t1; t1 = t2; t2 = t3; t3 = 0;
    }
    r[0] = t0; r[1] = t1;
    if (t2 || ge<2>(r, n)) sub_n<2>(r, r, n);
}

template <>
__device__ __forceinline__ void montmul<3>(uint32_t (&r)[3], const uint32_t (&a)[3],
                                           const uint32_t (&b)[3], const uint32_t (&n)[3],
                                           uint32_t ninv) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const uint32_t ai = a[i];
        asm(
            "mad.lo.cc.u32 %0, %5, %6, %0;\n\t"
            "madc.lo.cc.u32 %1, %5, %7, %1;\n\t"
            "madc.lo.cc.u32 %2, %5, %8, %2;\n\t"
            "addc.cc.u32 %3, %3, 0;\n\t"
            "addc.u32 %4, %4, 0;\n\t"
            "mad.hi.cc.u32 %1, %5, %6, %1;\n\t"
            "madc.hi.cc.u32 %2, %5, %7, %2;\n\t"
            "madc.hi.cc.u32 %3, %5, %8, %3;\n\t"
            "addc.u32 %4, %4, 0;\n\t"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4)
            : "r"(ai), "r"(b[0]), "r"(b[1]), "r"(b[2]));
        const uint32_t m = t0 * ninv;
        asm(
            "mad.lo.cc.u32 %0, %5, %6, %0;\n\t"
            "madc.lo.cc.u32 %1, %5, %7, %1;\n\t"
            "madc.lo.cc.u32 %2, %5, %8, %2;\n\t"
            "addc.cc.u32 %3, %3, 0;\n\t"
            "addc.u32 %4, %4, 0;\n\t"
            "mad.hi.cc.u32 %1, %5, %6, %1;\n\t"
            "madc.hi.cc.u32 %2, %5, %7, %2;\n\t"
            "madc.hi.cc.u32 %3, %5, %8, %3;\n\t"
            "addc.u32 %4, %4, 0;\n\t"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4)
            : "r"(m), "r"(n[0]), "r"(n[1]), "r"(n[2]));
        t0 = t1; t1 = t2; t2 = t3; t3 = t4; t4 = 0;
    }
    r[0] = t0; r[1] = t1; r[2] = t2;
    if (t3 || ge<3>(r, n)) sub_n<3>(r, r, n);
}

template <>
__device__ __forceinline__ void montmul<4>(uint32_t (&r)[4], const uint32_t (&a)[4],
                                           const uint32_t (&b)[4], const uint32_t (&n)[4],
                                           uint32_t ninv) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const uint32_t ai = a[i];
        asm(
            "mad.lo.cc.u32 %0, %6, %7, %0;\n\t"
            "madc.lo.cc.u32 %1, %6, %8, %1;\n\t"
            "madc.lo.cc.u32 %2, %6, %9, %2;\n\t"
            "madc.lo.cc.u32 %3, %6, %10, %3;\n\t"
            "addc.cc.u32 %4, %4, 0;\n\t"
            "addc.u32 %5, %5, 0;\n\t"
            "mad.hi.cc.u32 %1, %6, %7, %1;\n\t"
            "madc.hi.cc.u32 %2, %6, %8, %2;\n\t"
            "madc.hi.cc.u32 %3, %6, %9, %3;\n\t"
            "madc.hi.cc.u32 %4, %6, %10, %4;\n\t"
            "addc.u32 %5, %5, 0;\n\t"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5)
            : "r"(ai), "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]));
        const uint32_t m = t0 * ninv;
        asm(
            "mad.lo.cc.u32 %0, %6, %7, %0;\n\t"
            "madc.lo.cc.u32 %1, %6, %8, %1;\n\t"
            "madc.lo.cc.u32 %2, %6, %9, %2;\n\t"
            "madc.lo.cc.u32 %3, %6, %10, %3;\n\t"
            "addc.cc.u32 %4, %4, 0;\n\t"
            "addc.u32 %5, %5, 0;\n\t"
            "mad.hi.cc.u32 %1, %6, %7, %1;\n\t"
            "madc.hi.cc.u32 %2, %6, %8, %2;\n\t"
            "madc.hi.cc.u32 %3, %6, %9, %3;\n\t"
            "madc.hi.cc.u32 %4, %6, %10, %4;\n\t"
            "addc.u32 %5, %5, 0;\n\t"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5)
            : "r"(m), "r"(n[0]), "r"(n[1]), "r"(n[2]), "r"(n[3]));
        t0 = t1; t1 = t2; t2 = t3; t3 = t4; t4 = t5; t5 = 0;
    }
    r[0] = t0; r[1] = t1; r[2] = t2; r[3] = t3;
    if (t4 || ge<4>(r, n)) sub_n<4>(r, r, n);
}

template <>
__device__ __forceinline__ void montmul<5>(uint32_t (&r)[5], const uint32_t (&a)[5],
                                           const uint32_t (&b)[5], const uint32_t (&n)[5],
                                           uint32_t ninv) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0;
#pragma unroll
    for (int i = 0; i < 5; i++) {
        const uint32_t ai = a[i];
        asm(
            "mad.lo.cc.u32 %0, %7, %8, %0;\n\t"
            "madc.lo.cc.u32 %1, %7, %9, %1;\n\t"
            "madc.lo.cc.u32 %2, %7, %10, %2;\n\t"
            "madc.lo.cc.u32 %3, %7, %11, %3;\n\t"
            "madc.lo.cc.u32 %4, %7, %12, %4;\n\t"
            "addc.cc.u32 %5, %5, 0;\n\t"
            "addc.u32 %6, %6, 0;\n\t"
            "mad.hi.cc.u32 %1, %7, %8, %1;\n\t"
            "madc.hi.cc.u32 %2, %7, %9, %2;\n\t"
            "madc.hi.cc.u32 %3, %7, %10, %3;\n\t"
            "madc.hi.cc.u32 %4, %7, %11, %4;\n\t"
            "madc.hi.cc.u32 %5, %7, %12, %5;\n\t"
            "addc.u32 %6, %6, 0;\n\t"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6)
            : "r"(ai), "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]));
        const uint32_t m = t0 * ninv;
        asm(
            "mad.lo.cc.u32 %0, %7, %8, %0;\n\t"
            "madc.lo.cc.u32 %1, %7, %9, %1;\n\t"
            "madc.lo.cc.u32 %2, %7, %10, %2;\n\t"
            "madc.lo.cc.u32 %3, %7, %11, %3;\n\t"
            "madc.lo.cc.u32 %4, %7, %12, %4;\n\t"
            "addc.cc.u32 %5, %5, 0;\n\t"
            "addc.u32 %6, %6, 0;\n\t"
            "mad.hi.cc.u32 %1, %7, %8, %1;\n\t"
            "madc.hi.cc.u32 %2, %7, %9, %2;\n\t"
            "madc.hi.cc.u32 %3, %7, %10, %3;\n\t"
            "madc.hi.cc.u32 %4, %7, %11, %4;\n\t"
            "madc.hi.cc.u32 %5, %7, %12, %5;\n\t"
            "addc.u32 %6, %6, 0;\n\t"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6)
            : "r"(m), "r"(n[0]), "r"(n[1]), "r"(n[2]), "r"(n[3]), "r"(n[4]));
        t0 = t1; t1 = t2; t2 = t3; t3 = t4; t4 = t5; t5 = t6; t6 = 0;
    }
    r[0] = t0; r[1] = t1; r[2] = t2; r[3] = t3; r[4] = t4;
    if (t5 || ge<5>(r, n)) sub_n<5>(r, r, n);
}

template <>
__device__ __forceinline__ void montmul<6>(uint32_t (&r)[6], const uint32_t (&a)[6],
                                           const uint32_t (&b)[6], const uint32_t (&n)[6],
                                           uint32_t ninv) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        const uint32_t ai = a[i];
        asm(
            "mad.lo.cc.u32 %0, %8, %9, %0;\n\t"
            "madc.lo.cc.u32 %1, %8, %10, %1;\n\t"
            "madc.lo.cc.u32 %2, %8, %11, %2;\n\t"
            "madc.lo.cc.u32 %3, %8, %12, %3;\n\t"
            "madc.lo.cc.u32 %4, %8, %13, %4;\n\t"
            "madc.lo.cc.u32 %5, %8, %14, %5;\n\t"
            "addc.cc.u32 %6, %6, 0;\n\t"
            "addc.u32 %7, %7, 0;\n\t"
            "mad.hi.cc.u32 %1, %8, %9, %1;\n\t"
            "madc.hi.cc.u32 %2, %8, %10, %2;\n\t"
            "madc.hi.cc.u32 %3, %8, %11, %3;\n\t"
            "madc.hi.cc.u32 %4, %8, %12, %4;\n\t"
            "madc.hi.cc.u32 %5, %8, %13, %5;\n\t"
            "madc.hi.cc.u32 %6, %8, %14, %6;\n\t"
            "addc.u32 %7, %7, 0;\n\t"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7)
            : "r"(ai), "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]));
        const uint32_t m = t0 * ninv;
        asm(
            "mad.lo.cc.u32 %0, %8, %9, %0;\n\t"
            "madc.lo.cc.u32 %1, %8, %10, %1;\n\t"
            "madc.lo.cc.u32 %2, %8, %11, %2;\n\t"
            "madc.lo.cc.u32 %3, %8, %12, %3;\n\t"
            "madc.lo.cc.u32 %4, %8, %13, %4;\n\t"
            "madc.lo.cc.u32 %5, %8, %14, %5;\n\t"
            "addc.cc.u32 %6, %6, 0;\n\t"
            "addc.u32 %7, %7, 0;\n\t"
            "mad.hi.cc.u32 %1, %8, %9, %1;\n\t"
            "madc.hi.cc.u32 %2, %8, %10, %2;\n\t"
            "madc.hi.cc.u32 %3, %8, %11, %3;\n\t"
            "madc.hi.cc.u32 %4, %8, %12, %4;\n\t"
            "madc.hi.cc.u32 %5, %8, %13, %5;\n\t"
            "madc.hi.cc.u32 %6, %8, %14, %6;\n\t"
            "addc.u32 %7, %7, 0;\n\t"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7)
            : "r"(m), "r"(n[0]), "r"(n[1]), "r"(n[2]), "r"(n[3]), "r"(n[4]), "r"(n[5]));
        t0 = t1; t1 = t2; t2 = t3; t3 = t4; t4 = t5; t5 = t6; t6 = t7; t7 = 0;
    }
    r[0] = t0; r[1] = t1; r[2] = t2; r[3] = t3; r[4] = t4; r[5] = t5;
    if (t6 || ge<6>(r, n)) sub_n<6>(r, r, n);
}

// Montgomery square r = a^2 R^{-1} mod n (a < n): the full square first (each
// cross product a_i a_j, i < j, once, the sum doubled, the squares a_i^2 added
// on the diagonal), then the NL reduction rows.  NL (NL - 1)/2 + NL word
// products for the square against NL^2 for a product.  A reduction row adds
// m n at word i as one carry chain over the low halves and one over the high
// halves; the carry out of word i + NL is kept in a register and added by the
// next row (at its own word i + NL), so no row walks the carry to the top.
// Specialised for 3 and 4 limbs (the members of 65..128 bits); the other
// limb counts use the product.
template <int NL>
__device__ __forceinline__ void montsqr(uint32_t (&r)[NL], const uint32_t (&a)[NL],
                                        const uint32_t (&n)[NL], uint32_t ninv) {
    montmul<NL>(r, a, a, n, ninv);
}

// one reduction row of montsqr<3>: t_i..t_i+3 += m n, p into t_i+3, carry out in q
#define CCS_SQR_ROW3(T0, T1, T2, T3)                                            \
    {                                                                           \
        const uint32_t m = T0 * ninv;                                           \
        uint32_t q = 0;                                                         \
        asm("mad.lo.cc.u32 %0, %6, %7, %0;\n\t"                                 \
            "madc.lo.cc.u32 %1, %6, %8, %1;\n\t"                                \
            "madc.lo.cc.u32 %2, %6, %9, %2;\n\t"                                \
            "addc.cc.u32 %3, %3, %5;\n\t"                                       \
            "addc.u32 %4, %4, 0;\n\t"                                           \
            "mad.hi.cc.u32 %1, %6, %7, %1;\n\t"                                 \
            "madc.hi.cc.u32 %2, %6, %8, %2;\n\t"                                \
            "madc.hi.cc.u32 %3, %6, %9, %3;\n\t"                                \
            "addc.u32 %4, %4, 0;\n\t"                                           \
            : "+r"(T0), "+r"(T1), "+r"(T2), "+r"(T3), "+r"(q)                   \
            : "r"(p), "r"(m), "r"(n[0]), "r"(n[1]), "r"(n[2]));                 \
        p = q;                                                                  \
    }

template <>
__device__ __forceinline__ void montsqr<3>(uint32_t (&r)[3], const uint32_t (&a)[3],
                                           const uint32_t (&n)[3], uint32_t ninv) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0;
    asm("mul.lo.u32 %1, %6, %7;\n\t"              // cross products
        "mul.lo.u32 %2, %6, %8;\n\t"
        "mad.hi.cc.u32 %2, %6, %7, %2;\n\t"
        "madc.hi.u32 %3, %6, %8, %3;\n\t"
        "mad.lo.cc.u32 %3, %7, %8, %3;\n\t"
        "madc.hi.u32 %4, %7, %8, %4;\n\t"
        "add.cc.u32 %1, %1, %1;\n\t"              // doubled
        "addc.cc.u32 %2, %2, %2;\n\t"
        "addc.cc.u32 %3, %3, %3;\n\t"
        "addc.cc.u32 %4, %4, %4;\n\t"
        "addc.u32 %5, %5, 0;\n\t"
        "mul.lo.u32 %0, %6, %6;\n\t"              // the diagonal
        "mad.hi.cc.u32 %1, %6, %6, %1;\n\t"
        "madc.lo.cc.u32 %2, %7, %7, %2;\n\t"
        "madc.hi.cc.u32 %3, %7, %7, %3;\n\t"
        "madc.lo.cc.u32 %4, %8, %8, %4;\n\t"
        "madc.hi.u32 %5, %8, %8, %5;\n\t"
        : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]));
    uint32_t p = 0;
    CCS_SQR_ROW3(t0, t1, t2, t3)
    CCS_SQR_ROW3(t1, t2, t3, t4)
    CCS_SQR_ROW3(t2, t3, t4, t5)
    r[0] = t3; r[1] = t4; r[2] = t5;
    if (p || ge<3>(r, n)) sub_n<3>(r, r, n);
}
#undef CCS_SQR_ROW3

// one reduction row of montsqr<4>: t_i..t_i+4 += m n, p into t_i+4, carry out in q
#define CCS_SQR_ROW4(T0, T1, T2, T3, T4)                                        \
    {                                                                           \
        const uint32_t m = T0 * ninv;                                           \
        uint32_t q = 0;                                                         \
        asm("mad.lo.cc.u32 %0, %7, %8, %0;\n\t"                                 \
            "madc.lo.cc.u32 %1, %7, %9, %1;\n\t"                                \
            "madc.lo.cc.u32 %2, %7, %10, %2;\n\t"                               \
            "madc.lo.cc.u32 %3, %7, %11, %3;\n\t"                               \
            "addc.cc.u32 %4, %4, %6;\n\t"                                       \
            "addc.u32 %5, %5, 0;\n\t"                                           \
            "mad.hi.cc.u32 %1, %7, %8, %1;\n\t"                                 \
            "madc.hi.cc.u32 %2, %7, %9, %2;\n\t"                                \
            "madc.hi.cc.u32 %3, %7, %10, %3;\n\t"                               \
            "madc.hi.cc.u32 %4, %7, %11, %4;\n\t"                               \
            "addc.u32 %5, %5, 0;\n\t"                                           \
            : "+r"(T0), "+r"(T1), "+r"(T2), "+r"(T3), "+r"(T4), "+r"(q)         \
            : "r"(p), "r"(m), "r"(n[0]), "r"(n[1]), "r"(n[2]), "r"(n[3]));       \
        p = q;                                                                  \
    }

template <>
__device__ __forceinline__ void montsqr<4>(uint32_t (&r)[4], const uint32_t (&a)[4],
                                           const uint32_t (&n)[4], uint32_t ninv) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0;
    asm("mul.lo.u32 %1, %8, %9;\n\t"              // cross products
        "mul.lo.u32 %2, %8, %10;\n\t"
        "mul.lo.u32 %3, %8, %11;\n\t"
        "mad.hi.cc.u32 %2, %8, %9, %2;\n\t"
        "madc.hi.cc.u32 %3, %8, %10, %3;\n\t"
        "madc.hi.u32 %4, %8, %11, %4;\n\t"
        "mad.lo.cc.u32 %3, %9, %10, %3;\n\t"
        "madc.lo.cc.u32 %4, %9, %11, %4;\n\t"
        "addc.u32 %5, %5, 0;\n\t"
        "mad.hi.cc.u32 %4, %9, %10, %4;\n\t"
        "madc.hi.u32 %5, %9, %11, %5;\n\t"
        "mad.lo.cc.u32 %5, %10, %11, %5;\n\t"
        "madc.hi.u32 %6, %10, %11, %6;\n\t"
        "add.cc.u32 %1, %1, %1;\n\t"              // doubled
        "addc.cc.u32 %2, %2, %2;\n\t"
        "addc.cc.u32 %3, %3, %3;\n\t"
        "addc.cc.u32 %4, %4, %4;\n\t"
        "addc.cc.u32 %5, %5, %5;\n\t"
        "addc.cc.u32 %6, %6, %6;\n\t"
        "addc.u32 %7, %7, 0;\n\t"
        "mul.lo.u32 %0, %8, %8;\n\t"              // the diagonal
        "mad.hi.cc.u32 %1, %8, %8, %1;\n\t"
        "madc.lo.cc.u32 %2, %9, %9, %2;\n\t"
        "madc.hi.cc.u32 %3, %9, %9, %3;\n\t"
        "madc.lo.cc.u32 %4, %10, %10, %4;\n\t"
        "madc.hi.cc.u32 %5, %10, %10, %5;\n\t"
        "madc.lo.cc.u32 %6, %11, %11, %6;\n\t"
        "madc.hi.u32 %7, %11, %11, %7;\n\t"
        : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]));
    uint32_t p = 0;
    CCS_SQR_ROW4(t0, t1, t2, t3, t4)
    CCS_SQR_ROW4(t1, t2, t3, t4, t5)
    CCS_SQR_ROW4(t2, t3, t4, t5, t6)
    CCS_SQR_ROW4(t3, t4, t5, t6, t7)
    r[0] = t4; r[1] = t5; r[2] = t6; r[3] = t7;
    if (p || ge<4>(r, n)) sub_n<4>(r, r, n);
}
#undef CCS_SQR_ROW4


template <int NL>
__device__ __forceinline__ void mont_setup(Mont<NL>& M, const Big& nb, int nbits) {
#pragma unroll
    for (int i = 0; i < NL; i++) M.n[i] = nb.w[i];
    uint32_t n0 = M.n[0];
    uint32_t inv = n0;                       // 3 correct bits
#pragma unroll
    for (int k = 0; k < 4; k++) inv *= 2u - n0 * inv;
    M.ninv = 0u - inv;
    // R mod n: start at 2^nbits - n (< n), double 32 NL - nbits times
    uint32_t x[NL];
    uint32_t zero[NL];
#pragma unroll
    for (int i = 0; i < NL; i++) zero[i] = 0;
    sub_n<NL>(x, zero, M.n);                 // 2^(32NL) - n (as NL limbs, wraps)
    // 2^nbits - n = (2^(32NL) - n) mod 2^nbits
    if (nbits < 32 * NL) {
        int wi = nbits >> 5, bi = nbits & 31;
#pragma unroll
        for (int i = 0; i < NL; i++) {
            if (i > wi) x[i] = 0;
            else if (i == wi) x[i] &= (bi ? ((1u << bi) - 1u) : 0u);
        }
        for (int k = nbits; k < 32 * NL; k++) dblmod<NL>(x, x, M.n);
    }
#pragma unroll
    for (int i = 0; i < NL; i++) M.one[i] = x[i];
    sub_n<NL>(M.mone, M.n, M.one);
}

// a R mod n for a small a (double-and-add from the top bit of a)
template <int NL>
__device__ __forceinline__ void to_mont_small(uint32_t (&r)[NL], uint32_t a, const Mont<NL>& M) {
    uint32_t acc[NL];
#pragma unroll
    for (int i = 0; i < NL; i++) acc[i] = 0;
    for (int b = 31 - __clz(a); b >= 0; b--) {
        dblmod<NL>(acc, acc, M.n);
        if ((a >> b) & 1u) addmod<NL>(acc, acc, M.one, M.n);
    }
#pragma unroll
    for (int i = 0; i < NL; i++) r[i] = acc[i];
}

// strong probable-prime test to base a (n odd, n > a).  SYNC: every lane of
// the warp runs the test (the walk kernels give idle lanes a copy of a live
// lane's number) and the lanes are reconverged after the set-up loops, so the
// exponent loop runs once for the whole warp.
template <int NL, bool SYNC = false>
__device__ bool strong_prp(Mont<NL>& M, const Big& nb, uint32_t a) {
    // n - 1 = d 2^s
    Big d = nb;
    d.w[0] -= 1;                              // n odd: no borrow
    int s = 0;
    {
        int lz = 0;
        for (int i = 0; i < kMaxLimbs; i++) {
            if (d.w[i] == 0) { lz += 32; continue; }
            lz += __ffs(d.w[i]) - 1;
            break;
        }
        s = lz;
        // d >>= s: whole limbs first, then bits (static limb indices)
        const int ws = s >> 5, bs = s & 31;
        for (int k = 0; k < ws; k++) {
#pragma unroll
            for (int i = 0; i < kMaxLimbs; i++) d.w[i] = (i + 1 < kMaxLimbs) ? d.w[i + 1] : 0u;
        }
        if (bs) {
#pragma unroll
            for (int i = 0; i < kMaxLimbs; i++) {
                const uint32_t hi = (i + 1 < kMaxLimbs) ? d.w[i + 1] : 0u;
                d.w[i] = (d.w[i] >> bs) | (hi << (32 - bs));
            }
        }
    }
    if (SYNC) __syncwarp();
    uint32_t am[NL], x[NL];
    to_mont_small<NL>(am, a, M);
    if (SYNC) __syncwarp();
#pragma unroll
    for (int i = 0; i < NL; i++) x[i] = am[i];
    // left-to-right over the bits of d below its top bit; the limb loop is
    // unrolled so d stays in registers
    const int top = big_bits(d) - 1;
#pragma unroll
    for (int wi = kMaxLimbs - 1; wi >= 0; wi--) {
        if (32 * wi > top - 1) continue;
        const uint32_t word = d.w[wi];
        const int hb = (32 * wi + 31 > top - 1) ? (top - 1 - 32 * wi) : 31;
        for (int b = hb; b >= 0; b--) {
            montsqr<NL>(x, x, M.n, M.ninv);
            M.count++;
            M.sq++;
            if ((word >> b) & 1u) {
                if (a == 2) dblmod<NL>(x, x, M.n);
                else { montmul<NL>(x, x, am, M.n, M.ninv); M.count++; }
            }
        }
    }
    if (SYNC) __syncwarp();
    if (eq<NL>(x, M.one) || eq<NL>(x, M.mone)) return true;
    for (int r = 1; r < s; r++) {
        montsqr<NL>(x, x, M.n, M.ninv);
        M.count++;
        M.sq++;
        if (eq<NL>(x, M.mone)) return true;
        if (eq<NL>(x, M.one)) return false;
    }
    return false;
}

// Jacobi symbol (D / n) for small signed D, n odd
__device__ int jacobi_small(int D, const Big& nb) {
    int sign = 1;
    uint32_t a;
    if (D < 0) {
        a = (uint32_t)(-D);
        if ((nb.w[0] & 3u) == 3u) sign = -sign;
    } else {
        a = (uint32_t)D;
    }
    while (a && (a & 1u) == 0) {
        a >>= 1;
        uint32_t r8 = nb.w[0] & 7u;
        if (r8 == 3u || r8 == 5u) sign = -sign;
    }
    if (a == 0) return 0;
    if (a == 1) return sign;
    if ((a & 3u) == 3u && (nb.w[0] & 3u) == 3u) sign = -sign;
    uint32_t x = big_mod_small(nb, a), y = a;
    while (x) {
        while ((x & 1u) == 0) {
            x >>= 1;
            if ((y & 7u) == 3u || (y & 7u) == 5u) sign = -sign;
        }
        uint32_t t = x; x = y; y = t;
        if ((x & 3u) == 3u && (y & 3u) == 3u) sign = -sign;
        x %= y;
    }
    return y == 1 ? sign : 0;
}

// strong Lucas probable-prime test, Selfridge method A (P = 1, Q = (1 - D)/4).
// SYNC as in strong_prp: a lane whose D search decides the verdict still runs
// the ladder (on its last D) with the warp and returns its decided verdict.
// Q2: the caller has found the search's answer to be D = -7 ((5/n) = 1,
// (-7/n) = -1), so Q = 2 and Q^(k+1) = 2 Q^k is a modular doubling instead of
// a product: three products per bit instead of four, the same verdict.  Every
// member of a first-kind chain on a lattice with 5 in its CRT primes is -1 mod
// 5, so (5/n) = 1 and D = -7 is the parameter of about half of them.
template <int NL, bool SYNC = false, bool Q2 = false>
__device__ bool strong_lucas(Mont<NL>& M, const Big& nb) {
    int D = Q2 ? -7 : 5;
    int tries = 0;
    bool decided = false, dres = false;
    for (; !Q2;) {
        int j = jacobi_small(D, nb);
        if (j == -1) break;
        if (j == 0) {
            uint32_t ad = (uint32_t)(D < 0 ? -D : D);
            dres = big_lt_u32(nb, ad + 1) && nb.w[0] == ad;   // n == |D|
            decided = true;
            break;
        }
        D = D > 0 ? -(D + 2) : -(D - 2);
        // no D with (D/n) = -1 among the first 64 candidates: n is (almost
        // surely) a perfect square; squares are composite
        if (++tries > 64) { decided = true; dres = false; break; }
    }
    if (!SYNC && decided) return dres;
    if (SYNC) __syncwarp();
    const int Qs = (1 - D) / 4;
    uint32_t Qm[NL];
    if (Qs >= 0) to_mont_small<NL>(Qm, (uint32_t)Qs, M);
    else { uint32_t t[NL]; to_mont_small<NL>(t, (uint32_t)(-Qs), M); uint32_t z[NL];
#pragma unroll
        for (int i = 0; i < NL; i++) z[i] = 0;
        submod<NL>(Qm, z, t, M.n); }
    if (SYNC) __syncwarp();
    // n + 1 = d 2^s
    Big d = nb;
    {
        uint32_t c = 1;
#pragma unroll
        for (int i = 0; i < kMaxLimbs; i++) {
            uint64_t s2 = (uint64_t)d.w[i] + c;
            d.w[i] = (uint32_t)s2;
            c = (uint32_t)(s2 >> 32);
        }
    }
    int s = 0;
    while ((d.w[0] & 1u) == 0) {
#pragma unroll
        for (int i = 0; i < kMaxLimbs; i++) {
            uint32_t hi = (i + 1 < kMaxLimbs) ? d.w[i + 1] : 0;
            d.w[i] = (d.w[i] >> 1) | (hi << 31);
        }
        s++;
    }
    // V ladder (P = 1): keep (V_k, V_{k+1}, Q^k) from k = 1 over the bits of d,
    //   bit 0: V_2k   = V_k^2 - 2 Q^k,          V_2k+1 = V_k V_k+1 - Q^k,  Q^2k
    //   bit 1: V_2k+1 = V_k V_k+1 - Q^k,        V_2k+2 = V_k+1^2 - 2 Q^(k+1),  Q^(2k+1)
    // done branch-free (the same four products for either bit value, so a
    // warp never runs both); then D U_d = 2 V_(d+1) - V_d with D a unit mod n
    // ((D/n) = -1), so U_d = 0 exactly when 2 V_(d+1) = V_d.
    uint32_t V0[NL], V1[NL], Qk[NL], t1[NL], t2[NL];
#pragma unroll
    for (int i = 0; i < NL; i++) { V0[i] = M.one[i]; Qk[i] = Qm[i]; }
    dblmod<NL>(t1, Qm, M.n);
    submod<NL>(V1, M.one, t1, M.n);                 // V_2 = P^2 - 2Q
    const int top = big_bits(d) - 1;
#pragma unroll
    for (int wi = kMaxLimbs - 1; wi >= 0; wi--) {
      if (32 * wi > top - 1) continue;
      const uint32_t word = d.w[wi];
      const int hb = (32 * wi + 31 > top - 1) ? (top - 1 - 32 * wi) : 31;
      for (int b = hb; b >= 0; b--) {
        const bool bit = (word >> b) & 1u;
        uint32_t X[NL], Y[NL], S[NL];
        montmul<NL>(t1, V0, V1, M.n, M.ninv);
        submod<NL>(t1, t1, Qk, M.n);                // V_2k+1
        if (Q2) dblmod<NL>(t2, Qk, M.n);            // Q^(k+1)
        else montmul<NL>(t2, Qk, Qm, M.n, M.ninv);
#pragma unroll
        for (int i = 0; i < NL; i++) { X[i] = bit ? V1[i] : V0[i]; Y[i] = bit ? t2[i] : Qk[i]; }
        montsqr<NL>(S, X, M.n, M.ninv);
        dblmod<NL>(X, Y, M.n);
        submod<NL>(S, S, X, M.n);                   // V_2k (bit 0) or V_2k+2 (bit 1)
        if (Q2) {                                   // Q^2k, or 2 Q^2k = Q^(2k+1)
            montsqr<NL>(Qk, Qk, M.n, M.ninv);
            dblmod<NL>(X, Qk, M.n);
#pragma unroll
            for (int i = 0; i < NL; i++) Qk[i] = bit ? X[i] : Qk[i];
        } else {
            montmul<NL>(Qk, Qk, Y, M.n, M.ninv);    // Q^2k or Q^(2k+1)
        }
#pragma unroll
        for (int i = 0; i < NL; i++) { V0[i] = bit ? t1[i] : S[i]; V1[i] = bit ? S[i] : t1[i]; }
        M.count += Q2 ? 3 : 4;
        M.sq += Q2 ? 2 : 1;
      }
    }
    // V0 = V_d, V1 = V_(d+1), Qk = Q^d
    if (SYNC) __syncwarp();
    bool res = false;
    dblmod<NL>(t1, V1, M.n);
    if (eq<NL>(t1, V0) || is_zero<NL>(V0)) {
        res = true;
    } else {
        for (int r = 1; r < s; r++) {
            montsqr<NL>(t1, V0, M.n, M.ninv);
            dblmod<NL>(t2, Qk, M.n);
            submod<NL>(V0, t1, t2, M.n);
            if (is_zero<NL>(V0)) { res = true; break; }
            montsqr<NL>(Qk, Qk, M.n, M.ninv);
            M.count += 2;
            M.sq += 2;
        }
    }
    return decided ? dres : res;
}

// Fermat test to base 2: 2^(n-1) == 1 (mod n), n odd > 2 (the link test of
// the reference CPU engine, is_prime_pocklington_native, v33:1290-1302)
template <int NL, bool SYNC = false>
__device__ bool fermat2(Mont<NL>& M, const Big& nb) {
    Big e = nb;
    e.w[0] -= 1;                              // n odd: no borrow
    if (SYNC) __syncwarp();
    uint32_t x[NL];
#pragma unroll
    for (int i = 0; i < NL; i++) x[i] = M.one[i];
    dblmod<NL>(x, x, M.n);                    // 2 R mod n: the top bit of n - 1
    const int top = big_bits(e) - 1;
#pragma unroll
    for (int wi = kMaxLimbs - 1; wi >= 0; wi--) {
        if (32 * wi > top - 1) continue;
        const uint32_t word = e.w[wi];
        const int hb = (32 * wi + 31 > top - 1) ? (top - 1 - 32 * wi) : 31;
        for (int b = hb; b >= 0; b--) {
            montsqr<NL>(x, x, M.n, M.ninv);
            M.count++;
            M.sq++;
            if ((word >> b) & 1u) dblmod<NL>(x, x, M.n);
        }
    }
    return eq<NL>(x, M.one);
}

template <int NL>
__device__ bool prp_suite(const Big& nb, int nbits, uint32_t pred, const ProveConst& pc,
                          uint32_t& mm) {
    Mont<NL> M;
    mont_setup<NL>(M, nb, nbits);
    M.count = 0;
    M.sq = 0;
    bool r = true;
    if (pred == kPredBPSW) {
        r = strong_prp<NL>(M, nb, 2) && strong_lucas<NL>(M, nb);
    } else if (pred == kPredMR235) {
        r = strong_prp<NL>(M, nb, 2) && strong_prp<NL>(M, nb, 3) && strong_prp<NL>(M, nb, 5);
    } else if (pred == kPredFermat2) {
        r = fermat2<NL>(M, nb);
    } else {
        for (uint32_t i = 0; i < pc.n_wit && r; i++) r = strong_prp<NL>(M, nb, pc.wit[i]);
    }
    mm += M.count;
    return r;
}

__constant__ uint32_t c_small_primes[27] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47,
                                            53, 59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 1093, 3511};
// the trial primes in five groups whose products fit 32 bits: one multi-limb
// reduction per group, then 32-bit reductions per prime (groups 0..2 are the
// 19 primes 3..71 of the MR predicate)
__constant__ uint32_t c_group_prod[5] = {3234846615u, 95041567u, 907383479u, 4132280413u, 387589823u};
__constant__ uint8_t c_group_end[5] = {9, 14, 19, 24, 27};
#define CCS_M(p) (0xFFFFFFFFu / (p))
__constant__ uint32_t c_small_magic[27] = {
    CCS_M(3), CCS_M(5), CCS_M(7), CCS_M(11), CCS_M(13), CCS_M(17), CCS_M(19), CCS_M(23), CCS_M(29),
    CCS_M(31), CCS_M(37), CCS_M(41), CCS_M(43), CCS_M(47), CCS_M(53), CCS_M(59), CCS_M(61), CCS_M(67),
    CCS_M(71), CCS_M(73), CCS_M(79), CCS_M(83), CCS_M(89), CCS_M(97), CCS_M(101), CCS_M(1093),
    CCS_M(3511)};
#undef CCS_M

// Trial stage of the primality predicate (every branch of v13 gpu_is_prime,
// v13:1428-1452, and of the BPSW screen): returns 0 = composite, 1 = prime
// without a probable-prime test, or the Montgomery limb count (2..6) of the
// test that decides.
__device__ int prime_screen(const Big& nb, uint32_t pred, int& nbits_out) {
    const int nbits = big_bits(nb);
    nbits_out = nbits;
    if (nbits <= 1) return 0;
    const uint32_t lo = nb.w[0];
    if (pred == kPredMR235 || pred == kPredFermat2) {
        // the reference's native tests: 2, 3, 5 directly, even numbers out,
        // no trial division (its callers divide before, v33:1290-1339)
        if (nbits <= 3) return (lo == 2 || lo == 3 || lo == 5) ? 1 : (lo == 7 ? 2 : 0);
        if ((lo & 1u) == 0) return 0;
        const int nl = (nbits + 31) >> 5;
        return nl <= 2 ? 2 : nl;
    }
    const bool mr = pred == kPredMR;
    const int ntrial = mr ? 19 : 27;
    if (mr) {
        if (nbits <= 64 && nb.w[1] == 0) {
            if (lo < 2) return 0;
            if (lo == 2 || lo == 3) return 1;
            if ((lo & 1u) == 0) return 0;
            if (lo < 9) return 1;
        }
        if ((lo & 1u) == 0) return 0;
    } else {
        if (nbits <= 32 && lo == 2) return 1;
        if ((lo & 1u) == 0) return 0;
    }
    if (nbits <= 32) {
        // small n: the prime list in order (n may equal one of them)
        for (int i = 0; i < ntrial; i++) {
            const uint32_t p = c_small_primes[i];
            if (mr) {
                if (lo % p == 0) return lo == p ? 1 : 0;
            } else {
                if (lo == p) return 1;
                if (lo % p == 0) return 0;
            }
        }
        if (!mr && lo < 103u * 103u) return 1;
    } else {
        const int ngroups = mr ? 3 : 5;
        int i = 0;
        for (int g = 0; g < ngroups; g++) {
            const uint32_t G = c_group_prod[g];
            const uint32_t rg = big_mod_u32(nb, G, ~0ull / G);
            for (; i < c_group_end[g]; i++)
                if (mod_m32(rg, c_small_primes[i], c_small_magic[i]) == 0) return 0;
        }
    }
    const int nl = (nbits + 31) >> 5;
    return nl <= 2 ? 2 : nl;
}

// one primality test for any n < 2^192; mm counts the Montgomery products
// spent
__device__ bool is_prime_pred(const Big& nb, uint32_t pred, const ProveConst& pc, uint32_t& mm) {
    int nbits;
    const int v = prime_screen(nb, pred, nbits);
    if (v < 2) return v == 1;
    switch (v) {
        case 2: return prp_suite<2>(nb, nbits, pred, pc, mm);
        case 3: return prp_suite<3>(nb, nbits, pred, pc, mm);
        case 4: return prp_suite<4>(nb, nbits, pred, pc, mm);
        case 5: return prp_suite<5>(nb, nbits, pred, pc, mm);
        default: return prp_suite<6>(nb, nbits, pred, pc, mm);
    }
}

// the profile's test for a number that is neither n's root test nor a
// forward link (the reference CPU engine tests those with is_prime_fast:
// Baillie-PSW)
__device__ __forceinline__ uint32_t other_pred(const ProveConst& pc) {
    return pc.primality == CCS_PRIME_V33 ? (uint32_t)kPredBPSW : pc.primality;
}

__device__ bool is_prime_dev(const Big& nb, const ProveConst& pc, uint32_t& mm) {
    return is_prime_pred(nb, other_pred(pc), pc, mm);
}

__device__ bool screen_composite(const Big& nb);

// forward walk p -> 2p + 1 (second kind 2p - 1) while prime, counting p
// (v13:1519-1528, 1873-1881; v13b:1527-1535, 1878-1886).  With screen, a
// link first ends the walk when it has more than cap_bits bits or a zero
// residue mod a screen prime (v33:1540-1562).
__device__ int walk_forward(Big cur, const ProveConst& pc, uint32_t link_pred, bool screen,
                            uint32_t cap_bits, uint32_t& mm) {
    int len = 1;
    while (len < kMaxChain) {
        if (big_bits(cur) >= 32 * kMaxLimbs) break;   // next member would exceed 192 bits
        Big nx = cur;
        big_next(nx, pc.kind);
        if (screen) {
            if (cap_bits && big_bits(nx) > (int)cap_bits) break;
            if (screen_composite(nx)) break;
        }
        if (!is_prime_pred(nx, link_pred, pc, mm)) break;
        len++;
        cur = nx;
    }
    return len;
}

// staged prove: per-survivor flag set by the seed kernel (cleared to the
// record flags when n tests prime)
constexpr uint32_t kFlagCertificate = 1u << 8;

__constant__ uint32_t c_screen[132] = {
    67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113, 127, 131, 137, 139, 149, 151,
    157, 163, 167, 173, 179, 181, 191, 193, 197, 199, 211, 223, 227, 229, 233, 239, 241,
    251, 257, 263, 269, 271, 277, 281, 283, 293, 307, 311, 313, 317, 331, 337, 347, 349,
    353, 359, 367, 373, 379, 383, 389, 397, 401, 409, 419, 421, 431, 433, 439, 443, 449,
    457, 461, 463, 467, 479, 487, 491, 499, 503, 509, 521, 523, 541, 547, 557, 563, 569,
    571, 577, 587, 593, 599, 601, 607, 613, 617, 619, 631, 641, 643, 647, 653, 659, 661,
    673, 677, 683, 691, 701, 709, 719, 727, 733, 739, 743, 751, 757, 761, 769, 773, 787,
    797, 809, 811, 821, 823, 827, 829, 839, 853, 857, 859, 863};

// a zero residue mod any of the 132 screen primes 67..863 (the reference CPU
// engine's link screen counts a link equal to a screen prime as composite
// too, v33:1551-1562)
__device__ bool screen_composite(const Big& nb) {
    for (int t = 0; t < 132; t++)
        if (big_mod_small(nb, c_screen[t]) == 0) return true;
    return false;
}

// The tests of one range under the profile's predicate: the root test of n,
// and the forward-link rules (v33: native path up to bits + target = 127,
// wide path above, v33:3095-3101)
struct RangePreds {
    uint32_t root, link, cap;
    bool screen;
};
__device__ __forceinline__ RangePreds range_preds(const ProveConst& pc, uint32_t bits, uint32_t target) {
    RangePreds r;
    if (pc.primality == CCS_PRIME_V33) {
        const bool wide = bits + target > 127;
        r.root = wide ? (uint32_t)kPredBPSW : (uint32_t)kPredMR235;
        r.link = wide ? (uint32_t)kPredBPSW : (uint32_t)kPredFermat2;
        r.cap = wide ? bits + 2 * target : 127u;
        r.screen = true;
    } else {
        r.root = r.link = pc.primality;
        r.cap = 0;
        r.screen = false;
    }
    return r;
}

// trial division of n before its root test: v13 K2's 132 primes (roots
// mode), its CPU prover's 62 (full mode), or v33's 101..409 (v33:2112-2128)
__device__ __forceinline__ void trial_list(const ProveConst& pc, uint32_t& t0, uint32_t& t1) {
    if (pc.primality == CCS_PRIME_V33) { t0 = 7; t1 = 62; }
    else { t0 = 0; t1 = pc.prove_mode == CCS_PROVE_ROOTS ? 132u : 62u; }   // v13:1499 / 1832
}

// Trial division of n before its root test, together with the birth
// certificate of v34 (v34:70-77, 2598-2612): when n == 1 (mod q) for a screen
// prime q (second kind: n == -1), q divides the predecessor (n -/+ 1) / 2,
// which is then composite (it is larger than q for every n above 1727), so n
// is a root without a primality test of its predecessor.  Returns false when
// trial division rejects n; *cert receives the certificate.
__device__ __forceinline__ bool trial_and_certificate(const Big& nb, const ProveConst& pc, uint32_t t0,
                                                      uint32_t t1, bool& cert) {
    cert = false;
    for (uint32_t t = 0; t < 132; t++) {
        const uint32_t q = c_screen[t];
        const uint32_t r = big_mod_small(nb, q);
        if (r == 0 && t >= t0 && t < t1) return false;
        cert |= r == (pc.kind == 2 ? q - 1 : 1u);
    }
    cert &= !big_lt_u32(nb, 1728);
    return true;
}

// ---------------------------------------------------------------------------
// prove kernel: one thread per survivor
// ---------------------------------------------------------------------------
// n = ((T0 + tile_idx) * WP + k) * M + base   (v13:1479-1492)
__device__ __forceinline__ Big survivor_number(const uint4 s, const ProveRange& R, const ProveConst& pc) {
    Big nb;
    uint64_t c = s.z;
#pragma unroll
    for (int w = 0; w < 4; w++) {
        const uint64_t v = (uint64_t)R.T0[w] + c;
        nb.w[w] = (uint32_t)v;
        c = v >> 32;
    }
    nb.w[4] = (uint32_t)c;
    nb.w[5] = 0;
    c = s.y;
#pragma unroll
    for (int w = 0; w < kMaxLimbs; w++) {
        const uint64_t v = (uint64_t)nb.w[w] * pc.WP + c;
        nb.w[w] = (uint32_t)v;
        c = v >> 32;
    }
    c = (s.x < pc.n_bases) ? pc.bases[s.x] : 0;
#pragma unroll
    for (int w = 0; w < kMaxLimbs; w++) {
        const uint64_t v = (uint64_t)nb.w[w] * pc.M + c;
        nb.w[w] = (uint32_t)v;
        c = v >> 32;
    }
    return nb;
}

// p_0 = (q_base + offset) * D_V * 2^E - 1 for a q-iteration survivor
// {offset, seg, variant} (v16:2576-2620); the caller keeps p_0 < 2^160
__device__ __forceinline__ Big qiter_number(const uint4 s, const QiterProve& q) {
    const uint32_t* sg = q.seg + (size_t)s.y * 6;
    uint32_t Q[5];
    uint64_t c = s.x;
#pragma unroll
    for (int w = 0; w < 4; w++) {
        const uint64_t v = (uint64_t)sg[w] + c;
        Q[w] = (uint32_t)v;
        c = v >> 32;
    }
    Q[4] = (uint32_t)c;
    const uint32_t* d = q.dv + (size_t)sg[5] * 4;               // the segment's variant
    uint32_t prod[kMaxLimbs];
#pragma unroll
    for (int w = 0; w < kMaxLimbs; w++) prod[w] = 0;
#pragma unroll
    for (int i = 0; i < 5; i++) {
        uint64_t carry = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (i + j < kMaxLimbs) {
                const uint64_t v = (uint64_t)Q[i] * d[j] + prod[i + j] + carry;
                prod[i + j] = (uint32_t)v;
                carry = v >> 32;
            }
        }
        if (i + 4 < kMaxLimbs) prod[i + 4] = (uint32_t)carry;
    }
    Big b;
    const uint32_t E = q.exp_start;
    const uint32_t ws = E >> 5, bs = E & 31;
#pragma unroll
    for (int w = kMaxLimbs - 1; w >= 0; w--) {
        const int src = w - (int)ws;
        const uint32_t lo = src >= 0 ? prod[src] : 0u;
        const uint32_t lo2 = src >= 1 ? prod[src - 1] : 0u;
        b.w[w] = bs ? (lo << bs) | (lo2 >> (32 - bs)) : lo;
    }
    // - 1 (p + 1 >= 2 always: Q >= 1, D_V >= 1)
#pragma unroll
    for (int w = 0; w < kMaxLimbs; w++) {
        const uint32_t old = b.w[w];
        b.w[w] = old - 1u;
        if (old != 0u) break;
    }
    return b;
}

__global__ void __launch_bounds__(128)
prove_kernel(ProveArgs a) {
    uint32_t n = a.n_surv_dev ? *a.n_surv_dev : a.n_surv;
    if (n > a.surv_cap) n = a.surv_cap;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint4 s = reinterpret_cast<const uint4*>(a.surv)[i];
        const ProveRange& R = a.ranges[a.range_from_pad ? s.w : 0u];
        const ProveConst& pc = c_prove[R.profile];
        // n = ((T0 + tile_idx) * WP + k) * M + base   (v13:1479-1492), or a
        // q-iteration p_0 (no bit gate, v16:2620)
        Big nb;
        if (a.q.seg) {
            if (s.y >= a.q.n_segs) continue;
            nb = qiter_number(s, a.q);
        } else {
            uint64_t c = s.z;
#pragma unroll
            for (int w = 0; w < 4; w++) {
                uint64_t v = (uint64_t)R.T0[w] + c;
                nb.w[w] = (uint32_t)v;
                c = v >> 32;
            }
            nb.w[4] = (uint32_t)c;
            nb.w[5] = 0;
            c = s.y;
#pragma unroll
            for (int w = 0; w < kMaxLimbs; w++) {
                uint64_t v = (uint64_t)nb.w[w] * pc.WP + c;
                nb.w[w] = (uint32_t)v;
                c = v >> 32;
            }
            c = (s.x < pc.n_bases) ? pc.bases[s.x] : 0;
#pragma unroll
            for (int w = 0; w < kMaxLimbs; w++) {
                uint64_t v = (uint64_t)nb.w[w] * pc.M + c;
                nb.w[w] = (uint32_t)v;
                c = v >> 32;
            }
        }
        if (!a.q.seg && big_bits(nb) != (int)R.bits) continue;         // v13:1495, 1828
        // trial division only rejects composites that the primality test
        // rejects too (n > 863); q-iteration survivors passed the sieve at
        // position 0 already, so for them it is skipped
        uint32_t t0 = 0, t1 = 0;
        if (!a.q.seg) trial_list(pc, t0, t1);
        bool cert = false;
        if (!trial_and_certificate(nb, pc, t0, t1, cert)) continue;
        const RangePreds rp = range_preds(pc, R.bits, R.target);
        uint32_t mm = 0;
        if (pc.reverse) {
            // chain position target - 1 first (the largest member, the
            // likeliest composite; v15:1704-1708): pos applications of
            // p -> 2p + 1 (second kind 2p - 1)
            const int pos = R.target - 1 < 63 ? (int)R.target - 1 : 63;
            if (pos > 0 && big_bits(nb) + pos < 32 * kMaxLimbs) {
                Big top = nb;
                for (int k = 0; k < pos; k++) big_next(top, pc.kind);
                if (!is_prime_dev(top, pc, mm)) continue;
            }
        }
        if (!is_prime_pred(nb, rp.root, pc, mm)) continue;
        if (R.prime_count) atomicAdd(R.prime_count, 1u);
        Big root = nb;
        bool is_root = true;
        Big pred = nb;
        big_prev(pred, pc.kind);
        if (!cert && !big_lt_u32(pred, 2) && is_prime_dev(pred, pc, mm)) {
            is_root = false;
            if (pc.prove_mode == CCS_PROVE_ROOTS) continue;              // v13:1513-1516
            root = pred;
            for (int back = 0; back < kMaxChain; back++) {            // v13:1855-1866
                Big p2 = root;
                big_prev(p2, pc.kind);
                if (big_lt_u32(p2, 2)) break;
                if (!is_prime_dev(p2, pc, mm)) break;
                root = p2;
            }
        }
        const int len = walk_forward(root, pc, rp.link, rp.screen, rp.cap, mm);
        if (R.chain_count) atomicAdd(R.chain_count, 1u);
        const uint32_t slot = atomicAdd(a.chain_count, 1u);
        if (slot < a.chain_cap) {
            uint32_t* o = a.chains + (size_t)slot * 12;
            o[0] = s.x; o[1] = s.y; o[2] = s.z; o[3] = (uint32_t)len;
#pragma unroll
            for (int w = 0; w < 6; w++) o[4 + w] = root.w[w];
            o[10] = (is_root ? CCS_CHAIN_IS_ROOT : 0u) |
                    ((uint32_t)len >= R.target ? CCS_CHAIN_TARGET : 0u);
            o[11] = i;
        }
    }
}

// ---------------------------------------------------------------------------
// breadth-first chain walk
//
// Every number of a walk batch is an item {member, index, primes so far}.
// A round tests the current member of every live item: a screen kernel runs
// the trial stage and sorts the items that need a probable-prime test into
// one region per Montgomery limb count, a test kernel per region runs the
// base-2 strong test (or the witness list), a second one the strong Lucas
// test of the base-2 probable primes; members found prime advance to 2p + 1
// for the next round, the others end their walk.  Warps therefore run one
// limb count and one test at a time, whatever the chain lengths.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, want);
    const uint32_t lane = threadIdx.x & 31;
    uint32_t base = 0;
    const int leader = __ffs(m) - 1;
    if (m && (int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader < 0 ? 0 : leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

__device__ __forceinline__ void walk_count_mm(uint32_t mm, uint32_t words) {
    const uint32_t tot = __reduce_add_sync(0xFFFFFFFFu, mm);
    const uint32_t wtot = __reduce_add_sync(0xFFFFFFFFu, words);
    if ((threadIdx.x & 31) == 0 && tot) {
        atomicAdd(&g_modmul_count, (unsigned long long)tot);
        atomicAdd(&g_wordmul_count, (unsigned long long)wtot);
    }
}

// member found prime: count it, continue with 2p + 1 or end the walk
// (MAX_CHAIN, or a next member beyond 192 bits; v13:1519-1528, 1873-1881)
__device__ __forceinline__ void walk_advance(const WalkItem& it, int nbits, bool live, WalkArgs& a,
                                             uint32_t kind) {
    const uint32_t len = it.len + 1;
    const bool more = live && len < a.max_len && nbits < 32 * kMaxLimbs;
    const uint32_t pos = warp_append(&a.st->n_next, more);
    if (!live) return;
    if (more) {
        WalkItem nx = it;
        Big b;
#pragma unroll
        for (int i = 0; i < kMaxLimbs; i++) b.w[i] = nx.x[i];
        big_next(b, kind);
#pragma unroll
        for (int i = 0; i < kMaxLimbs; i++) nx.x[i] = b.w[i];
        nx.len = len;
        a.next[pos] = nx;
    } else {
        a.lengths[it.idx] = len;
    }
}

__global__ void __launch_bounds__(256)
walk_load_kernel(const uint32_t* __restrict__ numbers, uint64_t first, uint32_t n, uint32_t limbs,
                 WalkItem* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        WalkItem it;
#pragma unroll
        for (int w = 0; w < kMaxLimbs; w++)
            it.x[w] = (w < (int)limbs) ? numbers[(first + i) * limbs + w] : 0u;
        it.idx = (uint32_t)(first + i);
        it.len = 0;
        out[i] = it;
    }
}

// trial stage; records the verdict code of every item and counts each region
__global__ void __launch_bounds__(256)
walk_screen_kernel(WalkArgs a) {
    const ProveConst& pc = c_prove[a.profile];
    const uint32_t n = a.st->n_act;
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        const bool live = i < n;
        WalkItem it;
        int nbits = 0, v = 0;
        if (live) {
            it = a.act[i];
            Big b;
#pragma unroll
            for (int w = 0; w < kMaxLimbs; w++) b.w[w] = it.x[w];
            const bool link = a.screen && it.len >= 1;
            if (link && ((a.cap_bits && big_bits(b) > (int)a.cap_bits) || screen_composite(b))) {
                nbits = big_bits(b);
                v = 0;                                   // the walk ends here (v33:1546-1562)
            } else {
                v = prime_screen(b, link ? a.link_pred : a.pred, nbits);
            }
            a.code[i] = (uint8_t)v;
            if (v == 0) a.lengths[it.idx] = it.len;
        }
        walk_advance(it, nbits, live && v == 1, a, pc.kind);
        // count the members that need a test per bit length (one atomic per
        // distinct length in the warp)
        const bool need = live && v >= 2;
        const uint32_t nm = __ballot_sync(0xFFFFFFFFu, need);
        if (need) {
            const uint32_t grp = __match_any_sync(nm, (uint32_t)nbits);
            if ((threadIdx.x & 31) == (uint32_t)(__ffs(grp) - 1)) atomicAdd(&a.st->n_bits[nbits], __popc(grp));
        }
    }
}

// limb count of the Montgomery arithmetic for a member of nbits bits (the
// trial stage's code)
__host__ __device__ constexpr int limbs_of_bits(int nbits) {
    return nbits <= 64 ? 2 : (nbits + 31) >> 5;
}

// members sorted by bit length: ascending lengths, so the regions of one
// limb count are contiguous, and the warps of a test run members of one
// length (the same exponent loop lengths).  One warp: each lane sums seven
// bit lengths, a warp scan gives the offsets.
__global__ void __launch_bounds__(32) walk_regions_kernel(WalkState* st) {
    constexpr int kPer = (kWalkBits + 31) / 32;
    const uint32_t lane = threadIdx.x;
    uint32_t v[kPer], sum = 0;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        const int b = (int)lane * kPer + k;
        v[k] = b < kWalkBits ? st->n_bits[b] : 0u;
        sum += v[k];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    uint32_t o = incl - sum;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        const int b = (int)lane * kPer + k;
        if (b < kWalkBits) {
            st->fill_bits[b] = o;
            if (b == 0 || limbs_of_bits(b) != limbs_of_bits(b - 1)) st->off_region[limbs_of_bits(b)] = o;
        }
        o += v[k];
    }
    __syncwarp();
    if (lane == 0) {
        // regions of limb counts 2..kMaxLimbs in ascending order (bit
        // lengths 0..64 take 2 limbs), each ending where the next begins
        st->n_region[0] = st->n_region[1] = 0;
        st->off_region[0] = st->off_region[1] = 0;
        for (int nl = limbs_of_bits(0); nl <= kMaxLimbs; nl++)
            st->n_region[nl] = (nl < kMaxLimbs ? st->off_region[nl + 1] : total) - st->off_region[nl];
    }
}

__global__ void __launch_bounds__(256)
walk_scatter_kernel(WalkArgs a) {
    const uint32_t n = a.st->n_act;
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        const int v = i < n ? a.code[i] : 0;
        const bool need = v >= 2;
        const uint32_t nm = __ballot_sync(0xFFFFFFFFu, need);
        if (need) {
            const WalkItem it = a.act[i];
            Big b;
#pragma unroll
            for (int w = 0; w < kMaxLimbs; w++) b.w[w] = it.x[w];
            const uint32_t nbits = (uint32_t)big_bits(b);
            const uint32_t grp = __match_any_sync(nm, nbits);
            const uint32_t leader = __ffs(grp) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(&a.st->fill_bits[nbits], __popc(grp));
            base = __shfl_sync(grp, base, leader);
            a.sorted[base + __popc(grp & ((1u << lane) - 1u))] = it;
        }
    }
}

template <int NL, uint32_t PRED>
__device__ __forceinline__ void walk_test_region(WalkArgs& a, const ProveConst& pc, int stage) {
    // stage 0: the sorted region; stage 1: the base-2 probable primes at the
    // bottom of the region; stage 2: those whose Selfridge parameter is
    // D = -7, at its top
    const uint32_t off0 = a.st->off_region[NL];
    const uint32_t n = stage == 0 ? a.st->n_region[NL] : stage == 1 ? a.st->n_lucas[NL] : a.st->n_lucas_q2[NL];
    const uint32_t off = stage == 2 ? off0 + a.st->n_region[NL] - n : off0;
    const WalkItem* src = stage == 0 ? a.sorted : a.lucas;
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        // whole warps: lanes past the end test a copy of the warp's first
        // member (and record nothing), so the tests reconverge the warp
        const uint32_t wbase = i0 + (threadIdx.x & ~31u);
        if (wbase >= n) continue;
        const uint32_t i = i0 + threadIdx.x;
        const bool live = i < n;
        const WalkItem it = src[off + (live ? i : wbase)];
        Big b;
#pragma unroll
        for (int w = 0; w < kMaxLimbs; w++) b.w[w] = it.x[w];
        const int nbits = big_bits(b);
        bool prime = false, to_lucas = false;
        Mont<NL> M;
        mont_setup<NL>(M, b, nbits);
        M.count = 0;
        M.sq = 0;
        __syncwarp();
        if (stage == 0) {
            // the first test for every member; the rest only for its
            // probable primes, in a second launch of uniform warps
            if (PRED == kPredBPSW || PRED == kPredMR235) {
                to_lucas = strong_prp<NL, true>(M, b, 2);
            } else if (PRED == kPredFermat2) {
                prime = fermat2<NL, true>(M, b);
            } else if (pc.n_wit <= 1) {
                prime = pc.n_wit == 0 || strong_prp<NL, true>(M, b, pc.wit[0]);
            } else {
                to_lucas = strong_prp<NL, true>(M, b, pc.wit[0]);
            }
        } else if (PRED == kPredBPSW && stage == 2) {
            prime = strong_lucas<NL, true, true>(M, b);
        } else if (PRED == kPredBPSW) {
            prime = strong_lucas<NL, true>(M, b);
        } else if (PRED == kPredMR235) {
            // both tests on every lane: a test reconverges the warp inside
            const bool r3 = strong_prp<NL, true>(M, b, 3);
            const bool r5 = strong_prp<NL, true>(M, b, 5);
            prime = r3 && r5;
        } else if (PRED == kPredMR) {
            prime = true;
            for (uint32_t k = 1; k < pc.n_wit; k++) {
                const bool r = strong_prp<NL, true>(M, b, pc.wit[k]);
                prime = prime && r;
                if (!__any_sync(0xFFFFFFFFu, live && prime)) break;
            }
        }
        prime = prime && live;
        to_lucas = to_lucas && live;
        const uint32_t mm = live ? M.count : 0u;
        const uint32_t msq = live ? M.sq : 0u;
        const uint32_t words = (mm - msq) * mul_words(NL) + msq * sqr_words(NL);
        if (live && !prime && !to_lucas) a.lengths[it.idx] = it.len;
        walk_count_mm(mm, words);
        if (stage == 0) {
            // BPSW: probable primes whose Selfridge parameter is D = -7
            // (Q = 2) take the three-product ladder in a launch of their own
            bool q2 = false;
            if (PRED == kPredBPSW && to_lucas) q2 = jacobi_small(5, b) == 1 && jacobi_small(-7, b) == -1;
            const uint32_t pos = warp_append(&a.st->n_lucas[NL], to_lucas && !q2);
            if (PRED == kPredBPSW) {
                const uint32_t pq = warp_append(&a.st->n_lucas_q2[NL], to_lucas && q2);
                if (to_lucas && q2) a.lucas[off + a.st->n_region[NL] - 1 - pq] = it;
            }
            if (to_lucas && !q2) a.lucas[off + pos] = it;
        }
        walk_advance(it, nbits, prime, a, pc.kind);
    }
}

// One kernel per test (PRED), stage (0 = base-2 strong test or the first
// witness, 1 = strong Lucas test or the other witnesses, 2 = the strong
// Lucas test of the members with D = -7) and limb count, one
// launch per limb count: an SM runs the code of one of them at a time.
template <uint32_t PRED, int STAGE, int NL>
__global__ void __launch_bounds__(128, 4)
walk_test_kernel(WalkArgs a) {
    const ProveConst& pc = c_prove[a.profile];
    walk_test_region<NL, PRED>(a, pc, STAGE);
}

template <uint32_t PRED, int STAGE>
static void launch_walk_tests(const WalkArgs& a, uint32_t grid, cudaStream_t st) {
    walk_test_kernel<PRED, STAGE, 2><<<grid, 128, 0, st>>>(a);
    walk_test_kernel<PRED, STAGE, 3><<<grid, 128, 0, st>>>(a);
    walk_test_kernel<PRED, STAGE, 4><<<grid, 128, 0, st>>>(a);
    walk_test_kernel<PRED, STAGE, 5><<<grid, 128, 0, st>>>(a);
    walk_test_kernel<PRED, STAGE, 6><<<grid, 128, 0, st>>>(a);
}

template <uint32_t PRED>
static void launch_walk_stage(const WalkArgs& a, int stage, uint32_t grid, cudaStream_t st) {
    if (stage == 0) launch_walk_tests<PRED, 0>(a, grid, st);
    else launch_walk_tests<PRED, 1>(a, grid, st);
    if (PRED == kPredBPSW && stage == 1) launch_walk_tests<kPredBPSW, 2>(a, grid, st);
}

cudaError_t launch_walk_load(const uint32_t* numbers, uint64_t first, uint32_t n, uint32_t limbs,
                             WalkItem* out, cudaStream_t st) {
    const uint32_t blocks = std::min<uint32_t>((n + 255) / 256, 148 * 8);
    walk_load_kernel<<<blocks ? blocks : 1, 256, 0, st>>>(numbers, first, n, limbs, out);
    return cudaGetLastError();
}

cudaError_t launch_walk_round(const WalkArgs& a, uint32_t n_act, bool two_stage, uint32_t round_pred,
                              cudaStream_t st) {
    const uint32_t blocks = std::min<uint32_t>((n_act + 255) / 256, 148 * 8);
    walk_screen_kernel<<<blocks ? blocks : 1, 256, 0, st>>>(a);
    walk_regions_kernel<<<1, 32, 0, st>>>(a.st);
    walk_scatter_kernel<<<blocks ? blocks : 1, 256, 0, st>>>(a);
    const uint32_t tb = std::min<uint32_t>((n_act + 127) / 128, 148 * 16);
    const uint32_t grid = tb ? tb : 1;
    for (int stage = 0; stage < (two_stage ? 2 : 1); stage++) {
        switch (round_pred) {
            case kPredBPSW: launch_walk_stage<kPredBPSW>(a, stage, grid, st); break;
            case kPredMR235: launch_walk_stage<kPredMR235>(a, stage, grid, st); break;
            case kPredFermat2: launch_walk_stage<kPredFermat2>(a, stage, grid, st); break;
            default: launch_walk_stage<kPredMR>(a, stage, grid, st); break;
        }
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// staged prove of a filter launch's survivors
//
// The same semantics as prove_kernel, run as breadth-first stages over all
// survivors so warps do one kind of test at a time: seed (reconstruction,
// bit gate, trial division; with the reverse order the top member), then
// primality of the members each stage asks for through the walk rounds
// above (max length 1), then the forward walk from every root.  Per survivor
// index: its number, its current root, and the stage's verdict in
// lengths[idx].
// ---------------------------------------------------------------------------
__device__ __forceinline__ void big_store(uint32_t* dst, const Big& b) {
#pragma unroll
    for (int w = 0; w < kMaxLimbs; w++) dst[w] = b.w[w];
}
__device__ __forceinline__ Big big_load(const uint32_t* src) {
    Big b;
#pragma unroll
    for (int w = 0; w < kMaxLimbs; w++) b.w[w] = src[w];
    return b;
}
__device__ __forceinline__ void item_put(WalkItem* out, uint32_t pos, const Big& x, uint32_t idx, uint32_t len) {
    WalkItem it;
#pragma unroll
    for (int w = 0; w < kMaxLimbs; w++) it.x[w] = x.w[w];
    it.idx = idx;
    it.len = len;
    out[pos] = it;
}

__global__ void __launch_bounds__(256)
prove_seed_kernel(StagedProve p) {
    const ProveConst& pc = c_prove[p.range->profile];
    const ProveRange& R = *p.range;
    uint32_t t0 = 0, t1 = 0;
    if (!p.q.seg) trial_list(pc, t0, t1);
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < p.n_surv; i0 += gridDim.x * blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        bool keep = false;
        Big nb, x;
        if (i < p.n_surv) {
            const uint4 sv = reinterpret_cast<const uint4*>(p.surv)[p.first + i];
            if (p.q.seg) {
                keep = sv.y < p.q.n_segs;                                        // no bit gate (v16:2620)
                if (keep) nb = qiter_number(sv, p.q);
            } else {
                nb = survivor_number(sv, R, pc);
                keep = big_bits(nb) == (int)R.bits;                              // v13:1495, 1828
            }
            bool cert = false;
            if (keep) keep = trial_and_certificate(nb, pc, t0, t1, cert);
            x = nb;
            if (keep) {
                big_store(p.nval + (size_t)i * kMaxLimbs, nb);
                p.flags[i] = cert ? kFlagCertificate : 0u;
                if (pc.reverse) {
                    // chain position target - 1 first (v15:1704-1708)
                    const int pos = R.target - 1 < 63 ? (int)R.target - 1 : 63;
                    if (pos > 0 && big_bits(nb) + pos < 32 * kMaxLimbs)
                        for (int k = 0; k < pos; k++) big_next(x, pc.kind);
                }
            }
        }
        const uint32_t pos = warp_append(p.count, keep);
        if (keep) item_put(p.out, pos, x, i, 0);
    }
}

// after a primality stage over the items of `in` (len: backward steps so far)
//   stage 0: the reverse order's top member -> test n itself
//   stage 1: n itself  -> count the prime; test its predecessor (or it is a root)
//   stage 2: a predecessor -> prime: not a root (roots-only mode drops it,
//            otherwise it becomes the root candidate and its own predecessor is
//            tested next); composite: the current root is final
__global__ void __launch_bounds__(256)
prove_select_kernel(StagedProve p, const WalkItem* in, uint32_t n_in, int stage) {
    const ProveConst& pc = c_prove[p.range->profile];
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n_in; i0 += gridDim.x * blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        bool emit = false, to_fwd = false;
        Big x;
        uint32_t idx = 0;
        if (i < n_in) {
            const WalkItem it = in[i];
            idx = it.idx;
            // the walk of one member leaves len + 1 when it is prime, len otherwise
            const bool prime = p.lengths[idx] == it.len + 1;
            if (stage == 0) {
                if (prime) { x = big_load(p.nval + (size_t)idx * kMaxLimbs); emit = true; }
            } else if (stage == 1) {
                if (prime) {
                    atomicAdd(p.primes, 1u);
                    const Big nb = big_load(p.nval + (size_t)idx * kMaxLimbs);
                    big_store(p.root + (size_t)idx * kMaxLimbs, nb);
                    const bool cert = p.flags[idx] & kFlagCertificate;
                    p.flags[idx] = CCS_CHAIN_IS_ROOT;
                    x = nb;
                    big_prev(x, pc.kind);
                    if (big_lt_u32(x, 2)) {
                        to_fwd = true;
                    } else if (cert) {
                        to_fwd = true;                     // birth certificate: the predecessor is composite
                        atomicAdd(p.certified, 1u);
                    } else {
                        emit = true;
                    }
                }
            } else {
                if (prime) {
                    if (pc.prove_mode != CCS_PROVE_ROOTS) {                       // v13:1855-1866
                        Big r;
#pragma unroll
                        for (int w = 0; w < kMaxLimbs; w++) r.w[w] = it.x[w];
                        big_store(p.root + (size_t)idx * kMaxLimbs, r);
                        p.flags[idx] = 0;
                        if (it.len >= (uint32_t)kMaxChain) {
                            to_fwd = true;                 // the backward walk's step cap
                        } else {
                            x = r;
                            big_prev(x, pc.kind);
                            if (big_lt_u32(x, 2)) to_fwd = true; else emit = true;
                        }
                    }                                        // roots-only: dropped (v13:1513-1516)
                } else {
                    to_fwd = true;
                }
            }
        }
        const uint32_t pos = warp_append(p.count, emit);
        if (emit) item_put(p.out, pos, x, idx, stage == 2 ? in[i].len + 1 : 0);
        const uint32_t fpos = warp_append(p.fwd_count, to_fwd);
        if (to_fwd) {
            // forward walk from the root: its next member, the root counted;
            // a root of 192 bits has no next member (0 ends the walk at 1)
            const Big r = big_load(p.root + (size_t)idx * kMaxLimbs);
            Big nx = r;
            if (big_bits(r) >= 32 * kMaxLimbs) {
#pragma unroll
                for (int w = 0; w < kMaxLimbs; w++) nx.w[w] = 0;
            } else {
                big_next(nx, pc.kind);
            }
            item_put(p.fwd, fpos, nx, idx, 1u);
        }
    }
}

// records of the walked roots: lengths[idx] = chain length
__global__ void __launch_bounds__(256)
prove_emit_kernel(StagedProve p, const WalkItem* roots, uint32_t n_roots) {
    const ProveRange& R = *p.range;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_roots; i += gridDim.x * blockDim.x) {
        const uint32_t idx = roots[i].idx;
        const uint32_t len = p.lengths[idx];
        const uint4 sv = reinterpret_cast<const uint4*>(p.surv)[p.first + idx];
        const uint32_t slot = atomicAdd(p.chain_count, 1u);
        if (slot < p.chain_cap) {
            uint32_t* o = p.chains + (size_t)slot * 12;
            o[0] = sv.x; o[1] = sv.y; o[2] = sv.z; o[3] = len;
#pragma unroll
            for (int w = 0; w < 6; w++) o[4 + w] = p.root[(size_t)idx * kMaxLimbs + w];
            o[10] = p.flags[idx] | (len >= R.target ? CCS_CHAIN_TARGET : 0u);
            o[11] = p.first + idx;
        }
    }
}

cudaError_t launch_prove_stage(int which, const StagedProve& p, const WalkItem* in, uint32_t n,
                               cudaStream_t st) {
    const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((n + 255) / 256, 148 * 8));
    switch (which) {
        case -1: prove_seed_kernel<<<blocks, 256, 0, st>>>(p); break;
        case 0: case 1: case 2: prove_select_kernel<<<blocks, 256, 0, st>>>(p, in, n, which); break;
        default: prove_emit_kernel<<<blocks, 256, 0, st>>>(p, in, n); break;
    }
    return cudaGetLastError();
}

cudaError_t modmul_count(uint64_t* out, uint64_t* words, bool reset) {
    unsigned long long v = 0, w = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_modmul_count, sizeof(v));
    if (e == cudaSuccess) e = cudaMemcpyFromSymbol(&w, g_wordmul_count, sizeof(w));
    if (e != cudaSuccess) return e;
    if (out) *out = v;
    if (words) *words = w;
    if (reset) {
        v = 0;
        e = cudaMemcpyToSymbol(g_modmul_count, &v, sizeof(v));
        if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_wordmul_count, &v, sizeof(v));
    }
    return e;
}

cudaError_t launch_prove(const ProveArgs& a, uint32_t grid, cudaStream_t st) {
    if (grid == 0) grid = 1;
    prove_kernel<<<grid, 128, 0, st>>>(a);
    return cudaGetLastError();
}


}  // namespace ccs
