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
// GMP 6.3 mpz_probab_prime_p(n, 1) used by the reference CPU prover.
#include "ccs_kernels.cuh"
#include "../../include/ccs.h"

namespace ccs {

__constant__ ProveConst c_prove[kMaxProfiles];

// Montgomery products executed by walk launches (one atomic per number)
__device__ unsigned long long g_modmul_count = 0;

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

__device__ __forceinline__ uint32_t big_mod_small(const Big& a, uint32_t q) {
    uint64_t acc = 0;
#pragma unroll
    for (int i = kMaxLimbs - 1; i >= 0; i--) acc = ((acc << 32) | a.w[i]) % q;
    return (uint32_t)acc;
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

// a = (a - 1) / 2 for odd a
__device__ __forceinline__ void big_pred(Big& a) {
#pragma unroll
    for (int i = 0; i < kMaxLimbs; i++) {
        uint32_t hi = (i + 1 < kMaxLimbs) ? a.w[i + 1] : 0;
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
};

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

// CIOS Montgomery product r = a b R^{-1} mod n (a, b < n)
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

// strong probable-prime test to base a (n odd, n > a)
template <int NL>
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
        // d >>= s
        int ws = s >> 5, bs = s & 31;
#pragma unroll
        for (int i = 0; i < kMaxLimbs; i++) {
            uint32_t lo = (i + ws < kMaxLimbs) ? d.w[i + ws] : 0;
            uint32_t hi = (i + ws + 1 < kMaxLimbs) ? d.w[i + ws + 1] : 0;
            d.w[i] = bs ? ((lo >> bs) | (hi << (32 - bs))) : lo;
        }
    }
    uint32_t am[NL], x[NL];
    to_mont_small<NL>(am, a, M);
#pragma unroll
    for (int i = 0; i < NL; i++) x[i] = am[i];
    const int top = big_bits(d) - 1;
    for (int b = top - 1; b >= 0; b--) {
        montmul<NL>(x, x, x, M.n, M.ninv);
        M.count++;
        if ((d.w[b >> 5] >> (b & 31)) & 1u) {
            if (a == 2) dblmod<NL>(x, x, M.n);
            else { montmul<NL>(x, x, am, M.n, M.ninv); M.count++; }
        }
    }
    if (eq<NL>(x, M.one) || eq<NL>(x, M.mone)) return true;
    for (int r = 1; r < s; r++) {
        montmul<NL>(x, x, x, M.n, M.ninv);
        M.count++;
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

// strong Lucas probable-prime test, Selfridge method A (P = 1, Q = (1 - D)/4)
template <int NL>
__device__ bool strong_lucas(Mont<NL>& M, const Big& nb) {
    int D = 5;
    int tries = 0;
    for (;;) {
        int j = jacobi_small(D, nb);
        if (j == -1) break;
        if (j == 0) {
            uint32_t ad = (uint32_t)(D < 0 ? -D : D);
            return big_lt_u32(nb, ad + 1) && nb.w[0] == ad;   // n == |D|
        }
        D = D > 0 ? -(D + 2) : -(D - 2);
        // no D with (D/n) = -1 among the first 64 candidates: n is (almost
        // surely) a perfect square; squares are composite
        if (++tries > 64) return false;
    }
    const int Qs = (1 - D) / 4;
    uint32_t Dm[NL], Qm[NL];
    if (D >= 0) to_mont_small<NL>(Dm, (uint32_t)D, M);
    else { uint32_t t[NL]; to_mont_small<NL>(t, (uint32_t)(-D), M); submod<NL>(Dm, M.n, t, M.n); }
    if (Qs >= 0) to_mont_small<NL>(Qm, (uint32_t)Qs, M);
    else { uint32_t t[NL]; to_mont_small<NL>(t, (uint32_t)(-Qs), M); uint32_t z[NL];
#pragma unroll
        for (int i = 0; i < NL; i++) z[i] = 0;
        submod<NL>(Qm, z, t, M.n); }
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
    uint32_t U[NL], V[NL], Qk[NL], t1[NL], t2[NL];
#pragma unroll
    for (int i = 0; i < NL; i++) { U[i] = M.one[i]; V[i] = M.one[i]; Qk[i] = Qm[i]; }
    for (int b = big_bits(d) - 2; b >= 0; b--) {
        montmul<NL>(U, U, V, M.n, M.ninv);
        montmul<NL>(t1, V, V, M.n, M.ninv);
        addmod<NL>(t2, Qk, Qk, M.n);
        submod<NL>(V, t1, t2, M.n);
        montmul<NL>(Qk, Qk, Qk, M.n, M.ninv);
        M.count += 3;
        if ((d.w[b >> 5] >> (b & 31)) & 1u) {
            uint32_t nu[NL], nv[NL];
            addmod<NL>(nu, U, V, M.n);
            halfmod<NL>(nu, M.n);
            montmul<NL>(t1, Dm, U, M.n, M.ninv);
            addmod<NL>(nv, t1, V, M.n);
            halfmod<NL>(nv, M.n);
#pragma unroll
            for (int i = 0; i < NL; i++) { U[i] = nu[i]; V[i] = nv[i]; }
            montmul<NL>(Qk, Qk, Qm, M.n, M.ninv);
            M.count += 2;
        }
    }
    if (is_zero<NL>(U) || is_zero<NL>(V)) return true;
    for (int r = 1; r < s; r++) {
        montmul<NL>(t1, V, V, M.n, M.ninv);
        addmod<NL>(t2, Qk, Qk, M.n);
        submod<NL>(V, t1, t2, M.n);
        if (is_zero<NL>(V)) return true;
        montmul<NL>(Qk, Qk, Qk, M.n, M.ninv);
        M.count += 2;
    }
    return false;
}

template <int NL>
__device__ bool prp_suite(const Big& nb, int nbits, uint32_t primality, const ProveConst& pc,
                          uint32_t& mm) {
    Mont<NL> M;
    mont_setup<NL>(M, nb, nbits);
    M.count = 0;
    bool r = true;
    if (primality == CCS_PRIME_BPSW) {
        r = strong_prp<NL>(M, nb, 2) && strong_lucas<NL>(M, nb);
    } else {
        for (uint32_t i = 0; i < pc.n_wit && r; i++) r = strong_prp<NL>(M, nb, pc.wit[i]);
    }
    mm += M.count;
    return r;
}

__constant__ uint32_t c_small_primes[27] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47,
                                            53, 59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 1093, 3511};

// primality predicate of the profile for any n < 2^192; mm counts the
// Montgomery products spent
__device__ bool is_prime_dev(const Big& nb, const ProveConst& pc, uint32_t& mm) {
    const int nbits = big_bits(nb);
    if (nbits <= 1) return false;
    const uint32_t lo = nb.w[0];
    if (pc.primality == CCS_PRIME_MR) {
        // v13:1428-1452
        if (nbits <= 64 && nb.w[1] == 0) {
            if (lo < 2) return false;
            if (lo == 2 || lo == 3) return true;
            if ((lo & 1u) == 0) return false;
            if (lo < 9) return true;
        }
        if ((lo & 1u) == 0) return false;
        for (int i = 0; i < 19; i++) {
            uint32_t p = c_small_primes[i];
            if (big_mod_small(nb, p) == 0) return nbits <= 32 && lo == p;
        }
    } else {
        if (nbits <= 32 && lo == 2) return true;
        if ((lo & 1u) == 0) return false;
        for (int i = 0; i < 27; i++) {
            uint32_t p = c_small_primes[i];
            if (nbits <= 32 && lo == p) return true;
            if (big_mod_small(nb, p) == 0) return false;
        }
        if (nbits <= 32 && lo < 103u * 103u) return true;
    }
    const int nl = (nbits + 31) >> 5;
    switch (nl <= 2 ? 2 : nl) {
        case 2: return prp_suite<2>(nb, nbits, pc.primality, pc, mm);
        case 3: return prp_suite<3>(nb, nbits, pc.primality, pc, mm);
        case 4: return prp_suite<4>(nb, nbits, pc.primality, pc, mm);
        case 5: return prp_suite<5>(nb, nbits, pc.primality, pc, mm);
        default: return prp_suite<6>(nb, nbits, pc.primality, pc, mm);
    }
}

// forward walk p -> 2p + 1 while prime, counting p (v13:1519-1528, 1873-1881)
__device__ int walk_forward(Big cur, const ProveConst& pc, uint32_t& mm) {
    int len = 1;
    while (len < kMaxChain) {
        if (big_bits(cur) >= 32 * kMaxLimbs) break;   // next member would exceed 192 bits
        Big nx = cur;
        big_shl1_inc(nx);
        if (!is_prime_dev(nx, pc, mm)) break;
        len++;
        cur = nx;
    }
    return len;
}

__constant__ uint32_t c_screen[132] = {
    67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113, 127, 131, 137, 139, 149, 151,
    157, 163, 167, 173, 179, 181, 191, 193, 197, 199, 211, 223, 227, 229, 233, 239, 241,
    251, 257, 263, 269, 271, 277, 281, 283, 293, 307, 311, 313, 317, 331, 337, 347, 349,
    353, 359, 367, 373, 379, 383, 389, 397, 401, 409, 419, 421, 431, 433, 439, 443, 449,
    457, 461, 463, 467, 479, 487, 491, 499, 503, 509, 521, 523, 541, 547, 557, 563, 569,
    571, 577, 587, 593, 599, 601, 607, 613, 617, 619, 631, 641, 643, 647, 653, 659, 661,
    673, 677, 683, 691, 701, 709, 719, 727, 733, 739, 743, 751, 757, 761, 769, 773, 787,
    797, 809, 811, 821, 823, 827, 829, 839, 853, 857, 859, 863};

// ---------------------------------------------------------------------------
// prove kernel: one thread per survivor
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
prove_kernel(ProveArgs a) {
    uint32_t n = a.n_surv_dev ? *a.n_surv_dev : a.n_surv;
    if (n > a.surv_cap) n = a.surv_cap;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint4 s = reinterpret_cast<const uint4*>(a.surv)[i];
        const ProveRange& R = a.ranges[a.range_from_pad ? s.w : 0u];
        const ProveConst& pc = c_prove[R.profile];
        // n = ((T0 + tile_idx) * WP + k) * M + base   (v13:1479-1492)
        Big nb;
        {
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
        if (big_bits(nb) != (int)R.bits) continue;                     // v13:1495, 1828
        const int ntd = (pc.prove_mode == CCS_PROVE_ROOTS) ? 132 : 62;  // v13:1499 / 1832
        bool comp = false;
        for (int t = 0; t < ntd && !comp; t++) comp = big_mod_small(nb, c_screen[t]) == 0;
        if (comp) continue;
        uint32_t mm = 0;
        if (!is_prime_dev(nb, pc, mm)) continue;
        if (R.prime_count) atomicAdd(R.prime_count, 1u);
        Big root = nb;
        bool is_root = true;
        Big pred = nb;
        big_pred(pred);
        if (!big_lt_u32(pred, 2) && is_prime_dev(pred, pc, mm)) {
            is_root = false;
            if (pc.prove_mode == CCS_PROVE_ROOTS) continue;              // v13:1513-1516
            root = pred;
            for (int back = 0; back < kMaxChain; back++) {            // v13:1855-1866
                Big p2 = root;
                big_pred(p2);
                if (big_lt_u32(p2, 2)) break;
                if (!is_prime_dev(p2, pc, mm)) break;
                root = p2;
            }
        }
        const int len = walk_forward(root, pc, mm);
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
// walk kernel: chain length from each given number
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
walk_kernel(const uint32_t* __restrict__ numbers, uint64_t n, uint32_t limbs,
            uint32_t* __restrict__ lengths, int profile) {
    const ProveConst& pc = c_prove[profile];
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        Big x;
#pragma unroll
        for (int w = 0; w < kMaxLimbs; w++) x.w[w] = (w < (int)limbs) ? numbers[i * limbs + w] : 0u;
        uint32_t mm = 0;
        lengths[i] = is_prime_dev(x, pc, mm) ? (uint32_t)walk_forward(x, pc, mm) : 0u;
        atomicAdd(&g_modmul_count, (unsigned long long)mm);
    }
}

cudaError_t modmul_count(uint64_t* out, bool reset) {
    unsigned long long v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_modmul_count, sizeof(v));
    if (e != cudaSuccess) return e;
    *out = v;
    if (reset) {
        v = 0;
        e = cudaMemcpyToSymbol(g_modmul_count, &v, sizeof(v));
    }
    return e;
}

cudaError_t launch_prove(const ProveArgs& a, uint32_t grid, cudaStream_t st) {
    if (grid == 0) grid = 1;
    prove_kernel<<<grid, 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_walk(const uint32_t* numbers, uint64_t n, uint32_t limbs, uint32_t* lengths,
                        int profile, cudaStream_t st) {
    uint64_t blocks = (n + 127) / 128;
    if (blocks == 0) blocks = 1;
    if (blocks > 148 * 64) blocks = 148 * 64;
    walk_kernel<<<(unsigned)blocks, 128, 0, st>>>(numbers, n, limbs, lengths, profile);
    return cudaGetLastError();
}

}  // namespace ccs
