/*
 * ccs_oracle.c -- CPU restatement of the reference's Cunningham-chain hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * liboracle.so, and only as the checker.
 *
 * What is restated (reference = nmicic/cunningham-chain-search):
 *   - forbidden root residues       src/cuda/cc18_filter_cuda_CpC_v13.cu:771-787,
 *                                   src/cpu/cc_gmp_v33_03.c:585-609
 *   - CRT bases, wheels, mod-6 buckets
 *                                   v13:907-1059, v33:636-793
 *   - three-stage depth filter (L2 mask, ext-L2 bytes, line sieve), evaluated
 *     per candidate in the reference kernel's (tile, base, k) order
 *                                   v13:1570-1711 (K1), v33:1795-1960
 *   - n reconstruction, bit gate, trial division, Miller-Rabin with a witness
 *     list (v13:1428-1452), Baillie-PSW (the GMP 6.3 mpz_probab_prime_p(n,1)
 *     semantics the CPU prover relies on, v13:1841-1881), root check,
 *     backward walk and forward chain walk with MAX_CHAIN = 64
 *                                   v13:1479-1538 (K2), v13:1814-1881 (CPU prover)
 *
 * Arithmetic here is deliberately different from the product's: the product
 * uses 32-bit-limb Montgomery on the GPU; this file uses 64-bit limbs, plain
 * schoolbook products and shift-subtract reduction, so a shared bug is
 * unlikely.  Numbers are held in ORC_LIMBS x 64-bit little-endian limbs.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

typedef uint64_t u64;
typedef uint32_t u32;
typedef unsigned __int128 u128;

#define ORC_LIMBS 4          /* 256-bit numbers: roots <= 127 bits + 64 links */
#define ORC_MAX_CHAIN 64     /* v13:164 MAX_CHAIN */
#define ORC_MAX_STAGES 4
#define ORC_MAX_BASES 16384

/* ------------------------------------------------------------------------ */
/* small modular helpers                                                     */
/* ------------------------------------------------------------------------ */

static u64 powmod_u64(u64 b, u64 e, u64 m) {
    u128 r = 1 % m, x = b % m;
    while (e) {
        if (e & 1) r = (r * x) % m;
        x = (x * x) % m;
        e >>= 1;
    }
    return (u64)r;
}

/* inverse of a mod prime q via Fermat (q prime, a != 0 mod q) */
static u64 inv_mod_prime(u64 a, u64 q) { return powmod_u64(a % q, q - 2, q); }

/* Chain kind: 1 = first kind (p -> 2p + 1), 2 = second kind (p -> 2p - 1,
 * the reference's v13b).  Process-wide setting of the test oracle. */
static int g_kind = 1;
void orc_set_kind(int kind) { g_kind = (kind == 2) ? 2 : 1; }
int orc_get_kind(void) { return g_kind; }

/* Forbidden residues of n mod q for positions i in [pos_lo, min(L, q)):
 * p_i = 2^i (n + 1) - 1 == 0 (mod q)  <=>  n == 2^{-i} - 1 (mod q);
 * second kind: p_i = 2^i (n - 1) + 1 == 0  <=>  n == 1 - 2^{-i} (v13b:779-850).
 * For pos_lo = 0 the reference caps at min(L, q - 1) (v13:774); position
 * q - 1 yields residue 0, the same as position 0, so the set is identical.
 * For pos_lo = 1 the reference caps at min(L, q) (v13:838, "pos < q"). */
int orc_forbidden(u32 q, int L, int pos_lo, u32* out) {
    int cnt = 0;
    int hi = L < (int)q ? L : (int)q;
    for (int i = pos_lo; i < hi; i++) {
        u64 inv = inv_mod_prime(powmod_u64(2, (u64)i, q), q);
        u64 r = (g_kind == 2) ? (1 + q - inv) % q : (inv + q - 1) % q;
        int dup = 0;
        for (int k = 0; k < cnt; k++) if (out[k] == (u32)r) { dup = 1; break; }
        if (!dup) out[cnt++] = (u32)r;
    }
    return cnt;
}

/* ------------------------------------------------------------------------ */
/* lattice                                                                   */
/* ------------------------------------------------------------------------ */

typedef struct {
    int n_primes;
    u32* primes;
    int pos_lo;
    u32** fset;        /* per prime: membership bitmap of q bits (as bytes) */
} orc_stage;

typedef struct {
    u64 M;             /* product of CRT primes */
    u32 WP;            /* product of wheel primes */
    int lattice_len;
    int depth;
    int n_bases;
    u64* bases;
    u32 tkm6[ORC_MAX_BASES];
    u32* bucket[ORC_MAX_BASES][6];
    int bucket_n[ORC_MAX_BASES][6];
    int wheel_total[ORC_MAX_BASES];
    int n_stages;
    orc_stage st[ORC_MAX_STAGES];
} orc_lattice;

static int admissible(u64 v, const u32* primes, int np, int L) {
    u32 f[64];
    for (int i = 0; i < np; i++) {
        u32 q = primes[i];
        int nf = orc_forbidden(q, L, 0, f);
        u32 r = (u32)(v % q);
        for (int j = 0; j < nf; j++) if (f[j] == r) return 0;
    }
    return 1;
}

/* Build bases (ascending residues mod M admissible for all CRT primes at
 * lattice_len), per-base wheels over k in [0, WP) admissible for the wheel
 * primes, and the mod-6 buckets.  max_bases > 0 reproduces v13's MAX_BASES
 * cap (v13:163, 966); 0 keeps every base (v33). */
orc_lattice* orc_lattice_create(const u32* crt, int n_crt, const u32* wheel, int n_wheel,
                                int lattice_len, int max_bases) {
    orc_lattice* L = (orc_lattice*)calloc(1, sizeof(orc_lattice));
    if (!L) return NULL;
    L->M = 1;
    for (int i = 0; i < n_crt; i++) L->M *= crt[i];
    L->WP = 1;
    for (int i = 0; i < n_wheel; i++) L->WP *= wheel[i];
    L->lattice_len = lattice_len;
    L->bases = (u64*)malloc(sizeof(u64) * ORC_MAX_BASES);
    u32 inv_m6 = (L->M % 6 == 1) ? 1 : 5;       /* v33:722 */
    for (u64 r = 0; r < L->M; r++) {
        if (!admissible(r, crt, n_crt, lattice_len)) continue;
        if (max_bases > 0 && L->n_bases >= max_bases) break;
        if (L->n_bases >= ORC_MAX_BASES) break;
        int b = L->n_bases;
        u32 tmp[6] = {0};
        u32* wl = (u32*)malloc(sizeof(u32) * L->WP);
        int nw = 0;
        for (u32 k = 0; k < L->WP; k++) {
            u64 v = r + (u64)k * L->M;       /* only its residues mod wheel primes matter */
            if (admissible(v, wheel, n_wheel, lattice_len)) wl[nw++] = k;
        }
        if (nw == 0) { free(wl); continue; }
        L->bases[b] = r;
        /* n == 5 (mod 6) for the first kind, n == 1 for the second (v13b:983) */
        const u32 nres = (g_kind == 2) ? 1 : 5;
        L->tkm6[b] = (u32)(((nres + 6 - r % 6) % 6) * inv_m6 % 6);
        for (int i = 0; i < nw; i++) tmp[wl[i] % 6]++;
        for (int m = 0; m < 6; m++) {
            L->bucket[b][m] = (u32*)malloc(sizeof(u32) * (tmp[m] ? tmp[m] : 1));
            L->bucket_n[b][m] = 0;
        }
        for (int i = 0; i < nw; i++) {
            int m = wl[i] % 6;
            L->bucket[b][m][L->bucket_n[b][m]++] = wl[i];
        }
        L->wheel_total[b] = nw;
        free(wl);
        L->n_bases++;
    }
    return L;
}

void orc_lattice_free(orc_lattice* L) {
    if (!L) return;
    for (int b = 0; b < L->n_bases; b++)
        for (int m = 0; m < 6; m++) free(L->bucket[b][m]);
    for (int s = 0; s < L->n_stages; s++) {
        for (int i = 0; i < L->st[s].n_primes; i++) free(L->st[s].fset[i]);
        free(L->st[s].fset);
        free(L->st[s].primes);
    }
    free(L->bases);
    free(L);
}

int orc_num_bases(const orc_lattice* L) { return L->n_bases; }
u64 orc_base(const orc_lattice* L, int b) { return L->bases[b]; }
u32 orc_tkm6(const orc_lattice* L, int b) { return L->tkm6[b]; }
int orc_bucket_size(const orc_lattice* L, int b, int m) { return L->bucket_n[b][m]; }
int orc_wheel_total(const orc_lattice* L, int b) { return L->wheel_total[b]; }
/* copies bucket m of base b into out (caller sizes it with orc_bucket_size) */
void orc_bucket(const orc_lattice* L, int b, int m, u32* out) {
    memcpy(out, L->bucket[b][m], sizeof(u32) * (size_t)L->bucket_n[b][m]);
}

/* Adds one filter stage: primes tested at positions [pos_lo, min(depth, q)). */
int orc_add_stage(orc_lattice* L, const u32* primes, int n, int pos_lo, int depth) {
    if (L->n_stages >= ORC_MAX_STAGES) return -1;
    orc_stage* s = &L->st[L->n_stages++];
    L->depth = depth;
    s->n_primes = n;
    s->pos_lo = pos_lo;
    s->primes = (u32*)malloc(sizeof(u32) * (n ? n : 1));
    s->fset = (u32**)malloc(sizeof(u32*) * (n ? n : 1));
    u32 f[64];
    for (int i = 0; i < n; i++) {
        u32 q = primes[i];
        s->primes[i] = q;
        s->fset[i] = (u32*)calloc((q + 31) / 32, sizeof(u32));
        int nf = orc_forbidden(q, depth, pos_lo, f);
        for (int j = 0; j < nf; j++) s->fset[i][f[j] >> 5] |= 1u << (f[j] & 31);
    }
    return 0;
}

/* bucket chosen for (tile, base): k == tkm6 - tile*WP (mod 6); for WP == 1
 * (mod 6) this is v13:1589-1590 exactly. */
static int bucket_of(const orc_lattice* L, int b, u32 tile_mod6) {
    u32 wp6 = L->WP % 6;
    return (int)((L->tkm6[b] + 36 - (tile_mod6 * wp6) % 6) % 6);
}

/* residue of n = (tile*WP + k)*M + base modulo a small q, tile a u128 */
static u32 n_mod_q(const orc_lattice* L, u128 tile, u32 k, u64 base, u32 q) {
    u64 t = (u64)(tile % q);
    u64 v = (t * (L->WP % q) + k % q) % q;
    v = (v * (L->M % q) + base % q) % q;
    return (u32)v;
}

/* Filter one candidate.  Returns the stage index that killed it, or -1 when it
 * survives every stage (v13:1634-1686 test order: stage by stage, prime by
 * prime, first hit rejects). */
static int filter_one(const orc_lattice* L, u128 tile, u32 k, u64 base) {
    for (int s = 0; s < L->n_stages; s++) {
        const orc_stage* st = &L->st[s];
        for (int i = 0; i < st->n_primes; i++) {
            u32 q = st->primes[i];
            u32 r = n_mod_q(L, tile, k, base, q);
            if ((st->fset[i][r >> 5] >> (r & 31)) & 1u) return s;
        }
    }
    return -1;
}

/* Survivors of tiles [tile_start, tile_start + n_tiles) in reference record
 * layout {base_idx, k_offset, tile_idx, 0}, in (tile, base, k) order.  Writes
 * at most cap records; returns the total number of survivors.  stage_pass
 * (optional, n_stages + 1 entries) receives: [0] candidates tested,
 * [s + 1] candidates passing stage s. */
u64 orc_filter_range(const orc_lattice* L, u64 ts_lo, u64 ts_hi, u64 n_tiles,
                     u32* out, u64 cap, u64* stage_pass) {
    u128 ts = ((u128)ts_hi << 64) | ts_lo;
    u64 n_out = 0;
    if (stage_pass) memset(stage_pass, 0, sizeof(u64) * (size_t)(L->n_stages + 1));
    for (u64 t = 0; t < n_tiles; t++) {
        u128 tile = ts + t;
        u32 tm6 = (u32)(tile % 6);
        for (int b = 0; b < L->n_bases; b++) {
            int m = bucket_of(L, b, tm6);
            for (int w = 0; w < L->bucket_n[b][m]; w++) {
                u32 k = L->bucket[b][m][w];
                int killed = filter_one(L, tile, k, L->bases[b]);
                if (stage_pass) {
                    stage_pass[0]++;
                    int last = killed < 0 ? L->n_stages : killed;
                    for (int s = 0; s < last; s++) stage_pass[s + 1]++;
                }
                if (killed >= 0) continue;
                if (n_out < cap) {
                    out[4 * n_out + 0] = (u32)b;
                    out[4 * n_out + 1] = k;
                    out[4 * n_out + 2] = (u32)t;
                    out[4 * n_out + 3] = 0;
                }
                n_out++;
            }
        }
    }
    return n_out;
}

/* ------------------------------------------------------------------------ */
/* multi-precision (ORC_LIMBS x u64) arithmetic                              */
/* ------------------------------------------------------------------------ */

typedef struct { u64 w[ORC_LIMBS]; } big;

static void big_set_u64(big* a, u64 v) { memset(a, 0, sizeof(*a)); a->w[0] = v; }
static int big_cmp(const big* a, const big* b) {
    for (int i = ORC_LIMBS - 1; i >= 0; i--) {
        if (a->w[i] != b->w[i]) return a->w[i] < b->w[i] ? -1 : 1;
    }
    return 0;
}
static int big_is_zero(const big* a) {
    for (int i = 0; i < ORC_LIMBS; i++) if (a->w[i]) return 0;
    return 1;
}
static int big_bits(const big* a) {
    for (int i = ORC_LIMBS - 1; i >= 0; i--)
        if (a->w[i]) return 64 * i + 64 - __builtin_clzll(a->w[i]);
    return 0;
}
static int big_bit(const big* a, int i) { return (int)((a->w[i >> 6] >> (i & 63)) & 1); }
static u64 big_add(big* r, const big* a, const big* b) {
    u64 c = 0;
    for (int i = 0; i < ORC_LIMBS; i++) {
        u128 s = (u128)a->w[i] + b->w[i] + c;
        r->w[i] = (u64)s; c = (u64)(s >> 64);
    }
    return c;
}
static u64 big_sub(big* r, const big* a, const big* b) {
    u64 br = 0;
    for (int i = 0; i < ORC_LIMBS; i++) {
        u128 d = (u128)a->w[i] - b->w[i] - br;
        r->w[i] = (u64)d; br = (u64)(d >> 64) & 1;
    }
    return br;
}
static void big_add_u64(big* r, const big* a, u64 v) { big t; big_set_u64(&t, v); big_add(r, a, &t); }
static void big_sub_u64(big* r, const big* a, u64 v) { big t; big_set_u64(&t, v); big_sub(r, a, &t); }
static void big_shr1(big* a) {
    for (int i = 0; i < ORC_LIMBS; i++) {
        u64 hi = (i + 1 < ORC_LIMBS) ? a->w[i + 1] : 0;
        a->w[i] = (a->w[i] >> 1) | (hi << 63);
    }
}
static u64 big_shl1(big* a) {
    u64 out = a->w[ORC_LIMBS - 1] >> 63;
    for (int i = ORC_LIMBS - 1; i > 0; i--) a->w[i] = (a->w[i] << 1) | (a->w[i - 1] >> 63);
    a->w[0] <<= 1;
    return out;
}
static u32 big_mod_u32(const big* a, u32 q) {
    u128 r = 0;
    for (int i = ORC_LIMBS - 1; i >= 0; i--) r = ((r << 64) | a->w[i]) % q;
    return (u32)r;
}

/* (a + b) mod n, a, b < n */
static void addmod(big* r, const big* a, const big* b, const big* n) {
    big t;
    u64 c = big_add(&t, a, b);
    if (c || big_cmp(&t, n) >= 0) big_sub(&t, &t, n);
    *r = t;
}
static void submod(big* r, const big* a, const big* b, const big* n) {
    big t;
    if (big_sub(&t, a, b)) big_add(&t, &t, n);
    *r = t;
}

/* (a * b) mod n by double-and-add over the bits of b: slow, obviously right.
 * Requires a, b < n and n < 2^(64*ORC_LIMBS - 1). */
static void mulmod(big* r, const big* a, const big* b, const big* n) {
    big acc; big_set_u64(&acc, 0);
    for (int i = big_bits(b) - 1; i >= 0; i--) {
        big_shl1(&acc);
        if (big_cmp(&acc, n) >= 0) big_sub(&acc, &acc, n);
        if (big_bit(b, i)) addmod(&acc, &acc, a, n);
    }
    *r = acc;
}

/* a mod n for arbitrary a (shift-subtract) */
static void big_mod(big* r, const big* a, const big* n) {
    big rem; big_set_u64(&rem, 0);
    for (int i = big_bits(a) - 1; i >= 0; i--) {
        big_shl1(&rem);
        rem.w[0] |= (u64)big_bit(a, i);
        if (big_cmp(&rem, n) >= 0) big_sub(&rem, &rem, n);
    }
    *r = rem;
}

static void powmod(big* r, const big* b, const big* e, const big* n) {
    big acc, x;
    big_set_u64(&acc, 1);
    if (big_cmp(&acc, n) >= 0) big_set_u64(&acc, 0);
    big_mod(&x, b, n);
    for (int i = big_bits(e) - 1; i >= 0; i--) {
        mulmod(&acc, &acc, &acc, n);
        if (big_bit(e, i)) mulmod(&acc, &acc, &x, n);
    }
    *r = acc;
}

/* strong probable-prime test to base a (n odd, n > a) */
static int strong_prp(const big* n, u64 a) {
    big nm1, d, x, one, base;
    big_sub_u64(&nm1, n, 1);
    d = nm1;
    int s = 0;
    while ((d.w[0] & 1) == 0) { big_shr1(&d); s++; }
    big_set_u64(&base, a);
    big_set_u64(&one, 1);
    powmod(&x, &base, &d, n);
    if (big_cmp(&x, &one) == 0 || big_cmp(&x, &nm1) == 0) return 1;
    for (int i = 1; i < s; i++) {
        mulmod(&x, &x, &x, n);
        if (big_cmp(&x, &nm1) == 0) return 1;
        if (big_cmp(&x, &one) == 0) return 0;
    }
    return 0;
}

/* v13 gpu_is_prime semantics (v13:1428-1452): small cases, trial division by
 * {3..71}, then strong-PRP for every witness in the list. */
static const u64 V13_SMALL[19] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71};
static int is_prime_mr(const big* n, const u64* wit, int nw) {
    int bits = big_bits(n);
    if (bits <= 64) {
        u64 v = n->w[0];
        if (v < 2) return 0;
        if (v == 2 || v == 3) return 1;
        if ((v & 1) == 0) return 0;
        if (v < 9) return 1;
    }
    if ((n->w[0] & 1) == 0) return 0;
    for (int i = 0; i < 19; i++) {
        if (big_mod_u32(n, (u32)V13_SMALL[i]) == 0)
            return (bits <= 64 && n->w[0] == V13_SMALL[i]) ? 1 : 0;
    }
    for (int i = 0; i < nw; i++)
        if (!strong_prp(n, wit[i])) return 0;
    return 1;
}

/* Jacobi symbol (a / n), n odd positive, a signed small */
static int jacobi_small(long long a, const big* n) {
    u64 nm = 0;
    /* reduce: (a/n) with |a| small: use reciprocity on (n mod |a|) */
    int sign = 1;
    if (a < 0) {
        a = -a;
        /* (-1/n) = (-1)^((n-1)/2) */
        if ((n->w[0] & 3) == 3) sign = -sign;
    }
    u64 aa = (u64)a;
    while (aa && (aa & 1) == 0) {
        aa >>= 1;
        u64 r8 = n->w[0] & 7;
        if (r8 == 3 || r8 == 5) sign = -sign;
    }
    if (aa == 0) return 0;
    if (aa == 1) return sign;
    /* (aa / n) = (n / aa) * (-1)^((aa-1)/2 (n-1)/2) */
    if ((aa & 3) == 3 && (n->w[0] & 3) == 3) sign = -sign;
    nm = big_mod_u32(n, (u32)aa);
    /* now small Jacobi (nm / aa) */
    u64 x = nm, y = aa;
    while (x) {
        while ((x & 1) == 0) {
            x >>= 1;
            if ((y & 7) == 3 || (y & 7) == 5) sign = -sign;
        }
        u64 t = x; x = y; y = t;
        if ((x & 3) == 3 && (y & 3) == 3) sign = -sign;
        x %= y;
    }
    return y == 1 ? sign : 0;
}

static int big_is_square(const big* n) {
    /* integer sqrt by bisection on bits; fine for <= 256-bit oracle inputs */
    int bits = big_bits(n);
    big lo, hi, mid, sq, one;
    big_set_u64(&lo, 0);
    big_set_u64(&hi, 0);
    int hb = bits / 2 + 1;
    hi.w[hb >> 6] |= 1ull << (hb & 63);
    big_set_u64(&one, 1);
    while (big_cmp(&lo, &hi) < 0) {
        big_add(&mid, &lo, &hi);
        big_add_u64(&mid, &mid, 1);
        big_shr1(&mid);
        /* sq = mid^2 (no modulus) via shift-add */
        big_set_u64(&sq, 0);
        int overflow = 0;
        for (int i = big_bits(&mid) - 1; i >= 0; i--) {
            if (big_shl1(&sq)) overflow = 1;
            if (big_bit(&mid, i) && big_add(&sq, &sq, &mid)) overflow = 1;
        }
        if (!overflow && big_cmp(&sq, n) <= 0) lo = mid;
        else big_sub(&hi, &mid, &one);
    }
    big_set_u64(&sq, 0);
    for (int i = big_bits(&lo) - 1; i >= 0; i--) {
        big_shl1(&sq);
        if (big_bit(&lo, i)) big_add(&sq, &sq, &lo);
    }
    return big_cmp(&sq, n) == 0;
}

/* halve x mod n (n odd) */
static void halfmod(big* x, const big* n) {
    if (x->w[0] & 1) {
        u64 c = big_add(x, x, n);
        big_shr1(x);
        if (c) x->w[ORC_LIMBS - 1] |= 1ull << 63;
    } else {
        big_shr1(x);
    }
}

/* strong Lucas probable-prime test with Selfridge's method A parameters:
 * D in 5, -7, 9, -11, ... first with (D/n) = -1, P = 1, Q = (1 - D)/4. */
static int strong_lucas(const big* n) {
    long long D = 5;
    int guard = 0;
    for (;;) {
        int j = jacobi_small(D, n);
        if (j == -1) break;
        if (j == 0) {
            /* gcd(D, n) > 1: n composite unless n == |D| */
            big t; big_set_u64(&t, (u64)(D < 0 ? -D : D));
            return big_cmp(&t, n) == 0;
        }
        D = D > 0 ? -(D + 2) : -(D - 2);
        if (++guard == 20 && big_is_square(n)) return 0;
    }
    long long Qs = (1 - D) / 4;
    big Dm, Qm, d;
    /* D mod n, Q mod n (n > |D|, |Q| for all inputs that reach here) */
    if (D >= 0) big_set_u64(&Dm, (u64)D);
    else { big t; big_set_u64(&t, (u64)(-D)); big_sub(&Dm, n, &t); }
    if (Qs >= 0) big_set_u64(&Qm, (u64)Qs);
    else { big t; big_set_u64(&t, (u64)(-Qs)); big_sub(&Qm, n, &t); }
    /* n + 1 = d * 2^s */
    big_add_u64(&d, n, 1);
    int s = 0;
    while ((d.w[0] & 1) == 0) { big_shr1(&d); s++; }
    /* left-to-right binary ladder over d: U_k, V_k, Q^k */
    big U, V, Qk, t1, t2;
    big_set_u64(&U, 1);          /* U_1 */
    big_set_u64(&V, 1);          /* V_1 = P = 1 */
    Qk = Qm;                     /* Q^1 */
    for (int i = big_bits(&d) - 2; i >= 0; i--) {
        /* double: U_2k = U V, V_2k = V^2 - 2 Q^k, Q^2k */
        mulmod(&U, &U, &V, n);
        mulmod(&t1, &V, &V, n);
        addmod(&t2, &Qk, &Qk, n);
        submod(&V, &t1, &t2, n);
        mulmod(&Qk, &Qk, &Qk, n);
        if (big_bit(&d, i)) {
            /* increment: U_{k+1} = (P U + V)/2, V_{k+1} = (D U + P V)/2 */
            big nu, nv;
            addmod(&nu, &U, &V, n);
            halfmod(&nu, n);
            mulmod(&t1, &Dm, &U, n);
            addmod(&nv, &t1, &V, n);
            halfmod(&nv, n);
            U = nu; V = nv;
            mulmod(&Qk, &Qk, &Qm, n);
        }
    }
    if (big_is_zero(&U) || big_is_zero(&V)) return 1;
    for (int r = 1; r < s; r++) {
        mulmod(&t1, &V, &V, n);
        addmod(&t2, &Qk, &Qk, n);
        submod(&V, &t1, &t2, n);
        if (big_is_zero(&V)) return 1;
        mulmod(&Qk, &Qk, &Qk, n);
    }
    return 0;
}

/* Baillie-PSW: small-prime trial division, strong PRP base 2, strong Lucas. */
static const u32 SMALL_PRIMES[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53,
                                   59, 61, 67, 71, 73, 79, 83, 89, 97};
static int is_prime_bpsw(const big* n) {
    int bits = big_bits(n);
    if (bits <= 1) return 0;
    for (unsigned i = 0; i < sizeof(SMALL_PRIMES) / sizeof(SMALL_PRIMES[0]); i++) {
        u32 p = SMALL_PRIMES[i];
        if (bits <= 32 && n->w[0] == p) return 1;
        if (big_mod_u32(n, p) == 0) return 0;
    }
    if (bits <= 32 && n->w[0] < 97 * 97) return 1;
    if (!strong_prp(n, 2)) return 0;
    return strong_lucas(n);
}

/* ------------------------------------------------------------------------ */
/* predicates exported for tests                                             */
/* ------------------------------------------------------------------------ */

static void big_from_words(big* a, const u64* w, int nw) {
    memset(a, 0, sizeof(*a));
    for (int i = 0; i < nw && i < ORC_LIMBS; i++) a->w[i] = w[i];
}

int orc_is_prime_mr(const u64* n_words, int nw, const u64* wit, int n_wit) {
    big n; big_from_words(&n, n_words, nw);
    return is_prime_mr(&n, wit, n_wit);
}
int orc_is_prime_bpsw(const u64* n_words, int nw) {
    big n; big_from_words(&n, n_words, nw);
    return is_prime_bpsw(&n);
}
int orc_strong_prp(const u64* n_words, int nw, u64 a) {
    big n; big_from_words(&n, n_words, nw);
    return strong_prp(&n, a);
}
void orc_powmod(const u64* b, const u64* e, const u64* m, int nw, u64* out) {
    big B, E, Mo, R;
    big_from_words(&B, b, nw); big_from_words(&E, e, nw); big_from_words(&Mo, m, nw);
    powmod(&R, &B, &E, &Mo);
    memcpy(out, R.w, sizeof(u64) * (size_t)nw);
}

/* ------------------------------------------------------------------------ */
/* chain semantics                                                           */
/* ------------------------------------------------------------------------ */

enum { ORC_PRIME_MR = 0, ORC_PRIME_BPSW = 1 };

typedef struct {
    int primality;       /* ORC_PRIME_MR | ORC_PRIME_BPSW */
    const u64* wit;
    int n_wit;
} orc_pred;

static int is_prime_p(const big* n, const orc_pred* p) {
    if (p->primality == ORC_PRIME_BPSW) return is_prime_bpsw(n);
    return is_prime_mr(n, p->wit, p->n_wit);
}

/* forward walk p -> 2p + 1 (second kind: 2p - 1) while prime, counting p
 * itself (v13:1873-1881, v13b:1878-1886) */
static int walk_forward(const big* root, const orc_pred* p) {
    int len = 1;
    big cur = *root, nx;
    while (len < ORC_MAX_CHAIN) {
        nx = cur;
        big_shl1(&nx);
        if (g_kind == 2) big_sub_u64(&nx, &nx, 1);
        else big_add_u64(&nx, &nx, 1);
        if (!is_prime_p(&nx, p)) break;
        len++;
        cur = nx;
    }
    return len;
}

/* Length of the chain started at the given number (config-3 semantics: the
 * number is walked as given, 0 when it is not prime). */
int orc_chain_from(const u64* n_words, int nw, int primality, const u64* wit, int n_wit) {
    big n; big_from_words(&n, n_words, nw);
    orc_pred p = {primality, wit, n_wit};
    if (!is_prime_p(&n, &p)) return 0;
    return walk_forward(&n, &p);
}

/* Prove one survivor.  mode 0 = reference GPU K2 (v13:1479-1537): 132-prime
 * trial division, root check drops non-roots, forward walk.  mode 1 =
 * reference CPU prover (v13:1819-1881): 62-prime trial division, backward walk
 * to the true root, forward walk from there.
 * Returns -1 when the survivor yields no chain record, else the chain length;
 * root_out (ORC_LIMBS words) receives the chain root, flags bit0 = survivor
 * was itself the root. */
static const u32 CHAIN_SCREEN[132] = {
    67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113, 127, 131, 137, 139, 149, 151,
    157, 163, 167, 173, 179, 181, 191, 193, 197, 199, 211, 223, 227, 229, 233, 239, 241,
    251, 257, 263, 269, 271, 277, 281, 283, 293, 307, 311, 313, 317, 331, 337, 347, 349,
    353, 359, 367, 373, 379, 383, 389, 397, 401, 409, 419, 421, 431, 433, 439, 443, 449,
    457, 461, 463, 467, 479, 487, 491, 499, 503, 509, 521, 523, 541, 547, 557, 563, 569,
    571, 577, 587, 593, 599, 601, 607, 613, 617, 619, 631, 641, 643, 647, 653, 659, 661,
    673, 677, 683, 691, 701, 709, 719, 727, 733, 739, 743, 751, 757, 761, 769, 773, 787,
    797, 809, 811, 821, 823, 827, 829, 839, 853, 857, 859, 863};

int orc_prove_n(const u64* n_words, int nw, int bits, int mode, int primality,
                const u64* wit, int n_wit, u64* root_out, int* flags, int* is_prime_out) {
    big n; big_from_words(&n, n_words, nw);
    orc_pred p = {primality, wit, n_wit};
    *flags = 0;
    *is_prime_out = 0;
    if (big_bits(&n) != bits) return -1;
    int ntd = (mode == 0) ? 132 : 62;
    for (int i = 0; i < ntd; i++)
        if (big_mod_u32(&n, CHAIN_SCREEN[i]) == 0) return -1;
    if (!is_prime_p(&n, &p)) return -1;
    *is_prime_out = 1;
    big pred, root = n, two;
    big_set_u64(&two, 2);
    /* predecessor (n - 1) / 2; second kind (n + 1) / 2 (v13b:1522, 1860) */
    if (g_kind == 2) big_add_u64(&pred, &n, 1); else big_sub_u64(&pred, &n, 1);
    big_shr1(&pred);
    int is_root = 1;
    if (big_cmp(&pred, &two) >= 0 && is_prime_p(&pred, &p)) {
        is_root = 0;
        if (mode == 0) return -1;      /* K2 emits roots only (v13:1513-1516) */
        root = pred;
        int back = 0;
        while (back < ORC_MAX_CHAIN) {
            if (g_kind == 2) big_add_u64(&pred, &root, 1); else big_sub_u64(&pred, &root, 1);
            big_shr1(&pred);
            if (big_cmp(&pred, &two) < 0) break;
            if (!is_prime_p(&pred, &p)) break;
            root = pred;
            back++;
        }
    }
    int len = walk_forward(&root, &p);
    memcpy(root_out, root.w, sizeof(u64) * ORC_LIMBS);
    *flags = is_root ? 1 : 0;
    return len;
}

/* ---- the reference CPU engine's own tests (v33), first kind ------------ */

/* is_prime_root_native (v33:1326-1339): 2, 3, 5 prime, even composite, then
 * strong PRP to bases 2, 3 and 5 */
static int v33_root_test(const big* n) {
    if (big_bits(n) <= 3) {
        u64 v = n->w[0];
        if (v == 2 || v == 3 || v == 5) return 1;
        if (v != 7) return 0;
    }
    if (!(n->w[0] & 1)) return 0;
    return strong_prp(n, 2) && strong_prp(n, 3) && strong_prp(n, 5);
}

/* is_prime_pocklington_native (v33:1290-1302): n <= 5 -> n in {2, 3, 5};
 * else 2^(n-1) == 1 (mod n) */
static int v33_fermat2(const big* n) {
    if (big_bits(n) <= 3 && n->w[0] <= 5) return n->w[0] == 2 || n->w[0] == 3 || n->w[0] == 5;
    big e, two, r, one;
    big_sub_u64(&e, n, 1);
    big_set_u64(&two, 2);
    big_set_u64(&one, 1);
    powmod(&r, &two, &e, n);
    return big_cmp(&r, &one) == 0;
}

/* follow_chain_first_screened / its wide twin from a known-prime root
 * (v33:1512-1577, 1594-1656): a link of more than cap bits ends the walk,
 * then a zero residue mod any chain-screen prime, then the link test
 * (Fermat base 2 on the native path, Baillie-PSW on the wide one) */
static int v33_walk(const big* root, int wide, int cap_bits) {
    int len = 1;
    big cur = *root, nx;
    while (len < ORC_MAX_CHAIN) {
        nx = cur;
        big_shl1(&nx);
        big_add_u64(&nx, &nx, 1);
        if (big_bits(&nx) > cap_bits) break;
        int comp = 0;
        for (int i = 0; i < 132 && !comp; i++) comp = big_mod_u32(&nx, CHAIN_SCREEN[i]) == 0;
        if (comp) break;
        if (!(wide ? is_prime_bpsw(&nx) : v33_fermat2(&nx))) break;
        len++;
        cur = nx;
    }
    return len;
}

/* One survivor through the reference CPU engine's proving path
 * (worker_sequential, v33:2112-2215; wide path v33:1982-2098): trial division
 * by 101..409, root test (native: v33_root_test; wide, bits + target > 127:
 * Baillie-PSW), backward walk with Baillie-PSW from n, at most MAX_CHAIN
 * steps (is_chain_root_first / follow_chain_backward_first, v33:1489-1495,
 * 1665-1676), forward walk from the root (v33_walk; cap 2^127 native,
 * 2^(bits + 2 target) wide).  Returns -1 when the survivor yields no
 * record, else the chain length. */
int orc_prove_v33(const u64* n_words, int nw, int bits, int target, u64* root_out, int* flags,
                  int* is_prime_out) {
    big n; big_from_words(&n, n_words, nw);
    *flags = 0;
    *is_prime_out = 0;
    if (big_bits(&n) != bits) return -1;
    for (int i = 7; i < 62; i++)
        if (big_mod_u32(&n, CHAIN_SCREEN[i]) == 0) return -1;
    const int wide = bits + target > 127;
    const int cap = wide ? bits + 2 * target : 127;
    if (!(wide ? is_prime_bpsw(&n) : v33_root_test(&n))) return -1;
    *is_prime_out = 1;
    big pred, root = n, two;
    big_set_u64(&two, 2);
    for (int steps = 0; steps < ORC_MAX_CHAIN; steps++) {
        big_sub_u64(&pred, &root, 1);
        big_shr1(&pred);
        if (big_cmp(&pred, &two) < 0) break;
        if (!is_prime_bpsw(&pred)) break;
        root = pred;
    }
    const int is_root = big_cmp(&root, &n) == 0;
    int len = v33_walk(&root, wide, cap);
    memcpy(root_out, root.w, sizeof(u64) * ORC_LIMBS);
    *flags = is_root ? 1 : 0;
    return len;
}

/* The walk of a given number under those rules (follow_chain_first: the
 * number itself by Baillie-PSW, v33:1535-1540): 0 when it is not prime */
int orc_chain_from_v33(const u64* n_words, int nw, int wide, int cap_bits) {
    big n; big_from_words(&n, n_words, nw);
    if (!is_prime_bpsw(&n)) return 0;
    return v33_walk(&n, wide, cap_bits);
}

/* n = ((tile_start + tile_idx) * WP + k) * M + base as ORC_LIMBS words */
void orc_reconstruct(const orc_lattice* L, u64 ts_lo, u64 ts_hi, u32 base_idx, u32 k,
                     u32 tile_idx, u64* out) {
    u128 tile = (((u128)ts_hi << 64) | ts_lo) + tile_idx;
    /* full_k = tile*WP + k may exceed 128 bits only for absurd tiles; keep
     * the whole product in big arithmetic */
    big t, acc, wp;
    memset(&t, 0, sizeof(t));
    t.w[0] = (u64)tile; t.w[1] = (u64)(tile >> 64);
    big_set_u64(&wp, L->WP);
    big_set_u64(&acc, 0);
    for (int i = big_bits(&wp) - 1; i >= 0; i--) {
        big_shl1(&acc);
        if (big_bit(&wp, i)) big_add(&acc, &acc, &t);
    }
    big_add_u64(&acc, &acc, k);
    big m, prod;
    big_set_u64(&m, L->M);
    big_set_u64(&prod, 0);
    for (int i = big_bits(&m) - 1; i >= 0; i--) {
        big_shl1(&prod);
        if (big_bit(&m, i)) big_add(&prod, &prod, &acc);
    }
    big_add_u64(&prod, &prod, L->bases[base_idx]);
    memcpy(out, prod.w, sizeof(u64) * ORC_LIMBS);
}

/* ------------------------------------------------------------------------
 * Fingerprint-pool Q iteration (experimental/cc20_first_kind_immune_v16.cu)
 *   p_0 = Q * D_V * 2^E - 1,  p_j = 2^(E+j) * Q * D_V - 1.
 * ------------------------------------------------------------------------ */
static u32 orc_inv_mod(u32 a, u32 q) {
    long long t = 0, nt = 1, r = q, nr = a % q;
    while (nr) {
        long long f = r / nr, x;
        x = t - f * nt; t = nt; nt = x;
        x = r - f * nr; r = nr; nr = x;
    }
    return (u32)(t < 0 ? t + q : t);
}

static u32 orc_pow2_mod(int e, u32 q) {
    u64 r = 1 % q;
    for (int i = 0; i < e; i++) r = (r * 2) % q;
    return (u32)r;
}

/* Forbidden residues of Q mod q (v16:1244-1266): inv(D mod q) * inv(2^(E+j))
 * for j < depth, deduplicated, in order of first appearance.  Returns the
 * count, 0 when q divides D (immune: the prime sieves nothing). */
int orc_qiter_forbidden(u32 q, u64 d_lo, u64 d_hi, int E, int depth, u32* out) {
    u128 D = ((u128)d_hi << 64) | d_lo;
    u32 dm = (u32)(D % q);
    if (dm == 0) return 0;
    u32 inv_d = orc_inv_mod(dm, q);
    int n = 0;
    for (int j = 0; j < depth; j++) {
        u32 r = (u32)((u64)inv_d * orc_inv_mod(orc_pow2_mod(E + j, q), q) % q);
        int dup = 0;
        for (int k = 0; k < n; k++) if (out[k] == r) { dup = 1; break; }
        if (!dup) out[n++] = r;
    }
    return n;
}

/* Survivors of one segment Q = q_base + off, off < n_q, in increasing off
 * (the per-Q probe of v16_q_iter_kernel, v16:2104-2134, every prime whose
 * mask is non-empty).  Residues are advanced by one per Q.  Returns the
 * survivor count; offsets beyond cap are counted, not written. */
u64 orc_qiter_filter_seg(u64 qb_lo, u64 qb_hi, u32 n_q, u64 d_lo, u64 d_hi, int E, int depth,
                         const u32* primes, int n_primes, u32* out, u64 cap) {
    u128 qb = ((u128)qb_hi << 64) | qb_lo;
    unsigned char** bad = calloc((size_t)n_primes, sizeof(unsigned char*));
    u32* res = calloc((size_t)n_primes, sizeof(u32));
    u32* fb = malloc(sizeof(u32) * (size_t)(depth > 0 ? depth : 1));
    int* act = malloc(sizeof(int) * (size_t)(n_primes > 0 ? n_primes : 1));
    int n_act = 0;
    for (int i = 0; i < n_primes; i++) {
        int n = orc_qiter_forbidden(primes[i], d_lo, d_hi, E, depth, fb);
        if (n == 0) continue;
        bad[i] = calloc(primes[i], 1);
        for (int k = 0; k < n; k++) bad[i][fb[k]] = 1;
        res[i] = (u32)(qb % primes[i]);
        act[n_act++] = i;
    }
    u64 cnt = 0;
    for (u64 off = 0; off < n_q; off++) {
        int ok = 1;
        for (int a = 0; a < n_act; a++) {
            int i = act[a];
            if (bad[i][res[i]]) { ok = 0; break; }
        }
        if (ok) {
            if (cnt < cap) out[cnt] = (u32)off;
            cnt++;
        }
        for (int a = 0; a < n_act; a++) {
            int i = act[a];
            if (++res[i] == primes[i]) res[i] = 0;
        }
    }
    for (int i = 0; i < n_primes; i++) free(bad[i]);
    free(bad); free(res); free(fb); free(act);
    return cnt;
}

/* Prove one q-iteration survivor (the q-iter path of cpu_prove_worker,
 * v16:2540-2722): p_0 from (Q, D_V, E); with reverse != 0 chain position
 * target - 1 must be prime first (v16:2658-2673); p_0 prime (counted in
 * *is_prime_out); root check on (p_0 - 1)/2 (v16:2693-2711; the birth
 * certificate there only skips a test whose answer is already known);
 * mode 0 drops non-roots, mode 1 walks back to the true root; forward walk.
 * Returns the chain length or -1 when there is no record. */
int orc_qiter_prove(u64 q_lo, u64 q_hi, u64 d_lo, u64 d_hi, int E, int target, int reverse, int mode,
                    int primality, const u64* wit, int n_wit, u64* root_out, int* flags,
                    int* is_prime_out) {
    orc_pred pr = {primality, wit, n_wit};
    big Q, D, n, two;
    memset(&Q, 0, sizeof(Q)); memset(&D, 0, sizeof(D));
    Q.w[0] = q_lo; Q.w[1] = q_hi;
    D.w[0] = d_lo; D.w[1] = d_hi;
    big_set_u64(&n, 0);
    for (int i = big_bits(&D) - 1; i >= 0; i--) {          /* n = Q * D, shift-add */
        big_shl1(&n);
        if (big_bit(&D, i)) big_add(&n, &n, &Q);
    }
    for (int i = 0; i < E; i++) big_shl1(&n);
    big_sub_u64(&n, &n, 1);
    *flags = 0;
    *is_prime_out = 0;
    if (reverse && target > 1) {
        big top = n;
        for (int k = 0; k < target - 1; k++) { big_shl1(&top); big_add_u64(&top, &top, 1); }
        if (!is_prime_p(&top, &pr)) return -1;
    }
    if (!is_prime_p(&n, &pr)) return -1;
    *is_prime_out = 1;
    big pred, root = n;
    big_set_u64(&two, 2);
    big_sub_u64(&pred, &n, 1);
    big_shr1(&pred);
    int is_root = 1;
    if (big_cmp(&pred, &two) >= 0 && is_prime_p(&pred, &pr)) {
        is_root = 0;
        if (mode == 0) return -1;
        root = pred;
        for (int back = 0; back < ORC_MAX_CHAIN; back++) {
            big_sub_u64(&pred, &root, 1);
            big_shr1(&pred);
            if (big_cmp(&pred, &two) < 0) break;
            if (!is_prime_p(&pred, &pr)) break;
            root = pred;
        }
    }
    int len = walk_forward(&root, &pr);
    memcpy(root_out, root.w, sizeof(u64) * ORC_LIMBS);
    *flags = is_root ? 1 : 0;
    return len;
}
