/*
 * In-process harness around the reference's CPU/GMP engine v33
 * (src/cpu/cc_gmp_v33_03.c), compiled from the reference source where it
 * lies.  TEST INFRASTRUCTURE ONLY: exposes its lattice builder (v33:636-793),
 * filter tables (v33:799-962), native Montgomery Miller-Rabin
 * (v33:1238-1274), GMP predicates (v33:1345-1362, 1489-1495) and chain
 * walkers (v33:1511-1690), plus GMP's own mpz_probab_prime_p, so the tests can
 * pin the oracle against the reference and against GMP 6.3.0 itself.
 */
#define main v33_reference_main
#include "cc_gmp_v33_03.c"
#undef main

int ref33_setup(int target, int line_depth) {
    g_quiet_mode = 1;
    generate_optimized_wheels(target);
    compute_filter_bitmasks(target > MAX_SIEVE_CHAIN_LEN ? MAX_SIEVE_CHAIN_LEN : target);
    init_prefilter_tables();
    init_trial_batches();
    g_line_depth = line_depth;
    if (g_line_depth > target - 1) g_line_depth = target - 1;
    init_line_sieve(g_line_depth);
    return g_num_bases;
}

int ref33_num_bases(void) { return g_num_bases; }
unsigned long long ref33_base(int b) { return g_base_wheels[b].base; }
unsigned ref33_tkm6(int b) { return g_base_wheels[b].target_k_mod6; }
int ref33_bucket_size(int b, int m) { return g_base_wheels[b].wheel_size_by_mod6[m]; }
void ref33_bucket(int b, int m, unsigned* out) {
    memcpy(out, g_base_wheels[b].wheel_by_mod6[m], sizeof(u32) * g_base_wheels[b].wheel_size_by_mod6[m]);
}
unsigned long long ref33_l2_mask(int p_idx, int L) { return g_filter_mask_first[p_idx][L]; }
int ref33_ext(int p_idx, int L, int r) { return g_ext_filter_first[p_idx][L][r]; }
int ref33_line_kill(int idx, int r) { return g_line_kill_first[idx][r]; }
int ref33_line_depth(void) { return g_line_depth; }

/* GMP 6.3.0 mpz_probab_prime_p(n, reps) on a hex string */
int ref33_gmp_probab_prime(const char* hex, int reps) {
    mpz_t n; mpz_init(n);
    mpz_set_str(n, hex, 16);
    int r = mpz_probab_prime_p(n, reps);
    mpz_clear(n);
    return r;
}

/* GMP powm: writes hex of b^e mod m into out (size >= 130) */
void ref33_gmp_powm(const char* b, const char* e, const char* m, char* out) {
    mpz_t B, E, Mo, R;
    mpz_init(B); mpz_init(E); mpz_init(Mo); mpz_init(R);
    mpz_set_str(B, b, 16); mpz_set_str(E, e, 16); mpz_set_str(Mo, m, 16);
    mpz_powm(R, B, E, Mo);
    mpz_get_str(out, 16, R);
    mpz_clear(B); mpz_clear(E); mpz_clear(Mo); mpz_clear(R);
}

/* v33 native Montgomery strong-PRP (n < 2^127, odd) */
int ref33_mr_mont(unsigned long long lo, unsigned long long hi, unsigned long long a) {
    u128 n = ((u128)hi << 64) | lo;
    MontCtx ctx;
    mont_ctx_init(&ctx, n);
    return miller_rabin_mont(n, a, &ctx);
}

int ref33_is_prime_fast(const char* hex) {
    mpz_t n, t; mpz_init(n); mpz_init(t);
    mpz_set_str(n, hex, 16);
    int r = is_prime_fast(n, t);
    mpz_clear(n); mpz_clear(t);
    return r;
}

/* get_full_chain_length (backward walk + forward walk, GMP wide mode so no
 * 2^127 cap): writes the root hex into root_out, returns the length */
int ref33_full_chain(const char* hex, char* root_out) {
    mpz_t n, maxv, root, pred, cur, t, t2, pp;
    mpz_init(n); mpz_init(maxv); mpz_init(root); mpz_init(pred);
    mpz_init(cur); mpz_init(t); mpz_init(t2); mpz_init(pp);
    mpz_set_str(n, hex, 16);
    mpz_ui_pow_ui(maxv, 2, 400);
    int saved = g_wide_mode;
    g_wide_mode = 1;
    int len = get_full_chain_length(n, maxv, root, pred, cur, t, t2, pp);
    g_wide_mode = saved;
    mpz_get_str(root_out, 16, root);
    mpz_clear(n); mpz_clear(maxv); mpz_clear(root); mpz_clear(pred);
    mpz_clear(cur); mpz_clear(t); mpz_clear(t2); mpz_clear(pp);
    return len;
}

/* follow_chain_first_gmp from the number as given (forward only, BPSW) */
int ref33_forward_chain(const char* hex) {
    mpz_t n, maxv, cur, t, t2, pp;
    mpz_init(n); mpz_init(maxv); mpz_init(cur); mpz_init(t); mpz_init(t2); mpz_init(pp);
    mpz_set_str(n, hex, 16);
    mpz_ui_pow_ui(maxv, 2, 400);
    int len = follow_chain_first_gmp(n, maxv, cur, t, t2, pp);
    mpz_clear(n); mpz_clear(maxv); mpz_clear(cur); mpz_clear(t); mpz_clear(t2); mpz_clear(pp);
    return len;
}

int ref33_is_root(const char* hex) {
    mpz_t n, p, t; mpz_init(n); mpz_init(p); mpz_init(t);
    mpz_set_str(n, hex, 16);
    int r = is_chain_root_first(n, p, t);
    mpz_clear(n); mpz_clear(p); mpz_clear(t);
    return r;
}

/* Forward walk exactly as the reference CPU prover does it (v13:1870-1881):
 * count n, then 2p+1 while mpz_probab_prime_p(., 1) != 0, up to MAX_CHAIN.
 * Returns 0 when n itself is not prime. */
int ref_gmp_forward_chain(const char* hex) {
    mpz_t cur, t; mpz_init(cur); mpz_init(t);
    mpz_set_str(cur, hex, 16);
    int len = 0;
    if (mpz_probab_prime_p(cur, 1) != 0) {
        len = 1;
        while (len < MAX_CHAIN) {
            mpz_mul_2exp(t, cur, 1);
            mpz_add_ui(t, t, 1);
            if (mpz_probab_prime_p(t, 1) == 0) break;
            len++;
            mpz_set(cur, t);
        }
    }
    mpz_clear(cur); mpz_clear(t);
    return len;
}

/* The same walk for second-kind chains (p -> 2p - 1), the v13b CPU prover's
 * loop (v13b:1878-1888): count n, then 2p - 1 while mpz_probab_prime_p(., 1)
 * != 0, up to MAX_CHAIN.  Returns 0 when n itself is not prime. */
int ref_gmp_forward_chain2(const char* hex) {
    mpz_t cur, t; mpz_init(cur); mpz_init(t);
    mpz_set_str(cur, hex, 16);
    int len = 0;
    if (mpz_probab_prime_p(cur, 1) != 0) {
        len = 1;
        while (len < MAX_CHAIN) {
            mpz_mul_2exp(t, cur, 1);
            mpz_sub_ui(t, t, 1);
            if (mpz_probab_prime_p(t, 1) == 0) break;
            len++;
            mpz_set(cur, t);
        }
    }
    mpz_clear(cur); mpz_clear(t);
    return len;
}

/* ---- the native (u128) prove path of worker_sequential, per candidate ---- */

/* follow_chain_first_screened on the native path (v33:1512-1577) from n, cap
 * 2^127, no prefilter residues; root_known_prime as given (0: n is tested
 * with is_prime_fast first) */
int ref33_follow_native(unsigned long long lo, unsigned long long hi, int root_known_prime) {
    mpz_t n, maxv, cur, t, t2, pp;
    mpz_init(n); mpz_init(maxv); mpz_init(cur); mpz_init(t); mpz_init(t2); mpz_init(pp);
    u128_to_mpz(n, ((u128)hi << 64) | lo);
    mpz_ui_pow_ui(maxv, 2, 127);
    int len = follow_chain_first_screened(n, maxv, cur, t, t2, pp, NULL, root_known_prime, NULL, NULL);
    mpz_clear(n); mpz_clear(maxv); mpz_clear(cur); mpz_clear(t); mpz_clear(t2); mpz_clear(pp);
    return len;
}

int ref33_root_native(unsigned long long lo, unsigned long long hi) {
    return is_prime_root_native(((u128)hi << 64) | lo);
}

int ref33_fermat2_native(unsigned long long lo, unsigned long long hi) {
    u128 n = ((u128)hi << 64) | lo;
    MontCtx ctx;
    if (n > 5) mont_ctx_init(&ctx, n);
    return is_prime_pocklington_native(n, &ctx);
}

/* One candidate n (< 2^127) through the native proving path of
 * worker_sequential (v33:2112-2215) with the given log threshold: trial
 * division by 101..409, root test, root check, then the forward walk from n
 * (root) or the full chain from its true root (non-root).  Returns -1 when
 * trial division rejects n, 0 when the root test does, -2 when the
 * prefilter skips a root (its predicted ceiling is below log_threshold),
 * else the chain length; root_out receives the root's hex, *is_root the
 * root check.  Call ref33_setup first (trial batches, prefilter tables). */
int ref33_prove_native(unsigned long long lo, unsigned long long hi, int log_threshold, char* root_out,
                       int* is_root_out) {
    u128 n128 = ((u128)hi << 64) | lo;
    *is_root_out = 0;
    root_out[0] = 0;
    for (int tb = 0; tb < g_num_batches_extl2; tb++) {
        unsigned long r = (unsigned long)(n128 % g_trial_batches_extl2[tb].product);
        for (int j = 0; j < g_trial_batches_extl2[tb].count; j++)
            if (r % TRIAL_PRIMES[g_trial_batches_extl2[tb].start + j] == 0) return -1;
    }
    if (!is_prime_root_native(n128)) return 0;
    mpz_t n, pred, temp, temp2, root, cur, maxv, pp;
    mpz_init(n); mpz_init(pred); mpz_init(temp); mpz_init(temp2); mpz_init(root); mpz_init(cur);
    mpz_init(maxv); mpz_init(pp);
    mpz_ui_pow_ui(maxv, 2, 127);
    u128_to_mpz(n, n128);
    int saved = g_wide_mode;
    g_wide_mode = 0;
    int len;
    int is_root = is_chain_root_first(n, pred, temp);
    if (!is_root) {
        len = get_full_chain_length(n, maxv, root, pred, cur, temp, temp2, pp);
        mpz_get_str(root_out, 16, root);
    } else {
        u32 pf[PREFILTER_PRIMES_COUNT];
        int ceiling = prefilter_predict_ceiling(n, log_threshold, pf);
        if (ceiling < log_threshold) {
            len = -2;
        } else {
            len = follow_chain_first_screened(n, maxv, cur, temp, temp2, pp, pf, 1, NULL, NULL);
        }
        mpz_get_str(root_out, 16, n);
    }
    g_wide_mode = saved;
    *is_root_out = is_root;
    mpz_clear(n); mpz_clear(pred); mpz_clear(temp); mpz_clear(temp2); mpz_clear(root); mpz_clear(cur);
    mpz_clear(maxv); mpz_clear(pp);
    return len;
}
