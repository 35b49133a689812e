/*
 * In-process harness around the reference's v16 fingerprint-pool engine
 * (src/cuda/experimental/cc20_first_kind_immune_v16.cu), compiled from the
 * reference source where it lies.  TEST INFRASTRUCTURE ONLY: it exposes the
 * reference's forbidden-residue function (v16:1244-1266), builds one
 * variant's forbid mask and active-prime list the way its main() does
 * (v16:5104-5178, 5229-5299) and launches its v16_q_iter_kernel as the
 * dispatch loop does (v16:5807-5881, Q_per_thread = 16).  Built into
 * oracle/_ref/ by oracle/Makefile; never part of the product.
 */
#define main v16_reference_main
#include "cc20_first_kind_immune_v16.cu"
#undef main

extern "C" {

int ref16_forbidden(unsigned q, unsigned long long d_lo, unsigned long long d_hi, int E, int depth,
                    unsigned* out, int max_out) {
    u128 D = ((u128)d_hi << 64) | d_lo;
    return v16_forbidden_residues(q, D, E, depth, out, max_out);
}

/* One variant, one launch of n_q Q values from q_base; offsets of the
 * survivors (device order) into out; returns the raw device count. */
unsigned ref16_qiter_filter(const unsigned* primes, int n_qp, unsigned long long d_lo,
                            unsigned long long d_hi, int E, int depth, unsigned long long qb_lo,
                            unsigned long long qb_hi, unsigned n_q, unsigned* out, unsigned cap) {
    u128 D = ((u128)d_hi << 64) | d_lo;
    u128 Q_base = ((u128)qb_hi << 64) | qb_lo;
    BarrettQ qb[V16_MAX_SIEVE];
    u64 mask[V16_MAX_SIEVE * V16_Q_MASK_WORDS];
    u32 base_mod[V16_MAX_SIEVE];
    u8 active[V16_MAX_SIEVE];
    u32 n_act = 0;
    memset(mask, 0, sizeof(mask));
    for (int i = 0; i < n_qp; i++) {
        u32 q = primes[i];
        qb[i].q = q;
        qb[i].magic = barrett_magic_u32(q);
        base_mod[i] = (u32)(Q_base % (u128)q);
        u32 D_mod_q = (u32)(D % (u128)q);
        if (D_mod_q == 0) continue;
        for (int j = 0; j < depth; j++) {
            u32 p2 = pow2_mod_u32(E + j, q);
            u32 m = (u32)(((u64)D_mod_q * (u64)p2) % (u64)q);
            u32 inv = mod_inv_u32(m, q);
            mask[(size_t)i * V16_Q_MASK_WORDS + (inv >> 6)] |= (1ULL << (inv & 63u));
        }
        active[n_act++] = (u8)i;
    }
    u32 *d_primes, *d_base_mod, *d_count, *d_overflow;
    BarrettQ* d_qb;
    u64* d_mask;
    u8* d_act;
    QSurvivor* d_surv;
    unsigned long long *d_total, *d_pass;
    u32 surv_cap = V16_Q_MAX_SURVIVORS;
    CUDA_CHECK(cudaMalloc(&d_primes, n_qp * sizeof(u32)));
    CUDA_CHECK(cudaMalloc(&d_base_mod, n_qp * sizeof(u32)));
    CUDA_CHECK(cudaMalloc(&d_qb, n_qp * sizeof(BarrettQ)));
    CUDA_CHECK(cudaMalloc(&d_mask, (size_t)n_qp * V16_Q_MASK_WORDS * sizeof(u64)));
    CUDA_CHECK(cudaMalloc(&d_act, V16_MAX_SIEVE));
    CUDA_CHECK(cudaMalloc(&d_surv, (size_t)surv_cap * sizeof(QSurvivor)));
    CUDA_CHECK(cudaMalloc(&d_count, sizeof(u32)));
    CUDA_CHECK(cudaMalloc(&d_overflow, sizeof(u32)));
    CUDA_CHECK(cudaMalloc(&d_total, sizeof(unsigned long long)));
    CUDA_CHECK(cudaMalloc(&d_pass, sizeof(unsigned long long)));
    CUDA_CHECK(cudaMemcpy(d_primes, primes, n_qp * sizeof(u32), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_base_mod, base_mod, n_qp * sizeof(u32), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_qb, qb, n_qp * sizeof(BarrettQ), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_mask, mask, (size_t)n_qp * V16_Q_MASK_WORDS * sizeof(u64), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_act, active, V16_MAX_SIEVE, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemset(d_count, 0, sizeof(u32)));
    CUDA_CHECK(cudaMemset(d_overflow, 0, sizeof(u32)));
    CUDA_CHECK(cudaMemset(d_total, 0, sizeof(unsigned long long)));
    CUDA_CHECK(cudaMemset(d_pass, 0, sizeof(unsigned long long)));
    const u32 Q_per_thread = 16;
    u64 threads_needed = ((u64)n_q + Q_per_thread - 1) / Q_per_thread;
    u64 blocks = (threads_needed + V16_THREADS - 1) / V16_THREADS;
    if (blocks == 0) blocks = 1;
    v16_q_iter_kernel<<<(u32)blocks, V16_THREADS>>>(
        n_q, Q_per_thread, 0u, (u32)n_qp, d_primes, d_qb, d_mask, d_base_mod, (u32)depth,
        d_surv, d_count, surv_cap, d_total, d_pass, d_act, n_act, d_overflow);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaDeviceSynchronize());
    u32 cnt = 0;
    CUDA_CHECK(cudaMemcpy(&cnt, d_count, sizeof(u32), cudaMemcpyDeviceToHost));
    u32 take = cnt < cap ? cnt : cap;
    if (take > surv_cap) take = surv_cap;
    if (take) {
        QSurvivor* h = (QSurvivor*)malloc((size_t)take * sizeof(QSurvivor));
        CUDA_CHECK(cudaMemcpy(h, d_surv, (size_t)take * sizeof(QSurvivor), cudaMemcpyDeviceToHost));
        for (u32 i = 0; i < take; i++) out[i] = h[i].thread_offset;
        free(h);
    }
    cudaFree(d_primes); cudaFree(d_base_mod); cudaFree(d_qb); cudaFree(d_mask); cudaFree(d_act);
    cudaFree(d_surv); cudaFree(d_count); cudaFree(d_overflow); cudaFree(d_total); cudaFree(d_pass);
    return cnt;
}

/* Elapsed device time (ms, CUDA events) of `reps` launches of the reference
 * kernel over one variant's n_q Q values (the bench's reference arm). */
float ref16_qiter_time(const unsigned* primes, int n_qp, unsigned long long d_lo, unsigned long long d_hi,
                       int E, int depth, unsigned long long qb_lo, unsigned long long qb_hi, unsigned n_q,
                       int reps, unsigned* count_out) {
    u128 D = ((u128)d_hi << 64) | d_lo;
    u128 Q_base = ((u128)qb_hi << 64) | qb_lo;
    BarrettQ qb[V16_MAX_SIEVE];
    u64 mask[V16_MAX_SIEVE * V16_Q_MASK_WORDS];
    u32 base_mod[V16_MAX_SIEVE];
    u8 active[V16_MAX_SIEVE];
    u32 n_act = 0;
    memset(mask, 0, sizeof(mask));
    for (int i = 0; i < n_qp; i++) {
        u32 q = primes[i];
        qb[i].q = q;
        qb[i].magic = barrett_magic_u32(q);
        base_mod[i] = (u32)(Q_base % (u128)q);
        u32 D_mod_q = (u32)(D % (u128)q);
        if (D_mod_q == 0) continue;
        for (int j = 0; j < depth; j++) {
            u32 p2 = pow2_mod_u32(E + j, q);
            u32 m = (u32)(((u64)D_mod_q * (u64)p2) % (u64)q);
            u32 inv = mod_inv_u32(m, q);
            mask[(size_t)i * V16_Q_MASK_WORDS + (inv >> 6)] |= (1ULL << (inv & 63u));
        }
        active[n_act++] = (u8)i;
    }
    u32 *d_primes, *d_base_mod, *d_count, *d_overflow;
    BarrettQ* d_qb;
    u64* d_mask;
    u8* d_act;
    QSurvivor* d_surv;
    unsigned long long *d_total, *d_pass;
    u32 surv_cap = V16_Q_MAX_SURVIVORS;
    CUDA_CHECK(cudaMalloc(&d_primes, n_qp * sizeof(u32)));
    CUDA_CHECK(cudaMalloc(&d_base_mod, n_qp * sizeof(u32)));
    CUDA_CHECK(cudaMalloc(&d_qb, n_qp * sizeof(BarrettQ)));
    CUDA_CHECK(cudaMalloc(&d_mask, (size_t)n_qp * V16_Q_MASK_WORDS * sizeof(u64)));
    CUDA_CHECK(cudaMalloc(&d_act, V16_MAX_SIEVE));
    CUDA_CHECK(cudaMalloc(&d_surv, (size_t)surv_cap * sizeof(QSurvivor)));
    CUDA_CHECK(cudaMalloc(&d_count, sizeof(u32)));
    CUDA_CHECK(cudaMalloc(&d_overflow, sizeof(u32)));
    CUDA_CHECK(cudaMalloc(&d_total, sizeof(unsigned long long)));
    CUDA_CHECK(cudaMalloc(&d_pass, sizeof(unsigned long long)));
    CUDA_CHECK(cudaMemcpy(d_primes, primes, n_qp * sizeof(u32), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_base_mod, base_mod, n_qp * sizeof(u32), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_qb, qb, n_qp * sizeof(BarrettQ), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_mask, mask, (size_t)n_qp * V16_Q_MASK_WORDS * sizeof(u64), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_act, active, V16_MAX_SIEVE, cudaMemcpyHostToDevice));
    const u32 Q_per_thread = 16;
    u64 threads_needed = ((u64)n_q + Q_per_thread - 1) / Q_per_thread;
    u64 blocks = (threads_needed + V16_THREADS - 1) / V16_THREADS;
    if (blocks == 0) blocks = 1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float ms = 0;
    for (int r = -1; r < reps; r++) {
        if (r == 0) cudaEventRecord(e0);
        CUDA_CHECK(cudaMemsetAsync(d_count, 0, sizeof(u32)));
        v16_q_iter_kernel<<<(u32)blocks, V16_THREADS>>>(
            n_q, Q_per_thread, 0u, (u32)n_qp, d_primes, d_qb, d_mask, d_base_mod, (u32)depth,
            d_surv, d_count, surv_cap, d_total, d_pass, d_act, n_act, d_overflow);
    }
    cudaEventRecord(e1);
    CUDA_CHECK(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    u32 cnt = 0;
    CUDA_CHECK(cudaMemcpy(&cnt, d_count, sizeof(u32), cudaMemcpyDeviceToHost));
    if (count_out) *count_out = cnt;
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaFree(d_primes); cudaFree(d_base_mod); cudaFree(d_qb); cudaFree(d_mask); cudaFree(d_act);
    cudaFree(d_surv); cudaFree(d_count); cudaFree(d_overflow); cudaFree(d_total); cudaFree(d_pass);
    return ms;
}

/* The reference's q-iter checkpoint writer and reader on a configuration
 * given field by field (v16:4108-4390).  The sieve list hashed is q_primes;
 * its "sieve_primes=" line lists the q_primes above the default wheel bound
 * 53 (select_wheel_sieve with --wheel-max 53, v16:1408-1451).  pool_csv:
 * D_V in decimal, comma-separated. */
static void ref16_cfg(v16_cfg* c, int target, int depth, int bits_min, int bits_max, const char* seed_name,
                      const unsigned* immune, int n_immune, int E, unsigned sieve_max, const unsigned* q_primes,
                      int n_qp, int q_random, unsigned long long q_seed, unsigned q_chunk, int exhaustive,
                      int xbits) {
    memset(c, 0, sizeof(*c));
    c->target_len = target;
    c->sieve_depth = depth;
    c->bits_min = bits_min;
    c->bits_max = bits_max;
    strncpy(c->seed_name, seed_name, sizeof(c->seed_name) - 1);
    c->D = 1;
    for (int i = 0; i < n_immune; i++) { c->D_primes[i] = immune[i]; c->D *= immune[i]; }
    c->n_D_primes = n_immune;
    u128_to_dec(c->D, c->D_dec, sizeof(c->D_dec));
    c->exp_start = E;
    c->sieve_prime_max = sieve_max;
    c->wheel_prime_max = 53;
    for (int i = 0; i < n_qp; i++)
        if (q_primes[i] > 53) c->sieve_primes[c->n_sieve_primes++] = q_primes[i];
    c->q_iter = 1;
    c->q_order_random = q_random;
    c->q_seed = q_seed;
    c->q_chunk = q_chunk;
    c->q_band_mode_exhaustive = exhaustive;
    c->exhaustive_max_q_bits = xbits;
}

static v16_pool_seed* ref16_pool(const char* pool_csv, int n_v) {
    v16_pool_seed* ps = (v16_pool_seed*)calloc((size_t)n_v, sizeof(v16_pool_seed));
    const char* p = pool_csv;
    for (int v = 0; v < n_v; v++) {
        int k = 0;
        while (*p && *p != ',' && k < 79) ps[v].D_dec[k++] = *p++;
        if (*p == ',') p++;
    }
    return ps;
}

int ref16_ckpt_save(const char* path, int target, int depth, int bits_min, int bits_max, const char* seed_name,
                    const unsigned* immune, int n_immune, int E, unsigned sieve_max, const unsigned* q_primes,
                    int n_qp, int q_random, unsigned long long q_seed, unsigned q_chunk, int exhaustive,
                    int xbits, const char* pool_csv, int n_v, const unsigned long long* cur_lo,
                    const unsigned long long* cur_hi, const unsigned long long* qmin_lo,
                    const unsigned long long* qmin_hi) {
    static v16_cfg c;
    ref16_cfg(&c, target, depth, bits_min, bits_max, seed_name, immune, n_immune, E, sieve_max, q_primes,
              n_qp, q_random, q_seed, q_chunk, exhaustive, xbits);
    strncpy(c.checkpoint_file, path, sizeof(c.checkpoint_file) - 1);
    v16_pool_seed* ps = ref16_pool(pool_csv, n_v);
    int r = save_q_iter_checkpoint(&c, (const u64*)cur_lo, (const u64*)cur_hi, (const u64*)qmin_lo,
                                   (const u64*)qmin_hi, n_v, q_iter_sieve_fnv1a64(q_primes, n_qp),
                                   q_iter_pool_fnv1a64(ps, n_v));
    free(ps);
    return r;
}

/* 0 and the cursors found (others left as given), or -1 when the reference
 * refuses the file */
int ref16_ckpt_load(const char* path, int target, int depth, int bits_min, int bits_max, const char* seed_name,
                    const unsigned* immune, int n_immune, int E, unsigned sieve_max, const unsigned* q_primes,
                    int n_qp, int q_random, unsigned long long q_seed, unsigned q_chunk, int exhaustive,
                    int xbits, const char* pool_csv, int n_v, unsigned long long* cur_lo,
                    unsigned long long* cur_hi) {
    static v16_cfg c;
    ref16_cfg(&c, target, depth, bits_min, bits_max, seed_name, immune, n_immune, E, sieve_max, q_primes,
              n_qp, q_random, q_seed, q_chunk, exhaustive, xbits);
    strncpy(c.resume_file, path, sizeof(c.resume_file) - 1);
    v16_pool_seed* ps = ref16_pool(pool_csv, n_v);
    int r = load_q_iter_checkpoint(&c, (u64*)cur_lo, (u64*)cur_hi, n_v, q_iter_sieve_fnv1a64(q_primes, n_qp),
                                   q_iter_pool_fnv1a64(ps, n_v));
    free(ps);
    return r;
}

}  // extern "C"
