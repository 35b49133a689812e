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

}  // extern "C"
