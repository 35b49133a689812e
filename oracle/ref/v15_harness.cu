/*
 * In-process harness around the reference's v15 engine
 * (src/cuda/cc18_filter_cuda_CpC_v15.cu), compiled from the reference source
 * where it lies.  TEST INFRASTRUCTURE ONLY: it runs the reference's table
 * builders, its v15 filter kernel K1 (v15:1753-1929) and its prove kernel K2
 * (v15:1620-1740) in either prove order (--prove-order forward | reverse,
 * v15:1666-1730) with the launch sequence of its main loop (v15:4040-4105),
 * and reads the results back.  Built into oracle/_ref/ by oracle/Makefile;
 * never part of the product.
 */
#define main v15_reference_main
#include "cc18_filter_cuda_CpC_v15.cu"
#undef main

extern "C" {

/* init_filter_tables(depth) + generate_bases(target), FULL coverage */
int ref15_setup(int target, int depth) {
    for (int b = 0; b < h_num_bases; b++)
        for (int m = 0; m < 6; m++) { free(h_bases[b].wheel_by_mod6[m]); h_bases[b].wheel_by_mod6[m] = NULL; }
    h_num_bases = 0;
    g_coverage_mode = COVERAGE_FULL;
    init_filter_tables(depth);
    generate_bases(target);
    return h_num_bases;
}

/* gpu_upload_tables with the prove order and target, + d_target_bits */
int ref15_upload(int depth, int bits, int target, int prove_forward) {
    g_target_len = target;
    g_prove_forward = prove_forward;
    gpu_upload_tables(depth);
    CUDA_CHECK(cudaMemcpyToSymbol(d_target_bits, &bits, sizeof(int)));
    return 0;
}

/* One K1 batch as the v15 main loop issues it; copies survivors back and
 * returns the raw device count. */
unsigned ref15_filter(unsigned long long ts_lo, unsigned long long ts_hi, unsigned n_tiles,
                      int blocks_per_sm, unsigned* out, unsigned cap) {
    u128 ts = ((u128)ts_hi << 64) | ts_lo;
    static u16 hl2[MAX_BASES * FILTER_PRIMES_COUNT];
    static u16 hext[MAX_BASES * EXT_FILTER_PRIMES_COUNT];
    static u16 hline[MAX_BASES * LINE_SIEVE_COUNT];
    prepare_batch(ts, hl2, hext, hline);
    CUDA_CHECK(cudaMemcpy(d_batch_l2[0], hl2, h_num_bases * FILTER_PRIMES_COUNT * sizeof(u16), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_batch_ext[0], hext, h_num_bases * EXT_FILTER_PRIMES_COUNT * sizeof(u16), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_batch_line[0], hline, h_num_bases * LINE_SIEVE_COUNT * sizeof(u16), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemset(d_survivor_count[0], 0, sizeof(u32)));
    cudaDeviceProp prop;
    CUDA_CHECK(cudaGetDeviceProperties(&prop, 0));
    int num_blocks = prop.multiProcessorCount * blocks_per_sm;
    cc18_filter_kernel<<<num_blocks, THREADS_PER_BLOCK>>>(
        n_tiles, (u32)(ts % 6),
        d_kmod_filter, d_kmod_ext_filter, d_kmod_l2_interleaved, d_kmod_ext_interleaved,
        d_kM_mod_line, d_ext_filter_first, d_line_kill_first, d_line_kill_packed_g,
        d_batch_l2[0], d_batch_ext[0], d_batch_line[0],
        d_wheel_offsets, d_wheel_start_m6, d_wheel_count_m6,
        d_survivors[0], d_survivor_count[0]);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaDeviceSynchronize());
    u32 cnt = 0;
    CUDA_CHECK(cudaMemcpy(&cnt, d_survivor_count[0], sizeof(u32), cudaMemcpyDeviceToHost));
    u32 n = cnt < MAX_SURVIVORS_PER_BATCH ? cnt : MAX_SURVIVORS_PER_BATCH;
    if (n > cap) n = cap;
    if (n) CUDA_CHECK(cudaMemcpy(out, d_survivors[0], n * sizeof(Survivor), cudaMemcpyDeviceToHost));
    return cnt;
}

/* d_target_bits alone (the --bits of a later batch) */
int ref15_set_bits(int bits) {
    CUDA_CHECK(cudaMemcpyToSymbol(d_target_bits, &bits, sizeof(int)));
    return 0;
}

/* Times n_batches consecutive batches of batch_tiles tiles from ts with the
 * v15 main loop's launch sequence (v15:4040-4105): prepare_batch and the
 * residue uploads untimed, then K1 and, with with_k2, K2 (in the prove order
 * set by ref15_upload) on one stream, each bracketed by CUDA events.  k1_ms
 * / k2_ms receive the summed device times; counts = {survivors, chain
 * records, K2 primes}. */
int ref15_time_batches(unsigned long long ts_lo, unsigned long long ts_hi, unsigned batch_tiles,
                       int n_batches, int blocks_per_sm, int with_k2, float* k1_ms, float* k2_ms,
                       unsigned long long* counts) {
    u128 ts = ((u128)ts_hi << 64) | ts_lo;
    static u16 hl2[MAX_BASES * FILTER_PRIMES_COUNT];
    static u16 hext[MAX_BASES * EXT_FILTER_PRIMES_COUNT];
    static u16 hline[MAX_BASES * LINE_SIEVE_COUNT];
    cudaDeviceProp prop;
    CUDA_CHECK(cudaGetDeviceProperties(&prop, 0));
    const int num_blocks = prop.multiProcessorCount * blocks_per_sm;
    const int prove_blocks = (MAX_SURVIVORS_PER_BATCH + 255) / 256;
    cudaEvent_t e[3];
    for (int i = 0; i < 3; i++) cudaEventCreate(&e[i]);
    *k1_ms = 0; *k2_ms = 0;
    counts[0] = counts[1] = counts[2] = 0;
    for (int bi = 0; bi < n_batches; bi++) {
        u128 cur = ts + (u128)bi * batch_tiles;
        prepare_batch(cur, hl2, hext, hline);
        CUDA_CHECK(cudaMemcpy(d_batch_l2[0], hl2, h_num_bases * FILTER_PRIMES_COUNT * sizeof(u16), cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(d_batch_ext[0], hext, h_num_bases * EXT_FILTER_PRIMES_COUNT * sizeof(u16), cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(d_batch_line[0], hline, h_num_bases * LINE_SIEVE_COUNT * sizeof(u16), cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemset(d_survivor_count[0], 0, sizeof(u32)));
        CUDA_CHECK(cudaMemset(d_chain_result_count[0], 0, sizeof(u32)));
        CUDA_CHECK(cudaMemset(d_gpu_primes_count[0], 0, sizeof(u32)));
        CUDA_CHECK(cudaDeviceSynchronize());
        cudaEventRecord(e[0]);
        cc18_filter_kernel<<<num_blocks, THREADS_PER_BLOCK>>>(
            batch_tiles, (u32)(cur % 6),
            d_kmod_filter, d_kmod_ext_filter, d_kmod_l2_interleaved, d_kmod_ext_interleaved,
            d_kM_mod_line, d_ext_filter_first, d_line_kill_first, d_line_kill_packed_g,
            d_batch_l2[0], d_batch_ext[0], d_batch_line[0],
            d_wheel_offsets, d_wheel_start_m6, d_wheel_count_m6,
            d_survivors[0], d_survivor_count[0]);
        cudaEventRecord(e[1]);
        if (with_k2)
            cc18_prove_kernel<<<prove_blocks, 256>>>(d_survivors[0], d_survivor_count[0],
                                                     (u64)cur, (u64)(cur >> 64), d_chain_results[0],
                                                     d_chain_result_count[0], d_gpu_primes_count[0]);
        cudaEventRecord(e[2]);
        CUDA_CHECK(cudaGetLastError());
        CUDA_CHECK(cudaEventSynchronize(e[2]));
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, e[0], e[1]);
        cudaEventElapsedTime(&b, e[1], e[2]);
        *k1_ms += a;
        *k2_ms += b;
        u32 ns = 0, nc = 0, np = 0;
        CUDA_CHECK(cudaMemcpy(&ns, d_survivor_count[0], sizeof(u32), cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(&nc, d_chain_result_count[0], sizeof(u32), cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(&np, d_gpu_primes_count[0], sizeof(u32), cudaMemcpyDeviceToHost));
        counts[0] += ns; counts[1] += nc; counts[2] += np;
    }
    for (int i = 0; i < 3; i++) cudaEventDestroy(e[i]);
    return 0;
}

/* K2 over the survivors of the last ref15_filter; returns the record count */
unsigned ref15_prove_gpu(unsigned long long ts_lo, unsigned long long ts_hi,
                         unsigned* out, unsigned cap, unsigned* primes_out) {
    CUDA_CHECK(cudaMemset(d_chain_result_count[0], 0, sizeof(u32)));
    CUDA_CHECK(cudaMemset(d_gpu_primes_count[0], 0, sizeof(u32)));
    int prove_blocks = (MAX_SURVIVORS_PER_BATCH + 255) / 256;
    cc18_prove_kernel<<<prove_blocks, 256>>>(d_survivors[0], d_survivor_count[0], ts_lo, ts_hi,
                                             d_chain_results[0], d_chain_result_count[0],
                                             d_gpu_primes_count[0]);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaDeviceSynchronize());
    u32 n = 0, p = 0;
    CUDA_CHECK(cudaMemcpy(&n, d_chain_result_count[0], sizeof(u32), cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(&p, d_gpu_primes_count[0], sizeof(u32), cudaMemcpyDeviceToHost));
    u32 m = n < (u32)MAX_CHAIN_RESULTS ? n : (u32)MAX_CHAIN_RESULTS;
    if (m > cap) m = cap;
    if (m) CUDA_CHECK(cudaMemcpy(out, d_chain_results[0], m * sizeof(ChainResult), cudaMemcpyDeviceToHost));
    if (primes_out) *primes_out = p;
    return n;
}

}  // extern "C"
