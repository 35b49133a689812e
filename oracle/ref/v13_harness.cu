/*
 * In-process harness around the reference's own v13 engine
 * (src/cuda/cc18_filter_cuda_CpC_v13.cu), compiled from the reference source
 * where it lies.  TEST INFRASTRUCTURE ONLY: it lets the tests call the
 * reference's table builders (v13:793-1059), its filter kernel K1
 * (v13:1551-1714), its prove kernel K2 (v13:1462-1538) and its CPU GMP prover
 * pool (v13:1967-2068) with exactly the reference launch sequence of
 * v13:3764-3815, and read the results back.  Built into oracle/_ref/ by
 * oracle/Makefile; never part of the product.
 */
/* The same harness builds over the second-kind variant v13b
 * (-DREF13_SOURCE='"cc18_filter_cuda_CpC_v13b.cu"', oracle/Makefile). */
#ifndef REF13_SOURCE
#define REF13_SOURCE "cc18_filter_cuda_CpC_v13.cu"
#endif
#define main v13_reference_main
#include REF13_SOURCE
#undef main

extern "C" {

/* init_filter_tables(depth) + generate_bases(target), FULL coverage */
int ref13_setup(int target, int depth) {
    for (int b = 0; b < h_num_bases; b++)
        for (int m = 0; m < 6; m++) { free(h_bases[b].wheel_by_mod6[m]); h_bases[b].wheel_by_mod6[m] = NULL; }
    h_num_bases = 0;
    g_coverage_mode = COVERAGE_FULL;
    init_filter_tables(depth);
    generate_bases(target);
    return h_num_bases;
}

int ref13_num_bases(void) { return h_num_bases; }
unsigned long long ref13_base(int b) { return h_bases[b].base; }
unsigned ref13_tkm6(int b) { return h_bases[b].target_k_mod6; }
int ref13_bucket_size(int b, int m) { return h_bases[b].wheel_size_by_mod6[m]; }
void ref13_bucket(int b, int m, unsigned* out) {
    memcpy(out, h_bases[b].wheel_by_mod6[m], sizeof(u32) * h_bases[b].wheel_size_by_mod6[m]);
}
unsigned long long ref13_l2_mask(int p_idx, int L) { return h_filter_mask_first[p_idx][L]; }
int ref13_ext_forbidden(int p_idx, int L, int r) { return h_ext_filter_first[p_idx][L][r]; }
int ref13_line_kill(int idx, int r) { return h_line_kill_first[idx][r]; }

/* gpu_upload_tables + d_target_bits for the tables built by ref13_setup.
 * Each call uploads afresh (the reference allocates new buffers per call). */
int ref13_upload(int depth, int bits) {
    gpu_upload_tables(depth);
    CUDA_CHECK(cudaMemcpyToSymbol(d_target_bits, &bits, sizeof(int)));
    return 0;
}

/* One K1 batch exactly as the reference main loop issues it (v13:3764-3795):
 * prepare_batch on the host, upload residues, zero the count, launch
 * cc18_filter_kernel<<<SMs*blocks_per_sm, 256>>>.  Copies survivors back.
 * Returns the raw device survivor count (may exceed cap / 2^20). */
unsigned ref13_filter(unsigned long long ts_lo, unsigned long long ts_hi, unsigned n_tiles,
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
        d_kmod_filter, d_kmod_ext_filter, d_kM_mod_line,
        d_ext_filter_first, d_line_kill_first,
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

/* Times one K1 batch with CUDA events (same launch as ref13_filter); returns ms */
float ref13_time_filter(unsigned long long ts_lo, unsigned long long ts_hi, unsigned n_tiles,
                        int blocks_per_sm, int reps) {
    u128 ts = ((u128)ts_hi << 64) | ts_lo;
    static u16 hl2[MAX_BASES * FILTER_PRIMES_COUNT];
    static u16 hext[MAX_BASES * EXT_FILTER_PRIMES_COUNT];
    static u16 hline[MAX_BASES * LINE_SIEVE_COUNT];
    prepare_batch(ts, hl2, hext, hline);
    CUDA_CHECK(cudaMemcpy(d_batch_l2[0], hl2, h_num_bases * FILTER_PRIMES_COUNT * sizeof(u16), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_batch_ext[0], hext, h_num_bases * EXT_FILTER_PRIMES_COUNT * sizeof(u16), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_batch_line[0], hline, h_num_bases * LINE_SIEVE_COUNT * sizeof(u16), cudaMemcpyHostToDevice));
    cudaDeviceProp prop;
    CUDA_CHECK(cudaGetDeviceProperties(&prop, 0));
    int num_blocks = prop.multiProcessorCount * blocks_per_sm;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int r = 0; r < reps; r++) {
        cudaMemsetAsync(d_survivor_count[0], 0, sizeof(u32));
        cc18_filter_kernel<<<num_blocks, THREADS_PER_BLOCK>>>(
            n_tiles, (u32)(ts % 6),
            d_kmod_filter, d_kmod_ext_filter, d_kM_mod_line,
            d_ext_filter_first, d_line_kill_first,
            d_batch_l2[0], d_batch_ext[0], d_batch_line[0],
            d_wheel_offsets, d_wheel_start_m6, d_wheel_count_m6,
            d_survivors[0], d_survivor_count[0]);
    }
    cudaEventRecord(e1);
    CUDA_CHECK(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    return ms / reps;
}

/* d_target_bits alone (the --bits of a later batch, v13:3092) */
int ref13_set_bits(int bits) {
    CUDA_CHECK(cudaMemcpyToSymbol(d_target_bits, &bits, sizeof(int)));
    return 0;
}

/* Times n_batches consecutive batches of batch_tiles tiles from ts with the
 * reference main loop's launch sequence (v13:3764-3815): prepare_batch on the
 * host and the residue uploads (untimed), then K1 and, with with_k2, K2 on
 * one stream, each bracketed by CUDA events.  k1_ms / k2_ms receive the
 * summed device times; counts = {survivors, chain records, K2 primes}. */
int ref13_time_batches(unsigned long long ts_lo, unsigned long long ts_hi, unsigned batch_tiles,
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
            d_kmod_filter, d_kmod_ext_filter, d_kM_mod_line,
            d_ext_filter_first, d_line_kill_first,
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

/* K2 over survivors already placed by ref13_filter in d_survivors[0]
 * (v13:3797-3815).  Writes ChainResult records; returns their count. */
unsigned ref13_prove_gpu(unsigned long long ts_lo, unsigned long long ts_hi,
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

/* The reference CPU GMP prover pool on host survivors (v13:1967-2068), one
 * worker, every chain logged (log threshold 1) into the given file in the
 * reference's own output-line format (v13:2030-2033). */
int ref13_prove_cpu(const unsigned* surv, int count, unsigned long long ts_lo,
                    unsigned long long ts_hi, int target, int bits, const char* out_path,
                    unsigned long long* primes, unsigned long long* chains) {
    g_num_prove_threads = 1;
    if (prover_pool_start() != 0) return -1;
    FILE* fp = fopen(out_path, "w");
    if (!fp) return -2;
    u128 ts = ((u128)ts_hi << 64) | ts_lo;
    u64 p = 0, c = 0;
    int best = 0;
    /* the pool logs at most 256 entries per worker per batch: feed <= 200 */
    for (int off = 0; off < count; off += 200) {
        int n = count - off < 200 ? count - off : 200;
        prove_survivors_mt((const Survivor*)(surv + 4 * off), n, ts, target, bits, 1, fp,
                           &p, &c, &best);
    }
    fclose(fp);
    *primes = p;
    *chains = c;
    return 0;
}

}  /* extern "C" */

/* ---- campaign shell pins: generator and checkpoint file (v13:540-722) ---- */
extern "C" {

/* n outputs of the reference generator rng_next after rng_seed(seed) */
void ref13_rng(unsigned long long seed, int n, unsigned long long* out) {
    rng_seed(seed);
    for (int i = 0; i < n; i++) out[i] = rng_next();
}

static void ref13_set_prefix(const char* prefix, int lanes, int lane_id) {
    g_use_prefix = (prefix && prefix[0] && strcmp(prefix, "none") != 0);
    snprintf(g_prefix_str, sizeof(g_prefix_str), "%s", g_use_prefix ? prefix : "");
    g_prefix_lanes = lanes;
    g_prefix_lane_id = lane_id;
}

/* reference checkpoint_save with the given campaign identity and cursor */
int ref13_checkpoint_save(const char* path, int bits, int target, int depth, const char* prefix,
                          int lanes, int lane_id, unsigned long long tile_hi, unsigned long long tile_lo,
                          unsigned long long tiles, unsigned long long primes, unsigned long long chains,
                          int best) {
    ref13_set_prefix(prefix, lanes, lane_id);
    u128 t = ((u128)tile_hi << 64) | tile_lo;
    return checkpoint_save(path, bits, target, depth, t, tiles, primes, chains, best);
}

/* reference checkpoint_load; out = {tile_hi, tile_lo, tiles, primes, chains, best} */
int ref13_checkpoint_load(const char* path, int bits, int target, int depth, const char* prefix,
                          int lanes, int lane_id, unsigned long long* out) {
    ref13_set_prefix(prefix, lanes, lane_id);
    u128 t = 0;
    u64 tiles = 0, primes = 0, chains = 0;
    int best = 0;
    int r = checkpoint_load(path, bits, target, depth, &t, &tiles, &primes, &chains, &best);
    out[0] = (unsigned long long)(t >> 64);
    out[1] = (unsigned long long)t;
    out[2] = tiles; out[3] = primes; out[4] = chains; out[5] = (unsigned long long)best;
    return r;
}

}  // extern "C"
