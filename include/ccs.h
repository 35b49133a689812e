/*
 * ccs.h -- C ABI of the B200 Cunningham-chain search engine.
 *
 * The engine replaces the data-parallel hot path of nmicic/cunningham-chain-search
 * (first-kind chains p, 2p+1, 4p+3, ...): CRT-lattice/wheel candidate
 * enumeration, the three-stage forbidden-residue depth filter, and the
 * Miller-Rabin prove / chain walk.  Reference paths below are relative to the
 * reference repository; "v13" is src/cuda/cc18_filter_cuda_CpC_v13.cu, "v33"
 * is src/cpu/cc_gmp_v33_03.c.
 *
 * Conventions
 *   - every entry point returns a ccs_status; nothing calls exit() (the
 *     reference's CUDA_CHECK exits, v13:142-149);
 *   - a ccs_engine owns all of its device memory; caller buffers are passed as
 *     plain pointers plus capacities; the *_dev arguments are device pointers,
 *     the *_host arguments host pointers;
 *   - "stream" is a cudaStream_t passed as void* (NULL = legacy default);
 *   - an engine is not thread-safe: use one engine per host thread;
 *   - capacity overflow returns CCS_OVERFLOW together with the true count;
 *     records beyond the capacity are not written (the reference truncates
 *     with a warning, v13:3846-3863).
 */
#ifndef CCS_H
#define CCS_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCS_ABI_VERSION 1

typedef enum {
    CCS_OK = 0,
    CCS_ERR_INVALID = 1,      /* bad argument or parameter set */
    CCS_ERR_CUDA = 2,         /* a CUDA call failed; see ccs_last_error() */
    CCS_OVERFLOW = 3,         /* output capacity exceeded; count is exact */
    CCS_ERR_NOMEM = 4,        /* device or host allocation failed */
    CCS_ERR_TIMEOUT = 5,      /* a bounded device wait gave up */
    CCS_ERR_BUSY = 6,         /* admission refused: no slot or memory free */
    CCS_ERR_NOT_FOUND = 7,    /* unknown request id */
    CCS_ERR_CANCELLED = 8,    /* request was cancelled */
    CCS_PENDING = 9           /* request still running */
} ccs_status;

/* One filter stage: the listed primes are tested at chain positions
 * [pos_lo, min(depth, q)).  The reference's L2 and ext-L2 stages use
 * pos_lo = 0 (v13:799-828); its line sieve uses pos_lo = 1 (v13:834-846). */
typedef struct {
    const uint32_t* primes;
    uint32_t n_primes;
    uint32_t pos_lo;
} ccs_stage;

/* Chain kind.  First kind: p, 2p + 1, 4p + 3, ... (v13).  Second kind:
 * p, 2p - 1, 4p - 3, ...: forbidden residues 1 - 2^-i instead of 2^-i - 1,
 * n == 1 (mod 6) instead of 5, predecessor (n + 1) / 2 (the reference's
 * v13b, v13b:6-14). */
enum { CCS_KIND_FIRST = 1, CCS_KIND_SECOND = 2 };

/* Primality predicate used by the prover. */
enum {
    CCS_PRIME_MR = 0,      /* strong-PRP for every witness (v13 gpu_is_prime, v13:1428-1452) */
    CCS_PRIME_BPSW = 1,    /* Baillie-PSW: GMP 6.3 mpz_probab_prime_p(n, 1) (v13:1841) */
    CCS_PRIME_V33 = 2      /* the reference CPU engine's own tests (first kind, CCS_PROVE_FULL):
                              n after trial division by 101..409 -> strong PRP to bases
                              2, 3, 5 (v33:1326-1339, 2112-2130); predecessors and backward
                              steps -> Baillie-PSW (is_prime_fast, v33:1345-1362, 1489-1495);
                              forward links -> zero residue mod any of the 132 screen primes
                              67..863 is composite (a link equal to a screen prime included),
                              then Fermat base 2 (v33:1512-1577, 1290-1302), walk stopped at
                              2^127.  Ranges with bits + target > 127 take the reference's
                              wide path instead: Baillie-PSW for n and the links, walk
                              stopped at 2^(bits + 2 target) (v33:1594-1656, 1694-1703,
                              1982-1997). */
};

/* Prove semantics. */
enum {
    CCS_PROVE_ROOTS = 0,   /* reference K2: 132-prime trial division, non-roots dropped (v13:1462-1538) */
    CCS_PROVE_FULL = 1     /* reference CPU prover: 62-prime trial division, backward walk
                              to the true root, forward walk (v13:1814-1881) */
};

/* Engine parameters.  Zero / NULL fields take the reference's values
 * (v13:155-201): CRT {5..19}, wheel {23,29,31}, stages 37..61 / 67..97 /
 * 101..863 (line sieve from position 1), target 18, depth = target, bits 89,
 * v13's 20 witnesses {2..71}, BPSW, full prove. */
typedef struct {
    uint32_t kind;                 /* CCS_KIND_FIRST (0 = first) | CCS_KIND_SECOND */
    uint32_t target;               /* chain length for CRT/wheel admissibility (v13 generate_bases) */
    uint32_t depth;                /* filter depth, clamped to [1, min(target, 32)] (v13:3238-3252) */
    uint32_t bits;                 /* bit width gate of the prover (v13:1495, 1828) */
    const uint32_t* crt_primes;    /* lattice modulus M = product */
    uint32_t n_crt;
    const uint32_t* wheel_primes;  /* wheel period WP = product */
    uint32_t n_wheel;
    const ccs_stage* stages;       /* up to 4 filter stages */
    uint32_t n_stages;
    uint32_t max_bases;            /* 0 = every admissible base (v33); 64 = v13's MAX_BASES cap */
    const uint64_t* witnesses;     /* CCS_PRIME_MR witnesses */
    uint32_t n_witnesses;
    uint32_t primality;            /* CCS_PRIME_MR | CCS_PRIME_BPSW */
    uint32_t prove_mode;           /* CCS_PROVE_ROOTS | CCS_PROVE_FULL */
    uint32_t flags;                /* CCS_FLAG_* */
} ccs_params;

/* ccs_params.flags */
#define CCS_FLAG_REVERSE_PROVE 1u  /* with CCS_PROVE_ROOTS: test chain position target - 1 first
                                      and drop the survivor when it is composite, then prove as
                                      usual (v15 --prove-order reverse, v15:1686-1730); exact
                                      arithmetic where the reference wraps at 2^128 */

/* Filter output: the reference's Survivor record (v13:207-212), 16 bytes.
 * tile_idx is relative to the tile_start of the call. */
typedef struct {
    uint32_t base_idx;
    uint32_t k_offset;
    uint32_t tile_idx;
    uint32_t _pad;         /* written as 0 */
} ccs_survivor;

/* Prove output.  The first four words are the reference's ChainResult
 * (v13:218-223); the rest carries the chain root (the reference CPU prover
 * prints it, v13:1895-1896).  48 bytes. */
typedef struct {
    uint32_t base_idx;
    uint32_t k_offset;
    uint32_t tile_idx;
    uint32_t chain_len;
    uint32_t root[6];      /* true root, little-endian 32-bit limbs (<= 192 bits) */
    uint32_t flags;        /* bit0: survivor is the root; bit1: chain_len >= target */
    uint32_t survivor;     /* index of the survivor this record came from */
} ccs_chain;

enum { CCS_CHAIN_IS_ROOT = 1u, CCS_CHAIN_TARGET = 2u };

typedef struct ccs_engine ccs_engine;

/* Lattice facts of an engine (host copy). */
typedef struct {
    uint64_t lattice_m;            /* M */
    uint32_t wheel_period;         /* WP */
    uint32_t n_bases;
    uint64_t n_lines;              /* admissible residues mod W = 6*M*WP */
    uint64_t candidates_per_tile;  /* sum of wheel sizes / 6 (v13:3980-3987) */
    uint32_t target, depth, bits;
    uint32_t n_filter_primes;
    double expected_tests;         /* E[residue tests per candidate] of the
                                      reference's stage-ordered early-exit test */
    double pass_rate;              /* product of per-prime pass fractions */
    uint64_t launches;             /* kernels this engine has launched so far */
} ccs_info;

/* ---- engine ---------------------------------------------------------------- */

/* Host-only: build the lattice and filter tables for params and report them
 * without touching a GPU.  bases (optional) receives up to cap base values. */
ccs_status ccs_describe(const ccs_params* params, ccs_info* out, uint64_t* bases, uint32_t cap);

/* Builds the lattice, filter tables and device state (replaces v13's
 * init_filter_tables / generate_bases / gpu_upload_tables, v13:793-1222).
 * device = CUDA ordinal. */
ccs_status ccs_create(const ccs_params* params, int device, ccs_engine** out);
ccs_status ccs_destroy(ccs_engine* eng);
ccs_status ccs_get_info(const ccs_engine* eng, ccs_info* out);
/* host copies of the lattice: bases[n_bases] */
ccs_status ccs_get_bases(const ccs_engine* eng, uint64_t* bases, uint32_t cap);
const char* ccs_last_error(void);
int ccs_abi_version(void);

/* ---- plain per-range path ------------------------------------------------ */

/* Filter tiles [tile_start, tile_start + n_tiles) (tile_start a u128 given as
 * lo/hi words) and write survivors to out_dev (device, capacity cap).  The
 * survivor SET equals the reference K1's for the same range (v13:1551-1714,
 * launched as v13:3764-3795); order is unspecified.  n_tiles < 2^32.
 * Replaces prepare_batch + cc18_filter_kernel (v13:1232-1259, 1551-1714). */
ccs_status ccs_filter_range(ccs_engine* eng, uint64_t tile_start_lo, uint64_t tile_start_hi,
                            uint64_t n_tiles, ccs_survivor* out_dev, uint64_t cap,
                            uint64_t* n_out, void* stream);

/* ccs_filter_range without any device allocation.  No counterpart in the
 * reference.  For callers that may not allocate device memory once they are
 * running: services whose GPU footprint is fixed and accounted for at
 * start-up, allocators that refuse to grow after initialisation, and hosts
 * that share the GPU with other tenants under a memory quota.  The working
 * memory is a 66,560-byte array compiled into the library; every GPU that
 * loads the library holds one copy until the process exits.  Limit: engines
 * with at most 16362 filter primes (larger ones return CCS_ERR_INVALID); any
 * n_tiles < 2^32.  The call is synchronous: it waits for its stream and
 * returns the exact survivor count.  The first call on a device looks up the
 * array's device address.  Every call on a device shares the one array:
 * calls that overlap on the GPU (other streams, other threads, other engines
 * on the same device) race and must be serialised by the caller.  Results
 * equal ccs_filter_range's. */
ccs_status ccs_filter_range_noalloc(ccs_engine* eng, uint64_t tile_start_lo, uint64_t tile_start_hi,
                                    uint64_t n_tiles, ccs_survivor* out_dev, uint64_t cap,
                                    uint64_t* n_out, void* stream);

/* Prove survivors (device array) of the range that started at tile_start.
 * Replaces cc18_prove_kernel (v13:1462-1538) and prove_survivors_mt
 * (v13:1967-2068), per params.prove_mode / params.primality.
 * primes_out (optional) counts survivors whose n tested prime. */
ccs_status ccs_prove(ccs_engine* eng, const ccs_survivor* surv_dev, uint64_t n_surv,
                     uint64_t tile_start_lo, uint64_t tile_start_hi, ccs_chain* out_dev,
                     uint64_t cap, uint64_t* n_out, uint64_t* primes_out, void* stream);

/* Sets the prover bit-width gate of this engine for subsequent ccs_prove /
 * ccs_search_range_host calls (the reference's --bits, v13:3092). */
ccs_status ccs_set_bits(ccs_engine* eng, uint32_t bits);

/* Same two steps on HOST buffers, copies included (the reference's per-batch
 * H2D/D2H boundary, v13:3769-3830). */
ccs_status ccs_search_range_host(ccs_engine* eng, uint64_t tile_start_lo, uint64_t tile_start_hi,
                                 uint64_t n_tiles, ccs_survivor* surv_host, uint64_t surv_cap,
                                 uint64_t* n_surv, ccs_chain* chains_host, uint64_t chain_cap,
                                 uint64_t* n_chains, uint64_t* primes_out);

/* Walk given numbers forward (p -> 2p+1 while prime) and write each chain
 * length (0 when the number itself is not prime).  numbers_dev holds n
 * numbers of limbs x 32-bit little-endian limbs (limbs <= 6).  Same
 * predicate as the prover. */
ccs_status ccs_walk_numbers(ccs_engine* eng, const uint32_t* numbers_dev, uint64_t n, uint32_t limbs,
                            uint32_t* lengths_dev, void* stream);

/* ---- batched path -------------------------------------------------------- */

/* One lattice range of a batch.  profile selects one of the engines passed to
 * ccs_batch_create (ranges may differ in depth, width and lattice). */
typedef struct {
    uint64_t tile_start_lo, tile_start_hi;
    uint64_t n_tiles;
    uint32_t profile;
    uint32_t bits;          /* prover bit gate for this range */
} ccs_range;

/* Per-range result of a batch. */
typedef struct {
    uint64_t n_survivors;   /* exact count (may exceed the slice given) */
    uint64_t n_chains;
    uint64_t n_primes;
    uint64_t candidates;
    uint64_t surv_offset;   /* first survivor of this range in the batch survivor array */
    uint64_t chain_offset;
    uint32_t status;        /* ccs_status of this range */
    uint32_t _pad;
} ccs_range_result;

typedef struct ccs_batch ccs_batch;

/* A batch executor over n_profiles engines (all on one device).  Runs every
 * range of a submission in one persistent filter launch and one prove launch,
 * recorded once into a CUDA graph and replayed. max_ranges bounds a
 * submission; surv_cap / chain_cap bound the whole batch. */
ccs_status ccs_batch_create(ccs_engine* const* profiles, uint32_t n_profiles, uint32_t max_ranges,
                            uint64_t surv_cap, uint64_t chain_cap, ccs_batch** out);
ccs_status ccs_batch_destroy(ccs_batch* b);
/* ranges are host records; results / survivors / chains are copied back to the
 * host arrays (surv_host / chains_host may be NULL). */
ccs_status ccs_batch_run(ccs_batch* b, const ccs_range* ranges, uint32_t n_ranges,
                         ccs_range_result* results, ccs_survivor* surv_host, ccs_chain* chains_host,
                         void* stream);
/* The same as ccs_batch_run in two halves, so that a caller can prepare
 * (and another batch can run) while the GPU works: ccs_batch_launch stages
 * the ranges and replays the graph without waiting; ccs_batch_wait waits for
 * that launch and fills results and the host records.  A batch holds one
 * launch at a time (CCS_ERR_BUSY otherwise); two batches over the same
 * engines may be in flight together. */
ccs_status ccs_batch_launch(ccs_batch* b, const ccs_range* ranges, uint32_t n_ranges);
ccs_status ccs_batch_wait(ccs_batch* b, ccs_range_result* results, ccs_survivor* surv_host,
                          ccs_chain* chains_host);
/* device-side timing of the last ccs_batch_run: filter+prove milliseconds */
ccs_status ccs_batch_last_ms(const ccs_batch* b, float* ms);

/* Batch tuning: the sweep block shape of the recorded graph and the work
 * unit length applied to every range (0: each engine's own unit_words). */
typedef struct {
    uint32_t block_threads;   /* 128 or 256 */
    uint32_t blocks_per_sm;   /* 0: as many as fit */
    uint32_t unit_words;
    uint32_t _pad;
} ccs_batch_tuning;

ccs_status ccs_batch_get_tuning(const ccs_batch* b, ccs_batch_tuning* out);
/* a new block shape re-records the batch graph */
ccs_status ccs_batch_set_tuning(ccs_batch* b, const ccs_batch_tuning* t);

/* ---- served path ------------------------------------------------------------ */

/* A request server with continuous batching: requests (lattice ranges) are
 * admitted as slots and device memory free up; every scheduling tick runs
 * one chunk of every admitted request together in one batched graph replay,
 * so new arrivals overlap with long-running requests on the device.  Ticks
 * alternate between two batch executors: tick k is on the GPU while the host
 * collects and routes tick k - 1.  Results are identical to a plain
 * ccs_filter_range + ccs_prove of the whole range. */
typedef struct ccs_server ccs_server;

typedef struct {
    uint32_t max_active;      /* admitted requests per tick (batch slots) */
    uint32_t chunk_tiles;     /* tiles of one request per tick */
    uint64_t mem_cap_bytes;   /* admission budget for result buffers */
    uint32_t max_pending;     /* submitted-but-not-admitted queue bound */
    uint32_t _pad;
} ccs_server_config;

typedef struct {
    uint64_t n_survivors, n_chains, n_primes, candidates;
    double submit_s, admit_s, done_s;   /* monotonic seconds */
    uint32_t status;                    /* CCS_OK / CCS_PENDING / CCS_ERR_CANCELLED / CCS_OVERFLOW */
    uint32_t ticks;                     /* scheduling ticks the request took part in */
} ccs_request_result;

ccs_status ccs_server_create(ccs_engine* const* profiles, uint32_t n_profiles,
                             const ccs_server_config* cfg, ccs_server** out);
ccs_status ccs_server_destroy(ccs_server* s);
/* queue a range; CCS_ERR_BUSY when the pending queue is full */
ccs_status ccs_submit(ccs_server* s, const ccs_range* range, uint64_t* id);
/* CCS_PENDING while running; otherwise fills res and copies up to the given
 * capacities of survivors / chains (tile_idx relative to the range start)
 * and forgets the request */
ccs_status ccs_poll(ccs_server* s, uint64_t id, ccs_request_result* res, ccs_survivor* surv_host,
                    uint64_t surv_cap, ccs_chain* chains_host, uint64_t chain_cap);
/* block until the request is done (or timeout_ms passes: CCS_ERR_TIMEOUT) */
ccs_status ccs_wait(ccs_server* s, uint64_t id, uint32_t timeout_ms);
ccs_status ccs_cancel(ccs_server* s, uint64_t id);
/* batch tuning of the server's executor (ccs_batch_set_tuning), applied
 * before its next tick */
ccs_status ccs_server_set_batch_tuning(ccs_server* s, const ccs_batch_tuning* t);
/* device bytes reserved by admitted requests (residue rows and survivor /
 * chain slots of two ticks in flight), now and at the peak, against
 * mem_cap_bytes */
ccs_status ccs_server_memory(ccs_server* s, uint64_t* reserved_now, uint64_t* reserved_peak);
/* counters: [0] submitted [1] admitted [2] completed [3] cancelled [4] ticks [5] pending now */
ccs_status ccs_server_stats(ccs_server* s, uint64_t* out6);

/* ---- tuning -------------------------------------------------------------- */

typedef struct {
    uint32_t block_threads;   /* threads per block of the filter sweep: 128 or 256 */
    uint32_t blocks_per_sm;   /* resident blocks requested per SM */
    uint32_t unit_words;      /* 64-position words each lane sweeps per work unit (one lane
                               * owns one lattice residue: residues-per-thread = 1, positions
                               * per thread and unit = 64 x unit_words) */
    uint32_t split_prime;     /* first prime tested by the deferred warp-cooperative stage
                               * (changing it rebuilds the engine's filter tables) */
    uint32_t ext_min_words;   /* ranges spanning at least this many 64-position words of
                               * the extended lattice (smallest bit-sliced filter prime
                               * absorbed into the modulus) are swept on it; 1 = every
                               * range, 0xFFFFFFFF = none.  Both lattices give identical
                               * survivors. */
    uint32_t table_primes;    /* bit-sliced primes above 96 read from a pattern table (7 or
                               * 22; 0 = chosen by the engine's cost rule; changing it
                               * rebuilds the filter tables) */
} ccs_tuning;

ccs_status ccs_get_tuning(const ccs_engine* eng, ccs_tuning* out);
/* Zero fields keep their value.  A new split_prime or table_primes rebuilds
 * the engine's tables and is refused (CCS_ERR_BUSY) while a batch or server
 * uses the engine. */
ccs_status ccs_set_tuning(ccs_engine* eng, const ccs_tuning* t);

/* ---- autotuner ------------------------------------------------------------- */

/* One configuration the autotuner measured: the tuning and the device time
 * of one filter launch over the probe range. */
typedef struct {
    ccs_tuning tuning;
    uint64_t n_tiles;         /* probe size of this measurement */
    float ms;
    uint32_t _pad;
} ccs_tune_point;

#define CCS_TUNE_LATTICE 1u   /* plain vs extended lattice: the ext_min_words threshold */
#define CCS_TUNE_STAGES 2u    /* stage-split thresholds: split_prime, table_primes */
#define CCS_TUNE_UNITS 4u     /* positions per thread and work unit: unit_words */
#define CCS_TUNE_SHAPE 8u     /* block shape: block_threads, blocks_per_sm */
#define CCS_TUNE_ALL 15u

/* Times the filter on [ts, ts + n_tiles) (and, for the lattice threshold, on
 * shorter prefixes of it) under candidate tunings, one group of knobs after
 * another, keeps the fastest and leaves it set on the engine.  Every measured
 * point is written to points (up to cap; n_points gets the total).  Results
 * of the engine do not depend on the tuning.  Not thread-safe with other
 * calls on the same engine; refused (CCS_ERR_BUSY) for CCS_TUNE_STAGES while
 * a batch or server uses the engine. */
ccs_status ccs_autotune(ccs_engine* eng, uint64_t ts_lo, uint64_t ts_hi, uint64_t n_tiles,
                        uint32_t what, ccs_tune_point* points, uint32_t cap, uint32_t* n_points,
                        ccs_tuning* chosen);

/* Batch autotuner: runs the batch on the given ranges (results discarded)
 * for each unit length (each engine's own, 1024, 2048, 4096, 8192 words) and
 * block shape (1-3 blocks of 256 or 2-6 blocks of 128 threads, those that
 * fit), keeps the one with the shortest device time and leaves it set on
 * the batch.  Points
 * carry block_threads, blocks_per_sm and unit_words in their tuning. */
ccs_status ccs_batch_autotune(ccs_batch* b, const ccs_range* ranges, uint32_t n_ranges,
                              ccs_tune_point* points, uint32_t cap, uint32_t* n_points,
                              ccs_batch_tuning* chosen);

/* ---- diagnostics ----------------------------------------------------------- */

/* How ccs_filter_range would sweep a range on this engine with its current
 * tuning (host-only; no GPU work): the lattice chosen, the work units and
 * the launch shape.  A work unit is 32 lines x unit_words 64-position words;
 * the line table and line phase rows are read once per unit. */
typedef struct {
    uint32_t extended;        /* 1: the extended lattice (q0 absorbed into the modulus) */
    uint32_t q0;              /* absorbed prime (1: plain lattice) */
    uint64_t n_lines;         /* lines (residue classes) of the lattice used */
    uint32_t n_words;         /* 64-position words each line spans */
    uint32_t unit_words;      /* words per work unit */
    uint64_t units;           /* work units of the launch */
    uint32_t grid;            /* sweep blocks launched */
    uint32_t block_threads;
} ccs_range_plan;

ccs_status ccs_plan_range(const ccs_engine* eng, uint64_t tile_start_lo, uint64_t tile_start_hi,
                          uint64_t n_tiles, ccs_range_plan* out);

/* Measured INT32 ALU issue rate of the device (tera ops/s): eight independent
 * IADD3/LOP3 chains per thread, all SMs.  The roofline denominator of the
 * integer filter kernels. */
ccs_status ccs_measure_int32_peak(int device, double* tops);

/* Measured 32-bit multiply-add issue rate (IMAD / IMAD.HI chains), tera
 * ops/s: the roofline denominator of the Montgomery prover. */
ccs_status ccs_measure_imad_peak(int device, double* tops);

/* Counters of the staged proves (ccs_prove from 256 survivors on) of this
 * engine since the last reset: [0] survivors, [1] survivors whose n tested
 * prime, [2] primality tests of those n's predecessors, [3] n found to be
 * roots by a birth certificate instead (n == 1 mod a screen prime 67..863 --
 * second kind: n == -1 -- makes the predecessor a multiple of it; v34:70-77,
 * 2598-2612). */
ccs_status ccs_prove_stats(ccs_engine* eng, uint64_t* out4, int reset);

/* Montgomery products executed by ccs_walk_numbers launches on this device
 * since the last reset (reset != 0 clears after reading). */
ccs_status ccs_walk_modmuls(ccs_engine* eng, uint64_t* count, int reset);

/* The same count together with the 32 x 32-bit word products those
 * Montgomery products executed (2 NL^2 + NL per product for NL limbs); each
 * word product is one IMAD lo/hi pair. */
ccs_status ccs_walk_word_products(ccs_engine* eng, uint64_t* modmuls, uint64_t* words, int reset);

/* ------------------------------------------------------------------------
 * Fingerprint-pool Q iteration (the reference's v16 engine,
 * experimental/cc20_first_kind_immune_v16.cu).
 *
 * Candidates are p_0 = Q * D_V * 2^E - 1 for the variants V of a pool of
 * fingerprints D_V and consecutive Q.  Chain position j is
 * p_j = 2^(E+j) * Q * D_V - 1, so a prime q not dividing D_V divides p_j
 * exactly when Q = (D_V * 2^(E+j))^-1 (mod q); a Q is a survivor when no
 * sieve prime divides any of p_0 .. p_(depth-1) (v16:1244-1266, the
 * per-(V, q) forbid mask of v16:5104-5178 and its probe in
 * v16_q_iter_kernel, v16:2038-2153).  Primes that divide D_V sieve nothing
 * for V (the reference's active-prime pruning, v16:5229-5299).
 * ------------------------------------------------------------------------ */
typedef struct ccs_qiter ccs_qiter;

typedef struct {
    uint32_t n_variants;
    const uint32_t* dv;        /* [n_variants][4]: D_V as little-endian 32-bit limbs (< 2^128) */
    uint32_t exp_start;        /* E (--exp-start) */
    uint32_t depth;            /* sieved chain positions 0 .. depth-1 (--depth) */
    uint32_t target;           /* chain length of interest (--target): reverse prove order, TARGET flag */
    uint32_t n_primes;
    const uint32_t* primes;    /* sieve primes, ascending, odd, < 8192: the reference's q-iter list
                                  (7..sieve-max, v16:4680-4720) and, optionally, its CPU-side
                                  extended primes 509..1009 (v16:174-187, 2595-2616) */
    uint32_t primality;        /* CCS_PRIME_BPSW = mpz_probab_prime_p (v16:2677-2722) */
    uint32_t prove_mode;       /* CCS_PROVE_ROOTS: the reference's q-iter prover reports roots only */
    uint32_t flags;            /* CCS_FLAG_REVERSE_PROVE: position target - 1 first (the default
                                  --prove-order reverse, v16:2658-2673) */
} ccs_qiter_params;

/* One run of consecutive Q: Q = q_base + offset for offset < n_q, one variant. */
typedef struct {
    uint32_t q_base[4];        /* little-endian 32-bit limbs */
    uint32_t n_q;              /* Q values (the reference's --q-chunk per launch) */
    uint32_t variant;
} ccs_qseg;

/* Filter output: the reference's QSurvivor {thread_offset, seed_idx}
 * (v16:2140-2150) with the segment index; 16 bytes. */
typedef struct {
    uint32_t offset;           /* Q - q_base of the segment */
    uint32_t seg;
    uint32_t variant;
    uint32_t _pad;             /* written as 0 */
} ccs_qsurvivor;

/* Builds the per-variant forbidden-Q windows and uploads them.  One filter
 * call and one prove call may run at the same time on one object (two host
 * threads): they stage segments and run on separate streams. */
ccs_status ccs_qiter_create(const ccs_qiter_params* params, int device, ccs_qiter** out);
ccs_status ccs_qiter_destroy(ccs_qiter* qe);

/* Survivors of all segments (host array, n_segs <= 2^20) into a
 * caller-owned device buffer; CCS_OVERFLOW with the exact count in *n_out
 * when cap is too small.  Replaces v16_q_iter_kernel launched once per
 * (variant, chunk) (v16:5837-5881). */
ccs_status ccs_qiter_filter(ccs_qiter* qe, const ccs_qseg* segs, uint32_t n_segs, ccs_qsurvivor* out_dev,
                            uint64_t cap, uint64_t* n_out, void* stream);

/* Proves survivors on the device (BPSW predicate, reverse order, roots
 * only: the q-iter path of cpu_prove_worker, v16:2540-2722).  Records are
 * ccs_chain with base_idx = offset, k_offset = seg, tile_idx = variant and
 * root = p_0.  Every (Q + n_q) * D_V * 2^E of the segments must stay below
 * 2^160.  *primes_out counts survivors whose p_0 tested prime (after the
 * reverse gate). */
ccs_status ccs_qiter_prove(ccs_qiter* qe, const ccs_qseg* segs, uint32_t n_segs,
                           const ccs_qsurvivor* surv_dev, uint64_t n_surv, ccs_chain* out_dev,
                           uint64_t cap, uint64_t* n_out, uint64_t* primes_out, void* stream);

/* For variant v: counts[i] = how many residues of Q mod primes[i] are
 * forbidden (0 when primes[i] divides D_V: the prime is pruned), as the
 * uploaded windows hold them. */
ccs_status ccs_qiter_forbidden_count(const ccs_qiter* qe, uint32_t variant, uint32_t* counts, uint32_t cap);

#ifdef __cplusplus
}
#endif
#endif /* CCS_H */
