// Device-side records and launch helpers shared by the engine translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/ccs.h"
#include "ccs_internal.h"

namespace ccs {

constexpr int kSweepThreads = 256;

// device buffer owned by a host object (freed explicitly)
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count) {
        free_();
        n = count;
        return cudaMalloc((void**)&p, sizeof(T) * (count ? count : 1));
    }
    void free_() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// One lattice range as the device sees it.
struct RangeDev {
    uint32_t J0[4];          // floor(floor(tile_start / 6) / q0), u128 limbs
    uint32_t e0;             // tile_start mod 6
    uint32_t e1;             // floor(tile_start / 6) mod q0 (0 on a plain profile)
    uint32_t n_tiles;        // tiles in the range (< 2^32)
    uint32_t n_words;        // 64-position words spanned by the range's lines
    uint32_t unit_words;     // words per work unit
    uint32_t profile;        // constant-memory profile slot
    uint32_t prime_base;     // offset of this profile's prime list (range setup)
    uint32_t n_range_primes; // kNumA + nB + nC
    uint32_t surv_cap;       // capacity of surv
    uint32_t* surv_count;    // device counter (exact count, may exceed cap)
    uint32_t* surv;          // 4 x u32 records
    uint32_t* range_count;   // per-range survivor counter (may be null)
    uint32_t range_id;       // written into the record's last word (0 on the plain path)
    uint32_t tile_bias;      // added to tile_idx (chunked plain calls)
};

// header of a sweep launch, read on the device so graphs can be replayed
struct SweepHeader {
    uint32_t n_ranges;
    uint32_t _pad;
    uint64_t total_units;
};


// Prove-side description of one range.
struct ProveRange {
    uint32_t T0[4];          // tile_start (u128 limbs)
    uint32_t bits;
    uint32_t profile;
    uint32_t target;
    uint32_t _pad;
    uint32_t* chain_count;   // per-range chain counter (may be null)
    uint32_t* prime_count;   // per-range prime counter
};

// q-iteration survivors {offset, seg, variant} in a staged prove:
// p_0 = (q_base[seg] + offset) * D_V * 2^E - 1
struct QiterProve {
    const uint32_t* seg;                 // [n_segs][6]: q_base limbs, n_q, variant (null: lattice survivors)
    const uint32_t* dv;                  // [n_variants][4]
    uint32_t exp_start;
    uint32_t n_segs;                     // survivors naming another segment are skipped
};

// Prove launch: survivors of one or many ranges in one flat array.
struct ProveArgs {
    const ProveRange* ranges;
    const uint32_t* surv;          // 4 x u32 records
    const uint32_t* n_surv_dev;    // device count (null: use n_surv)
    uint32_t n_surv;
    uint32_t surv_cap;             // records readable
    uint32_t range_from_pad;       // 1: record word 3 holds the range index
    uint32_t* chains;              // 12 x u32 records
    uint32_t* chain_count;         // global counter
    uint32_t chain_cap;
    QiterProve q = {nullptr, nullptr, 0, 0};   // q-iteration survivors (seg null: lattice)
};

// Prover constants per profile (constant memory).
struct ProveConst {
    const uint64_t* bases;   // device copy of the base list
    uint32_t n_bases;
    uint32_t WP;
    uint32_t M;
    uint32_t primality;      // CCS_PRIME_MR / CCS_PRIME_BPSW
    uint32_t prove_mode;     // CCS_PROVE_ROOTS / CCS_PROVE_FULL
    uint32_t reverse;        // 1: test chain position target - 1 first (v15 --prove-order reverse)
    uint32_t kind;           // 1: p -> 2p + 1, 2: p -> 2p - 1 (v13b)
    uint32_t n_wit;
    uint32_t wit[32];
};

cudaError_t upload_profile_const(int slot, const ProfileConst& pc, cudaStream_t st);
cudaError_t upload_prove_const(int slot, const ProveConst& pc, cudaStream_t st);
cudaError_t launch_phase_table(const Line* lines, uint32_t n_lines, const SlotConst* pq, uint32_t n_slots,
                               uint16_t* tab, cudaStream_t st);
cudaError_t launch_range_setup(const RangeDev* ranges, const SweepHeader* hdr, uint32_t max_ranges,
                               const uint32_t* primes, uint32_t max_primes, uint32_t* jmod,
                               uint32_t stride, cudaStream_t st);
// merged: the launch stages the merged table windows of one profile per
// block (and keeps no per-warp table-window copies)
size_t sweep_smem_bytes(uint32_t block_threads, uint32_t b_stride, bool merged);
// lowreg: the register-capped variant (needed for more than the default
// variant's resident blocks; sweep_needs_lowreg tells); merge_slot: the
// profile slot whose merged table windows the launch uses (every range of the
// launch must be of that profile, a 22-prime standard set), or -1
cudaError_t launch_sweep(const RangeDev* ranges, const uint64_t* unit_prefix,
                         const SweepHeader* hdr, const uint32_t* jmod, uint32_t stride,
                         uint32_t b_stride, uint32_t grid, uint32_t block_threads, bool lowreg,
                         int merge_slot, cudaStream_t st);
bool sweep_needs_lowreg(uint32_t b_stride, uint32_t block_threads, uint32_t blocks_per_sm, bool merged);
cudaError_t launch_prove(const ProveArgs& a, uint32_t grid, cudaStream_t st);
// breadth-first chain walk (prove.cu)
struct WalkItem {
    uint32_t x[kMaxLimbs];   // current chain member
    uint32_t idx;            // position in the caller's batch
    uint32_t len;            // primes found so far
};
constexpr int kWalkBits = 32 * kMaxLimbs + 1;   // bit lengths 0..192
struct WalkState {
    uint32_t n_act;                      // items tested this round
    uint32_t n_next;                     // items for the next round
    uint32_t n_region[kMaxLimbs + 1];    // items per Montgomery limb count
    uint32_t off_region[kMaxLimbs + 1];
    uint32_t n_lucas[kMaxLimbs + 1];     // base-2 probable primes per limb count (from the
                                         // bottom of the region)
    uint32_t n_lucas_q2[kMaxLimbs + 1];  // of them with Selfridge D = -7 (BPSW; from the top)
    uint32_t n_bits[kWalkBits];          // items needing a test, per bit length
    uint32_t fill_bits[kWalkBits];       // next slot of each bit length in the sorted list
};
// Primality tests a walk round can apply (CCS_PRIME_MR / CCS_PRIME_BPSW,
// plus the two native tests of the reference CPU engine v33)
enum : uint32_t {
    kPredMR = 0,                         // strong PRP for every witness of the profile
    kPredBPSW = 1,                       // Baillie-PSW (GMP mpz_probab_prime_p(n, 1))
    kPredMR235 = 3,                      // strong PRP to bases 2, 3, 5 (v33 is_prime_root_native)
    kPredFermat2 = 4                     // 2^(n-1) == 1 (mod n) (v33 is_prime_pocklington_native)
};

struct WalkArgs {
    uint32_t max_len;                    // walks end at this length (chain lengths cap)
    uint32_t pred;                       // test of members that start a walk (len 0) or are
                                         // tested alone (stage tests)
    uint32_t link_pred;                  // test of forward links (len >= 1) when screen is set
    uint32_t screen;                     // 1: links are first screened by the 132 primes
                                         // 67..863 (a zero residue is composite) and capped
    uint32_t cap_bits;                   // with screen: a link of more bits ends the walk (0: none)
    WalkState* st;
    const WalkItem* act;
    WalkItem* sorted;                    // act, grouped by limb count
    WalkItem* lucas;                     // same regions as sorted
    WalkItem* next;
    uint8_t* code;                       // trial-stage verdict per act item
    uint32_t* lengths;
    int profile;
};
cudaError_t launch_walk_load(const uint32_t* numbers, uint64_t first, uint32_t n, uint32_t limbs,
                             WalkItem* out, cudaStream_t st);
// round_pred: the test of this round's members (every member of a round is
// either a walk start / stage member or a forward link)
cudaError_t launch_walk_round(const WalkArgs& a, uint32_t n_act, bool two_stage, uint32_t round_pred,
                              cudaStream_t st);

// staged prove of one range's survivors (prove.cu)
struct StagedProve {
    QiterProve q;
    const ProveRange* range;
    const uint32_t* surv;                // survivor records (4 x u32)
    uint32_t first, n_surv;              // this chunk: records [first, first + n_surv)
    uint32_t* nval;                      // [n_surv][kMaxLimbs] survivor numbers
    uint32_t* root;                      // [n_surv][kMaxLimbs] current root
    uint32_t* flags;                     // [n_surv] CCS_CHAIN_IS_ROOT
    uint32_t* lengths;                   // [n_surv] verdict of the last stage / chain length
    WalkItem* out;                       // members for the next primality stage
    uint32_t* count;
    WalkItem* fwd;                       // roots ready for the forward walk
    uint32_t* fwd_count;
    uint32_t* primes;
    uint32_t* chains;
    uint32_t* chain_count;
    uint32_t chain_cap;
    uint32_t* certified;                 // roots decided by a birth certificate (no predecessor test)
};
// which: -1 seed, 0 after the top member, 1 after n, 2 after a predecessor, 3 emit
cudaError_t launch_prove_stage(int which, const StagedProve& p, const WalkItem* in, uint32_t n,
                               cudaStream_t st);
int sweep_blocks_per_sm(uint32_t b_stride, uint32_t block_threads, bool merged = false);

// engine services used by the q-iteration object (engine.cu); set_error
// records the message ccs_last_error returns
ccs_status set_error(ccs_status st, const char* msg);
ccs_status engine_create_prover(int device, uint32_t primality, uint32_t prove_mode, bool reverse,
                                uint32_t target, ccs_engine** out);
ccs_status engine_prove_staged(ccs_engine* E, const ccs_survivor* surv_dev, uint64_t n_surv,
                               const ProveRange& pr, const QiterProve* q, ccs_chain* out_dev,
                               uint64_t cap, uint64_t* n_out, uint64_t* primes_out, cudaStream_t st);
cudaStream_t engine_stream(ccs_engine* E);
int engine_slot(const ccs_engine* E);
cudaError_t modmul_count(uint64_t* out, uint64_t* words, bool reset);

}  // namespace ccs
