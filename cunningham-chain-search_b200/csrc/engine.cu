// C-ABI implementation: engine lifetime, plain per-range path, host-buffer
// path, number walks and the batched (graph-replayed) executor.
//
// Reference behaviour replaced: gpu_upload_tables (v13:1065-1222), the
// per-batch launch/copy sequence of the main loop (v13:3719-3906) and the
// error policy (CUDA_CHECK -> exit, v13:142-149): every failure here is a
// returned status plus a message in ccs_last_error().
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ccs.h"
#include "ccs_internal.h"
#include "ccs_kernels.cuh"

using namespace ccs;

namespace {

thread_local std::string g_err;

ccs_status fail(ccs_status st, const std::string& msg) {
    g_err = msg;
    return st;
}

#define CU(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(e_ == cudaErrorMemoryAllocation ? CCS_ERR_NOMEM : CCS_ERR_CUDA,   \
                        std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)

// survivor counts from which ccs_prove runs the staged (breadth-first) prove
constexpr uint64_t kStagedProveMin = 256;
// largest extended lattice built (lines of 16 bytes)
constexpr uint64_t kExtLinesMax = 1ull << 26;

// constant-memory profile slots, per device
std::mutex g_slot_mu;
uint32_t g_slots_used[64] = {0};

int alloc_slot(int dev) {
    std::lock_guard<std::mutex> lk(g_slot_mu);
    for (int s = 0; s < kMaxProfiles; s++)
        if (!(g_slots_used[dev] & (1u << s))) { g_slots_used[dev] |= 1u << s; return s; }
    return -1;
}

void free_slot(int dev, int s) {
    std::lock_guard<std::mutex> lk(g_slot_mu);
    if (s >= 0) g_slots_used[dev] &= ~(1u << s);
}

const uint32_t kRefCrt[] = {5, 7, 11, 13, 17, 19};
const uint32_t kRefWheel[] = {23, 29, 31};
const uint32_t kRefL2[] = {37, 41, 43, 47, 53, 59, 61};
const uint32_t kRefExt[] = {67, 71, 73, 79, 83, 89, 97};
const uint64_t kRefWit[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71};

// One filter variant of a profile: the lattice lines and the per-prime tables
// the sweep reads, plus the constant-memory slot they are registered in.
struct FilterSet {
    HostProfile hp;
    int slot = -1;
    DevBuf<Line> lines;
    DevBuf<PrimeC> primesB, primesC;
    DevBuf<PrimeB> packB;
    DevBuf<uint32_t> bitmapB, listC, bitmapC, range_primes, patT, patM;
    DevBuf<uint16_t> ptab;           // line phase table (may stay empty)
    DevBuf<SlotConst> pq;
    void free_() {
        lines.free_(); primesB.free_(); primesC.free_(); packB.free_();
        bitmapB.free_(); listC.free_(); bitmapC.free_(); range_primes.free_(); patT.free_();
        patM.free_();
        ptab.free_(); pq.free_();
    }
};

}  // namespace

// fs[0] is the profile as given (the lattice of the reference); fs[1], when
// present, is the same profile with its smallest bit-sliced filter prime q0
// absorbed into the modulus (W' = q0 W, lines r + d W for the d in [0, q0)
// that q0 does not kill).  Long ranges are swept on fs[1]; both produce the
// same survivors in the same (base, k, tile) coordinates.
struct ccs_engine {
    int device = 0;
    FilterSet fs[2];
    int n_fs = 1;
    ccs_tuning tune{};
    int sms = 148;
    cudaStream_t own_stream = nullptr;
    int slot = -1;                   // == fs[0].slot: prove-side constants
    HostProfile& hp = fs[0].hp;      // the profile as given
    int users = 0;                   // batches / servers referencing the tables

    DevBuf<uint64_t> bases;

    // plain-path working state
    DevBuf<RangeDev> d_range;
    DevBuf<ProveRange> d_prange;
    DevBuf<uint64_t> d_prefix;
    DevBuf<SweepHeader> d_hdr;
    DevBuf<uint32_t> d_jmod;
    DevBuf<uint32_t> d_counters;     // [0] surv, [1] spare, [2] chains, [3] primes
    // host-path scratch
    DevBuf<uint32_t> d_surv_scratch, d_chain_scratch;
    // chain-walk rounds: items, sorted / Lucas regions, next round, codes, state
    DevBuf<WalkItem> w_act, w_next, w_sorted, w_lucas;
    DevBuf<uint8_t> w_code;
    DevBuf<WalkState> w_state;
    // staged prove: per-survivor numbers, roots, flags, verdicts; item lists
    DevBuf<uint32_t> p_nval, p_root, p_flags, p_len, p_ctr;
    DevBuf<WalkItem> p_items0, p_items1, p_fwd;
    // pinned staging
    void* h_stage = nullptr;
    size_t h_stage_bytes = 0;
    uint64_t launches = 0;           // kernels launched by this engine
    // staged proves: survivors, primes n, predecessor tests, roots decided
    // by a birth certificate
    uint64_t stats[4] = {0, 0, 0, 0};
};

struct ccs_batch {
    std::vector<ccs_engine*> prof;
    int device = 0;
    uint32_t max_ranges = 0;
    uint64_t surv_cap = 0, chain_cap = 0;
    uint32_t jstride = 0;
    DevBuf<RangeDev> d_ranges;
    DevBuf<ProveRange> d_pranges;
    DevBuf<uint64_t> d_prefix;
    DevBuf<SweepHeader> d_hdr;
    DevBuf<uint32_t> d_jmod, d_primes;   // concatenated range-prime lists of all profiles
    DevBuf<uint32_t> d_surv, d_chains;
    DevBuf<uint32_t> d_counts;           // [0] surv [1] spare [2] chains [3] spare, then 3 per range
    std::vector<uint32_t> prime_base;    // offset into d_primes per (profile i, filter set v): [2 i + v]
    uint32_t max_range_primes = 0;
    uint32_t b_stride = 0;
    // pinned staging: ranges, prefix, header, counts
    RangeDev* h_ranges = nullptr;
    ProveRange* h_pranges = nullptr;
    uint64_t* h_prefix = nullptr;
    SweepHeader* h_hdr = nullptr;
    uint32_t* h_counts = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0;
    uint32_t grid = 0;
    uint32_t nc = 0;                     // counters in d_counts
    // batch tuning: sweep block shape (captured in the graph) and the work
    // unit length of every range (0: each engine's own)
    uint32_t block_threads = 0, blocks_per_sm = 0, unit_words = 0;
    uint32_t req_blocks_per_sm = 0;      // requested (0: as many as fit)
    bool in_flight = false;              // launched, not yet waited for
    std::vector<ccs_range> cur_ranges;   // ranges of the launch in flight
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
namespace {

struct U128 {
    uint64_t lo, hi;
};

inline unsigned __int128 mk128(uint64_t lo, uint64_t hi) {
    return ((unsigned __int128)hi << 64) | lo;
}

void fill_J0(uint32_t (&J0)[4], unsigned __int128 v) {
    for (int i = 0; i < 4; i++) J0[i] = (uint32_t)(v >> (32 * i));
}

uint32_t words_for(uint32_t e0, uint64_t n_tiles) {
    uint64_t span = (e0 + n_tiles + 5) / 6;
    return (uint32_t)((span + 63) / 64);
}

ccs_status upload_filter(FilterSet& f, cudaStream_t st) {
    const HostProfile& hp = f.hp;
    CU(f.lines.alloc(hp.lines.size()));
    CU(cudaMemcpy(f.lines.p, hp.lines.data(), sizeof(Line) * hp.lines.size(), cudaMemcpyHostToDevice));
    CU(f.primesB.alloc(hp.primesB.size()));
    if (!hp.primesB.empty())
        CU(cudaMemcpy(f.primesB.p, hp.primesB.data(), sizeof(PrimeC) * hp.primesB.size(), cudaMemcpyHostToDevice));
    CU(f.primesC.alloc(hp.primesC.size()));
    if (!hp.primesC.empty())
        CU(cudaMemcpy(f.primesC.p, hp.primesC.data(), sizeof(PrimeC) * hp.primesC.size(), cudaMemcpyHostToDevice));
    CU(f.packB.alloc(hp.packB.size()));
    if (!hp.packB.empty())
        CU(cudaMemcpy(f.packB.p, hp.packB.data(), sizeof(PrimeB) * hp.packB.size(), cudaMemcpyHostToDevice));
    CU(f.bitmapB.alloc(hp.bitmapB.size()));
    if (!hp.bitmapB.empty())
        CU(cudaMemcpy(f.bitmapB.p, hp.bitmapB.data(), 4 * hp.bitmapB.size(), cudaMemcpyHostToDevice));
    CU(f.listC.alloc(hp.listC.size()));
    if (!hp.listC.empty())
        CU(cudaMemcpy(f.listC.p, hp.listC.data(), 4 * hp.listC.size(), cudaMemcpyHostToDevice));
    CU(f.bitmapC.alloc(hp.bitmapC.size()));
    if (!hp.bitmapC.empty())
        CU(cudaMemcpy(f.bitmapC.p, hp.bitmapC.data(), 4 * hp.bitmapC.size(), cudaMemcpyHostToDevice));
    CU(f.patM.alloc(hp.patM.size()));
    if (!hp.patM.empty())
        CU(cudaMemcpy(f.patM.p, hp.patM.data(), 4 * hp.patM.size(), cudaMemcpyHostToDevice));
    CU(f.patT.alloc(hp.patT.size()));
    CU(cudaMemcpy(f.patT.p, hp.patT.data(), 4 * hp.patT.size(), cudaMemcpyHostToDevice));
    CU(f.range_primes.alloc(hp.range_primes.size()));
    CU(cudaMemcpy(f.range_primes.p, hp.range_primes.data(), 4 * hp.range_primes.size(), cudaMemcpyHostToDevice));

    ProfileConst pc;
    memset(&pc, 0, sizeof(pc));
    pc.W = hp.W;
    pc.q0 = hp.q0;
    pc.n_lines = (uint32_t)hp.lines.size();
    pc.nB = (uint32_t)hp.primesB.size();
    pc.nBpad = (uint32_t)hp.packB.size();
    pc.nC = (uint32_t)hp.primesC.size();
    memcpy(pc.A, hp.A, sizeof(pc.A));
    pc.patT = f.patT.p;
    pc.patT_words = (uint32_t)hp.patT.size();
    pc.lines = f.lines.p;
    pc.primesB = f.primesB.p;
    pc.packB = f.packB.p;
    pc.bitmapB = f.bitmapB.p;
    pc.std_a = hp.std_a;
    pc.primesC = f.primesC.p;
    pc.listC = f.listC.p;
    pc.bitmapC = f.bitmapC.p;
    pc.nCb = hp.nCb;
    pc.patM = hp.patM.empty() ? nullptr : f.patM.p;
    // line phase table for every level-A slot and level-B prime, when it fits
    {
        const uint32_t nb = hp.primesB.empty() ? 1u : (uint32_t)hp.primesB.size();
        const uint32_t n_slots = kSlotB + ((nb + 7) & ~7u);           // level-B rows as in shared memory
        const size_t bytes = 2ull * n_slots * hp.lines.size();
        if (bytes <= kPhaseTableMax && !hp.lines.empty()) {
            std::vector<SlotConst> pq(n_slots, SlotConst{2u, 0xFFFFFFFFu / 2, 0u, 0u});   // pads: phase 0
            for (int i = 0; i < kNumA; i++) pq[i] = SlotConst{hp.A[i].q, hp.A[i].magic, hp.A[i].c32, hp.A[i].winv};
            for (int i = kNumA; i < kSlotB; i++) pq[i] = SlotConst{1u, 0xFFFFFFFFu, 0u, 0u};
            for (size_t p = 0; p < hp.primesB.size(); p++) {
                const PrimeC& b = hp.primesB[p];
                pq[kSlotB + p] = SlotConst{b.q, b.magic, b.c32, b.winv};
            }
            CU(f.pq.alloc(n_slots));
            CU(cudaMemcpy(f.pq.p, pq.data(), sizeof(SlotConst) * n_slots, cudaMemcpyHostToDevice));
            CU(f.ptab.alloc((size_t)n_slots * hp.lines.size()));
            CU(launch_phase_table(f.lines.p, (uint32_t)hp.lines.size(), f.pq.p, n_slots, f.ptab.p, st));
            pc.ptab = f.ptab.p;
            pc.pq = f.pq.p;
            pc.ptab_stride = n_slots;
        }
    }
    CU(upload_profile_const(f.slot, pc, st));
    CU(cudaStreamSynchronize(st));
    return CCS_OK;
}

ccs_status upload_prove(ccs_engine* E, cudaStream_t st) {
    const HostProfile& hp = E->hp;
    CU(E->bases.alloc(hp.bases.size()));
    CU(cudaMemcpy(E->bases.p, hp.bases.data(), 8 * hp.bases.size(), cudaMemcpyHostToDevice));
    ProveConst pv;
    memset(&pv, 0, sizeof(pv));
    pv.bases = E->bases.p;
    pv.n_bases = (uint32_t)hp.bases.size();
    pv.WP = hp.WP;
    pv.M = (uint32_t)hp.M;
    pv.primality = hp.primality;
    pv.prove_mode = hp.prove_mode;
    pv.reverse = hp.reverse_prove;
    pv.kind = hp.kind;
    pv.n_wit = (uint32_t)std::min<size_t>(hp.witnesses.size(), 32);
    for (uint32_t i = 0; i < pv.n_wit; i++) pv.wit[i] = (uint32_t)hp.witnesses[i];
    CU(upload_prove_const(E->slot, pv, st));
    CU(cudaStreamSynchronize(st));
    return CCS_OK;
}

// level-B phase rows per lane column in shared memory: the level-B records
// padded to a whole number of rounds (the rows the rounds read), rounded up
// to 8 rows (the phase-table rows are read 8 at a time)
uint32_t b_stride_of(uint32_t nB) {
    uint32_t s = nB ? nB : 1;
    s = (s + kLevelBRound - 1) / kLevelBRound * kLevelBRound;
    return (s + 7) & ~7u;
}

uint32_t max_level_b(const ccs_engine* E) {
    uint32_t nb = 0;
    for (int v = 0; v < E->n_fs; v++) nb = std::max<uint32_t>(nb, (uint32_t)E->fs[v].hp.primesB.size());
    return nb;
}

// resident sweep blocks per SM for a block size (at least 1)
uint32_t max_blocks_per_sm(const ccs_engine* E, uint32_t block_threads) {
    const int bps = sweep_blocks_per_sm(b_stride_of(max_level_b(E)), block_threads);
    return bps > 0 ? (uint32_t)bps : 1u;
}

// A one-range sweep of filter set f uses the merged table windows when the
// profile has them (22-prime standard sets) and the tuned resident-block
// count still fits with their per-block copy in shared memory.
static bool use_merged(const ccs_engine* E, const FilterSet& f, uint32_t b_stride) {
    return f.hp.patM.size() == kPatMWords && f.slot >= 0 &&
           sweep_blocks_per_sm(b_stride, E->tune.block_threads, true) >= (int)E->tune.blocks_per_sm;
}

// (Re)builds the engine's filter sets for a level-B/C split prime and a
// table-window count: the profile as given (fs[0]) and, when its smallest
// bit-sliced prime q0 is below 64, the extended lattice that absorbs q0
// (fs[1]).  Tables are uploaded into the engine's constant-memory slots
// (allocated on first use).  The engine stream is drained first.
ccs_status build_filters(ccs_engine* E, uint32_t split, uint32_t t_count) {
    HostProfile nh[2];
    auto params_of = [&](HostProfile& d) {
        const HostProfile& s = E->fs[0].hp;
        d.target = s.target; d.depth = s.depth; d.bits = s.bits;
        d.crt = s.crt; d.wheel = s.wheel; d.stages = s.stages;
        d.max_bases = s.max_bases; d.witnesses = s.witnesses;
        d.primality = s.primality; d.prove_mode = s.prove_mode;
        d.reverse_prove = s.reverse_prove;
        d.kind = s.kind;
        d.t_count = t_count;
    };
    params_of(nh[0]);
    std::string err = build_profile(nh[0], split);
    if (!err.empty()) return fail(CCS_ERR_INVALID, err);
    if (nh[0].primesB.size() > (size_t)kMaxLevelB) return fail(CCS_ERR_INVALID, "too many level-B primes");
    int n_new = 1;
    // the extended lattice multiplies the lines by q0 - |F_q0|; it is built
    // while its line table stays within kExtLinesMax lines (1 GiB)
    uint64_t ext_lines = 0;
    if (nh[0].A[0].q > 1 && nh[0].A[0].q < 64) {
        for (const auto& fp : nh[0].fprimes)
            if (fp.q == nh[0].A[0].q) ext_lines = (uint64_t)nh[0].lines.size() * (fp.q - fp.forb.size());
    }
    if (ext_lines && ext_lines <= kExtLinesMax) {
        params_of(nh[1]);
        if (build_profile(nh[1], split, nh[0].A[0].q).empty() && nh[1].primesB.size() <= (size_t)kMaxLevelB)
            n_new = 2;
    }
    if (E->own_stream) CU(cudaStreamSynchronize(E->own_stream));
    for (int v = 0; v < 2; v++) {
        if (v < n_new && E->fs[v].slot < 0) {
            E->fs[v].slot = alloc_slot(E->device);
            if (E->fs[v].slot < 0)
                return fail(CCS_ERR_BUSY, "all constant-memory profile slots in use (max 16 filter profiles per device)");
        }
        if (v >= n_new && E->fs[v].slot >= 0) { free_slot(E->device, E->fs[v].slot); E->fs[v].slot = -1; }
        E->fs[v].free_();
    }
    uint32_t max_np = 0;
    for (int v = 0; v < n_new; v++) {
        E->fs[v].hp = nh[v];
        ccs_status st = upload_filter(E->fs[v], E->own_stream);
        if (st != CCS_OK) return st;
        max_np = std::max<uint32_t>(max_np, (uint32_t)nh[v].range_primes.size());
    }
    E->n_fs = n_new;
    E->slot = E->fs[0].slot;
    if (E->d_jmod.n < max_np) CU(E->d_jmod.alloc(max_np));
    E->tune.split_prime = split;
    E->tune.table_primes = t_count;
    return CCS_OK;
}

// work units for one range
uint64_t units_of(const FilterSet& f, uint32_t n_words, uint32_t unit_words) {
    uint64_t groups = (f.hp.lines.size() + 31) / 32;
    uint64_t chunks = (n_words + unit_words - 1) / unit_words;
    return groups * chunks;
}

// words per work unit: the tuned length; when the range runs alone on the
// GPU (fill_gpu) it is shortened so every resident warp gets several units
uint32_t choose_unit_words(const ccs_engine* E, const FilterSet& f, uint32_t n_words, bool fill_gpu) {
    uint32_t uw = E->tune.unit_words ? E->tune.unit_words : 1024;
    uint64_t groups = (f.hp.lines.size() + 31) / 32;
    uint64_t warps = (uint64_t)E->sms * std::max<uint32_t>(E->tune.blocks_per_sm, 1) * (E->tune.block_threads / 32);
    uint64_t chunks_wanted = (4 * warps + groups - 1) / groups;
    if (fill_gpu && chunks_wanted > 1) {
        uint64_t fit = (n_words + chunks_wanted - 1) / chunks_wanted;
        if (fit < uw) uw = (uint32_t)std::max<uint64_t>(fit, 32);
    }
    if (uw > n_words) uw = n_words ? n_words : 1;
    return uw;
}

// Places a range of n_tiles tiles from ts on one of the engine's filter sets:
// the extended one when the range spans at least ext_min_words 64-position
// words of it.  Fills J0, e0, e1, n_tiles, n_words, unit_words, profile and
// n_range_primes; returns the filter set used.
const FilterSet& place_range(const ccs_engine* E, unsigned __int128 ts, uint64_t n_tiles, RangeDev& R,
                             bool fill_gpu = true) {
    const unsigned __int128 J = ts / 6;
    R.e0 = (uint32_t)(ts % 6);
    R.n_tiles = (uint32_t)n_tiles;
    const uint64_t span = n_tiles ? (R.e0 + n_tiles + 5) / 6 : 0;     // blocks touched
    int v = 0;
    if (E->n_fs > 1 && E->tune.ext_min_words != 0xFFFFFFFFu) {
        const uint32_t q0 = E->fs[1].hp.q0;
        if (((span + q0 - 1) / q0 + 63) / 64 >= E->tune.ext_min_words) v = 1;
    }
    const FilterSet& f = E->fs[v];
    const uint32_t q0 = f.hp.q0;
    fill_J0(R.J0, J / q0);
    R.e1 = (uint32_t)(J % q0);
    const uint64_t positions = (span + R.e1 + q0 - 1) / q0;
    R.n_words = n_tiles ? (uint32_t)((positions + 63) / 64) : 0;
    R.unit_words = choose_unit_words(E, f, R.n_words, fill_gpu);
    R.profile = (uint32_t)f.slot;
    R.n_range_primes = (uint32_t)f.hp.range_primes.size();
    return f;
}

}  // namespace

// ---------------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------------
extern "C" {

const char* ccs_last_error(void) { return g_err.c_str(); }
int ccs_abi_version(void) { return CCS_ABI_VERSION; }

static ccs_status params_to_profile(const ccs_params* params, HostProfile& hp) {
    ccs_params def;
    memset(&def, 0, sizeof(def));
    const ccs_params& p = params ? *params : def;
    if (p.kind != 0 && p.kind != CCS_KIND_FIRST && p.kind != CCS_KIND_SECOND)
        return fail(CCS_ERR_INVALID, "kind must be CCS_KIND_FIRST or CCS_KIND_SECOND");
    hp.kind = p.kind == CCS_KIND_SECOND ? 2u : 1u;
    hp.target = p.target ? p.target : 18;
    hp.depth = p.depth ? p.depth : hp.target;
    hp.bits = p.bits ? p.bits : 89;
    if (p.crt_primes && p.n_crt) hp.crt.assign(p.crt_primes, p.crt_primes + p.n_crt);
    else hp.crt.assign(kRefCrt, kRefCrt + 6);
    if (p.wheel_primes && p.n_wheel) hp.wheel.assign(p.wheel_primes, p.wheel_primes + p.n_wheel);
    else hp.wheel.assign(kRefWheel, kRefWheel + 3);
    hp.stages.clear();
    if (p.stages && p.n_stages) {
        if (p.n_stages > (uint32_t)kMaxStages) return fail(CCS_ERR_INVALID, "too many stages");
        for (uint32_t s = 0; s < p.n_stages; s++) {
            HostProfile::Stage st;
            if (p.stages[s].n_primes && !p.stages[s].primes) return fail(CCS_ERR_INVALID, "stage primes null");
            st.primes.assign(p.stages[s].primes, p.stages[s].primes + p.stages[s].n_primes);
            st.pos_lo = p.stages[s].pos_lo;
            hp.stages.push_back(st);
        }
    } else {
        HostProfile::Stage a, b, c;
        a.primes.assign(kRefL2, kRefL2 + 7); a.pos_lo = 0;
        b.primes.assign(kRefExt, kRefExt + 7); b.pos_lo = 0;
        for (uint32_t q = 101; q <= 863; q++)
            if (is_prime_u32(q)) c.primes.push_back(q);
        c.pos_lo = 1;
        hp.stages = {a, b, c};
    }
    hp.max_bases = p.max_bases;
    if (p.witnesses && p.n_witnesses) {
        if (p.n_witnesses > 32) return fail(CCS_ERR_INVALID, "at most 32 witnesses");
        for (uint32_t i = 0; i < p.n_witnesses; i++)
            if (p.witnesses[i] < 2 || p.witnesses[i] > 0xFFFFFFFFull)
                return fail(CCS_ERR_INVALID, "witnesses must be in [2, 2^32)");
        hp.witnesses.assign(p.witnesses, p.witnesses + p.n_witnesses);
    } else {
        hp.witnesses.assign(kRefWit, kRefWit + 20);
    }
    hp.primality = p.primality;
    hp.prove_mode = p.prove_mode;
    if (hp.primality > CCS_PRIME_V33 || hp.prove_mode > 1) return fail(CCS_ERR_INVALID, "bad primality / prove_mode");
    if (hp.primality == CCS_PRIME_V33 && (hp.prove_mode != CCS_PROVE_FULL || hp.kind != 1))
        return fail(CCS_ERR_INVALID, "CCS_PRIME_V33 is the reference CPU engine's first-kind full prove "
                                     "(CCS_PROVE_FULL, first kind)");
    if (p.flags & ~CCS_FLAG_REVERSE_PROVE) return fail(CCS_ERR_INVALID, "unknown flags");
    hp.reverse_prove = (p.flags & CCS_FLAG_REVERSE_PROVE) ? 1u : 0u;
    if (hp.reverse_prove && hp.prove_mode != CCS_PROVE_ROOTS)
        return fail(CCS_ERR_INVALID, "reverse prove order is a CCS_PROVE_ROOTS option (the reference K2's)");
    std::string err = build_profile(hp, 1024);
    if (!err.empty()) return fail(CCS_ERR_INVALID, err);
    if (hp.primesB.size() > (size_t)kMaxLevelB) return fail(CCS_ERR_INVALID, "too many level-B primes");
    return CCS_OK;
}

static void fill_info(const HostProfile& hp, ccs_info* o) {
    o->lattice_m = hp.M;
    o->wheel_period = hp.WP;
    o->n_bases = (uint32_t)hp.bases.size();
    o->n_lines = hp.lines.size();
    uint64_t tot = 0;
    for (uint32_t w : hp.wheel_total) tot += w;
    o->candidates_per_tile = tot / 6;
    o->target = hp.target;
    o->depth = hp.depth;
    o->bits = hp.bits;
    o->n_filter_primes = (uint32_t)hp.fprimes.size();
    o->expected_tests = hp.expected_tests;
    o->pass_rate = hp.pass_rate;
    o->launches = 0;
}

ccs_status ccs_describe(const ccs_params* params, ccs_info* out, uint64_t* bases, uint32_t cap) {
    if (!out) return fail(CCS_ERR_INVALID, "out is null");
    HostProfile hp;
    ccs_status s = params_to_profile(params, hp);
    if (s != CCS_OK) return s;
    fill_info(hp, out);
    if (bases) {
        uint32_t n = (uint32_t)std::min<size_t>(cap, hp.bases.size());
        memcpy(bases, hp.bases.data(), 8 * n);
        if (cap < hp.bases.size()) return fail(CCS_OVERFLOW, "bases capacity exceeded");
    }
    return CCS_OK;
}

ccs_status ccs_create(const ccs_params* params, int device, ccs_engine** out) {
    if (!out) return fail(CCS_ERR_INVALID, "out is null");
    *out = nullptr;
    int ndev = 0;
    CU(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev || device >= 64) return fail(CCS_ERR_INVALID, "bad device ordinal");
    CU(cudaSetDevice(device));
    ccs_engine* E = new ccs_engine();
    E->device = device;
    HostProfile& hp = E->hp;
    {
        ccs_status s = params_to_profile(params, hp);
        if (s != CCS_OK) { delete E; return s; }
    }
    E->tune.block_threads = kSweepThreads;
    E->tune.unit_words = 1024;
    E->tune.split_prime = 1024;
    E->tune.ext_min_words = 256;
    E->tune.table_primes = 0;
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    E->sms = prop.multiProcessorCount;
    CU(cudaStreamCreateWithFlags(&E->own_stream, cudaStreamNonBlocking));
    {
        ccs_status st = build_filters(E, 1024, 0);
        if (st != CCS_OK) { ccs_destroy(E); return st; }
        st = upload_prove(E, E->own_stream);
        if (st != CCS_OK) { ccs_destroy(E); return st; }
    }
    E->tune.blocks_per_sm = max_blocks_per_sm(E, E->tune.block_threads);

    // plain-path state
    if (E->d_range.alloc(1) || E->d_prange.alloc(1) || E->d_prefix.alloc(2) || E->d_hdr.alloc(1) ||
        E->d_counters.alloc(8)) {
        ccs_destroy(E);
        return fail(CCS_ERR_NOMEM, "device allocation failed");
    }
    E->h_stage_bytes = 1 << 16;
    if (cudaMallocHost(&E->h_stage, E->h_stage_bytes) != cudaSuccess) {
        ccs_destroy(E);
        return fail(CCS_ERR_NOMEM, "pinned allocation failed");
    }
    *out = E;
    return CCS_OK;
}

ccs_status ccs_destroy(ccs_engine* E) {
    if (!E) return CCS_OK;
    cudaSetDevice(E->device);
    if (E->own_stream) cudaStreamSynchronize(E->own_stream);
    for (auto& f : E->fs) f.free_();
    E->bases.free_();
    E->d_range.free_(); E->d_prange.free_(); E->d_prefix.free_(); E->d_hdr.free_();
    E->d_jmod.free_(); E->d_counters.free_();
    E->d_surv_scratch.free_(); E->d_chain_scratch.free_();
    E->w_act.free_(); E->w_next.free_(); E->w_sorted.free_(); E->w_lucas.free_();
    E->w_code.free_(); E->w_state.free_();
    E->p_nval.free_(); E->p_root.free_(); E->p_flags.free_(); E->p_len.free_(); E->p_ctr.free_();
    E->p_items0.free_(); E->p_items1.free_(); E->p_fwd.free_();
    if (E->h_stage) cudaFreeHost(E->h_stage);
    if (E->own_stream) cudaStreamDestroy(E->own_stream);
    for (auto& f : E->fs) free_slot(E->device, f.slot);
    delete E;
    return CCS_OK;
}

ccs_status ccs_get_info(const ccs_engine* E, ccs_info* o) {
    if (!E || !o) return fail(CCS_ERR_INVALID, "null argument");
    fill_info(E->hp, o);
    o->launches = E->launches;
    return CCS_OK;
}

ccs_status ccs_get_bases(const ccs_engine* E, uint64_t* bases, uint32_t cap) {
    if (!E || !bases) return fail(CCS_ERR_INVALID, "null argument");
    uint32_t n = (uint32_t)std::min<size_t>(cap, E->hp.bases.size());
    memcpy(bases, E->hp.bases.data(), 8 * n);
    return cap < E->hp.bases.size() ? CCS_OVERFLOW : CCS_OK;
}

ccs_status ccs_get_tuning(const ccs_engine* E, ccs_tuning* t) {
    if (!E || !t) return fail(CCS_ERR_INVALID, "null argument");
    *t = E->tune;
    return CCS_OK;
}

ccs_status ccs_set_tuning(ccs_engine* E, const ccs_tuning* t) {
    if (!E || !t) return fail(CCS_ERR_INVALID, "null argument");
    if (t->block_threads && t->block_threads != 128 && t->block_threads != 256)
        return fail(CCS_ERR_INVALID, "block_threads must be 128 or 256");
    if (t->unit_words > (1u << 20)) return fail(CCS_ERR_INVALID, "unit_words too large");
    if (t->split_prime && (t->split_prime < 128 || t->split_prime > (1u << 16)))
        return fail(CCS_ERR_INVALID, "split_prime must be in [128, 65536]");
    if (t->table_primes && t->table_primes != 7 && t->table_primes != (uint32_t)kNumT)
        return fail(CCS_ERR_INVALID, "table_primes must be 0, 7 or 22");
    const uint32_t split = t->split_prime ? t->split_prime : E->tune.split_prime;
    const uint32_t tabl = t->table_primes ? t->table_primes : E->tune.table_primes;
    if (split != E->tune.split_prime || tabl != E->tune.table_primes) {
        if (E->users) return fail(CCS_ERR_BUSY, "engine tables are in use by a batch or server");
        CU(cudaSetDevice(E->device));
        ccs_status st = build_filters(E, split, tabl);
        if (st != CCS_OK) return st;
    }
    if (t->block_threads) E->tune.block_threads = t->block_threads;
    if (t->unit_words) E->tune.unit_words = t->unit_words;
    if (t->blocks_per_sm) E->tune.blocks_per_sm = t->blocks_per_sm;
    if (t->ext_min_words) E->tune.ext_min_words = t->ext_min_words;
    const uint32_t mx = max_blocks_per_sm(E, E->tune.block_threads);
    if (E->tune.blocks_per_sm > mx) E->tune.blocks_per_sm = mx;
    return CCS_OK;
}

// ---------------------------------------------------------------------------
// plain path
// ---------------------------------------------------------------------------
static ccs_status filter_chunk(ccs_engine* E, unsigned __int128 ts, uint64_t n_tiles, uint32_t bias,
                               ccs_survivor* out, uint64_t cap, cudaStream_t st) {
    RangeDev* hr = (RangeDev*)E->h_stage;
    uint64_t* hpre = (uint64_t*)((char*)E->h_stage + 1024);
    SweepHeader* hh = (SweepHeader*)((char*)E->h_stage + 2048);
    memset(hr, 0, sizeof(RangeDev));
    const FilterSet& f = place_range(E, ts, n_tiles, *hr);
    const HostProfile& hp = f.hp;
    hr->prime_base = 0;
    hr->surv_cap = (uint32_t)std::min<uint64_t>(cap, 0xFFFFFFFFull);
    hr->surv_count = E->d_counters.p;
    hr->surv = (uint32_t*)out;
    hr->range_count = nullptr;
    hr->range_id = 0;
    hr->tile_bias = bias;
    uint64_t units = units_of(f, hr->n_words, hr->unit_words);
    hpre[0] = 0;
    hpre[1] = units;
    hh->n_ranges = 1;
    hh->total_units = units;
    CU(cudaMemcpyAsync(E->d_range.p, hr, sizeof(RangeDev), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(E->d_prefix.p, hpre, 16, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(E->d_hdr.p, hh, sizeof(SweepHeader), cudaMemcpyHostToDevice, st));
    E->launches += 2;
    CU(launch_range_setup(E->d_range.p, E->d_hdr.p, 1, f.range_primes.p,
                          (uint32_t)hp.range_primes.size(), E->d_jmod.p,
                          (uint32_t)hp.range_primes.size(), st));
    uint32_t grid = (uint32_t)E->sms * E->tune.blocks_per_sm;
    const uint32_t wpb = E->tune.block_threads / 32;
    uint64_t need = (units + wpb - 1) / wpb;
    if (need < grid) grid = (uint32_t)std::max<uint64_t>(need, 1);
    const uint32_t bs = b_stride_of((uint32_t)hp.primesB.size());
    const bool mg = use_merged(E, f, bs);
    CU(launch_sweep(E->d_range.p, E->d_prefix.p, E->d_hdr.p, E->d_jmod.p,
                    (uint32_t)hp.range_primes.size(), bs, grid, E->tune.block_threads,
                    sweep_needs_lowreg(bs, E->tune.block_threads, E->tune.blocks_per_sm, mg),
                    mg ? f.slot : -1, st));
    return CCS_OK;
}

ccs_status ccs_filter_range(ccs_engine* E, uint64_t ts_lo, uint64_t ts_hi, uint64_t n_tiles,
                            ccs_survivor* out_dev, uint64_t cap, uint64_t* n_out, void* stream) {
    if (!E || !n_out) return fail(CCS_ERR_INVALID, "null argument");
    if (cap && !out_dev) return fail(CCS_ERR_INVALID, "out_dev is null");
    if (n_tiles >= (1ull << 32)) return fail(CCS_ERR_INVALID, "n_tiles must be < 2^32");
    unsigned __int128 ts = mk128(ts_lo, ts_hi);
    if (ts + n_tiles < ts) return fail(CCS_ERR_INVALID, "tile range wraps 2^128");
    CU(cudaSetDevice(E->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : E->own_stream;
    CU(cudaMemsetAsync(E->d_counters.p, 0, 4, st));
    *n_out = 0;
    if (n_tiles) {
        ccs_status s = filter_chunk(E, ts, n_tiles, 0, out_dev, cap, st);
        if (s != CCS_OK) return s;
    }
    uint32_t cnt = 0;
    CU(cudaMemcpyAsync(E->h_stage, E->d_counters.p, 4, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    cnt = *(uint32_t*)E->h_stage;
    *n_out = cnt;
    if (cnt > cap) return fail(CCS_OVERFLOW, "survivor capacity exceeded");
    return CCS_OK;
}

static ccs_status prove_staged(ccs_engine* E, const ccs_survivor* surv_dev, uint64_t n_surv,
                               const ProveRange* pr_dev, uint32_t bits, const QiterProve* q, ccs_chain* out_dev,
                               uint64_t cap, uint64_t* n_out, uint64_t* primes_out, cudaStream_t st);

ccs_status ccs_prove(ccs_engine* E, const ccs_survivor* surv_dev, uint64_t n_surv, uint64_t ts_lo,
                     uint64_t ts_hi, ccs_chain* out_dev, uint64_t cap, uint64_t* n_out,
                     uint64_t* primes_out, void* stream) {
    if (!E || !n_out) return fail(CCS_ERR_INVALID, "null argument");
    if (n_surv && !surv_dev) return fail(CCS_ERR_INVALID, "surv_dev is null");
    if (cap && !out_dev) return fail(CCS_ERR_INVALID, "out_dev is null");
    if (n_surv >= (1ull << 32)) return fail(CCS_ERR_INVALID, "n_surv must be < 2^32");
    CU(cudaSetDevice(E->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : E->own_stream;
    ProveRange* pr = (ProveRange*)((char*)E->h_stage + 4096);
    memset(pr, 0, sizeof(ProveRange));
    fill_J0(pr->T0, mk128(ts_lo, ts_hi));
    pr->bits = E->hp.bits;
    pr->profile = (uint32_t)E->slot;
    pr->target = E->hp.target;
    pr->chain_count = nullptr;
    pr->prime_count = E->d_counters.p + 3;
    CU(cudaMemcpyAsync(E->d_prange.p, pr, sizeof(ProveRange), cudaMemcpyHostToDevice, st));
    if (n_surv >= kStagedProveMin)
        return prove_staged(E, surv_dev, n_surv, E->d_prange.p, E->hp.bits, nullptr, out_dev, cap, n_out,
                            primes_out, st);
    CU(cudaMemsetAsync(E->d_counters.p + 2, 0, 8, st));
    ProveArgs a;
    a.ranges = E->d_prange.p;
    a.surv = (const uint32_t*)surv_dev;
    a.n_surv_dev = nullptr;
    a.n_surv = (uint32_t)n_surv;
    a.surv_cap = (uint32_t)n_surv;
    a.range_from_pad = 0;
    a.chains = (uint32_t*)out_dev;
    a.chain_count = E->d_counters.p + 2;
    a.chain_cap = (uint32_t)std::min<uint64_t>(cap, 0xFFFFFFFFull);
    uint32_t grid = (uint32_t)std::min<uint64_t>((n_surv + 127) / 128, (uint64_t)E->sms * 16);
    CU(launch_prove(a, grid, st));
    E->launches += 1;
    uint32_t* hc = (uint32_t*)((char*)E->h_stage + 8192);
    CU(cudaMemcpyAsync(hc, E->d_counters.p + 2, 8, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    *n_out = hc[0];
    if (primes_out) *primes_out = hc[1];
    if (hc[0] > cap) return fail(CCS_OVERFLOW, "chain capacity exceeded");
    return CCS_OK;
}

ccs_status ccs_set_bits(ccs_engine* E, uint32_t bits) {
    if (!E) return fail(CCS_ERR_INVALID, "null engine");
    if (bits < 21 || bits > 160) return fail(CCS_ERR_INVALID, "bits out of range [21, 160]");
    E->hp.bits = bits;
    return CCS_OK;
}

ccs_status ccs_search_range_host(ccs_engine* E, uint64_t ts_lo, uint64_t ts_hi, uint64_t n_tiles,
                                 ccs_survivor* surv_host, uint64_t surv_cap, uint64_t* n_surv,
                                 ccs_chain* chains_host, uint64_t chain_cap, uint64_t* n_chains,
                                 uint64_t* primes_out) {
    if (!E || !n_surv || !n_chains) return fail(CCS_ERR_INVALID, "null argument");
    CU(cudaSetDevice(E->device));
    uint64_t scap = std::max<uint64_t>(surv_cap, 1 << 16);
    uint64_t ccap = std::max<uint64_t>(chain_cap, 1 << 16);
    if (E->d_surv_scratch.n < 4 * scap) CU(E->d_surv_scratch.alloc(4 * scap));
    if (E->d_chain_scratch.n < 12 * ccap) CU(E->d_chain_scratch.alloc(12 * ccap));
    ccs_survivor* ds = (ccs_survivor*)E->d_surv_scratch.p;
    ccs_chain* dc = (ccs_chain*)E->d_chain_scratch.p;
    uint64_t ns = 0;
    ccs_status s = ccs_filter_range(E, ts_lo, ts_hi, n_tiles, ds, scap, &ns, nullptr);
    *n_surv = ns;
    if (s != CCS_OK && s != CCS_OVERFLOW) return s;
    uint64_t use = std::min(ns, scap);
    uint64_t nc = 0;
    ccs_status s2 = ccs_prove(E, ds, use, ts_lo, ts_hi, dc, ccap, &nc, primes_out, nullptr);
    *n_chains = nc;
    if (s2 != CCS_OK && s2 != CCS_OVERFLOW) return s2;
    cudaStream_t st = E->own_stream;
    if (surv_host && surv_cap)
        CU(cudaMemcpyAsync(surv_host, ds, sizeof(ccs_survivor) * std::min(use, surv_cap),
                           cudaMemcpyDeviceToHost, st));
    if (chains_host && chain_cap)
        CU(cudaMemcpyAsync(chains_host, dc, sizeof(ccs_chain) * std::min(nc, chain_cap),
                           cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (ns > surv_cap || nc > chain_cap) return fail(CCS_OVERFLOW, "host capacity exceeded");
    return s != CCS_OK ? s : s2;
}

// capacity for n items of per-batch scratch: the next power of two, so that
// batches of slightly varying size do not reallocate
static uint64_t scratch_items(uint64_t n) {
    uint64_t c = 1024;
    while (c < n) c <<= 1;
    return c;
}

// walk scratch for up to n items
static ccs_status walk_reserve(ccs_engine* E, uint64_t n) {
    n = scratch_items(n);
    if (E->w_act.n < n) {
        CU(E->w_act.alloc(n)); CU(E->w_next.alloc(n));
        CU(E->w_sorted.alloc(n)); CU(E->w_lucas.alloc(n));
        CU(E->w_code.alloc(n));
    }
    if (!E->w_state.p) CU(E->w_state.alloc(1));
    return CCS_OK;
}

// Breadth-first walk rounds over the n items already in E->w_act: every walk
// ends at its first composite member or at max_len; lengths[idx] receives
// the count (the items' len included).
// The tests a walk applies: pred to members that start a walk (or are tested
// alone), link_pred to forward links; with screen, links are screened by the
// 132 primes 67..863 and capped at cap bits first.
struct WalkPreds {
    uint32_t pred, link_pred;
    bool screen;
    uint32_t cap;
};

// the profile's tests for stage members (root_role: n itself) and for the
// forward links of a range of bit width `bits`
static WalkPreds walk_preds(const HostProfile& hp, bool root_role, uint32_t bits) {
    WalkPreds w;
    if (hp.primality == CCS_PRIME_V33) {
        const bool wide = bits + hp.target > 127;                 // v33:3095-3101
        w.pred = (root_role && !wide) ? kPredMR235 : kPredBPSW;
        w.link_pred = wide ? kPredBPSW : kPredFermat2;
        w.screen = true;
        w.cap = wide ? bits + 2 * hp.target : 127u;               // v33:1694-1703
    } else {
        w.pred = w.link_pred = hp.primality;
        w.screen = false;
        w.cap = 0;
    }
    return w;
}

// first_len: the chain length the members of round 0 carry (0: walk starts,
// 1: forward links from a root); members of round r carry first_len + r
static ccs_status walk_rounds(ccs_engine* E, uint32_t n, uint32_t* lengths, uint32_t max_len,
                              const WalkPreds& wp, uint32_t first_len, cudaStream_t st) {
    WalkState* hs = (WalkState*)((char*)E->h_stage + 12288);

    WalkItem* act = E->w_act.p;
    WalkItem* nxt = E->w_next.p;
    uint32_t n_act = n;
    for (int round = 0; n_act && round <= kMaxChain; round++) {
        memset(hs, 0, sizeof(WalkState));
        hs->n_act = n_act;
        CU(cudaMemcpyAsync(E->w_state.p, hs, sizeof(WalkState), cudaMemcpyHostToDevice, st));
        WalkArgs a;
        a.max_len = max_len;
        a.pred = wp.pred;
        a.link_pred = wp.link_pred;
        a.screen = wp.screen ? 1u : 0u;
        a.cap_bits = wp.cap;
        a.st = E->w_state.p;
        a.act = act;
        a.sorted = E->w_sorted.p;
        a.lucas = E->w_lucas.p;
        a.next = nxt;
        a.code = E->w_code.p;
        a.lengths = lengths;
        a.profile = E->slot;
        const uint32_t rp = (wp.screen && first_len + round >= 1) ? wp.link_pred : wp.pred;
        const bool second = rp == kPredBPSW || rp == kPredMR235 ||
                            (rp == kPredMR && E->hp.witnesses.size() > 1);
        CU(launch_walk_round(a, n_act, second, rp, st));
        E->launches += 3 + (second ? 10 : 5) + (rp == kPredBPSW ? 5 : 0);
        CU(cudaMemcpyAsync(hs, &E->w_state.p->n_next, 4, cudaMemcpyDeviceToHost, st));
        CU(cudaStreamSynchronize(st));
        n_act = hs->n_act;
        std::swap(act, nxt);
    }
    return CCS_OK;
}

ccs_status ccs_walk_numbers(ccs_engine* E, const uint32_t* numbers_dev, uint64_t n, uint32_t limbs,
                            uint32_t* lengths_dev, void* stream) {
    if (!E) return fail(CCS_ERR_INVALID, "null engine");
    if (limbs < 1 || limbs > (uint32_t)kMaxLimbs) return fail(CCS_ERR_INVALID, "limbs must be 1..6");
    if (n && (!numbers_dev || !lengths_dev)) return fail(CCS_ERR_INVALID, "null buffer");
    CU(cudaSetDevice(E->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : E->own_stream;
    if (!n) return CCS_OK;
    // numbers are walked in chunks of up to 2^24 (32 bytes per item in each
    // of four lists), each in rounds until every walk has ended (at most
    // MAX_CHAIN rounds); the late rounds of a chunk hold few walks and cost
    // about their launches, so fewer, larger chunks pay
    const uint64_t chunk = std::min<uint64_t>(n, 1ull << 24);
    {
        ccs_status s = walk_reserve(E, chunk);
        if (s != CCS_OK) return s;
    }
    for (uint64_t first = 0; first < n; first += chunk) {
        const uint32_t cn = (uint32_t)std::min<uint64_t>(chunk, n - first);
        CU(launch_walk_load(numbers_dev, first, cn, limbs, E->w_act.p, st));
        E->launches += 1;
        // the walk of a given number tests it as a walk start (v33
        // follow_chain_first: is_prime_fast, v33:1535-1540), then its links
        ccs_status s = walk_rounds(E, cn, lengths_dev, kMaxChain, walk_preds(E->hp, false, E->hp.bits), 0, st);
        if (s != CCS_OK) return s;
    }
    CU(cudaStreamSynchronize(st));
    return CCS_OK;
}

// Staged prove of n survivors of one range (the prove_kernel semantics, in
// breadth-first stages; see prove.cu).  pr_dev: the range's ProveRange on
// the device; counters: chains at hc[0], primes at hc[1].
static ccs_status prove_staged(ccs_engine* E, const ccs_survivor* surv_dev, uint64_t n_surv,
                               const ProveRange* pr_dev, uint32_t bits, const QiterProve* q, ccs_chain* out_dev,
                               uint64_t cap, uint64_t* n_out, uint64_t* primes_out, cudaStream_t st) {
    if (n_surv == 0) {
        *n_out = 0;
        if (primes_out) *primes_out = 0;
        return CCS_OK;
    }
    const uint64_t chunk = std::min<uint64_t>(n_surv, 1ull << 22);
    {
        ccs_status s = walk_reserve(E, chunk);
        if (s != CCS_OK) return s;
    }
    const uint64_t cap_items = scratch_items(chunk);
    if (E->p_len.n < cap_items) {
        CU(E->p_nval.alloc(cap_items * kMaxLimbs)); CU(E->p_root.alloc(cap_items * kMaxLimbs));
        CU(E->p_flags.alloc(cap_items)); CU(E->p_len.alloc(cap_items));
        CU(E->p_items0.alloc(cap_items)); CU(E->p_items1.alloc(cap_items)); CU(E->p_fwd.alloc(cap_items));
    }
    if (!E->p_ctr.p) CU(E->p_ctr.alloc(8));
    uint32_t* hc = (uint32_t*)((char*)E->h_stage + 16384);
    uint32_t* ctr = E->p_ctr.p;                   // [0] items [1] roots [2] primes [3] chains
    CU(cudaMemsetAsync(ctr, 0, 32, st));
    StagedProve p;
    p.q = q ? *q : QiterProve{nullptr, nullptr, 0, 0};
    p.range = pr_dev;
    p.surv = (const uint32_t*)surv_dev;
    p.nval = E->p_nval.p;
    p.root = E->p_root.p;
    p.flags = E->p_flags.p;
    p.lengths = E->p_len.p;
    p.count = ctr;
    p.fwd = E->p_fwd.p;
    p.fwd_count = ctr + 1;
    p.primes = ctr + 2;
    p.chains = (uint32_t*)out_dev;
    p.chain_count = ctr + 3;
    p.chain_cap = (uint32_t)std::min<uint64_t>(cap, 0xFFFFFFFFull);
    p.certified = ctr + 4;
    uint64_t pred_tests = 0;
    auto read_ctr = [&](int i) -> uint32_t {
        cudaMemcpyAsync(hc, ctr + i, 4, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        return *hc;
    };
    for (uint64_t first = 0; first < n_surv; first += chunk) {
        p.first = (uint32_t)first;
        p.n_surv = (uint32_t)std::min<uint64_t>(chunk, n_surv - first);
        CU(cudaMemsetAsync(ctr, 0, 8, st));                       // items, roots
        WalkItem* lists[2] = {E->p_items0.p, E->p_items1.p};
        int cur = 0;
        p.out = lists[cur];
        CU(launch_prove_stage(-1, p, nullptr, p.n_surv, st));
        uint32_t n = read_ctr(0);
        // primality stages: the top member (reverse order), n, then predecessors
        int stage = E->hp.reverse_prove ? 0 : 1;
        while (n) {
            CU(cudaMemcpyAsync(E->w_act.p, lists[cur], sizeof(WalkItem) * n, cudaMemcpyDeviceToDevice, st));
            {
                // stage 1 tests n itself (the root test), the others the top
                // member and predecessors
                WalkPreds wp = walk_preds(E->hp, stage == 1, bits);
                wp.screen = false;
                ccs_status s = walk_rounds(E, n, p.lengths, 1, wp, 0, st);
                if (s != CCS_OK) return s;
            }
            CU(cudaMemsetAsync(ctr, 0, 4, st));
            p.out = lists[cur ^ 1];
            CU(launch_prove_stage(stage, p, lists[cur], n, st));
            E->launches += 1;
            n = read_ctr(0);
            if (stage == 1) pred_tests += n;                    // predecessors of the primes n
            cur ^= 1;
            if (stage < 2) stage++;
        }
        // forward walks from the roots, then their records
        const uint32_t nr = read_ctr(1);
        if (nr) {
            CU(cudaMemcpyAsync(E->w_act.p, E->p_fwd.p, sizeof(WalkItem) * nr, cudaMemcpyDeviceToDevice, st));
            ccs_status s = walk_rounds(E, nr, p.lengths, kMaxChain, walk_preds(E->hp, false, bits), 1, st);
            if (s != CCS_OK) return s;
            CU(launch_prove_stage(3, p, E->p_fwd.p, nr, st));
            E->launches += 1;
        }
    }
    CU(cudaMemcpyAsync(hc, ctr + 2, 12, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    *n_out = hc[1];
    if (primes_out) *primes_out = hc[0];
    E->stats[0] += n_surv;
    E->stats[1] += hc[0];
    E->stats[2] += pred_tests;
    E->stats[3] += hc[2];
    if (hc[1] > cap) return fail(CCS_OVERFLOW, "chain capacity exceeded");
    return CCS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// engine services for the q-iteration object
// ---------------------------------------------------------------------------
namespace ccs {

ccs_status set_error(ccs_status st, const char* msg) { return fail(st, msg); }

// An engine with no filter tables: one prove-constant slot (the predicate,
// prove mode and order; no lattice), the walk scratch and the staging.
ccs_status engine_create_prover(int device, uint32_t primality, uint32_t prove_mode, bool reverse,
                                uint32_t target, ccs_engine** out) {
    *out = nullptr;
    if (primality > 1 || prove_mode > 1) return fail(CCS_ERR_INVALID, "bad primality / prove_mode");
    if (reverse && prove_mode != CCS_PROVE_ROOTS)
        return fail(CCS_ERR_INVALID, "reverse prove order is a CCS_PROVE_ROOTS option");
    CU(cudaSetDevice(device));
    ccs_engine* E = new ccs_engine();
    E->device = device;
    HostProfile& hp = E->hp;
    hp.target = target;
    hp.depth = target;
    hp.bits = 0;
    hp.primality = primality;
    hp.prove_mode = prove_mode;
    hp.reverse_prove = reverse ? 1u : 0u;
    hp.kind = 1;
    hp.witnesses.assign(kRefWit, kRefWit + 20);
    E->fs[0].slot = alloc_slot(device);
    if (E->fs[0].slot < 0) { delete E; return fail(CCS_ERR_INVALID, "no free constant-memory slot"); }
    E->slot = E->fs[0].slot;
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    E->sms = prop.multiProcessorCount;
    // proves run beside long filter launches: their blocks go first
    int lo_prio = 0, hi_prio = 0;
    CU(cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio));
    CU(cudaStreamCreateWithPriority(&E->own_stream, cudaStreamNonBlocking, hi_prio));
    ccs_status st = upload_prove(E, E->own_stream);
    if (st != CCS_OK) { ccs_destroy(E); return st; }
    if (E->d_prange.alloc(1) || E->d_counters.alloc(8)) {
        ccs_destroy(E);
        return fail(CCS_ERR_NOMEM, "device allocation failed");
    }
    E->h_stage_bytes = 1 << 16;
    if (cudaMallocHost(&E->h_stage, E->h_stage_bytes) != cudaSuccess) {
        ccs_destroy(E);
        return fail(CCS_ERR_NOMEM, "pinned allocation failed");
    }
    *out = E;
    return CCS_OK;
}

ccs_status engine_prove_staged(ccs_engine* E, const ccs_survivor* surv_dev, uint64_t n_surv,
                               const ProveRange& pr, const QiterProve* q, ccs_chain* out_dev,
                               uint64_t cap, uint64_t* n_out, uint64_t* primes_out, cudaStream_t st) {
    ProveRange* h = (ProveRange*)((char*)E->h_stage + 4096);
    *h = pr;
    h->profile = (uint32_t)E->slot;
    h->chain_count = nullptr;
    h->prime_count = E->d_counters.p + 3;
    CU(cudaMemcpyAsync(E->d_prange.p, h, sizeof(ProveRange), cudaMemcpyHostToDevice, st));
    if (n_surv >= kStagedProveMin)
        return prove_staged(E, surv_dev, n_surv, E->d_prange.p, pr.bits, q, out_dev, cap, n_out, primes_out, st);
    // few survivors: one thread each, one launch
    CU(cudaMemsetAsync(E->d_counters.p + 2, 0, 8, st));
    ProveArgs a;
    a.ranges = E->d_prange.p;
    a.surv = (const uint32_t*)surv_dev;
    a.n_surv_dev = nullptr;
    a.n_surv = (uint32_t)n_surv;
    a.surv_cap = (uint32_t)n_surv;
    a.range_from_pad = 0;
    a.chains = (uint32_t*)out_dev;
    a.chain_count = E->d_counters.p + 2;
    a.chain_cap = (uint32_t)std::min<uint64_t>(cap, 0xFFFFFFFFull);
    if (q) a.q = *q;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, (n_surv + 127) / 128);
    CU(launch_prove(a, grid, st));
    E->launches += 1;
    uint32_t* hc = (uint32_t*)((char*)E->h_stage + 8192);
    CU(cudaMemcpyAsync(hc, E->d_counters.p + 2, 8, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    *n_out = hc[0];
    if (primes_out) *primes_out = hc[1];
    if (hc[0] > cap) return fail(CCS_OVERFLOW, "chain capacity exceeded");
    return CCS_OK;
}

cudaStream_t engine_stream(ccs_engine* E) { return E->own_stream; }
int engine_slot(const ccs_engine* E) { return E->slot; }

}  // namespace ccs

extern "C" {

ccs_status ccs_plan_range(const ccs_engine* E, uint64_t ts_lo, uint64_t ts_hi, uint64_t n_tiles,
                          ccs_range_plan* out) {
    if (!E || !out) return fail(CCS_ERR_INVALID, "null argument");
    if (n_tiles >= (1ull << 32)) return fail(CCS_ERR_INVALID, "n_tiles must be < 2^32");
    memset(out, 0, sizeof(*out));
    RangeDev R;
    memset(&R, 0, sizeof(R));
    const FilterSet& f = place_range(E, mk128(ts_lo, ts_hi), n_tiles, R);
    out->extended = &f == &E->fs[1] ? 1u : 0u;
    out->q0 = f.hp.q0;
    out->n_lines = f.hp.lines.size();
    out->n_words = R.n_words;
    out->unit_words = R.unit_words;
    out->units = n_tiles ? units_of(f, R.n_words, R.unit_words) : 0;
    uint32_t grid = (uint32_t)E->sms * E->tune.blocks_per_sm;
    const uint32_t wpb = E->tune.block_threads / 32;
    const uint64_t need = (out->units + wpb - 1) / wpb;
    if (need < grid) grid = (uint32_t)std::max<uint64_t>(need, 1);
    out->grid = grid;
    out->block_threads = E->tune.block_threads;
    return CCS_OK;
}

ccs_status ccs_prove_stats(ccs_engine* E, uint64_t* out4, int reset) {
    if (!E || !out4) return fail(CCS_ERR_INVALID, "null argument");
    for (int i = 0; i < 4; i++) out4[i] = E->stats[i];
    if (reset) for (int i = 0; i < 4; i++) E->stats[i] = 0;
    return CCS_OK;
}

ccs_status ccs_walk_modmuls(ccs_engine* E, uint64_t* count, int reset) {
    if (!E || !count) return fail(CCS_ERR_INVALID, "null argument");
    CU(cudaSetDevice(E->device));
    CU(modmul_count(count, nullptr, reset != 0));
    return CCS_OK;
}

ccs_status ccs_walk_word_products(ccs_engine* E, uint64_t* modmuls, uint64_t* words, int reset) {
    if (!E || !modmuls || !words) return fail(CCS_ERR_INVALID, "null argument");
    CU(cudaSetDevice(E->device));
    CU(modmul_count(modmuls, words, reset != 0));
    return CCS_OK;
}

// ---------------------------------------------------------------------------
// filter without allocation
//
// For callers that may not allocate device memory once they are running:
// services whose GPU footprint is fixed and accounted for at start-up,
// allocators that refuse to grow after initialisation, and hosts that share
// the device with other tenants under a memory quota.  The engine's tables
// were allocated by ccs_create; this entry point uses only a fixed scratch
// area that lives in the library image itself.  It is synchronous: it waits
// for its stream before returning the survivor count.
// ---------------------------------------------------------------------------

// Scratch layout (bytes):
//   [0, 1024)            range descriptor, unit prefix, sweep header, counters
//   [1024, +64 KiB)      per-range residues J0 mod q (kNoAllocMaxPrimes x u32)
constexpr uint32_t kNoAllocMaxPrimes = 16384;
constexpr size_t kNoAllocJmodOff = 1024;
constexpr size_t kNoAllocBytes = kNoAllocJmodOff + 4ull * kNoAllocMaxPrimes;   // 66,560 B
constexpr int kNoAllocMaxDevices = 64;
static_assert(sizeof(RangeDev) <= 256, "range descriptor must fit its 256-byte scratch slot");
static_assert(sizeof(SweepHeader) <= 256, "sweep header must fit its 256-byte scratch slot");

// One copy per device that loads the library, held until process exit.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on `device` (which must be current).
// Resolved once per device; the host-side name of the array is not a device
// address and is never passed to a kernel.
ccs_status noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(CCS_ERR_INVALID, "bad device ordinal");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return fail(CCS_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_ptr[device] = (unsigned char*)p;
    }
    *out = g_noalloc_ptr[device];
    return CCS_OK;
}
}  // namespace

ccs_status ccs_filter_range_noalloc(ccs_engine* E, uint64_t ts_lo, uint64_t ts_hi, uint64_t n_tiles,
                                    ccs_survivor* out_dev, uint64_t cap, uint64_t* n_out, void* stream) {
    if (!E || !n_out) return fail(CCS_ERR_INVALID, "null argument");
    if (cap && !out_dev) return fail(CCS_ERR_INVALID, "out_dev is null");
    if (n_tiles >= (1ull << 32)) return fail(CCS_ERR_INVALID, "n_tiles must be < 2^32");
    for (int v = 0; v < E->n_fs; v++) {
        const uint32_t np = (uint32_t)E->fs[v].hp.range_primes.size();
        if (np > kNoAllocMaxPrimes)
            return fail(CCS_ERR_INVALID, "ccs_filter_range_noalloc supports at most " +
                                             std::to_string(kNoAllocMaxPrimes - kNumA) +
                                             " filter primes per engine (this engine has " +
                                             std::to_string(np - kNumA) + ")");
    }
    unsigned __int128 ts = mk128(ts_lo, ts_hi);
    if (ts + n_tiles < ts) return fail(CCS_ERR_INVALID, "tile range wraps 2^128");
    CU(cudaSetDevice(E->device));
    unsigned char* base = nullptr;
    {
        ccs_status s = noalloc_scratch(E->device, &base);
        if (s != CCS_OK) return s;
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : E->own_stream;
    RangeDev* d_range = (RangeDev*)(base + 0);
    uint64_t* d_prefix = (uint64_t*)(base + 256);
    SweepHeader* d_hdr = (SweepHeader*)(base + 512);
    uint32_t* d_cnt = (uint32_t*)(base + 768);                 // [0] survivors
    uint32_t* d_jmod = (uint32_t*)(base + kNoAllocJmodOff);
    // the array keeps the previous call's contents: zero the counter
    CU(cudaMemsetAsync(d_cnt, 0, 4, st));
    // descriptors are staged through the engine's pinned buffer (the same
    // slots the plain path uses; the call waits for its copies below)
    RangeDev* hr = (RangeDev*)E->h_stage;
    uint64_t* hpre = (uint64_t*)((char*)E->h_stage + 1024);
    SweepHeader* hh = (SweepHeader*)((char*)E->h_stage + 2048);
    if (n_tiles) {
        memset(hr, 0, sizeof(RangeDev));
        // the same placement as ccs_filter_range (plain or extended lattice)
        const FilterSet& f = place_range(E, ts, n_tiles, *hr);
        const uint32_t np = (uint32_t)f.hp.range_primes.size();
        hr->prime_base = 0;
        hr->surv_cap = (uint32_t)std::min<uint64_t>(cap, 0xFFFFFFFFull);
        hr->surv_count = d_cnt;
        hr->surv = (uint32_t*)out_dev;
        hr->range_count = nullptr;
        hr->range_id = 0;
        hr->tile_bias = 0;
        const uint64_t units = units_of(f, hr->n_words, hr->unit_words);
        hpre[0] = 0;
        hpre[1] = units;
        memset(hh, 0, sizeof(SweepHeader));
        hh->n_ranges = 1;
        hh->total_units = units;
        CU(cudaMemcpyAsync(d_range, hr, sizeof(RangeDev), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(d_prefix, hpre, 16, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(d_hdr, hh, sizeof(SweepHeader), cudaMemcpyHostToDevice, st));
        CU(launch_range_setup(d_range, d_hdr, 1, f.range_primes.p, np, d_jmod, np, st));
        uint32_t grid = (uint32_t)E->sms * E->tune.blocks_per_sm;
        const uint32_t wpb = E->tune.block_threads / 32;
        const uint64_t need = (units + wpb - 1) / wpb;
        if (need < grid) grid = (uint32_t)std::max<uint64_t>(need, 1);
        const uint32_t bs = b_stride_of((uint32_t)f.hp.primesB.size());
        const bool mg = use_merged(E, f, bs);
        CU(launch_sweep(d_range, d_prefix, d_hdr, d_jmod, np, bs, grid, E->tune.block_threads,
                        sweep_needs_lowreg(bs, E->tune.block_threads, E->tune.blocks_per_sm, mg),
                        mg ? f.slot : -1, st));
        E->launches += 2;
    }
    uint32_t* hcnt = (uint32_t*)((char*)E->h_stage + 3072);
    CU(cudaMemcpyAsync(hcnt, d_cnt, 4, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    *n_out = *hcnt;
    if (*hcnt > cap) return fail(CCS_OVERFLOW, "survivor capacity exceeded");
    return CCS_OK;
}

// ---------------------------------------------------------------------------
// autotuner
// ---------------------------------------------------------------------------
namespace {

struct Tuner {
    ccs_engine* E;
    unsigned __int128 ts;
    ccs_tune_point* points;
    uint32_t cap, n = 0;
    DevBuf<uint32_t> out;
    uint64_t out_cap = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;

    // device time of one filter launch over n_tiles tiles (best of two after
    // a warm-up run); -1 on error
    float time(uint64_t n_tiles) {
        cudaStream_t st = E->own_stream;
        float best = -1.0f;
        for (int rep = 0; rep < 3; rep++) {
            if (cudaMemsetAsync(E->d_counters.p, 0, 4, st) != cudaSuccess) return -1.0f;
            if (cudaEventRecord(e0, st) != cudaSuccess) return -1.0f;
            if (filter_chunk(E, ts, n_tiles, 0, (ccs_survivor*)out.p, out_cap, st) != CCS_OK) return -1.0f;
            if (cudaEventRecord(e1, st) != cudaSuccess) return -1.0f;
            if (cudaEventSynchronize(e1) != cudaSuccess) return -1.0f;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0 && (best < 0 || ms < best)) best = ms;
        }
        return best;
    }
    float record(uint64_t n_tiles) {
        const float ms = time(n_tiles);
        if (n < cap && points) {
            points[n].tuning = E->tune;
            points[n].n_tiles = n_tiles;
            points[n].ms = ms;
            points[n]._pad = 0;
        }
        n++;
        return ms;
    }
};

}  // namespace

ccs_status ccs_autotune(ccs_engine* E, uint64_t ts_lo, uint64_t ts_hi, uint64_t n_tiles, uint32_t what,
                        ccs_tune_point* points, uint32_t cap, uint32_t* n_points, ccs_tuning* chosen) {
    if (!E) return fail(CCS_ERR_INVALID, "null engine");
    if (n_tiles == 0 || n_tiles >= (1ull << 32)) return fail(CCS_ERR_INVALID, "n_tiles must be in [1, 2^32)");
    if (cap && !points) return fail(CCS_ERR_INVALID, "points is null");
    if (what == 0) what = CCS_TUNE_ALL;
    if ((what & CCS_TUNE_STAGES) && E->users) return fail(CCS_ERR_BUSY, "engine tables are in use by a batch or server");
    const unsigned __int128 ts = mk128(ts_lo, ts_hi);
    if (ts + n_tiles < ts) return fail(CCS_ERR_INVALID, "tile range wraps 2^128");
    CU(cudaSetDevice(E->device));
    Tuner T;
    T.E = E;
    T.ts = ts;
    T.points = points;
    T.cap = cap;
    {
        // survivor buffer: 4x the expected count, at least 2^16, at most 2^24
        uint64_t cpt = 0;
        for (uint32_t w : E->hp.wheel_total) cpt += w;
        cpt /= 6;
        const double expect = (double)n_tiles * (double)cpt * E->hp.pass_rate;
        T.out_cap = (uint64_t)std::min(std::max(4.0 * expect, 65536.0), 16777216.0);
        CU(T.out.alloc(4 * T.out_cap));
    }
    CU(cudaEventCreate(&T.e0));
    CU(cudaEventCreate(&T.e1));
    ccs_status status = CCS_OK;
    auto finish = [&]() {
        cudaEventDestroy(T.e0);
        cudaEventDestroy(T.e1);
        T.out.free_();
    };
    auto set = [&](const ccs_tuning& t) {
        ccs_status s = ccs_set_tuning(E, &t);
        if (s != CCS_OK) status = s;
        return s == CCS_OK;
    };
    ccs_tuning best = E->tune;
    float best_ms = T.record(n_tiles);
    if (best_ms < 0) { finish(); return fail(CCS_ERR_CUDA, "probe launch failed"); }

    // stage-split thresholds: level-B/C split and table-window count
    if ((what & CCS_TUNE_STAGES) && status == CCS_OK) {
        const uint32_t splits[3] = {512, 1024, 2048};
        const uint32_t tables[2] = {7, (uint32_t)kNumT};
        for (uint32_t sp : splits)
            for (uint32_t tb : tables) {
                ccs_tuning t = best;
                t.split_prime = sp;
                t.table_primes = tb;
                if (!set(t)) { status = CCS_OK; continue; }   // e.g. too many level-B primes
                const float ms = T.record(n_tiles);
                if (ms > 0 && ms < best_ms) { best_ms = ms; best = E->tune; }
            }
        set(best);
    }
    // lattice threshold: the smallest probe prefix (n, n/4, n/16, n/64) on
    // which the extended lattice is faster sets ext_min_words
    if ((what & CCS_TUNE_LATTICE) && E->n_fs > 1 && status == CCS_OK) {
        uint32_t threshold = 0xFFFFFFFFu;
        for (uint64_t len = n_tiles; len >= 64; len /= 4) {
            ccs_tuning t = best;
            t.ext_min_words = 0xFFFFFFFFu;
            set(t);
            const float plain = T.record(len);
            t.ext_min_words = 1;
            set(t);
            const float ext = T.record(len);
            if (ext > 0 && plain > 0 && ext < plain) {
                const uint32_t q0 = E->fs[1].hp.q0;
                const uint64_t span = (len + 5) / 6 + 1;
                threshold = (uint32_t)(((span + q0 - 1) / q0 + 63) / 64);
            } else {
                break;
            }
            if (len / 4 < 64) break;
        }
        best.ext_min_words = threshold;
        set(best);
        best_ms = T.time(n_tiles);
    }
    // positions per thread and work unit
    if ((what & CCS_TUNE_UNITS) && status == CCS_OK) {
        const uint32_t units[6] = {128, 256, 512, 1024, 2048, 4096};
        const ccs_tuning base = best;
        for (uint32_t uw : units) {
            ccs_tuning t = base;
            t.unit_words = uw;
            set(t);
            const float ms = T.record(n_tiles);
            if (ms > 0 && ms < best_ms) { best_ms = ms; best = E->tune; }
        }
        set(best);
    }
    // block shape
    if ((what & CCS_TUNE_SHAPE) && status == CCS_OK) {
        const ccs_tuning base = best;
        for (uint32_t bt : {128u, 256u}) {
            const uint32_t mx = max_blocks_per_sm(E, bt);
            for (uint32_t b = 1; b <= mx; b++) {
                ccs_tuning t = base;
                t.block_threads = bt;
                t.blocks_per_sm = b;
                set(t);
                if (E->tune.block_threads != bt || E->tune.blocks_per_sm != b) continue;
                const float ms = T.record(n_tiles);
                if (ms > 0 && ms < best_ms) { best_ms = ms; best = E->tune; }
            }
        }
        set(best);
    }
    finish();
    if (status != CCS_OK) return status;
    if (n_points) *n_points = T.n;
    if (chosen) *chosen = E->tune;
    return CCS_OK;
}

// ---------------------------------------------------------------------------
// batched executor
// ---------------------------------------------------------------------------
ccs_status ccs_batch_destroy(ccs_batch* b) {
    if (!b) return CCS_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto* E : b->prof) E->users--;
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->d_ranges.free_(); b->d_pranges.free_(); b->d_prefix.free_(); b->d_hdr.free_();
    b->d_jmod.free_(); b->d_primes.free_(); b->d_surv.free_(); b->d_chains.free_();
    b->d_counts.free_();
    if (b->h_ranges) cudaFreeHost(b->h_ranges);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return CCS_OK;
}

static ccs_status batch_capture(ccs_batch* b);

ccs_status ccs_batch_create(ccs_engine* const* profiles, uint32_t n_profiles, uint32_t max_ranges,
                            uint64_t surv_cap, uint64_t chain_cap, ccs_batch** out) {
    if (!out || !profiles || !n_profiles || !max_ranges) return fail(CCS_ERR_INVALID, "bad argument");
    if (surv_cap >= (1ull << 32) || chain_cap >= (1ull << 32)) return fail(CCS_ERR_INVALID, "caps must be < 2^32");
    *out = nullptr;
    ccs_batch* b = new ccs_batch();
    b->device = profiles[0]->device;
    for (uint32_t i = 0; i < n_profiles; i++)
        if (!profiles[i] || profiles[i]->device != b->device) { delete b; return fail(CCS_ERR_INVALID, "profiles must share one device"); }
    for (uint32_t i = 0; i < n_profiles; i++) {
        b->prof.push_back(profiles[i]);
        profiles[i]->users++;
    }
    CU(cudaSetDevice(b->device));
    b->max_ranges = max_ranges;
    b->surv_cap = std::max<uint64_t>(surv_cap, 1);
    b->chain_cap = std::max<uint64_t>(chain_cap, 1);
    std::vector<uint32_t> allp;
    uint32_t maxnb = 0;
    for (auto* E : b->prof) {
        for (int v = 0; v < 2; v++) {
            const HostProfile& hp = E->fs[v < E->n_fs ? v : 0].hp;
            b->prime_base.push_back((uint32_t)allp.size());
            if (v >= E->n_fs) continue;
            allp.insert(allp.end(), hp.range_primes.begin(), hp.range_primes.end());
            b->max_range_primes = std::max<uint32_t>(b->max_range_primes, (uint32_t)hp.range_primes.size());
            maxnb = std::max<uint32_t>(maxnb, (uint32_t)hp.primesB.size());
        }
    }
    b->b_stride = b_stride_of(maxnb);
    b->jstride = b->max_range_primes;
    size_t nc = 4 + 3 * (size_t)max_ranges;
    if (b->d_ranges.alloc(max_ranges) || b->d_pranges.alloc(max_ranges) ||
        b->d_prefix.alloc(max_ranges + 1) || b->d_hdr.alloc(1) ||
        b->d_jmod.alloc((size_t)max_ranges * b->jstride) || b->d_primes.alloc(allp.size()) ||
        b->d_surv.alloc(4 * b->surv_cap) || b->d_chains.alloc(12 * b->chain_cap) ||
        b->d_counts.alloc(nc)) {
        ccs_batch_destroy(b);
        return fail(CCS_ERR_NOMEM, "batch device allocation failed");
    }
    CU(cudaMemcpy(b->d_primes.p, allp.data(), 4 * allp.size(), cudaMemcpyHostToDevice));
    size_t hb = sizeof(RangeDev) * max_ranges + sizeof(ProveRange) * max_ranges +
                8 * (max_ranges + 1) + sizeof(SweepHeader) + 4 * nc + 256;
    void* h = nullptr;
    if (cudaMallocHost(&h, hb) != cudaSuccess) { ccs_batch_destroy(b); return fail(CCS_ERR_NOMEM, "pinned alloc failed"); }
    char* c = (char*)h;
    b->h_ranges = (RangeDev*)c; c += sizeof(RangeDev) * max_ranges;
    b->h_pranges = (ProveRange*)c; c += sizeof(ProveRange) * max_ranges;
    b->h_prefix = (uint64_t*)c; c += 8 * (max_ranges + 1);
    b->h_hdr = (SweepHeader*)c; c += sizeof(SweepHeader);
    c = (char*)(((uintptr_t)c + 15) & ~(uintptr_t)15);
    b->h_counts = (uint32_t*)c;
    CU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CU(cudaEventCreate(&b->ev0));
    CU(cudaEventCreate(&b->ev1));
    b->nc = (uint32_t)nc;
    b->block_threads = kSweepThreads;
    {
        ccs_status s = batch_capture(b);
        if (s != CCS_OK) { ccs_batch_destroy(b); return s; }
    }
    *out = b;
    return CCS_OK;
}

// Records the whole batch once: H2D descriptors, setup, sweep (with the
// batch's block shape), prove, D2H counters.  Replays read the
// per-submission header on the device.
static ccs_status batch_capture(ccs_batch* b) {
    if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    const uint32_t bt = b->block_threads;
    const int mx = sweep_blocks_per_sm(b->b_stride, bt);
    if (mx <= 0) return fail(CCS_ERR_INVALID, "sweep does not fit the SM at this block size");
    b->blocks_per_sm = (b->req_blocks_per_sm == 0 || b->req_blocks_per_sm > (uint32_t)mx)
                           ? (uint32_t)mx : b->req_blocks_per_sm;
    b->grid = (uint32_t)b->prof[0]->sms * b->blocks_per_sm;
    const bool lowreg = sweep_needs_lowreg(b->b_stride, bt, b->blocks_per_sm, false);
    const uint32_t max_ranges = b->max_ranges;
    const size_t nc = b->nc;
    cudaStream_t st = b->stream;
    CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(b->d_ranges.p, b->h_ranges, sizeof(RangeDev) * max_ranges, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->d_pranges.p, b->h_pranges, sizeof(ProveRange) * max_ranges, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->d_prefix.p, b->h_prefix, 8 * (max_ranges + 1), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->d_hdr.p, b->h_hdr, sizeof(SweepHeader), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(b->d_counts.p, 0, 4 * nc, st);
    launch_range_setup(b->d_ranges.p, b->d_hdr.p, max_ranges, b->d_primes.p, b->max_range_primes,
                       b->d_jmod.p, b->jstride, st);
    launch_sweep(b->d_ranges.p, b->d_prefix.p, b->d_hdr.p, b->d_jmod.p, b->jstride, b->b_stride,
                 b->grid, bt, lowreg, -1, st);
    ProveArgs pa;
    pa.ranges = b->d_pranges.p;
    pa.surv = b->d_surv.p;
    pa.n_surv_dev = b->d_counts.p;
    pa.n_surv = 0;
    pa.surv_cap = (uint32_t)b->surv_cap;
    pa.range_from_pad = 1;
    pa.chains = b->d_chains.p;
    pa.chain_count = b->d_counts.p + 2;
    pa.chain_cap = (uint32_t)b->chain_cap;
    launch_prove(pa, (uint32_t)b->prof[0]->sms * 16, st);
    cudaMemcpyAsync(b->h_counts, b->d_counts.p, 4 * nc, cudaMemcpyDeviceToHost, st);
    cudaError_t ce = cudaStreamEndCapture(st, &b->graph);
    if (ce != cudaSuccess) return fail(CCS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&b->gexec, b->graph, 0);
    if (ce != cudaSuccess) return fail(CCS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    return CCS_OK;
}

ccs_status ccs_batch_get_tuning(const ccs_batch* b, ccs_batch_tuning* t) {
    if (!b || !t) return fail(CCS_ERR_INVALID, "null argument");
    t->block_threads = b->block_threads;
    t->blocks_per_sm = b->blocks_per_sm;
    t->unit_words = b->unit_words;
    t->_pad = 0;
    return CCS_OK;
}

ccs_status ccs_batch_set_tuning(ccs_batch* b, const ccs_batch_tuning* t) {
    if (!b || !t) return fail(CCS_ERR_INVALID, "null argument");
    if (t->block_threads && t->block_threads != 128 && t->block_threads != 256)
        return fail(CCS_ERR_INVALID, "block_threads must be 128 or 256");
    if (t->unit_words > (1u << 20)) return fail(CCS_ERR_INVALID, "unit_words too large");
    if (b->in_flight) return fail(CCS_ERR_BUSY, "the batch's previous launch has not been waited for");
    CU(cudaSetDevice(b->device));
    b->unit_words = t->unit_words;
    const uint32_t bt = t->block_threads ? t->block_threads : b->block_threads;
    if (bt != b->block_threads || t->blocks_per_sm != b->req_blocks_per_sm) {
        CU(cudaStreamSynchronize(b->stream));
        b->block_threads = bt;
        b->req_blocks_per_sm = t->blocks_per_sm;
        return batch_capture(b);
    }
    return CCS_OK;
}

ccs_status ccs_batch_launch(ccs_batch* b, const ccs_range* ranges, uint32_t n_ranges) {
    if (!b || (n_ranges && !ranges)) return fail(CCS_ERR_INVALID, "null argument");
    if (n_ranges > b->max_ranges) return fail(CCS_ERR_INVALID, "too many ranges for this batch");
    if (b->in_flight) return fail(CCS_ERR_BUSY, "the batch's previous launch has not been waited for");
    CU(cudaSetDevice(b->device));
    uint64_t total = 0;
    uint32_t* cnt = b->d_counts.p;
    for (uint32_t i = 0; i < n_ranges; i++) {
        if (ranges[i].profile >= b->prof.size()) return fail(CCS_ERR_INVALID, "bad profile index");
        if (ranges[i].n_tiles >= (1ull << 32)) return fail(CCS_ERR_INVALID, "n_tiles must be < 2^32");
    }
    // work units are laid out profile by profile, longest range first, so the
    // persistent sweep works through one profile's tables at a time and ends
    // on short units; records still carry the caller's range index
    std::vector<uint32_t> order(n_ranges);
    for (uint32_t i = 0; i < n_ranges; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        if (ranges[x].profile != ranges[y].profile) return ranges[x].profile < ranges[y].profile;
        return ranges[x].n_tiles > ranges[y].n_tiles;
    });
    b->cur_ranges.assign(ranges, ranges + n_ranges);
    for (uint32_t k = 0; k < n_ranges; k++) {
        const uint32_t i = order[k];
        const ccs_range& rg = ranges[i];
        ccs_engine* E = b->prof[rg.profile];
        unsigned __int128 ts = mk128(rg.tile_start_lo, rg.tile_start_hi);
        RangeDev& R = b->h_ranges[k];
        memset(&R, 0, sizeof(R));
        const FilterSet& f = place_range(E, ts, rg.n_tiles, R, false);   // ranges share the GPU
        if (b->unit_words) R.unit_words = std::max<uint32_t>(1, std::min(b->unit_words, R.n_words));
        R.prime_base = b->prime_base[2 * rg.profile + (&f == &E->fs[1] ? 1 : 0)];
        R.surv_cap = (uint32_t)b->surv_cap;
        R.surv_count = cnt;
        R.surv = b->d_surv.p;
        R.range_count = cnt + 4 + 3 * i;
        R.range_id = i;
        R.tile_bias = 0;
        ProveRange& P = b->h_pranges[i];
        memset(&P, 0, sizeof(P));
        fill_J0(P.T0, ts);
        P.bits = rg.bits ? rg.bits : E->hp.bits;
        P.profile = (uint32_t)E->slot;
        P.target = E->hp.target;
        P.chain_count = cnt + 4 + 3 * i + 1;
        P.prime_count = cnt + 4 + 3 * i + 2;
        b->h_prefix[k] = total;
        total += R.n_words ? units_of(f, R.n_words, R.unit_words) : 0;
    }
    b->h_prefix[n_ranges] = total;
    for (uint32_t i = n_ranges + 1; i <= b->max_ranges; i++) b->h_prefix[i] = total;
    b->h_hdr->n_ranges = n_ranges;
    b->h_hdr->total_units = total;
    CU(cudaEventRecord(b->ev0, b->stream));
    CU(cudaGraphLaunch(b->gexec, b->stream));
    CU(cudaEventRecord(b->ev1, b->stream));
    b->in_flight = true;
    return CCS_OK;
}

ccs_status ccs_batch_wait(ccs_batch* b, ccs_range_result* results, ccs_survivor* surv_host,
                          ccs_chain* chains_host) {
    if (!b) return fail(CCS_ERR_INVALID, "null argument");
    if (!b->in_flight) return fail(CCS_ERR_INVALID, "no batch launch to wait for");
    const uint32_t n_ranges = (uint32_t)b->cur_ranges.size();
    if (n_ranges && !results) return fail(CCS_ERR_INVALID, "results is null");
    CU(cudaSetDevice(b->device));
    b->in_flight = false;
    CU(cudaEventSynchronize(b->ev1));
    CU(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
    const uint32_t* hc = b->h_counts;
    ccs_status st = CCS_OK;
    uint64_t ns = hc[0], nch = hc[2];
    for (uint32_t i = 0; i < n_ranges; i++) {
        const ccs_range& rg = b->cur_ranges[i];
        ccs_range_result& r = results[i];
        memset(&r, 0, sizeof(r));
        r.n_survivors = hc[4 + 3 * i];
        r.n_chains = hc[4 + 3 * i + 1];
        r.n_primes = hc[4 + 3 * i + 2];
        ccs_engine* E = b->prof[rg.profile];
        // exact candidate count: lines of each tile class times their blocks
        uint32_t e0 = (uint32_t)(mk128(rg.tile_start_lo, rg.tile_start_hi) % 6);
        uint64_t cand = 0;
        for (uint32_t c6 = 0; c6 < 6; c6++) {
            uint64_t endc = (uint64_t)e0 + rg.n_tiles;
            uint64_t jhi = endc > c6 ? (endc - c6 + 5) / 6 : 0;
            uint64_t jlo = c6 < e0 ? 1 : 0;
            if (jhi > jlo) cand += (jhi - jlo) * E->hp.lines_per_class[c6];
        }
        r.candidates = cand;
        r.status = (ns > b->surv_cap || nch > b->chain_cap) ? CCS_OVERFLOW : CCS_OK;
    }
    // records are copied on the batch stream: a launch of another batch may
    // already be running on the GPU
    uint64_t ncopy = std::min<uint64_t>(ns, b->surv_cap);
    uint64_t ccopy = std::min<uint64_t>(nch, b->chain_cap);
    if (surv_host && ncopy)
        CU(cudaMemcpyAsync(surv_host, b->d_surv.p, 16 * ncopy, cudaMemcpyDeviceToHost, b->stream));
    if (chains_host && ccopy)
        CU(cudaMemcpyAsync(chains_host, b->d_chains.p, 48 * ccopy, cudaMemcpyDeviceToHost, b->stream));
    if ((surv_host && ncopy) || (chains_host && ccopy)) CU(cudaStreamSynchronize(b->stream));
    if (ns > b->surv_cap || nch > b->chain_cap) st = fail(CCS_OVERFLOW, "batch capacity exceeded");
    return st;
}

ccs_status ccs_batch_run(ccs_batch* b, const ccs_range* ranges, uint32_t n_ranges,
                         ccs_range_result* results, ccs_survivor* surv_host, ccs_chain* chains_host,
                         void* stream) {
    (void)stream;
    ccs_status st = ccs_batch_launch(b, ranges, n_ranges);
    if (st != CCS_OK) return st;
    return ccs_batch_wait(b, results, surv_host, chains_host);
}

ccs_status ccs_batch_autotune(ccs_batch* b, const ccs_range* ranges, uint32_t n_ranges,
                              ccs_tune_point* points, uint32_t cap, uint32_t* n_points,
                              ccs_batch_tuning* chosen) {
    if (!b || !ranges || !n_ranges) return fail(CCS_ERR_INVALID, "bad argument");
    if (n_ranges > b->max_ranges) return fail(CCS_ERR_INVALID, "too many ranges for this batch");
    if (cap && !points) return fail(CCS_ERR_INVALID, "points is null");
    std::vector<ccs_range_result> res(n_ranges);
    uint32_t n = 0;
    float best_ms = -1.0f;
    ccs_batch_tuning best{};
    ccs_batch_get_tuning(b, &best);
    auto measure = [&](const ccs_batch_tuning& t) -> ccs_status {
        ccs_status s = ccs_batch_set_tuning(b, &t);
        if (s != CCS_OK) return s;
        float ms = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
            s = ccs_batch_run(b, ranges, n_ranges, res.data(), nullptr, nullptr, nullptr);
            if (s != CCS_OK && s != CCS_OVERFLOW) return s;
            ms = std::min(ms, b->last_ms);
        }
        if (n < cap) {
            memset(&points[n], 0, sizeof(points[n]));
            points[n].tuning.block_threads = b->block_threads;
            points[n].tuning.blocks_per_sm = b->blocks_per_sm;
            points[n].tuning.unit_words = b->unit_words;
            points[n].ms = ms;
        }
        n++;
        if (best_ms < 0 || ms < best_ms) {
            best_ms = ms;
            best = t;
            best.block_threads = b->block_threads;
        }
        return CCS_OK;
    };
    // unit length at the default shape, then block shapes at that length
    const uint32_t units[5] = {0, 1024, 2048, 4096, 8192};
    for (uint32_t uw : units) {
        ccs_status s = measure(ccs_batch_tuning{256u, 0u, uw, 0u});
        if (s != CCS_OK) return s;
    }
    const uint32_t uw_best = best.unit_words;
    // 3 x 256 and 5-6 x 128 run the register-capped sweep variant
    const uint32_t shapes[8][2] = {{256, 1}, {256, 2}, {256, 3}, {128, 2}, {128, 3}, {128, 4}, {128, 5}, {128, 6}};
    for (const auto& sh : shapes) {
        if (sh[1] > (uint32_t)sweep_blocks_per_sm(b->b_stride, sh[0])) continue;
        ccs_status s = measure(ccs_batch_tuning{sh[0], sh[1], uw_best, 0u});
        if (s != CCS_OK) return s;
    }
    ccs_status s = ccs_batch_set_tuning(b, &best);
    if (s != CCS_OK) return s;
    if (n_points) *n_points = n;
    if (chosen) ccs_batch_get_tuning(b, chosen);
    return CCS_OK;
}

ccs_status ccs_batch_last_ms(const ccs_batch* b, float* ms) {
    if (!b || !ms) return fail(CCS_ERR_INVALID, "null argument");
    *ms = b->last_ms;
    return CCS_OK;
}

}  // extern "C"
