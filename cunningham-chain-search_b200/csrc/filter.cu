// Depth-filter kernels for sm_100a.
//
// Reference behaviour replaced: cc18_filter_kernel (v13:1551-1714, v15:1753-1929)
// and the host residue preparation prepare_batch (v13:1232-1259).
//
// Design (see ccs_internal.h for the line / phase model):
//   * one warp owns 32 lines (residues r mod W) and sweeps them along the
//     block index J, 64 blocks ("a word") per step;
//   * level A: every filter prime q < 128 is bit-sliced.  Its 64-position kill
//     word is a window of the q-periodic phase pattern, held in 2-4 registers
//     and advanced by two shifts and an OR per word -- no table lookups, no
//     per-candidate arithmetic;
//   * level B: surviving positions are tested one by one against the primes in
//     [128, split) using per-lane phases cached in shared memory and the G_q
//     bitmaps (early exit, ascending q);
//   * level C: the rare level-B survivors collect in a per-warp list and the
//     whole warp tests them against all primes >= split (32 primes per
//     round, ballot early exit) inside the same kernel;
//   * survivors are written as the reference's 16-byte Survivor records.
#include "ccs_kernels.cuh"

namespace ccs {

__constant__ ProfileConst c_prof[kMaxProfiles];

// x mod q for x < 2^32 with magic = floor(2^32 / q)
__device__ __forceinline__ uint32_t mod_magic(uint32_t x, uint32_t q, uint32_t magic) {
    uint32_t t = x - __umulhi(x, magic) * q;
    return t >= q ? t - q : t;
}

// x mod q for x < 2^64 with magic64 = floor(2^64 / q)
__device__ __forceinline__ uint32_t mod_magic64(uint64_t x, uint32_t q, uint64_t magic64) {
    uint64_t t = x - __umul64hi(x, magic64) * (uint64_t)q;
    while (t >= q) t -= q;
    return (uint32_t)t;
}

// ---------------------------------------------------------------------------
// per-range J0 mod q tables (replaces the host u128 prepare_batch)
// ---------------------------------------------------------------------------
__global__ void range_setup_kernel(const RangeDev* __restrict__ ranges,
                                   const SweepHeader* __restrict__ hdr,
                                   const uint32_t* __restrict__ primes, uint32_t n_primes,
                                   uint32_t* __restrict__ jmod, uint32_t jmod_stride) {
    const uint32_t n_ranges = hdr->n_ranges;
    for (uint32_t r = blockIdx.y; r < n_ranges; r += gridDim.y) {
    const RangeDev& R = ranges[r];
    const uint32_t* pr = primes + R.prime_base;
    uint32_t np = R.n_range_primes;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        uint32_t q = pr[i];
        uint64_t acc = 0;
#pragma unroll
        for (int w = 3; w >= 0; w--) acc = ((acc << 32) | R.J0[w]) % q;
        jmod[(uint64_t)r * jmod_stride + i] = (uint32_t)acc;
    }
    }
    (void)n_primes;
}

// line phases r W^-1 mod q for every (line, slot) of a profile, row per line
__global__ void phase_table_kernel(const Line* __restrict__ lines, uint32_t n_lines,
                                   const SlotConst* __restrict__ pq, uint32_t n_slots,
                                   uint16_t* __restrict__ tab) {
    const uint64_t total = (uint64_t)n_lines * n_slots;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t l = (uint32_t)(x / n_slots), s = (uint32_t)(x % n_slots);
        const SlotConst c = pq[s];
        const Line ln = lines[l];
        uint32_t a = mod_magic(ln.r_hi, c.q, c.magic) * c.c32 + mod_magic(ln.r_lo, c.q, c.magic);
        a = mod_magic(a, c.q, c.magic);
        tab[x] = (uint16_t)mod_magic(a * c.winv, c.q, c.magic);
    }
}

cudaError_t launch_phase_table(const Line* lines, uint32_t n_lines, const SlotConst* pq, uint32_t n_slots,
                               uint16_t* tab, cudaStream_t st) {
    phase_table_kernel<<<148 * 8, 256, 0, st>>>(lines, n_lines, pq, n_slots, tab);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// survivor emission
// ---------------------------------------------------------------------------
// p is the line's position (block index j on a plain profile; on an extended
// profile j = q0 p + d - e1)
__device__ __forceinline__ void emit_survivor(const RangeDev& R, const Line& ln, uint32_t p, uint32_t q0) {
    const uint32_t c = (ln.bc >> 16) & 7u;
    const uint32_t d = ln.bc >> 19;
    const uint32_t j = q0 * p + d - R.e1;
    uint32_t slot = atomicAdd(R.surv_count, 1u);
    if (R.range_count) atomicAdd(R.range_count, 1u);
    if (slot < R.surv_cap) {
        uint4 rec;
        rec.x = ln.bc & 0xFFFFu;
        rec.y = ln.k;
        rec.z = 6u * j + c - R.e0 + R.tile_bias;
        rec.w = R.range_id;
        reinterpret_cast<uint4*>(R.surv)[slot] = rec;
    }
}

// ---------------------------------------------------------------------------
// sweep kernel (levels A and B)
// ---------------------------------------------------------------------------
struct SweepArgs {
    const RangeDev* ranges;
    const uint64_t* unit_prefix;   // [n_ranges + 1] exclusive prefix of units
    const SweepHeader* hdr;
    const uint32_t* jmod;          // [n_ranges][jmod_stride]
    uint32_t jmod_stride;
    uint32_t b_stride;             // level-B primes per lane column in shared memory
    uint32_t merge_slot;           // profile whose merged table windows are staged per
                                   // block (every range of the launch has it), or kNone
};

// standard level-A sets, with compile-time primes: STD = 1, 2: primes
// 37..127 / 41..127 (37 absorbed into an extended lattice); STD = 3, 4: the
// same with table windows up to 199
#define CCS_STD_T7 97, 101, 103, 107, 109, 113, 127
#define CCS_STD_T22 CCS_STD_T7, 131, 137, 139, 149, 151, 157, 163, 167, 173, 179, 181, 191, 193, 197, 199
#define CCS_NO_T15 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1
__device__ constexpr uint32_t kStdQ[5][kNumA] = {
    {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
     1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    {37, 41, 43, 47, 53, 59, 61, 1, 1, 67, 71, 73, 79, 83, 89, CCS_STD_T7, CCS_NO_T15},
    {41, 43, 47, 53, 59, 61, 1, 1, 1, 67, 71, 73, 79, 83, 89, CCS_STD_T7, CCS_NO_T15},
    {37, 41, 43, 47, 53, 59, 61, 1, 1, 67, 71, 73, 79, 83, 89, CCS_STD_T22},
    {41, 43, 47, 53, 59, 61, 1, 1, 1, 67, 71, 73, 79, 83, 89, CCS_STD_T22}};
#undef CCS_STD_T7
#undef CCS_STD_T22
#undef CCS_NO_T15
__device__ constexpr int kStdA1[5] = {kNumA1, 7, 6, 7, 6};
__device__ constexpr MgTable kMg = make_mg_table();   // merged table windows
__device__ constexpr int kStdNT[5] = {kNumT, 7, 7, 22, 22};
// pattern-table offset of table-window slot i in a standard set (t_words(q)
// words per prime, in slot order)
__device__ constexpr uint32_t std_toff(int i) {
    uint32_t o = 0;
    for (int k = 0; k < i; k++) o += t_words(kStdQ[3][kNumAR + k]);
    return o;
}

constexpr int kQCap = 256;               // per-warp level-B queue (entries, power of two)
constexpr uint32_t kQLow = 64;           // level-B rounds run until at most this many are queued
constexpr int kCCap = 64;                // per-warp level-C list (entries)
constexpr int kBK = kLevelBRound;        // level-B primes tested per lane per round
constexpr int kPAWords = kNumAR * 8 + kPatTMax;   // per-warp copy of the level-A patterns (u32)
constexpr int kSAWords = kNumA * 8;      // per-warp level-A phases, [kNumA][32] u8
constexpr uint32_t kNone = 0xFFFFFFFFu;  // empty lane slot
constexpr uint32_t kFull = 0xFFFFFFFFu;

// x mod q for x < 2^32 via the profile's magic (fast init-time reductions)
__device__ __forceinline__ uint32_t phase_fast(uint32_t rl, uint32_t rh, uint32_t q, uint32_t magic,
                                               uint32_t c32, uint32_t winv, uint32_t j0q,
                                               uint32_t jb) {
    uint32_t a = mod_magic(rh, q, magic) * c32 + mod_magic(rl, q, magic);   // < q^2 + q
    a = mod_magic(a, q, magic);
    a = mod_magic(a * winv, q, magic);                                     // r * W^-1 mod q
    uint32_t v = a + j0q + mod_magic(jb, q, magic);                        // < 3q
    v = v >= q ? v - q : v;
    return v >= q ? v - q : v;
}

// Per-warp level-B machinery: a queue of (block offset, line lane) entries in
// shared memory and one candidate per lane, refilled whenever a lane's
// candidate is decided, so lanes stay busy whichever line produced the work.
struct LevelB {
    uint32_t* Q;                   // kQCap entries: (jrel << 5) | line lane
    uint32_t* Cl;                  // kCCap level-B survivors waiting for level C
    uint32_t cnum;                 // entries in Cl (warp-uniform)
    const uint16_t* S;             // [nB][32] phases of the unit's 32 lines at jbase
    const PrimeB* pb;
    const uint32_t* bm;
    uint32_t nB;                   // level-B primes, padded to a multiple of kBK
    uint32_t head, tail;           // warp-uniform
    uint32_t cur, pi;              // this lane's candidate and next prime index
};

// Level C, warp-cooperative: every lane takes 32 primes >= split per round
// for each listed candidate (phase from scratch, binary search in the sorted
// G_q list), ballot early exit; survivors are written by lane 0.
__device__ __forceinline__ void c_process(LevelB& B, const SweepArgs& a, const RangeDev& R,
                                       const ProfileConst& P, uint32_t cur_range, uint32_t g,
                                       uint32_t jbase, uint32_t lane) {
    __syncwarp();
    const uint32_t* jm = a.jmod + (uint64_t)cur_range * a.jmod_stride + kNumA + P.nB;
    for (uint32_t e = 0; e < B.cnum; e++) {
        const uint32_t ent = B.Cl[e];
        const uint32_t j = jbase + (ent >> 5);
        const Line ln = P.lines[g * 32 + (ent & 31u)];
        const uint64_t r = ((uint64_t)ln.r_hi << 32) | ln.r_lo;
        bool killed = false;
        for (uint32_t base = 0; base < P.nC && !killed; base += 32) {
            const uint32_t p = base + lane;
            bool kill = false;
            if (p < P.nCb) {
                // q < 2^13: the phase in 32-bit arithmetic, one bitmap word
                const PrimeC pc = P.primesC[p];
                const uint32_t q = pc.q;
                uint32_t rm = mod_magic(ln.r_hi, q, pc.magic) * pc.c32 + mod_magic(ln.r_lo, q, pc.magic);
                rm = mod_magic(rm, q, pc.magic);                          // r mod q
                const uint32_t rw = mod_magic(rm * pc.winv, q, pc.magic);
                uint32_t uph = rw + jm[p] + mod_magic(j, q, pc.magic);    // < 3q
                uph = uph >= q ? uph - q : uph;
                uph = uph >= q ? uph - q : uph;
                kill = (__ldg(P.bitmapC + pc.off + (uph >> 5)) >> (uph & 31)) & 1u;
            } else if (p < P.nC) {
                const PrimeC pc = P.primesC[p];
                const uint32_t rm = mod_magic64(r, pc.q, pc.magic64);
                const uint32_t rw = mod_magic64((uint64_t)rm * pc.winv, pc.q, pc.magic64);
                const uint32_t jq = mod_magic64(j, pc.q, pc.magic64);
                const uint32_t uph = mod_magic64((uint64_t)rw + jm[p] + jq, pc.q, pc.magic64);
                // the padded list, four entries per load, all loads independent
                const uint4* lst = reinterpret_cast<const uint4*>(P.listC + pc.off);
                const uint32_t n4 = (pc.cnt + 3) >> 2;
                for (uint32_t k = 0; k < n4; k++) {
                    const uint4 v = __ldg(lst + k);
                    kill |= (v.x == uph) | (v.y == uph) | (v.z == uph) | (v.w == uph);
                }
            }
            killed = __any_sync(kFull, kill);
        }
        if (!killed && lane == 0) emit_survivor(R, ln, j, P.q0);
    }
    B.cnum = 0;
    __syncwarp();
}

// One round: refill empty lanes from the queue, then test kBK primes of each
// lane's candidate.  The kBK tests are independent (their loads and
// reductions overlap); a candidate killed by any of them is dropped, so the
// outcome equals the one-prime-at-a-time test.
__device__ __forceinline__ void b_round(LevelB& B, const SweepArgs& a, const RangeDev& R,
                                        const ProfileConst& P, uint32_t cur_range, uint32_t g,
                                        uint32_t jbase, uint32_t lane_lt) {
    const bool needy = B.cur == kNone;
    const uint32_t nm = __ballot_sync(kFull, needy);
    const uint32_t avail = B.tail - B.head;
    if (needy) {
        const uint32_t rk = __popc(nm & lane_lt);
        if (rk < avail) { B.cur = B.Q[(B.head + rk) & (kQCap - 1)]; B.pi = 0; }
    }
    B.head += min((uint32_t)__popc(nm), avail);
    if (B.cur != kNone && B.pi < B.nB) {
        const uint32_t L = B.cur & 31u, jrel = B.cur >> 5;
        uint32_t hit = 0;
#pragma unroll
        for (int t = 0; t < kBK; t++) {
            const uint32_t idx = B.pi + t;
            const uint2 pr = __ldg(reinterpret_cast<const uint2*>(B.pb) + idx);
            const uint32_t q = pr.y & 0xFFFFu;
            const uint32_t u = mod_magic((uint32_t)B.S[idx * 32 + L] + jrel, q, pr.x);
            const uint32_t wv = __ldg(B.bm + (pr.y >> 16) + (u >> 5));
            hit |= wv >> (u & 31);
        }
        if (hit & 1u) B.cur = kNone; else B.pi += kBK;
    }
    // candidates that passed every level-B prime
    const bool pass = B.cur != kNone && B.pi >= B.nB;
    if (P.nC == 0) {
        if (pass) {
            emit_survivor(R, P.lines[g * 32 + (B.cur & 31u)], jbase + (B.cur >> 5), P.q0);
            B.cur = kNone;
        }
    } else {
        const uint32_t pm = __ballot_sync(kFull, pass);
        if (pass) {
            B.Cl[B.cnum + __popc(pm & lane_lt)] = B.cur;
            B.cur = kNone;
        }
        B.cnum += __popc(pm);
        if (B.cnum > (uint32_t)(kCCap - 32)) c_process(B, a, R, P, cur_range, g, jbase, threadIdx.x & 31);
    }
}

// One work unit: 32 lines of range cur_range, words [w0, w1).  STD selects
// the level-A variant: 1 = primes 37..127, 2 = 41..127 (37 absorbed), 0 =
// whatever the profile lists (shift amounts read from constant memory).
//
// The unit alternates two phases.  Level A sweeps words with the kill
// windows in registers and queues the surviving positions until the queue is
// full; level B then runs rounds until the queue is nearly empty.  The
// windows are rebuilt from the per-lane phases at the start of every level-A
// phase, so they are dead while level B runs and its independent tests have
// the registers.
//
// MG (standard 22-prime sets only): the table windows are the merged ones
// (kMgWin patterns of period q1 q2, staged per block at PM) instead of the 22
// per-prime patterns of the per-warp copy.
template <int STD, bool MG>
__device__ __forceinline__ void sweep_unit(const SweepArgs& a, const RangeDev& R, const ProfileConst& P,
                                           uint32_t cur_range, uint32_t g, uint32_t w0, uint32_t w1,
                                           uint32_t* Qw, uint32_t* Cw, uint32_t* PA, uint8_t* SA,
                                           uint16_t* S, const uint32_t* PM, uint32_t lane,
                                           uint32_t lane_lt) {
        static_assert(!MG || STD == 3 || STD == 4, "merged windows need the 22-prime standard set");
        const uint32_t* jm = a.jmod + (uint64_t)cur_range * a.jmod_stride;
        const uint32_t li = g * 32 + lane;
        const bool has_line = li < P.n_lines;
        if (P.ptab && has_line) {
            // start pulling this line's phase-table row toward L2 now; it is
            // read after the pattern copies and range offsets below
            const char* rp = reinterpret_cast<const char*>(P.ptab + (size_t)li * P.ptab_stride);
            const uint32_t bytes = P.ptab_stride * 2u;
            for (uint32_t off = 0; off < bytes; off += 128)
                asm volatile("prefetch.global.L2 [%0];" :: "l"(rp + off));
            asm volatile("prefetch.global.L2 [%0];" :: "l"(rp + bytes - 1));
        }
        const Line ln = has_line ? P.lines[li] : Line{0, 0, 0, 0};
        const uint32_t c = (ln.bc >> 16) & 7u;
        const uint32_t d = ln.bc >> 19;
        const uint32_t q0 = P.q0;
        // block range [jlo0, jhi0) of this line relative to floor(tile_start / 6)
        const uint32_t jlo0 = (c < R.e0) ? 1u : 0u;
        const uint64_t endc = (uint64_t)R.e0 + R.n_tiles;
        const uint64_t jhi0 = has_line && endc > c ? (endc - c + 5) / 6 : 0u;
        // positions p with j = q0 p + d - e1 in that range
        const uint32_t jlo = (jlo0 + R.e1 > d) ? (uint32_t)((jlo0 + R.e1 - d + q0 - 1) / q0) : 0u;
        const uint32_t jhi = (jhi0 + R.e1 > d) ? (uint32_t)((jhi0 + R.e1 - d + q0 - 1) / q0) : 0u;
        const uint32_t jbase = w0 * 64;

        // ---- per-warp pattern copy, per-lane phases at block jbase ----
        for (uint32_t x = lane; x < (uint32_t)kNumAR * 8; x += 32) PA[x] = P.A[x >> 3].ext[x & 7];
        uint32_t* PT = PA + kNumAR * 8;
        if (!MG)
            for (uint32_t x = lane; x < P.patT_words; x += 32) PT[x] = __ldg(P.patT + x);
        if (P.ptab) {
            // phase = line phase (one table row per line, read with 16-byte
            // loads) + (J0 + jbase) mod q; the second term is the same for
            // the warp's 32 lines: one slot per lane, parked as (q << 16 | o)
            // in the (still empty) queue
            const uint32_t stride = P.ptab_stride;
            for (uint32_t s = lane; s < stride; s += 32) {
                const uint4 c = __ldg(reinterpret_cast<const uint4*>(P.pq) + s);   // q, magic, ...
                uint32_t j0q = 0;
                if (s < (uint32_t)kNumA) j0q = jm[s];
                else if (s >= (uint32_t)kSlotB && s - kSlotB < P.nB) j0q = jm[kNumA + (s - kSlotB)];
                const uint32_t o = j0q + mod_magic(jbase, c.x, c.y);
                Qw[s] = (c.x << 16) | (o >= c.x ? o - c.x : o);
            }
            __syncwarp();
            if (has_line) {
                const uint4* row = reinterpret_cast<const uint4*>(P.ptab + (size_t)li * stride);
#pragma unroll
                for (int c = 0; c < kSlotB / 8; c++) {
                    const uint4 v = __ldg(row + c);
                    const uint32_t hw[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const int i = c * 8 + k;
                        if (i >= kNumA || (STD && i >= kNumAR + kStdNT[STD])) continue;
                        const uint32_t qo = Qw[i], q = qo >> 16;
                        uint32_t ph = ((hw[k >> 1] >> (16 * (k & 1))) & 0xFFFFu) + (qo & 0xFFFFu);
                        ph = ph >= q ? ph - q : ph;
                        SA[i * 32 + lane] = (uint8_t)ph;
                    }
                }
                const uint32_t nbc = (stride - kSlotB) / 8;
#pragma unroll 4
                for (uint32_t c = 0; c < nbc; c++) {
                    const uint4 v = __ldg(row + kSlotB / 8 + c);
                    const uint32_t hw[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const uint32_t p = c * 8 + k;
                        const uint32_t qo = Qw[kSlotB + p], q = qo >> 16;
                        uint32_t ph = ((hw[k >> 1] >> (16 * (k & 1))) & 0xFFFFu) + (qo & 0xFFFFu);
                        ph = ph >= q ? ph - q : ph;
                        S[p * 32 + lane] = (uint16_t)ph;
                    }
                }
            }
            __syncwarp();
        } else {
#pragma unroll
            for (int i = 0; i < kNumA; i++) {
                if (STD && i >= kNumAR + kStdNT[STD]) continue;
                const LevelA& la = P.A[i];
                const uint32_t q = STD ? kStdQ[STD][i] : la.q;
                uint32_t ph = 0;
                if (q > 1) ph = phase_fast(ln.r_lo, ln.r_hi, q, la.magic, la.c32, la.winv, jm[i], jbase);
                SA[i * 32 + lane] = (uint8_t)ph;
            }
#pragma unroll 4
            for (uint32_t p = 0; p < P.nBpad; p++) {
                uint32_t ph = 0;
                if (p < P.nB) {
                    const PrimeC pc = P.primesB[p];
                    ph = phase_fast(ln.r_lo, ln.r_hi, pc.q, pc.magic, pc.c32, pc.winv, jm[kNumA + p], jbase);
                }
                S[p * 32 + lane] = (uint16_t)ph;
            }
        }
        LevelB B;
        B.Q = Qw;
        B.Cl = Cw;
        B.cnum = 0;
        B.S = S;
        B.pb = P.packB;
        B.bm = P.bitmapB;
        B.nB = P.nBpad;
        B.head = 0;
        B.tail = 0;
        B.cur = kNone;
        B.pi = 0;
        __syncwarp();

        // positions of words wbm / wbm + 64 (relative to jbase) not yet queued
        uint64_t ma = 0, mb = 0;
        uint32_t wbm = 0;
        uint32_t w = w0;            // next word to sweep
        for (;;) {
            // ---- level A: windows at word w ----
            uint64_t A1w[kNumA1];
            uint32_t A2w[kNumA2][3];
            uint32_t Tph[kNumT];
            const uint32_t off = (w - w0) * 64;
#pragma unroll
            for (int i = 0; i < kNumA; i++) {
                if (STD && i >= kNumAR + kStdNT[STD]) continue;
                const uint32_t q = STD ? kStdQ[STD][i] : P.A[i].q;
                uint32_t ph = (uint32_t)SA[i * 32 + lane] + off;
                if (STD) ph = q > 1 ? ph % q : 0;
                else ph = q > 1 ? mod_magic(ph, q, P.A[i].magic) : 0u;
                if (i >= kNumAR) { Tph[i - kNumAR] = ph; continue; }
                const uint32_t* pa = PA + i * 8 + (ph >> 5);
                const uint32_t b = ph & 31;
                if (i < kNumA1) {
                    A1w[i] = ((uint64_t)__funnelshift_r(pa[1], pa[2], b) << 32) | __funnelshift_r(pa[0], pa[1], b);
                } else {
#pragma unroll
                    for (int m = 0; m < 3; m++) A2w[i - kNumA1][m] = __funnelshift_r(pa[m], pa[m + 1], b);
                }
            }
            // merged windows: the phase mod q1 q2 from the two phases (CRT)
            uint32_t Mph[kMgWin];
            if (MG) {
#pragma unroll
                for (int k = 0; k < kMgWin; k++) {
                    const uint32_t a1 = Tph[mg_slot1(k)];
                    if (k < kMgPairs) {
                        const uint32_t q2 = kMg.w[k].q2;
                        const uint32_t d = (Tph[mg_slot2(k)] + q2 - a1) * kMg.w[k].inv % q2;   // a1 < q1 < q2
                        Mph[k] = a1 + kMg.w[k].q1 * d;
                    } else {
                        Mph[k] = a1;
                    }
                }
            }
            for (;;) {
                if (!__any_sync(kFull, (ma | mb) != 0)) {
                    if (w >= w1) break;
                    // two words per step: kill words ka (word w) and kb (w + 1)
                    uint64_t ka = 0, kb = 0;
#pragma unroll
                    for (int i = 0; i < kNumA1; i++) {
                        if (STD && i >= kStdA1[STD]) continue;       // dummy slots of the standard sets
                        const uint32_t q = STD ? kStdQ[STD][i] : P.A[i].q;
                        const uint32_t s1 = STD ? (64u % q) : P.A[i].s;
                        const uint32_t t1 = STD ? (q - 64u % q) : P.A[i].t;
                        // 128 mod q < q < 64: the same shift rule over two words
                        const uint32_t s2 = STD ? (128u % q) : (s1 + s1 >= q ? s1 + s1 - q : s1 + s1);
                        const uint32_t t2 = q - s2;
                        const uint64_t W = A1w[i];
                        ka |= W;
                        kb |= (W >> s1) | (W << t1);
                        A1w[i] = (W >> s2) | (W << t2);
                    }
#pragma unroll
                    for (int i = 0; i < kNumA2; i++) {
                        const uint32_t t = STD ? (kStdQ[STD][kNumA1 + i] - 64u) : P.A[kNumA1 + i].t;
                        uint32_t o0 = A2w[i][0], o1 = A2w[i][1], o2 = A2w[i][2];
                        ka |= ((uint64_t)o1 << 32) | o0;
                        uint32_t p0 = o2 | (o0 << t), p1 = __funnelshift_l(o0, o1, t), p2 = __funnelshift_l(o1, o2, t);
                        kb |= ((uint64_t)p1 << 32) | p0;
                        A2w[i][0] = p2 | (p0 << t);
                        A2w[i][1] = __funnelshift_l(p0, p1, t);
                        A2w[i][2] = __funnelshift_l(p1, p2, t);
                    }
                    // table windows: 128 pattern bits from the phase, phase += 128 mod q
                    if (MG) {
#pragma unroll
                        for (int k = 0; k < kMgWin; k++) {
                            const uint32_t ph = Mph[k];
                            const uint32_t* pt = PM + kMg.w[k].off + (ph >> 5);
                            const uint32_t b = ph & 31;
                            const uint32_t x0 = pt[0], x1 = pt[1], x2 = pt[2], x3 = pt[3], x4 = pt[4];
                            ka |= ((uint64_t)__funnelshift_r(x1, x2, b) << 32) | __funnelshift_r(x0, x1, b);
                            kb |= ((uint64_t)__funnelshift_r(x3, x4, b) << 32) | __funnelshift_r(x2, x3, b);
                            // periods > 128: one subtraction
                            Mph[k] = min(ph + 128u, ph + 128u - kMg.w[k].period);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < kNumT; i++) {
                        if (MG || (STD && i >= kStdNT[STD])) continue;
                        const uint32_t q = STD ? kStdQ[STD][kNumAR + i] : P.A[kNumAR + i].q;
                        const uint32_t toff = STD ? std_toff(i) : P.A[kNumAR + i].toff;
                        const uint32_t ph = Tph[i];
                        const uint32_t* pt = PT + toff + (ph >> 5);
                        const uint32_t b = ph & 31;
                        const uint32_t x0 = pt[0], x1 = pt[1], x2 = pt[2], x3 = pt[3], x4 = pt[4];
                        ka |= ((uint64_t)__funnelshift_r(x1, x2, b) << 32) | __funnelshift_r(x0, x1, b);
                        kb |= ((uint64_t)__funnelshift_r(x3, x4, b) << 32) | __funnelshift_r(x2, x3, b);
                        // ph + 128 < 3q for the table primes (q > 96); one
                        // subtraction suffices from q = 128 on
                        uint32_t nx = min(ph + 128u, ph + 128u - q);
                        if (!STD || q < 128u) nx = min(nx, nx - q);
                        if (!STD) nx = q > 1 ? nx : 0u;
                        Tph[i] = nx;
                    }
                    // positions of words w, w + 1 inside [jlo, jhi) and this unit
                    const uint32_t wb = w * 64;
                    uint64_t va = ~0ull, vb = ~0ull;
                    if (jlo > wb || jhi < wb + 128 || w + 2 > w1) {
                        va = 0;
                        vb = 0;
                        if (jhi > wb && jlo < wb + 64) {
                            const uint32_t lo = jlo > wb ? jlo - wb : 0;
                            const uint32_t hi = jhi - wb < 64 ? jhi - wb : 64;
                            va = (hi >= 64 ? ~0ull : ((1ull << hi) - 1)) & ~((1ull << lo) - 1);
                        }
                        const uint32_t wb2 = wb + 64;
                        if (w + 1 < w1 && jhi > wb2 && jlo < wb2 + 64) {
                            const uint32_t lo = jlo > wb2 ? jlo - wb2 : 0;
                            const uint32_t hi = jhi - wb2 < 64 ? jhi - wb2 : 64;
                            vb = (hi >= 64 ? ~0ull : ((1ull << hi) - 1)) & ~((1ull << lo) - 1);
                        }
                    }
                    ma = ~ka & va;
                    mb = ~kb & vb;
                    wbm = wb - jbase;
                    w += 2;
                }
                // queue this lane's survivors: warp prefix sum of the counts
                const uint32_t cnt = __popcll(ma) + __popcll(mb);
                uint32_t incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(kFull, incl, o);
                    if (lane >= (uint32_t)o) incl += v;
                }
                const uint32_t total = __shfl_sync(kFull, incl, 31);
                const uint32_t room = (uint32_t)kQCap - (B.tail - B.head);
                // fill in warp order up to the room left; what does not fit
                // stays in ma / mb for the next segment
                const uint32_t lim = total <= room ? total : room;
                uint32_t pos = incl - cnt;
                while (ma && pos < lim) {
                    const uint32_t bit = __ffsll((long long)ma) - 1;
                    ma &= ma - 1;
                    B.Q[(B.tail + pos++) & (kQCap - 1)] = ((wbm + bit) << 5) | lane;
                }
                while (mb && pos < lim) {
                    const uint32_t bit = __ffsll((long long)mb) - 1;
                    mb &= mb - 1;
                    B.Q[(B.tail + pos++) & (kQCap - 1)] = ((wbm + 64 + bit) << 5) | lane;
                }
                B.tail += lim;
                if (total > room) break;
            }
            __syncwarp();
            if (w >= w1 && !__any_sync(kFull, (ma | mb) != 0)) break;
            // ---- level B until the queue has room again ----
            while (B.tail - B.head > kQLow) b_round(B, a, R, P, cur_range, g, jbase, lane_lt);
        }
        // drain before the unit's phases are replaced
        while (__any_sync(kFull, B.cur != kNone) || B.tail != B.head)
            b_round(B, a, R, P, cur_range, g, jbase, lane_lt);
        if (B.cnum) c_process(B, a, R, P, cur_range, g, jbase, lane);
        __syncwarp();
}

// MINB = 2: at most 128 registers per thread (2 blocks of
// 256 per SM); MINB = 3: at most 80 registers (3 blocks of 256, or 6 of 128,
// when shared memory allows), a few spills in exchange for 50 % more
// resident warps.  The engine picks by the resident-block count it is tuned
// for.
template <int MINB>
__global__ void __launch_bounds__(kSweepThreads, MINB)
sweep_kernel(SweepArgs a) {
    extern __shared__ uint32_t s_mem[];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lane_lt = (1u << lane) - 1u;
    const uint32_t warp_in_block = threadIdx.x >> 5;
    // per warp: level-B queue (kQCap u32), level-C list (kCCap u32), level-A
    // patterns (register windows, and the table windows unless merged),
    // level-A phases (kNumA * 32 u8), level-B phases (b_stride * 32 u16);
    // then, in a merged launch, the block's merged table windows
    const bool mlaunch = a.merge_slot < (uint32_t)kMaxProfiles;
    const uint32_t paw = mlaunch ? (uint32_t)kNumAR * 8 : (uint32_t)kPAWords;
    const uint32_t ww = kQCap + kCCap + paw + kSAWords + a.b_stride * 16;
    uint32_t* Qw = s_mem + (size_t)warp_in_block * ww;
    uint32_t* Cw = Qw + kQCap;
    uint32_t* PA = Cw + kCCap;
    uint8_t* SA = reinterpret_cast<uint8_t*>(PA + paw);
    uint16_t* S = reinterpret_cast<uint16_t*>(PA + paw + kSAWords);
    uint32_t* PM = s_mem + (size_t)(blockDim.x >> 5) * ww;
    if (mlaunch) {
        const uint32_t* src = c_prof[a.merge_slot].patM;
        for (uint32_t x = threadIdx.x; x < kPatMWords; x += blockDim.x) PM[x] = __ldg(src + x);
    }
    __syncthreads();
    const uint64_t gwarp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;

    const uint32_t n_ranges = a.hdr->n_ranges;
    const uint64_t total_units = a.hdr->total_units;
    uint32_t cur_range = 0;
    for (uint64_t u = gwarp; u < total_units; u += nwarps) {
        if (u >= a.unit_prefix[cur_range + 1] || u < a.unit_prefix[cur_range]) {
            uint32_t lo = 0, hi = n_ranges;                 // last prefix <= u
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (a.unit_prefix[mid] <= u) lo = mid; else hi = mid;
            }
            cur_range = lo;
        }
        const RangeDev& R = a.ranges[cur_range];
        const ProfileConst& P = c_prof[R.profile];
        const uint64_t local = u - a.unit_prefix[cur_range];
        const uint32_t n_groups = (P.n_lines + 31) >> 5;
        const uint32_t g = (uint32_t)(local % n_groups);
        const uint32_t wc = (uint32_t)(local / n_groups);
        const uint32_t w0 = wc * R.unit_words;
        const uint32_t w1 = min(w0 + R.unit_words, R.n_words);
        // a merged launch has no per-warp table-window copies: the host
        // gives it only ranges of the merged profile (a unit of any other
        // profile is not swept)
        if (mlaunch) {
            if (R.profile != a.merge_slot) continue;
            if (P.std_a == 3)
                sweep_unit<3, true>(a, R, P, cur_range, g, w0, w1, Qw, Cw, PA, SA, S, PM, lane, lane_lt);
            else if (P.std_a == 4)
                sweep_unit<4, true>(a, R, P, cur_range, g, w0, w1, Qw, Cw, PA, SA, S, PM, lane, lane_lt);
            continue;
        }
        switch (P.std_a) {
        case 1: sweep_unit<1, false>(a, R, P, cur_range, g, w0, w1, Qw, Cw, PA, SA, S, PM, lane, lane_lt); break;
        case 2: sweep_unit<2, false>(a, R, P, cur_range, g, w0, w1, Qw, Cw, PA, SA, S, PM, lane, lane_lt); break;
        case 3: sweep_unit<3, false>(a, R, P, cur_range, g, w0, w1, Qw, Cw, PA, SA, S, PM, lane, lane_lt); break;
        case 4: sweep_unit<4, false>(a, R, P, cur_range, g, w0, w1, Qw, Cw, PA, SA, S, PM, lane, lane_lt); break;
        default: sweep_unit<0, false>(a, R, P, cur_range, g, w0, w1, Qw, Cw, PA, SA, S, PM, lane, lane_lt); break;
        }
    }
}

// ---------------------------------------------------------------------------
// host-side launch helpers
// ---------------------------------------------------------------------------
cudaError_t upload_profile_const(int slot, const ProfileConst& pc, cudaStream_t st) {
    return cudaMemcpyToSymbolAsync(c_prof, &pc, sizeof(ProfileConst), slot * sizeof(ProfileConst),
                                   cudaMemcpyHostToDevice, st);
}

cudaError_t launch_range_setup(const RangeDev* ranges, const SweepHeader* hdr, uint32_t max_ranges,
                               const uint32_t* primes, uint32_t max_primes, uint32_t* jmod,
                               uint32_t stride, cudaStream_t st) {
    dim3 grid((max_primes + 255) / 256, max_ranges < 65535 ? max_ranges : 65535);
    if (grid.x == 0) grid.x = 1;
    if (grid.x > 64) grid.x = 64;
    if (grid.y == 0) grid.y = 1;
    range_setup_kernel<<<grid, 256, 0, st>>>(ranges, hdr, primes, max_primes, jmod, stride);
    return cudaGetLastError();
}

size_t sweep_smem_bytes(uint32_t block_threads, uint32_t b_stride, bool merged) {
    const size_t paw = merged ? (size_t)kNumAR * 8 : (size_t)kPAWords;
    return ((size_t)(block_threads / 32) * (kQCap + kCCap + paw + kSAWords + (size_t)b_stride * 16) +
            (merged ? kPatMWords : 0)) * sizeof(uint32_t);
}

static bool g_sweep_attr_set = false;

// raise the dynamic shared-memory limit of the sweep kernels once (never
// during stream capture: callers invoke this before capturing)
static cudaError_t ensure_sweep_attr() {
    if (g_sweep_attr_set) return cudaSuccess;
    const int lim = (int)std::max(sweep_smem_bytes(kSweepThreads, kMaxLevelB, false),
                                  sweep_smem_bytes(kSweepThreads, kMaxLevelB, true));
    cudaError_t e = cudaFuncSetAttribute(sweep_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(sweep_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    if (e == cudaSuccess) g_sweep_attr_set = true;
    return e;
}

// resident blocks per SM of one register variant
static int sweep_occupancy(bool lowreg, uint32_t b_stride, uint32_t block_threads, bool merged) {
    int nb = 0;
    if (ensure_sweep_attr() != cudaSuccess) return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, lowreg ? sweep_kernel<3> : sweep_kernel<2>,
                                                  (int)block_threads,
                                                  sweep_smem_bytes(block_threads, b_stride, merged));
    return nb;
}

int sweep_blocks_per_sm(uint32_t b_stride, uint32_t block_threads, bool merged) {
    const int a = sweep_occupancy(false, b_stride, block_threads, merged);
    const int b = sweep_occupancy(true, b_stride, block_threads, merged);
    return a > b ? a : b;
}

bool sweep_needs_lowreg(uint32_t b_stride, uint32_t block_threads, uint32_t blocks_per_sm, bool merged) {
    return (int)blocks_per_sm > sweep_occupancy(false, b_stride, block_threads, merged);
}

cudaError_t launch_sweep(const RangeDev* ranges, const uint64_t* unit_prefix,
                         const SweepHeader* hdr, const uint32_t* jmod, uint32_t stride,
                         uint32_t b_stride, uint32_t grid, uint32_t block_threads, bool lowreg,
                         int merge_slot, cudaStream_t st) {
    if (block_threads != 128 && block_threads != 256) return cudaErrorInvalidValue;
    if (merge_slot >= kMaxProfiles) return cudaErrorInvalidValue;
    const bool merged = merge_slot >= 0;
    size_t smem = sweep_smem_bytes(block_threads, b_stride, merged);
    cudaError_t e = ensure_sweep_attr();
    if (e != cudaSuccess) return e;
    SweepArgs a;
    a.ranges = ranges;
    a.unit_prefix = unit_prefix;
    a.hdr = hdr;
    a.jmod = jmod;
    a.jmod_stride = stride;
    a.b_stride = b_stride;
    a.merge_slot = merged ? (uint32_t)merge_slot : kNone;
    if (lowreg) sweep_kernel<3><<<grid, block_threads, smem, st>>>(a);
    else sweep_kernel<2><<<grid, block_threads, smem, st>>>(a);
    return cudaGetLastError();
}


}  // namespace ccs
