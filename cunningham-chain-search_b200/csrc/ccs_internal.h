// Internal definitions shared by the host builder and the CUDA kernels.
//
// Lattice model.  The reference enumerates n = (tile*WP + k)*M + base with a
// mod-6 bucket per (tile, base) (v13:1551-1630).  Writing tile = 6J + c shows
// that every candidate is n = r + J*W with W = 6*M*WP and r = (c*WP + k)*M +
// base, i.e. one residue r mod W (a "line") per admissible (base, k, c), and J
// the block index.  The engine sweeps lines along J; the survivor set for a
// tile range is identical to the reference's, only the visiting order differs.
//
// Residue arithmetic runs in "phase space": for a filter prime q with
// w = W^{-1} mod q, the phase of n is u = n*w mod q = (r*w + J) mod q, which
// advances by exactly 1 per block.  A candidate is killed by q when u lies in
// G_q = {f*w mod q : f forbidden}.
#pragma once
#include <stdint.h>
#include <vector>
#include <string>

namespace ccs {

constexpr int kMaxStages = 4;
constexpr int kMaxChain = 64;          // v13:164 MAX_CHAIN
constexpr int kMaxDepth = 32;          // v13:159 MAX_SIEVE_CHAIN_LEN
constexpr int kMaxLimbs = 6;           // 192-bit chain members
constexpr int kNumA1 = 9;              // bit-sliced primes q < 64 (64-bit register windows)
constexpr int kNumA2 = 6;              // bit-sliced primes 64 < q < 96 (96-bit register windows)
constexpr int kNumT = 22;              // bit-sliced primes 96 < q < kTLimit (table windows)
constexpr int kNumAR = kNumA1 + kNumA2;
constexpr int kNumA = kNumAR + kNumT;  // level-A slots
constexpr uint32_t kTLimit = 211;
constexpr int kPatTMax = 224;          // pattern-table words of the table-window primes
constexpr double kTAdmit = 0.18;       // table-window admission (level-A survivors per 64 positions)

// Pattern words of a table-window prime: a 128-bit window (two 64-position
// words, the sweep's step) at any phase < q lies inside them.
constexpr uint32_t t_words(uint32_t q) { return (q - 1) / 32 + 5; }

// Merged table windows of the standard 22-prime table set (97..199): table
// slots 2k and 2k + 1 (k < kMgPairs) share one pattern of period q1 q2 (bit t
// set when t mod q1 or t mod q2 is a kill phase), the last slots keep their
// own.  One merged window costs the same five shared loads and funnel shifts
// per 128 positions as a single prime.  The patterns (kPatMWords words) are
// staged once per block.
constexpr int kMgPairs = 9;
constexpr int kMgWin = kNumT - kMgPairs;          // windows of the merged set
constexpr uint32_t std_t_prime(int i) {           // table slot i of the standard set
    constexpr uint32_t t[kNumT] = {97, 101, 103, 107, 109, 113, 127, 131, 137, 139, 149,
                                   151, 157, 163, 167, 173, 179, 181, 191, 193, 197, 199};
    return t[i];
}
constexpr int mg_slot1(int k) { return k < kMgPairs ? 2 * k : kMgPairs + k; }
constexpr int mg_slot2(int k) { return k < kMgPairs ? 2 * k + 1 : -1; }
// Per-window constants, built once at compile time (device code indexes the
// table with unrolled loop counters, so every entry folds to an immediate).
struct MgWin {
    uint32_t q1, q2, period, off, inv;   // inv = q1^-1 mod q2 (pairs)
};
struct MgTable {
    MgWin w[kMgWin];
    uint32_t words;                      // total pattern words
};
constexpr MgTable make_mg_table() {
    MgTable t{};
    uint32_t off = 0;
    for (int k = 0; k < kMgWin; k++) {
        MgWin& m = t.w[k];
        m.q1 = std_t_prime(mg_slot1(k));
        m.q2 = k < kMgPairs ? std_t_prime(mg_slot2(k)) : 1u;
        m.period = m.q1 * m.q2;
        m.off = off;
        off += t_words(m.period);
        m.inv = 0;
        for (uint32_t x = 1; k < kMgPairs && x < m.q2; x++)
            if (x * m.q1 % m.q2 == 1) { m.inv = x; break; }
    }
    t.words = off;
    return t;
}
constexpr MgTable kMgHost = make_mg_table();
constexpr uint32_t kPatMWords = kMgHost.words;
constexpr int kMaxProfiles = 16;
constexpr int kMaxLevelB = 256;        // per-lane cached phases (shared memory)
constexpr int kLevelBRound = 6;        // level-B primes tested per lane per round
constexpr uint32_t kCBitmapMax = 65536; // level-C primes below this test a G_q bitmap with
                                        // 32-bit phase arithmetic (q^2 + q < 2^32)

// One bit-sliced ("level A") prime.  Register-window primes (A1, A2) keep
// their 64/96-bit kill window in registers and advance it by shifts per 64
// blocks; table-window primes (T) keep only their phase and read the window
// from a replicated pattern table in shared memory (see filter.cu).
struct LevelA {
    uint32_t q;          // 1: dummy slot (no kills)
    uint32_t s;          // A1: 64 mod q          A2, T: unused
    uint32_t t;          // A1: q - s             A2: q - 64    T: unused
    uint32_t winv;       // W^{-1} mod q
    uint32_t magic;      // floor(2^32 / q)
    uint32_t c32;        // 2^32 mod q
    uint32_t toff;       // T: first word of the pattern in the table
    uint32_t tnw;        // T: pattern words, t_words(q)
    uint32_t ext[8];     // A1, A2: 256 bits, bit x = [x mod q in G_q]; all zero = dummy
};

// Level-B prime record read per candidate test: x = floor(2^32/q),
// y = q | (bitmap word offset << 16).
struct PrimeB {
    uint32_t magic;
    uint32_t q_off;
};

// Per-prime constants for the per-candidate stages.
struct PrimeC {
    uint32_t q;
    uint32_t magic;      // floor(2^32 / q)
    uint32_t winv;       // W^{-1} mod q
    uint32_t c32;        // 2^32 mod q
    uint32_t off;        // level B: bitmap word offset; level C: list offset
    uint32_t cnt;        // level C: list length
    uint64_t magic64;    // floor(2^64 / q) (level C)
};

// Device line record: residue r mod W and its reference coordinates.  On an
// extended profile (a filter prime q0 absorbed into the modulus, W' = q0 W)
// r is the residue mod W' and d = (r div W) < q0 selects the block class.
struct Line {
    uint32_t r_lo, r_hi;
    uint32_t k;          // wheel offset (k_offset)
    uint32_t bc;         // base_idx | (c << 16) | (d << 19)   (c = tile mod 6)
};

// Per-slot constants of the line phase table.
struct alignas(16) SlotConst {
    uint32_t q, magic, c32, winv;   // magic = floor((2^32 - 1) / q), c32 = 2^32 mod q, winv = W^-1 mod q
};

// Constant-memory image of one profile (lattice + filter).
struct ProfileConst {
    uint64_t W;                      // 6*M*WP (times q0 on an extended profile)
    uint32_t q0;                     // absorbed prime (1: none)
    uint32_t _q0pad;
    uint32_t n_lines;
    uint32_t nB, nC;                 // counts of per-candidate primes
    uint32_t nBpad;                  // nB rounded up with never-killing dummies (packB length)
    LevelA A[kNumA];                 // A1 slots, A2 slots, T slots
    const uint32_t* patT;            // T pattern table (patT_words u32)
    uint32_t patT_words;
    const Line* lines;
    const PrimeC* primesB;           // level B primes (ascending)
    const PrimeB* packB;             // compact level B records for the per-candidate test
    const uint32_t* bitmapB;         // G_q bitmaps of level B primes
    uint32_t std_a;                  // 1: level-A slots hold the standard set 37..127
    const PrimeC* primesC;           // level C primes (ascending)
    const uint32_t* listC;           // sorted G_q lists of level C primes
    const uint32_t* bitmapC;         // G_q bitmaps of the first nCb level C primes (q < kCBitmapMax)
    uint32_t nCb;
    uint32_t _cpad;
    const uint32_t* patM;            // merged table-window patterns (standard 22-prime sets; else null)
    // line phases r W^-1 mod q, [line][ptab_stride] u16 (null: computed per
    // work unit): level-A slot i at i, level-B prime p at kSlotB + p; and the
    // constants of those ptab_stride slots
    const uint16_t* ptab;
    const SlotConst* pq;
    uint32_t ptab_stride;
    uint32_t _ptpad;
};

// First level-B slot of a line phase table row (level-A slots padded to 8).
constexpr int kSlotB = (kNumA + 7) / 8 * 8;

// Line phase tables are kept when they need at most this many bytes.
constexpr size_t kPhaseTableMax = 1ull << 30;

// Host-side profile (everything derived from ccs_params).
struct HostProfile {
    // parameters
    uint32_t target = 18, depth = 18, bits = 89;
    std::vector<uint32_t> crt, wheel;
    struct Stage { std::vector<uint32_t> primes; uint32_t pos_lo; };
    std::vector<Stage> stages;
    uint32_t max_bases = 0;
    std::vector<uint64_t> witnesses;
    uint32_t primality = 1, prove_mode = 1;
    uint32_t reverse_prove = 0;      // CCS_FLAG_REVERSE_PROVE
    uint32_t kind = 1;               // 1: p -> 2p + 1, 2: p -> 2p - 1
    uint32_t q0 = 1;                 // filter prime absorbed into the modulus (1: none)
    uint32_t t_count = 0;            // table-window primes wanted (0: by the admission rule)

    // lattice
    uint64_t M = 0, W = 0;
    uint32_t WP = 0;
    std::vector<uint64_t> bases;
    std::vector<uint32_t> tkm6;
    std::vector<uint32_t> wheel_total;
    std::vector<Line> lines;
    uint64_t lines_per_class[6] = {0, 0, 0, 0, 0, 0};

    // filter primes (merged over stages, ascending)
    struct FPrime { uint32_t q; std::vector<uint32_t> forb; };
    std::vector<FPrime> fprimes;
    double expected_tests = 0, pass_rate = 1;

    // device-facing tables
    LevelA A[kNumA];
    std::vector<uint32_t> patT;      // T pattern table: bit x of a prime's block = [x mod q in G_q]
    std::vector<PrimeC> primesB, primesC;
    std::vector<PrimeB> packB;
    uint32_t std_a = 0;
    std::vector<uint32_t> bitmapB, listC;
    std::vector<uint32_t> bitmapC;   // level C primes below kCBitmapMax (PrimeC.off: first word)
    std::vector<uint32_t> patM;      // merged table windows (std_a 3 or 4: kPatMWords words)
    uint32_t nCb = 0;
    // index of every level-A/B prime for the per-range J0 mod q table
    std::vector<uint32_t> range_primes;   // A slots (kNumA, dummies as 1) then B then C
};

// Builds the lattice and tables; returns "" or an error message.
std::string build_profile(HostProfile& hp, uint32_t split_prime, uint32_t q0 = 1);

uint32_t mod_inverse_u32(uint32_t a, uint32_t q);
bool is_prime_u32(uint32_t n);

}  // namespace ccs
