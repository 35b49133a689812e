// Host-side lattice and filter-table builder.
//
// Replaces the reference's one-time table construction: forbidden residues
// (v13:771-787, v33:585-609), CRT bases with mod-6 buckets (v13:907-1059,
// v33:636-793) and the per-stage filter tables (v13:793-901, v15:871-1011).
// Everything is parametric: any CRT / wheel / stage prime lists, depth up to
// 32, filter primes up to 2^24.
#include "ccs_internal.h"

#include <algorithm>
#include <map>
#include <set>
#include <cstring>

namespace ccs {

bool is_prime_u32(uint32_t n) {
    if (n < 2) return false;
    if (n % 2 == 0) return n == 2;
    for (uint32_t d = 3; (uint64_t)d * d <= n; d += 2)
        if (n % d == 0) return false;
    return true;
}

static uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t m) {
    return (uint64_t)((unsigned __int128)a * b % m);
}

static uint64_t powmod64(uint64_t b, uint64_t e, uint64_t m) {
    uint64_t r = 1 % m;
    b %= m;
    while (e) {
        if (e & 1) r = mulmod64(r, b, m);
        b = mulmod64(b, b, m);
        e >>= 1;
    }
    return r;
}

uint32_t mod_inverse_u32(uint32_t a, uint32_t q) {
    // extended Euclid
    int64_t t = 0, nt = 1, r = q, nr = a % q;
    while (nr) {
        int64_t qq = r / nr;
        int64_t tmp = t - qq * nt; t = nt; nt = tmp;
        tmp = r - qq * nr; r = nr; nr = tmp;
    }
    if (t < 0) t += q;
    return (uint32_t)t;
}

// Residues n mod q with q | p_i = 2^i (n+1) - 1 for some i in [pos_lo, min(L, q)):
// n = 2^{-i} - 1; second kind, p_i = 2^i (n-1) + 1: n = 1 - 2^{-i} (v13b:779).
// Walk x = 2^{-i} by repeated multiplication with 2^{-1}.
static std::vector<uint32_t> forbidden_set(uint32_t q, uint32_t L, uint32_t pos_lo, uint32_t kind) {
    std::set<uint32_t> s;
    uint64_t inv2 = (q + 1) / 2;                 // 2^{-1} mod odd q
    uint64_t x = 1;                               // 2^{-0}
    uint32_t hi = std::min<uint32_t>(L, q);
    for (uint32_t i = 0; i < hi; i++) {
        if (i >= pos_lo) s.insert((uint32_t)(kind == 2 ? (1 + q - x) % q : (x + q - 1) % q));
        x = x * inv2 % q;
    }
    return std::vector<uint32_t>(s.begin(), s.end());
}

std::string build_profile(HostProfile& hp, uint32_t split_prime, uint32_t q0) {
    // ---- validation -------------------------------------------------------
    if (hp.crt.empty() || hp.wheel.empty()) return "crt and wheel prime lists must be non-empty";
    if (hp.target < 1 || hp.target > (uint32_t)kMaxChain) return "target out of range [1, 64]";
    if (hp.depth < 1) hp.depth = 1;
    if (hp.depth > (uint32_t)kMaxDepth) hp.depth = kMaxDepth;
    if (hp.depth > hp.target) hp.depth = hp.target;     // v13:3248-3252
    if (hp.bits < 21 || hp.bits > 160) return "bits out of range [21, 160]";
    std::set<uint32_t> lattice_primes;
    unsigned __int128 M = 1, WP = 1;
    for (uint32_t p : hp.crt) {
        if (!is_prime_u32(p) || p < 5) return "crt primes must be primes >= 5";
        if (!lattice_primes.insert(p).second) return "duplicate lattice prime";
        M *= p;
    }
    for (uint32_t p : hp.wheel) {
        if (!is_prime_u32(p) || p < 5) return "wheel primes must be primes >= 5";
        if (!lattice_primes.insert(p).second) return "duplicate lattice prime";
        WP *= p;
    }
    if (M >= ((unsigned __int128)1 << 32)) return "product of crt primes must be < 2^32";
    if (WP >= ((unsigned __int128)1 << 24)) return "wheel period must be < 2^24";
    unsigned __int128 W = M * WP * 6;
    if (W >= ((unsigned __int128)1 << 62)) return "lattice modulus 6*M*WP must be < 2^62";
    hp.M = (uint64_t)M;
    hp.WP = (uint32_t)WP;
    hp.W = (uint64_t)W;
    if (hp.stages.empty() || hp.stages.size() > (size_t)kMaxStages) return "1..4 filter stages required";

    // ---- CRT bases: combine admissible residues of every CRT prime --------
    std::vector<uint64_t> combos = {0};
    uint64_t mod = 1;
    for (uint32_t q : hp.crt) {
        std::vector<uint32_t> f = forbidden_set(q, hp.target, 0, hp.kind);
        std::vector<uint64_t> next;
        uint64_t inv = mod_inverse_u32((uint32_t)(mod % q), q);   // mod^{-1} mod q
        for (uint64_t a : combos) {
            for (uint32_t v = 0; v < q; v++) {
                if (std::binary_search(f.begin(), f.end(), v)) continue;
                // x == a (mod mod), x == v (mod q)
                uint64_t d = (v + q - a % q) % q;
                uint64_t t = d * inv % q;
                next.push_back(a + mod * t);
            }
        }
        combos.swap(next);
        mod *= q;
    }
    std::sort(combos.begin(), combos.end());

    // ---- wheels and mod-6 classes -----------------------------------------
    const uint32_t m6 = (uint32_t)(hp.M % 6);
    const uint32_t inv_m6 = (m6 == 1) ? 1 : 5;             // units mod 6 are self-inverse
    const uint32_t wp6 = hp.WP % 6;
    std::vector<std::vector<uint32_t>> wf;
    for (uint32_t q : hp.wheel) wf.push_back(forbidden_set(q, hp.target, 0, hp.kind));
    hp.bases.clear(); hp.tkm6.clear(); hp.wheel_total.clear(); hp.lines.clear();
    for (int c = 0; c < 6; c++) hp.lines_per_class[c] = 0;
    for (uint64_t base : combos) {
        if (hp.max_bases && hp.bases.size() >= hp.max_bases) break;
        std::vector<uint32_t> rq(hp.wheel.size()), step(hp.wheel.size());
        for (size_t i = 0; i < hp.wheel.size(); i++) {
            rq[i] = (uint32_t)(base % hp.wheel[i]);
            step[i] = (uint32_t)(hp.M % hp.wheel[i]);
        }
        std::vector<uint32_t> ks;
        for (uint32_t k = 0; k < hp.WP; k++) {
            bool ok = true;
            for (size_t i = 0; i < hp.wheel.size() && ok; i++)
                if (std::binary_search(wf[i].begin(), wf[i].end(), rq[i])) ok = false;
            if (ok) ks.push_back(k);
            for (size_t i = 0; i < hp.wheel.size(); i++) {
                rq[i] += step[i];
                if (rq[i] >= hp.wheel[i]) rq[i] -= hp.wheel[i];
            }
        }
        if (ks.empty()) continue;
        uint32_t bidx = (uint32_t)hp.bases.size();
        if (bidx >= 65536) return "too many bases (> 65535)";
        // n == 5 (mod 6) for the first kind, n == 1 for the second (v13b:983)
        const uint32_t nres = hp.kind == 2 ? 1u : 5u;
        uint32_t t6 = (uint32_t)(((nres + 6 - base % 6) % 6) * inv_m6 % 6);
        hp.bases.push_back(base);
        hp.tkm6.push_back(t6);
        hp.wheel_total.push_back((uint32_t)ks.size());
        for (uint32_t k : ks) {
            // tile class c with k == t6 - c*WP (mod 6)
            uint32_t c = (uint32_t)(((t6 + 6 - k % 6) % 6) * wp6 % 6);
            unsigned __int128 r = ((unsigned __int128)c * hp.WP + k) * hp.M + base;
            Line ln;
            ln.r_lo = (uint32_t)r;
            ln.r_hi = (uint32_t)(r >> 32);
            ln.k = k;
            ln.bc = bidx | (c << 16);
            hp.lines.push_back(ln);
            hp.lines_per_class[c]++;
        }
    }
    if (hp.bases.empty()) return "no admissible bases";
    if (hp.lines.size() >= (1ull << 31)) return "too many lines";

    // ---- filter primes ----------------------------------------------------
    std::map<uint32_t, std::set<uint32_t>> fmap;
    hp.expected_tests = 0;
    double surv = 1.0;
    for (auto& st : hp.stages) {
        if (st.pos_lo > 1) return "stage pos_lo must be 0 or 1";
        for (uint32_t q : st.primes) {
            if (!is_prime_u32(q) || q < 5) return "filter primes must be primes >= 5";
            if (lattice_primes.count(q)) return "filter prime divides the lattice modulus";
            if (q >= (1u << 24)) return "filter primes must be < 2^24";
            std::vector<uint32_t> f = forbidden_set(q, hp.depth, st.pos_lo, hp.kind);
            // reference test order: stage by stage, prime by prime
            hp.expected_tests += surv;
            surv *= 1.0 - (double)f.size() / q;
            fmap[q].insert(f.begin(), f.end());
        }
    }
    hp.pass_rate = surv;
    hp.fprimes.clear();
    for (auto& kv : fmap) {
        HostProfile::FPrime fp;
        fp.q = kv.first;
        fp.forb.assign(kv.second.begin(), kv.second.end());
        hp.fprimes.push_back(fp);
    }

    // ---- optional extension: absorb filter prime q0 into the modulus ------
    hp.q0 = 1;
    if (q0 > 1) {
        const HostProfile::FPrime* fq = nullptr;
        for (auto& fp : hp.fprimes)
            if (fp.q == q0) fq = &fp;
        if (!fq) return "extension prime is not a filter prime";
        if ((unsigned __int128)hp.W * q0 >= ((unsigned __int128)1 << 62)) return "extended modulus too large";
        std::vector<Line> ext;
        ext.reserve(hp.lines.size() * (q0 - fq->forb.size()));
        for (const Line& ln : hp.lines) {
            const uint64_t r = ((uint64_t)ln.r_hi << 32) | ln.r_lo;
            for (uint32_t d = 0; d < q0; d++) {
                const uint64_t r2 = r + (uint64_t)d * hp.W;
                if (std::binary_search(fq->forb.begin(), fq->forb.end(), (uint32_t)(r2 % q0))) continue;
                Line e;
                e.r_lo = (uint32_t)r2;
                e.r_hi = (uint32_t)(r2 >> 32);
                e.k = ln.k;
                e.bc = ln.bc | (d << 19);
                ext.push_back(e);
            }
        }
        if (ext.size() >= (1ull << 31)) return "too many extended lines";
        hp.lines.swap(ext);
        hp.W *= q0;
        hp.q0 = q0;
    }

    // ---- level classification ----------------------------------------------
    memset(hp.A, 0, sizeof(hp.A));
    for (int i = 0; i < kNumA; i++) { hp.A[i].q = 1; hp.A[i].magic = 0xFFFFFFFFu; }   // dummy: no kills
    int nA1 = 0, nA2 = 0, nT = 0;
    hp.primesB.clear(); hp.primesC.clear(); hp.bitmapB.clear(); hp.listC.clear(); hp.packB.clear();
    hp.bitmapC.clear();
    hp.nCb = 0;
    hp.patT.clear();
    const uint64_t Wm = hp.W;
    // How many table-window primes: one costs about as much per 64-position
    // word as a fifth of a level-B test per lane, so the next prime is taken
    // while the expected level-A survivors per word (64 x product of the pass
    // fractions taken so far) stay above kTAdmit; the count is then rounded
    // to one of the two compiled standard sizes (7: primes < 128, or 22).
    int nT_max = 0;
    {
        double as = 64.0;
        int a1 = 0, a2 = 0, nt = 0, avail = 0;
        bool open = true;
        for (auto& fp : hp.fprimes) {
            const uint32_t q = fp.q;
            if (q == hp.q0) continue;
            const double pass = 1.0 - (double)fp.forb.size() / q;
            if (q < 64 && a1 < kNumA1) { a1++; as *= pass; }
            else if (q > 64 && q < 96 && a2 < kNumA2) { a2++; as *= pass; }
            else if (q > 96 && q < kTLimit && avail < kNumT) {
                avail++;
                if (open && as >= kTAdmit) { nt++; as *= pass; } else open = false;
            }
        }
        nT_max = nt <= 14 ? std::min(7, avail) : std::min(kNumT, avail);
        if (hp.t_count) nT_max = std::min<int>((int)hp.t_count, avail);
    }
    for (auto& fp : hp.fprimes) {
        uint32_t q = fp.q;
        if (q == hp.q0) continue;                       // absorbed into the lattice
        uint32_t winv = mod_inverse_u32((uint32_t)(Wm % q), q);
        std::vector<uint32_t> g;
        for (uint32_t f : fp.forb) g.push_back((uint32_t)((uint64_t)f * winv % q));
        std::sort(g.begin(), g.end());
        int slot = -1;
        if (q < 64 && nA1 < kNumA1) slot = nA1++;
        else if (q > 64 && q < 96 && nA2 < kNumA2) slot = kNumA1 + nA2++;
        else if (q > 96 && q < kTLimit && nT < nT_max &&
                 hp.patT.size() + t_words(q) + 5 <= (size_t)kPatTMax)
            slot = kNumAR + nT++;
        if (slot >= 0) {
            LevelA& a = hp.A[slot];
            a.q = q;
            a.winv = winv;
            a.magic = 0xFFFFFFFFu / q;
            a.c32 = (uint32_t)((1ull << 32) % q);
            if (slot < kNumA1) { a.s = 64 % q; a.t = q - a.s; }
            else if (slot < kNumAR) { a.s = 0; a.t = q - 64; }
            if (slot < kNumAR) {
                for (uint32_t x = 0; x < 256; x++)
                    if (std::binary_search(g.begin(), g.end(), x % q)) a.ext[x >> 5] |= 1u << (x & 31);
            } else {
                // replicated pattern: a 128-bit window at any phase < q lies in tnw words
                a.toff = (uint32_t)hp.patT.size();
                a.tnw = t_words(q);
                for (uint32_t wd = 0; wd < a.tnw; wd++) {
                    uint32_t v = 0;
                    for (uint32_t bit = 0; bit < 32; bit++)
                        if (std::binary_search(g.begin(), g.end(), (wd * 32 + bit) % q)) v |= 1u << bit;
                    hp.patT.push_back(v);
                }
            }
            continue;
        }
        PrimeC pc;
        memset(&pc, 0, sizeof(pc));
        pc.q = q;
        pc.magic = 0xFFFFFFFFu / q;
        pc.winv = winv;
        pc.c32 = (uint32_t)((1ull << 32) % q);
        pc.magic64 = ~0ull / q;
        if (q < split_prime && q < 65536 && hp.primesB.size() < (size_t)kMaxLevelB &&
            hp.bitmapB.size() + (q + 31) / 32 < 65536) {
            pc.off = (uint32_t)hp.bitmapB.size();
            pc.cnt = (uint32_t)g.size();
            std::vector<uint32_t> bm((q + 31) / 32, 0);
            for (uint32_t u : g) bm[u >> 5] |= 1u << (u & 31);
            hp.bitmapB.insert(hp.bitmapB.end(), bm.begin(), bm.end());
            hp.primesB.push_back(pc);
            PrimeB pb;
            pb.magic = pc.magic;
            pb.q_off = q | (pc.off << 16);
            hp.packB.push_back(pb);
        } else if (q < kCBitmapMax) {
            // small level-C primes (a prefix of the ascending list): G_q bitmap
            pc.off = (uint32_t)hp.bitmapC.size();
            pc.cnt = (uint32_t)g.size();
            std::vector<uint32_t> bm((q + 31) / 32, 0);
            for (uint32_t u : g) bm[u >> 5] |= 1u << (u & 31);
            hp.bitmapC.insert(hp.bitmapC.end(), bm.begin(), bm.end());
            hp.primesC.push_back(pc);
            hp.nCb = (uint32_t)hp.primesC.size();
        } else {
            // sorted list padded to a multiple of 4 entries (0xFFFFFFFF never
            // matches a phase), 16-byte aligned for vector loads
            pc.off = (uint32_t)hp.listC.size();
            pc.cnt = (uint32_t)g.size();
            hp.listC.insert(hp.listC.end(), g.begin(), g.end());
            while (hp.listC.size() % 4) hp.listC.push_back(0xFFFFFFFFu);
            hp.primesC.push_back(pc);
        }
    }
    // dummy table-window slots read an all-zero block (phase stays 0)
    {
        const uint32_t zoff = (uint32_t)hp.patT.size();
        for (int i = 0; i < 5; i++) hp.patT.push_back(0);
        for (int i = nT; i < kNumT; i++) { hp.A[kNumAR + i].toff = zoff; hp.A[kNumAR + i].tnw = 5; }
    }
    // pad the level-B records to a multiple of the per-round test count with
    // entries that never kill (q = 2, all-zero bitmap word)
    if (!hp.packB.empty() && hp.packB.size() % kLevelBRound) {
        if (hp.bitmapB.size() >= 65536) return "level-B bitmaps too large";
        const uint32_t zero_off = (uint32_t)hp.bitmapB.size();
        hp.bitmapB.push_back(0);
        while (hp.packB.size() % kLevelBRound) {
            PrimeB pb;
            pb.magic = 0xFFFFFFFFu / 2;
            pb.q_off = 2u | (zero_off << 16);
            hp.packB.push_back(pb);
        }
    }
    // the standard level-A sets (primes 37..127 or 37..199, with or without 37
    // absorbed into the lattice) have kernels with
    // compile-time shift amounts
    {
        static const uint32_t std_q[4][kNumA] = {
            {37, 41, 43, 47, 53, 59, 61, 1, 1, 67, 71, 73, 79, 83, 89,
             97, 101, 103, 107, 109, 113, 127, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
            {41, 43, 47, 53, 59, 61, 1, 1, 1, 67, 71, 73, 79, 83, 89,
             97, 101, 103, 107, 109, 113, 127, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
            {37, 41, 43, 47, 53, 59, 61, 1, 1, 67, 71, 73, 79, 83, 89,
             97, 101, 103, 107, 109, 113, 127, 131, 137, 139, 149, 151, 157, 163, 167, 173, 179, 181,
             191, 193, 197, 199},
            {41, 43, 47, 53, 59, 61, 1, 1, 1, 67, 71, 73, 79, 83, 89,
             97, 101, 103, 107, 109, 113, 127, 131, 137, 139, 149, 151, 157, 163, 167, 173, 179, 181,
             191, 193, 197, 199}};
        hp.std_a = 0;
        for (int v = 0; v < 4; v++) {
            bool same = true;
            for (int i = 0; i < kNumA; i++) same &= hp.A[i].q == std_q[v][i];
            if (same) hp.std_a = 1 + v;
        }
    }
    // merged table windows of the 22-prime standard sets: bit t of window k
    // is set when t mod q1 (or t mod q2) is a kill phase of that slot, read
    // from the slot's own pattern (bit x of it, x < q, is the phase x)
    hp.patM.clear();
    if (hp.std_a == 3 || hp.std_a == 4) {
        auto kill = [&](int slot, uint32_t x) {
            const LevelA& a = hp.A[kNumAR + slot];
            return (hp.patT[a.toff + (x >> 5)] >> (x & 31)) & 1u;
        };
        for (int k = 0; k < kMgWin; k++) {
            const uint32_t q1 = kMgHost.w[k].q1, q2 = kMgHost.w[k].q2, P = kMgHost.w[k].period;
            const int s1 = mg_slot1(k), s2 = mg_slot2(k);
            if (hp.A[kNumAR + s1].q != q1 || (s2 >= 0 && hp.A[kNumAR + s2].q != q2))
                return "merged table windows do not match the standard set";
            for (uint32_t wd = 0; wd < t_words(P); wd++) {
                uint32_t v = 0;
                for (uint32_t bit = 0; bit < 32; bit++) {
                    const uint32_t t = (wd * 32 + bit) % P;
                    if (kill(s1, t % q1) | (s2 >= 0 ? kill(s2, t % q2) : 0u)) v |= 1u << bit;
                }
                hp.patM.push_back(v);
            }
        }
        if (hp.patM.size() != kPatMWords) return "merged table windows: size mismatch";
    }
    hp.range_primes.clear();
    for (int i = 0; i < kNumA; i++) hp.range_primes.push_back(hp.A[i].q);
    for (auto& p : hp.primesB) hp.range_primes.push_back(p.q);
    for (auto& p : hp.primesC) hp.range_primes.push_back(p.q);
    (void)powmod64;
    return "";
}

}  // namespace ccs
