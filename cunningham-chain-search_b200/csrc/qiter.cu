// Fingerprint-pool Q iteration: p_0 = Q * D_V * 2^E - 1 over consecutive Q
// for every variant V of a pool (the reference's v16 engine,
// experimental/cc20_first_kind_immune_v16.cu).
//
// Sieve.  For a prime q not dividing D_V, chain position j is divisible by q
// exactly when Q = (D_V * 2^(E+j))^-1 (mod q) (v16:1244-1266); the reference
// ORs these residues into one mask per (V, q) and probes Q mod q for every Q
// of a launch, one thread per Q (v16:2038-2153).  Here a lane owns a word of
// 64 consecutive Q and a window kills a whole word at once: per variant, the
// primes (ordered by the share of Q they kill) are merged into runs whose
// product P stays within 8192, and each run's pattern (bit b set when b mod q
// is forbidden for some q of the run, b < P + 64 and beyond) is staged in
// shared memory; the 64-bit window starting at the word's phase u = Q mod P
// is three shared loads and two funnel shifts.  A warp leaves the window loop
// as soon as all 32 words are fully killed, which after a dozen windows is the
// common case.
//
// Work units are runs of unit_words words of one segment (one variant, one
// run of Q); blocks take units from a global counter and restage the pattern
// slab only when the variant changes; warps take 32-word blocks of a unit
// from a shared counter.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ccs.h"
#include "ccs_internal.h"
#include "ccs_kernels.cuh"

namespace ccs {
namespace {

ccs_status fail(ccs_status st, const std::string& msg) { return set_error(st, msg.c_str()); }

#define CU(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(e_ == cudaErrorMemoryAllocation ? CCS_ERR_NOMEM : CCS_ERR_CUDA,   \
                        std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)

constexpr uint32_t kQPrimeMax = 8192;        // sieve primes below this
constexpr uint32_t kQMaxPrimes = 1024;
constexpr uint32_t kQSlabMax = 16384;        // pattern words per variant (64 KB of shared memory)
constexpr uint32_t kQThreads = 256;
constexpr uint32_t kQUnitWords = 8192;       // 524,288 Q per work unit
constexpr uint32_t kQMaxSegs = 1u << 20;
constexpr uint64_t kQGroupMax = 8192;        // largest period of a merged window

inline uint32_t q_words(uint32_t q) { return (q - 1) / 32 + 3; }

struct QSweepArgs {
    const uint4* vhdr;                       // per variant: act_start, n_act, pat_start, pat_words
    const uint4* act;                        // per window: period, floor(2^32 / period), slab offset
    const uint32_t* pat;
    const ccs_qseg* segs;
    const uint64_t* unit_prefix;             // [n_segs + 1]
    uint32_t n_segs;
    uint32_t unit_words;
    uint32_t act_max;                        // shared-memory entries reserved
    uint32_t* out;                           // ccs_qsurvivor records
    uint32_t* count;                         // [0] survivors, [1] next work unit
    uint32_t cap;
};

__device__ __forceinline__ uint32_t qmod(uint32_t x, uint32_t q, uint32_t m) {
    uint32_t r = x - __umulhi(x, m) * q;       // < 2q
    return r >= q ? r - q : r;
}

// unit u -> segment, first word, word count (binary search on the unit prefix)
__device__ __forceinline__ void qiter_unit(const QSweepArgs& a, uint64_t u, uint32_t* info) {
    uint32_t lo = 0, hi = a.n_segs;                                  // last seg with prefix <= u
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.unit_prefix[mid] <= u) lo = mid; else hi = mid;
    }
    const ccs_qseg& sg = a.segs[lo];
    const uint32_t words = (uint32_t)(((uint64_t)sg.n_q + 63) >> 6);
    const uint32_t w0 = (uint32_t)(u - a.unit_prefix[lo]) * a.unit_words;
    info[0] = lo;
    info[1] = sg.variant;
    info[2] = w0;
    info[3] = min(a.unit_words, words - w0);
}

__global__ void __launch_bounds__(kQThreads)
qiter_sweep_kernel(QSweepArgs a) {
    extern __shared__ __align__(16) uint32_t qsm[];
    uint4* s_act = reinterpret_cast<uint4*>(qsm);                 // q, magic, phase, slab offset
    uint32_t* s_pat = qsm + 4 * a.act_max;
    // units are taken from a global counter; thread 0 resolves the next one
    // while the block sweeps the current one.  Inside a unit, warps take
    // 32-word blocks from a shared counter, so no warp waits on a slow one
    // at the next unit boundary for longer than one block.
    __shared__ uint32_t s_cur[4], s_next[4];
    __shared__ uint32_t s_blk;
    __shared__ uint32_t s_staged;
    __shared__ int s_has_next;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t total = a.unit_prefix[a.n_segs];
    if (threadIdx.x == 0) {
        s_staged = 0xFFFFFFFFu;
        const uint64_t u = atomicAdd(a.count + 1, 1u);
        s_has_next = u < total;
        if (u < total) qiter_unit(a, u, s_next);
    }
    __syncthreads();
    while (s_has_next) {
        if (threadIdx.x < 4) s_cur[threadIdx.x] = s_next[threadIdx.x];
        if (threadIdx.x == 0) s_blk = 0;
        __syncthreads();
        const uint32_t seg = s_cur[0], v = s_cur[1], w0 = s_cur[2], nw = s_cur[3];
        const uint4 vh = a.vhdr[v];
        if (s_staged != v) {
            for (uint32_t i = threadIdx.x; i < vh.w; i += blockDim.x) s_pat[i] = a.pat[vh.z + i];
        }
        const ccs_qseg& sg = a.segs[seg];
        for (uint32_t i = threadIdx.x; i < vh.y; i += blockDim.x) {
            const uint4 e = a.act[vh.x + i];
            const uint32_t q = e.x;
            // (q_base + 64 w0) mod q, limb by limb from the top
            uint32_t L[4];
            uint64_t c = (uint64_t)w0 << 6;
#pragma unroll
            for (int w = 0; w < 4; w++) {
                const uint64_t s = (uint64_t)sg.q_base[w] + c;
                L[w] = (uint32_t)s;
                c = s >> 32;
            }
            uint64_t r = c;                                          // a carry out of 2^128 is 1
#pragma unroll
            for (int w = 3; w >= 0; w--) r = ((r << 32) | L[w]) % q;
            s_act[i] = make_uint4(q, e.y, (uint32_t)r, e.z);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_staged = v;
            const uint64_t u = atomicAdd(a.count + 1, 1u);           // next unit, resolved
            s_has_next = u < total;                                  // while the block sweeps
            if (u < total) qiter_unit(a, u, s_next);
        }
        const uint32_t n_act = vh.y;
        const uint32_t n_q = sg.n_q;
        const uint32_t n_blk = (nw + 31) >> 5;
        for (;;) {
            uint32_t blk = 0;
            if (lane == 0) blk = atomicAdd(&s_blk, 1u);
            blk = __shfl_sync(0xFFFFFFFFu, blk, 0);
            if (blk >= n_blk) break;
            const uint32_t k = blk * 32 + lane;
            const uint32_t wg = w0 + k;                              // word index in the segment
            uint32_t klo = 0, khi = 0;
            if (k >= nw) {
                klo = khi = 0xFFFFFFFFu;
            } else {
                const uint64_t first = (uint64_t)wg << 6;
                const uint64_t left = (uint64_t)n_q - first;         // Q of this word in the segment
                if (left < 64) {
                    const uint64_t valid = (1ull << left) - 1;
                    klo = ~(uint32_t)valid;
                    khi = ~(uint32_t)(valid >> 32);
                }
            }
            const uint32_t k64 = k << 6;
            for (uint32_t i = 0; i < n_act; i++) {
                const uint4 e = s_act[i];
                const uint32_t ph = qmod(e.z + k64, e.x, e.y);
                const uint32_t* p = s_pat + e.w + (ph >> 5);
                const uint32_t x0 = p[0], x1 = p[1], x2 = p[2];
                const uint32_t sh = ph & 31;
                klo |= __funnelshift_r(x0, x1, sh);
                khi |= __funnelshift_r(x1, x2, sh);
                if (__all_sync(0xFFFFFFFFu, (klo & khi) == 0xFFFFFFFFu)) break;   // after every window
            }
            const uint32_t llo = ~klo, lhi = ~khi;
            const uint32_t cnt = __popc(llo) + __popc(lhi);
            if (__ballot_sync(0xFFFFFFFFu, cnt != 0) == 0) continue;
            uint32_t incl = cnt;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                if (lane >= (uint32_t)d) incl += t;
            }
            uint32_t base = 0;
            if (lane == 31) base = atomicAdd(a.count, incl);
            base = __shfl_sync(0xFFFFFFFFu, base, 31) + incl - cnt;
            uint64_t live = ((uint64_t)lhi << 32) | llo;
            while (live) {
                const int b = __ffsll((long long)live) - 1;
                live &= live - 1;
                if (base < a.cap) {
                    uint4* o = reinterpret_cast<uint4*>(a.out) + base;
                    *o = make_uint4((wg << 6) + (uint32_t)b, seg, v, 0u);
                }
                base++;
            }
        }
        __syncthreads();                                             // unit done: shared memory free
    }
}

}  // namespace
}  // namespace ccs

using namespace ccs;

struct ccs_qiter {
    int device = 0;
    int sms = 148;
    ccs_engine* pe = nullptr;                 // prover: constant slot, walk scratch, staging
    uint32_t n_variants = 0, exp_start = 0, depth = 0, target = 0;
    std::vector<uint32_t> primes;
    std::vector<uint32_t> dv;                 // [n_variants][4]
    std::vector<uint4> vhdr;
    std::vector<uint4> act;                   // window: period, floor(2^32 / period), slab offset
    std::vector<uint32_t> pat;
    std::vector<uint32_t> fcount;             // [variant][prime] forbidden residues
    uint32_t act_max = 0, slab_max = 0;
    size_t smem = 0;
    int blocks_per_sm = 1;
    DevBuf<uint4> d_vhdr, d_act;
    DevBuf<uint32_t> d_pat, d_dv, d_count;
    // segment staging, one set for filter calls and one for prove calls, so
    // that a filter and a prove may run at the same time from two host
    // threads (each on its own stream)
    struct Staging {
        DevBuf<ccs_qseg> d_segs;
        DevBuf<uint64_t> d_prefix;
        ccs_qseg* h_segs = nullptr;           // pinned
        uint64_t* h_prefix = nullptr;
        uint32_t h_cap = 0;
    } fst, pst;
    cudaStream_t fstream = nullptr;           // filter calls without a stream
    uint32_t* h_count = nullptr;
};

namespace {

uint32_t inv_mod(uint32_t a, uint32_t q) {
    int64_t t = 0, nt = 1, r = q, nr = a % q;
    while (nr) {
        const int64_t f = r / nr;
        int64_t x = t - f * nt; t = nt; nt = x;
        x = r - f * nr; r = nr; nr = x;
    }
    return (uint32_t)(t < 0 ? t + q : t);
}

uint32_t pow2_mod(uint32_t e, uint32_t q) {
    uint64_t r = 1 % q, b = 2 % q;
    while (e) {
        if (e & 1) r = r * b % q;
        b = b * b % q;
        e >>= 1;
    }
    return (uint32_t)r;
}

bool is_odd_prime(uint32_t q) {
    if (q < 3 || !(q & 1)) return false;
    for (uint32_t d = 3; d * d <= q; d += 2)
        if (q % d == 0) return false;
    return true;
}

unsigned __int128 dv_of(const ccs_qiter* Q, uint32_t v) {
    unsigned __int128 d = 0;
    for (int w = 3; w >= 0; w--) d = (d << 32) | Q->dv[4 * (size_t)v + w];
    return d;
}

int bits128(unsigned __int128 x) {
    int b = 0;
    while (x) { b++; x >>= 1; }
    return b;
}

ccs_status stage_segs(ccs_qiter::Staging& S, const ccs_qseg* segs, uint32_t n_segs, cudaStream_t st) {
    if (n_segs > S.h_cap) {
        uint32_t c = 1024;
        while (c < n_segs) c <<= 1;
        if (S.h_segs) cudaFreeHost(S.h_segs);
        if (S.h_prefix) cudaFreeHost(S.h_prefix);
        S.h_segs = nullptr; S.h_prefix = nullptr; S.h_cap = 0;
        if (cudaMallocHost(&S.h_segs, sizeof(ccs_qseg) * c) != cudaSuccess ||
            cudaMallocHost(&S.h_prefix, sizeof(uint64_t) * (c + 1)) != cudaSuccess)
            return fail(CCS_ERR_NOMEM, "pinned allocation failed");
        CU(S.d_segs.alloc(c));
        CU(S.d_prefix.alloc(c + 1));
        S.h_cap = c;
    }
    cudaStreamSynchronize(st);                // staging buffers may still feed a copy
    memcpy(S.h_segs, segs, sizeof(ccs_qseg) * n_segs);
    uint64_t acc = 0;
    S.h_prefix[0] = 0;
    for (uint32_t s = 0; s < n_segs; s++) {
        const uint64_t words = ((uint64_t)segs[s].n_q + 63) >> 6;
        acc += (words + kQUnitWords - 1) / kQUnitWords;
        S.h_prefix[s + 1] = acc;
    }
    if (n_segs) {
        CU(cudaMemcpyAsync(S.d_segs.p, S.h_segs, sizeof(ccs_qseg) * n_segs, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(S.d_prefix.p, S.h_prefix, sizeof(uint64_t) * (n_segs + 1),
                           cudaMemcpyHostToDevice, st));
    }
    return CCS_OK;
}

ccs_status check_segs(const ccs_qiter* Q, const ccs_qseg* segs, uint32_t n_segs) {
    if (n_segs && !segs) return fail(CCS_ERR_INVALID, "segs is null");
    if (n_segs > kQMaxSegs) return fail(CCS_ERR_INVALID, "at most 2^20 segments per call");
    for (uint32_t s = 0; s < n_segs; s++)
        if (segs[s].variant >= Q->n_variants) return fail(CCS_ERR_INVALID, "segment variant out of range");
    return CCS_OK;
}

}  // namespace

extern "C" {

ccs_status ccs_qiter_create(const ccs_qiter_params* p, int device, ccs_qiter** out) {
    if (!p || !out) return fail(CCS_ERR_INVALID, "null argument");
    *out = nullptr;
    if (!p->n_variants || !p->dv) return fail(CCS_ERR_INVALID, "empty pool");
    if (p->n_variants > (1u << 24)) return fail(CCS_ERR_INVALID, "at most 2^24 variants");
    if (!p->depth || p->depth > 64) return fail(CCS_ERR_INVALID, "depth must be in [1, 64]");
    if (!p->target || p->target > 64) return fail(CCS_ERR_INVALID, "target must be in [1, 64]");
    if (p->exp_start > 96) return fail(CCS_ERR_INVALID, "exp_start must be <= 96");
    if (!p->n_primes || !p->primes || p->n_primes > kQMaxPrimes)
        return fail(CCS_ERR_INVALID, "1 .. 1024 sieve primes required");
    for (uint32_t i = 0; i < p->n_primes; i++) {
        if (!is_odd_prime(p->primes[i]) || p->primes[i] >= kQPrimeMax)
            return fail(CCS_ERR_INVALID, "sieve primes must be odd primes below 8192");
        if (i && p->primes[i] <= p->primes[i - 1]) return fail(CCS_ERR_INVALID, "sieve primes must ascend");
    }
    if (p->flags & ~CCS_FLAG_REVERSE_PROVE) return fail(CCS_ERR_INVALID, "unknown flags");
    int ndev = 0;
    CU(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(CCS_ERR_INVALID, "bad device ordinal");
    CU(cudaSetDevice(device));
    ccs_qiter* Q = new ccs_qiter();
    Q->device = device;
    Q->n_variants = p->n_variants;
    Q->exp_start = p->exp_start;
    Q->depth = p->depth;
    Q->target = p->target;
    Q->primes.assign(p->primes, p->primes + p->n_primes);
    Q->dv.assign(p->dv, p->dv + 4 * (size_t)p->n_variants);
    // windows: per variant the active primes (q not dividing D_V) with their
    // forbidden residues, ordered by the share of Q they kill (the survivor
    // set does not depend on the order; words die after fewer tests), then
    // runs of consecutive primes whose product stays within kQGroupMax
    // merged into one window of that period: one lookup tests the run
    Q->fcount.assign((size_t)Q->n_variants * p->n_primes, 0);
    struct Pr { uint32_t q; double surv; std::vector<uint32_t> res; };
    std::vector<Pr> ps;
    std::vector<char> seen;
    for (uint32_t v = 0; v < Q->n_variants; v++) {
        const unsigned __int128 D = dv_of(Q, v);
        if (D == 0) { delete Q; return fail(CCS_ERR_INVALID, "D_V must be >= 1"); }
        ps.clear();
        for (uint32_t i = 0; i < p->n_primes; i++) {
            const uint32_t q = Q->primes[i];
            const uint32_t d = (uint32_t)(D % q);
            if (d == 0) continue;                                    // q | D_V: immune (v16:1247)
            Pr e{q, 0.0, {}};
            seen.assign(q, 0);
            for (uint32_t j = 0; j < p->depth; j++) {
                const uint32_t m = (uint32_t)((uint64_t)d * pow2_mod(p->exp_start + j, q) % q);
                const uint32_t r = inv_mod(m, q);                    // v16:1256-1258
                if (!seen[r]) { seen[r] = 1; e.res.push_back(r); }
            }
            Q->fcount[(size_t)v * p->n_primes + i] = (uint32_t)e.res.size();
            e.surv = (double)(q - e.res.size()) / q;
            ps.push_back(std::move(e));
        }
        std::stable_sort(ps.begin(), ps.end(), [](const Pr& a, const Pr& b) { return a.surv < b.surv; });
        const uint32_t act0 = (uint32_t)Q->act.size();
        const uint32_t pat0 = (uint32_t)Q->pat.size();
        for (size_t k = 0; k < ps.size();) {
            uint64_t P = ps[k].q;
            size_t e = k + 1;
            while (e < ps.size() && P * ps[e].q <= kQGroupMax) P *= ps[e++].q;
            const uint32_t off = (uint32_t)Q->pat.size() - pat0;
            const uint32_t nw = q_words((uint32_t)P);
            Q->pat.resize(Q->pat.size() + nw, 0u);
            uint32_t* w = Q->pat.data() + pat0 + off;
            for (size_t t = k; t < e; t++)
                for (uint32_t r : ps[t].res)
                    for (uint32_t b = r; b < 32 * nw; b += ps[t].q) w[b >> 5] |= 1u << (b & 31);
            Q->act.push_back(make_uint4((uint32_t)P, (uint32_t)(0xFFFFFFFFull / P), off, 0u));
            k = e;
        }
        const uint32_t n_act = (uint32_t)Q->act.size() - act0;
        const uint32_t words = (uint32_t)Q->pat.size() - pat0;
        if (words > kQSlabMax) { delete Q; return fail(CCS_ERR_INVALID, "sieve primes too large for one slab"); }
        Q->vhdr.push_back(make_uint4(act0, n_act, pat0, words));
        Q->act_max = std::max(Q->act_max, n_act);
        Q->slab_max = std::max(Q->slab_max, words);
    }
    Q->act_max = std::max<uint32_t>(Q->act_max, 1);
    Q->smem = (size_t)Q->act_max * 16 + (size_t)std::max<uint32_t>(Q->slab_max, 1) * 4;
    ccs_status s = engine_create_prover(device, p->primality, p->prove_mode,
                                        (p->flags & CCS_FLAG_REVERSE_PROVE) != 0, p->target, &Q->pe);
    if (s != CCS_OK) { delete Q; return s; }
    auto up = [&](auto& buf, const auto& vec) -> bool {
        if (buf.alloc(std::max<size_t>(vec.size(), 1)) != cudaSuccess) return false;
        return vec.empty() || cudaMemcpy(buf.p, vec.data(), sizeof(vec[0]) * vec.size(),
                                         cudaMemcpyHostToDevice) == cudaSuccess;
    };
    if (!up(Q->d_vhdr, Q->vhdr) || !up(Q->d_act, Q->act) || !up(Q->d_pat, Q->pat) ||
        !up(Q->d_dv, Q->dv) ||
        Q->d_count.alloc(2) != cudaSuccess || cudaMallocHost(&Q->h_count, 8) != cudaSuccess) {
        ccs_qiter_destroy(Q);
        return fail(CCS_ERR_NOMEM, "device allocation failed");
    }
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    Q->sms = prop.multiProcessorCount;
    CU(cudaStreamCreateWithFlags(&Q->fstream, cudaStreamNonBlocking));
    if (Q->smem > 48 * 1024)
        CU(cudaFuncSetAttribute(qiter_sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Q->smem));
    int bps = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, qiter_sweep_kernel, kQThreads, Q->smem));
    Q->blocks_per_sm = std::max(bps, 1);
    *out = Q;
    return CCS_OK;
}

ccs_status ccs_qiter_destroy(ccs_qiter* Q) {
    if (!Q) return CCS_OK;
    cudaSetDevice(Q->device);
    if (Q->pe) ccs_destroy(Q->pe);
    Q->d_vhdr.free_(); Q->d_act.free_(); Q->d_pat.free_();
    Q->d_dv.free_(); Q->d_count.free_();
    for (ccs_qiter::Staging* S : {&Q->fst, &Q->pst}) {
        S->d_segs.free_();
        S->d_prefix.free_();
        if (S->h_segs) cudaFreeHost(S->h_segs);
        if (S->h_prefix) cudaFreeHost(S->h_prefix);
    }
    if (Q->h_count) cudaFreeHost(Q->h_count);
    if (Q->fstream) { cudaStreamSynchronize(Q->fstream); cudaStreamDestroy(Q->fstream); }
    delete Q;
    return CCS_OK;
}

ccs_status ccs_qiter_filter(ccs_qiter* Q, const ccs_qseg* segs, uint32_t n_segs, ccs_qsurvivor* out_dev,
                            uint64_t cap, uint64_t* n_out, void* stream) {
    if (!Q || !n_out) return fail(CCS_ERR_INVALID, "null argument");
    if (cap && !out_dev) return fail(CCS_ERR_INVALID, "out_dev is null");
    {
        ccs_status s = check_segs(Q, segs, n_segs);
        if (s != CCS_OK) return s;
    }
    CU(cudaSetDevice(Q->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : Q->fstream;
    *n_out = 0;
    if (!n_segs) return CCS_OK;
    {
        ccs_status s = stage_segs(Q->fst, segs, n_segs, st);
        if (s != CCS_OK) return s;
    }
    const uint64_t units = Q->fst.h_prefix[n_segs];
    if (units >= (1ull << 31)) return fail(CCS_ERR_INVALID, "too many Q in one call (split the segments)");
    CU(cudaMemsetAsync(Q->d_count.p, 0, 8, st));
    if (units) {
        QSweepArgs a;
        a.vhdr = Q->d_vhdr.p;
        a.act = Q->d_act.p;
        a.pat = Q->d_pat.p;
        a.segs = Q->fst.d_segs.p;
        a.unit_prefix = Q->fst.d_prefix.p;
        a.n_segs = n_segs;
        a.unit_words = kQUnitWords;
        a.act_max = Q->act_max;
        a.out = (uint32_t*)out_dev;
        a.count = Q->d_count.p;
        a.cap = (uint32_t)std::min<uint64_t>(cap, 0xFFFFFFFFull);
        // one block slot per SM stays free for a prove running beside the filter
        const uint64_t per_sm = Q->blocks_per_sm > 2 ? Q->blocks_per_sm - 1 : Q->blocks_per_sm;
        const uint64_t grid = std::min<uint64_t>(units, (uint64_t)Q->sms * per_sm);
        qiter_sweep_kernel<<<(uint32_t)grid, kQThreads, Q->smem, st>>>(a);
        CU(cudaGetLastError());
    }
    CU(cudaMemcpyAsync(Q->h_count, Q->d_count.p, 4, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    *n_out = Q->h_count[0];
    if (*n_out > cap) return fail(CCS_OVERFLOW, "survivor capacity exceeded");
    return CCS_OK;
}

ccs_status ccs_qiter_prove(ccs_qiter* Q, const ccs_qseg* segs, uint32_t n_segs,
                           const ccs_qsurvivor* surv_dev, uint64_t n_surv, ccs_chain* out_dev,
                           uint64_t cap, uint64_t* n_out, uint64_t* primes_out, void* stream) {
    if (!Q || !n_out) return fail(CCS_ERR_INVALID, "null argument");
    if (n_surv && !surv_dev) return fail(CCS_ERR_INVALID, "surv_dev is null");
    if (cap && !out_dev) return fail(CCS_ERR_INVALID, "out_dev is null");
    if (n_surv >= (1ull << 32)) return fail(CCS_ERR_INVALID, "n_surv must be < 2^32");
    {
        ccs_status s = check_segs(Q, segs, n_segs);
        if (s != CCS_OK) return s;
    }
    // p_0 of every segment within [2^32, 2^160): exact multi-limb arithmetic
    // on the device, no trial-division prime equal to p_0
    for (uint32_t s = 0; s < n_segs; s++) {
        unsigned __int128 qb = 0;
        for (int w = 3; w >= 0; w--) qb = (qb << 32) | segs[s].q_base[w];
        const unsigned __int128 qe = qb + segs[s].n_q;
        const unsigned __int128 D = dv_of(Q, segs[s].variant);
        const int hi_bits = (qe < qb ? 129 : bits128(qe)) + bits128(D) + (int)Q->exp_start;
        const int lo_bits = bits128(qb) + bits128(D) + (int)Q->exp_start - 2;
        if (segs[s].n_q && (qb == 0 || hi_bits > 160 || lo_bits < 32))
            return fail(CCS_ERR_INVALID, "segment p_0 outside [2^32, 2^160)");
    }
    CU(cudaSetDevice(Q->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : engine_stream(Q->pe);
    {
        ccs_status s = stage_segs(Q->pst, segs, n_segs, st);
        if (s != CCS_OK) return s;
    }
    ProveRange pr;
    memset(&pr, 0, sizeof(pr));
    pr.target = Q->target;
    QiterProve qp;
    qp.seg = reinterpret_cast<const uint32_t*>(Q->pst.d_segs.p);
    qp.dv = Q->d_dv.p;
    qp.exp_start = Q->exp_start;
    qp.n_segs = n_segs;
    return engine_prove_staged(Q->pe, reinterpret_cast<const ccs_survivor*>(surv_dev), n_surv, pr, &qp,
                               out_dev, cap, n_out, primes_out, st);
}

ccs_status ccs_qiter_forbidden_count(const ccs_qiter* Q, uint32_t v, uint32_t* counts, uint32_t cap) {
    if (!Q || !counts) return fail(CCS_ERR_INVALID, "null argument");
    if (v >= Q->n_variants) return fail(CCS_ERR_INVALID, "variant out of range");
    const uint32_t n = (uint32_t)Q->primes.size();
    for (uint32_t i = 0; i < std::min(n, cap); i++) counts[i] = Q->fcount[(size_t)v * n + i];
    return CCS_OK;
}

}  // extern "C"
