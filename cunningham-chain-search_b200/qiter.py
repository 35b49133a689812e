"""Fingerprint-pool Q iteration: the host side of the reference's v16 engine
(src/cuda/experimental/cc20_first_kind_immune_v16.cu) over the ccs_qiter_*
C ABI.

Candidates are p_0 = Q * D_V * 2^E - 1 for every variant V of a pool of
fingerprints D_V (v16 DESIGN section 2).  This module reads pool files in the
reference's format, builds the reference's sieve prime lists, computes the
per-variant Q windows of a bit band, draws Q chunks (sequential cursors or
seeded random starts) and formats the reference's HIT lines; filtering and
proving run on the GPU.

Kept alike on purpose, so pools, bands and logs move between the engines:
  * pool lines "q1[^e1]*q2[^e2]*...  # comment" (v16:556-664, 709-748);
  * the sieve list: odd primes up to --sieve-max not dividing the immune
    product, then the extended primes 509..1009 (v16:1408-1451, 174-187);
  * Q windows [ceil(2^(N1-1) / (D_V 2^E)), floor((2^N2 - 1) / (D_V 2^E))]
    (v16:4405-4468);
  * "HIT seed=<name> len=<L> [fp={..}][ pool=[..]] A=<Q> p_0=0x<hex>" lines
    (v16:2838-2848).
"""
import ctypes as C
import re

import numpy as np

V16_SMALL_PRIMES = tuple(q for q in range(2, 504) if all(q % d for d in range(2, int(q ** 0.5) + 1)))
V16_EXT_PRIMES = tuple(q for q in range(509, 1010) if all(q % d for d in range(2, int(q ** 0.5) + 1)))

_TERM = re.compile(r"^(\d+)(?:\^(\d+))?$")


def _is_prime(q):
    return q >= 2 and all(q % d for d in range(2, int(q ** 0.5) + 1))


def parse_pool_spec(spec):
    """One pool entry (name, D, {q: e}) from "q1[^e1]*q2[^e2]*..." or the
    primorial form "Z#[/omit]..." (v16:556-654)."""
    spec = spec.strip()
    fac = {}
    if "#" in spec:
        z, _, rest = spec.partition("#")
        Z = int(z)
        if not 2 <= Z <= 500:
            raise ValueError(f"bad primorial {spec!r}")
        ps = [q for q in V16_SMALL_PRIMES if q <= Z]
        for o in filter(None, rest.replace(" ", "").split("/")):
            if int(o) not in ps:
                raise ValueError(f"prime {o} not in {Z}# ({spec!r})")
            ps.remove(int(o))
        fac = {q: 1 for q in ps}
    else:
        for term in filter(None, spec.split("*")):
            m = _TERM.match(term.strip())
            if not m:
                raise ValueError(f"bad pool term {term!r} in {spec!r}")
            q, e = int(m.group(1)), int(m.group(2) or 1)
            if not _is_prime(q) or not 1 <= e <= 16:
                raise ValueError(f"bad pool term {term!r} in {spec!r}")
            fac[q] = fac.get(q, 0) + e
    D = 1
    for q, e in fac.items():
        D *= q ** e
    if D >= 1 << 128:
        raise ValueError(f"D_V of {spec!r} exceeds 128 bits")
    return spec, D, fac


def parse_pool(lines):
    """Pool entries from pool-file lines: everything from '#' on is a
    comment, blank lines are skipped (v16:709-748)."""
    out = []
    for raw in lines:
        line = raw.split("#", 1)[0].strip()
        if line:
            out.append(parse_pool_spec(line))
    return out


def parse_pool_specs(text):
    """Pool entries from a comma-separated --seed-pool list (primorial
    forms allowed)."""
    return [parse_pool_spec(s) for s in text.split(",") if s.strip()]


def pool_from_text(text):
    return parse_pool(text.splitlines())


def qiter_sieve_primes(immune=(2, 3, 5), sieve_max=503, ext=True):
    """The reference's q-iter sieve list: primes <= sieve_max not in the
    immune set, ascending, plus the extended primes 509..1009 its prove
    workers apply before any primality test (on by default)."""
    base = [q for q in V16_SMALL_PRIMES if q <= sieve_max and q not in immune and q > 2]
    return base + (list(V16_EXT_PRIMES) if ext else [])


def q_window(D, E, bits_min, bits_max):
    """(Q_min, Q_max) with p_0 = Q * D * 2^E - 1 of bits_min .. bits_max bits;
    Q_min > Q_max when the band holds no Q for this D."""
    DE = D << E
    lo = 1 << (bits_min - 1)
    qmin = -(-lo // DE)
    qmax = ((1 << bits_max) - 1) // DE
    return qmin, qmax


def synthetic_pool(n=4248, seed=1, bits_lo=12.0, bits_hi=37.0):
    """n distinct seeded fingerprints shaped like the reference's empirical
    pools: the floor 2*3*5 times a random subset of the palette primes
    7..61, small exponents on 2, 3 and 5, D_V between 2^bits_lo and
    2^bits_hi.  A stand-in for pool files, which are data, not code."""
    import math
    import random
    r = random.Random(seed)
    palette = [7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61]
    seen, out = set(), []
    while len(out) < n:
        fac = {2: r.choice([1, 1, 1, 2, 3]), 3: r.choice([1, 1, 2, 3]), 5: r.choice([1, 1, 1, 2])}
        for q in palette:
            if r.random() < 0.3:
                fac[q] = 2 if r.random() < 0.05 else 1
        D = 1
        for q, e in fac.items():
            D *= q ** e
        if not bits_lo <= math.log2(D) <= bits_hi or D in seen:
            continue
        seen.add(D)
        spec = "*".join(f"{q}^{e}" if e > 1 else str(q) for q, e in sorted(fac.items()))
        out.append((spec, D, fac))
    return out


def format_hit_line(seed_name, chain_len, Q, p0, fp=None, pool=None):
    s = f"HIT seed={seed_name} len={chain_len} "
    if fp is not None:
        s += "fp={" + ",".join(str(q) for q in fp) + "}"
    if pool is not None:
        s += " pool=[" + ",".join(pool) + "]"
    return s + f" A={Q} p_0=0x{p0:x}"


class QIter:
    """Q iteration over one pool on one GPU.

    pool: parsed entries (parse_pool) or plain ints D_V.  depth defaults to
    target (the production runs pass --depth = --target)."""

    def __init__(self, pool, target=18, depth=None, exp_start=0, primes=None, reverse=True,
                 primality=None, prove_mode=None, device=0, seed_name="unnamed"):
        from . import (PRIME_BPSW, PROVE_ROOTS, FLAG_REVERSE_PROVE, _QIterParams, _check,
                       load_library)
        entries = [(str(p), int(p), None) if isinstance(p, int) else p for p in pool]
        self.names = [e[0] for e in entries]
        self.dv = [int(e[1]) for e in entries]
        self.target = target
        self.depth = depth or target
        self.exp_start = exp_start
        self.primes = list(primes) if primes is not None else qiter_sieve_primes()
        self.seed_name = seed_name
        self.device = device
        lib = load_library()
        dv = np.zeros((len(self.dv), 4), dtype=np.uint32)
        for i, d in enumerate(self.dv):
            for w in range(4):
                dv[i, w] = (d >> (32 * w)) & 0xFFFFFFFF
        self._dv_arr = dv
        pr = (C.c_uint32 * len(self.primes))(*self.primes)
        p = _QIterParams()
        p.n_variants = len(self.dv)
        p.dv = dv.ctypes.data_as(C.POINTER(C.c_uint32))
        p.exp_start = exp_start
        p.depth = self.depth
        p.target = target
        p.n_primes = len(self.primes)
        p.primes = pr
        p.primality = PRIME_BPSW if primality is None else primality
        p.prove_mode = PROVE_ROOTS if prove_mode is None else prove_mode
        p.flags = FLAG_REVERSE_PROVE if reverse else 0
        h = C.c_void_p()
        _check(lib.ccs_qiter_create(C.byref(p), device, C.byref(h)), "ccs_qiter_create")
        self.h = h

    def close(self):
        from . import load_library
        if getattr(self, "h", None):
            load_library().ccs_qiter_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- segments
    @staticmethod
    def pack(segs):
        """Segments [(q_base, n_q, variant)] as the C ABI's ccs_qseg array
        (a [n, 6] uint32 array); filter and prove take either form."""
        if isinstance(segs, np.ndarray):
            return segs
        arr = np.zeros((max(len(segs), 1), 6), dtype=np.uint32)
        for i, (qb, n_q, v) in enumerate(segs):
            qb = int(qb)
            if qb < 0 or qb >= 1 << 128 or not 0 <= int(n_q) < 1 << 32:
                raise ValueError("segment out of range")
            arr[i] = (qb & 0xFFFFFFFF, (qb >> 32) & 0xFFFFFFFF, (qb >> 64) & 0xFFFFFFFF, qb >> 96,
                      int(n_q), int(v))
        return arr

    @staticmethod
    def _segs(segs):
        from . import _QSeg
        arr = QIter.pack(segs)
        return arr, arr.ctypes.data_as(C.POINTER(_QSeg))

    @staticmethod
    def _nsegs(segs):
        return segs.shape[0] if isinstance(segs, np.ndarray) else len(segs)

    def windows(self, bits_min, bits_max):
        return [q_window(d, self.exp_start, bits_min, bits_max) for d in self.dv]

    def random_segments(self, n, chunk, bits_min, bits_max, seed=1, start_variant=0):
        """n chunks, round-robin over the variants with a non-empty window,
        each from a random start (the reference's --q-order random,
        v16:5667-5680, without the clock mixing so a seed reproduces)."""
        from .campaign import XorShift64
        rng = XorShift64(seed)                 # the reference's rng_next (v16:333-342)
        wins = self.windows(bits_min, bits_max)
        live = [v for v, (a, b) in enumerate(wins) if a <= b]
        if not live:
            raise ValueError("no variant has a Q window in this band")
        out = []
        k = start_variant % len(live)
        for _ in range(n):
            v = live[k]
            k = (k + 1) % len(live)
            qmn, qmx = wins[v]
            span = qmx - qmn + 1
            this = min(chunk, span)
            r = ((rng.next() << 64) | rng.next()) % (span - this + 1)
            out.append((qmn + r, this, v))
        return out

    # ---------------------------------------------------------------- device
    def filter(self, segs, cap=1 << 22, out=None, stream=None):
        """Survivors [n, 4] int32 (offset, seg, variant, 0) on the device."""
        from . import OVERFLOW, CCSError, _check, _torch, _u64, load_library
        torch = _torch()
        if out is None:
            out = torch.empty((cap, 4), dtype=torch.int32, device=f"cuda:{self.device}")
        cap = out.shape[0]
        keep, arr = self._segs(segs)
        n = _u64(0)
        st = load_library().ccs_qiter_filter(self.h, arr, self._nsegs(segs), out.data_ptr(), cap, C.byref(n),
                                             stream.cuda_stream if stream is not None else None)
        if st == OVERFLOW:
            raise CCSError(st, f"{n.value} survivors > cap {cap}")
        _check(st, "ccs_qiter_filter")
        return out[: n.value]

    def prove(self, segs, survivors, cap=1 << 16, out=None, stream=None):
        """Chain records [n, 12] int32 (offset, seg, variant, len, p_0 limbs,
        flags, survivor index) and the count of survivors whose p_0 tested
        prime."""
        from . import OVERFLOW, CCSError, _check, _torch, _u64, load_library
        torch = _torch()
        if out is None:
            out = torch.empty((cap, 12), dtype=torch.int32, device=f"cuda:{self.device}")
        cap = out.shape[0]
        keep, arr = self._segs(segs)
        sv = survivors.contiguous()
        n = _u64(0)
        pr = _u64(0)
        st = load_library().ccs_qiter_prove(self.h, arr, self._nsegs(segs), sv.data_ptr() if sv.numel() else None,
                                            sv.shape[0], out.data_ptr(), cap, C.byref(n), C.byref(pr),
                                            stream.cuda_stream if stream is not None else None)
        if st == OVERFLOW:
            raise CCSError(st, f"{n.value} chains > cap {cap}")
        _check(st, "ccs_qiter_prove")
        return out[: n.value], pr.value

    def run(self, plan, min_report_len=8, surv_cap=1 << 22, chain_cap=1 << 16, pool_primes=None,
            dedup_p0=True):
        """Filters and proves a list of steps (each a segment list), the
        prove of step i overlapping the filter of step i + 1 (two host
        threads, two streams, two survivor buffers), as the reference
        overlaps its sieve launches with its CPU prove pool (v16:5700-5800).
        Returns the totals and the sorted HIT lines."""
        import queue
        import threading
        from . import _torch
        torch = _torch()
        dev = f"cuda:{self.device}"
        bufs = [torch.empty((surv_cap, 4), dtype=torch.int32, device=dev) for _ in range(2)]
        chains = torch.empty((chain_cap, 12), dtype=torch.int32, device=dev)
        free = [threading.Semaphore(1), threading.Semaphore(1)]
        work = queue.Queue(maxsize=1)
        tot = {"steps": 0, "q": 0, "survivors": 0, "chains": 0, "primes": 0}
        lines, err = [], []
        seen = set() if dedup_p0 else None

        def prover():
            while True:
                item = work.get()
                if item is None:
                    return
                i, segs, surv = item
                try:
                    if not err:
                        c, pr = self.prove(segs, surv, out=chains)
                        tot["chains"] += c.shape[0]
                        tot["primes"] += pr
                        lines.extend(self.hit_lines(segs, c, min_report_len, pool_primes, seen))
                except Exception as ex:                   # reported to the caller below
                    err.append(ex)
                finally:
                    free[i % 2].release()

        th = threading.Thread(target=prover, daemon=True)
        th.start()
        try:
            for i, segs in enumerate(plan):
                packed = self.pack(segs)
                free[i % 2].acquire()
                if err:
                    free[i % 2].release()
                    break
                s_ = self.filter(packed, out=bufs[i % 2])
                tot["steps"] += 1
                tot["q"] += int(packed[: self._nsegs(segs), 4].astype(np.int64).sum())
                tot["survivors"] += s_.shape[0]
                work.put((i, packed, s_))
        finally:
            work.put(None)
            th.join()
        if err:
            raise err[0]
        return tot, sorted(lines)

    def forbidden_counts(self, variant):
        from . import _check, load_library
        arr = (C.c_uint32 * len(self.primes))()
        _check(load_library().ccs_qiter_forbidden_count(self.h, variant, arr, len(self.primes)),
               "ccs_qiter_forbidden_count")
        return list(arr)

    # ---------------------------------------------------------------- output
    def hit_lines(self, segs, chains, min_report_len=8, pool_primes=None, seen=None):
        """The reference's HIT lines for records of at least min_report_len,
        sorted; fp lists the pool primes dividing p_0 + 1 and pool the
        variants whose D_V divides it (v16:2775-2848).  With a set `seen`
        (its --dedup-p0, v16:2826-2848), a p_0 already in it gives the short
        "HIT-DUP seed=.. len=.. A=.. p_0=0x.." line instead, and new p_0 are
        added."""
        recs = np.asarray(chains.cpu().numpy() if hasattr(chains, "cpu") else chains).astype(np.int64) & 0xFFFFFFFF
        lines = []
        for r in recs:
            L = int(r[3])
            if L < min_report_len:
                continue
            sg = segs[int(r[1])]
            qb = sum(int(sg[w]) << (32 * w) for w in range(4)) if isinstance(segs, np.ndarray) else int(sg[0])
            Q = qb + int(r[0])
            p0 = sum(int(x) << (32 * i) for i, x in enumerate(r[4:10]))
            if seen is not None and p0 in seen:
                lines.append(f"HIT-DUP seed={self.seed_name} len={L} A={Q} p_0=0x{p0:x}")
                continue
            if seen is not None:
                seen.add(p0)
            fp = [q for q in pool_primes if (p0 + 1) % q == 0] if pool_primes else None
            pool = [self.names[i] for i, d in enumerate(self.dv) if (p0 + 1) % d == 0]
            lines.append(format_hit_line(self.seed_name, L, Q, p0, fp, pool))
        return sorted(lines)
