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
            dedup_p0=True, prove_steps=2, prove_survivors=2048):
        """Filters and proves a list of steps (each a segment list) as a
        pipeline of three host threads: the caller's thread packs step i + 1
        while a filter thread runs the filter of step i on its own stream,
        and a prover thread proves the survivors of earlier steps beside it,
        as the reference overlaps its sieve launches with its CPU prove pool
        (v16:5700-5800).  Survivors are proved in groups of up to
        `prove_steps` steps (or once `prove_survivors` have collected): a
        step may hold only a few dozen survivors, whose prove costs about
        the latency of the longest walk, so a group's prove costs about one
        step's and still ends beside the next group's filters.  Returns the
        totals and the sorted HIT lines."""
        import queue
        import threading
        from . import _torch
        torch = _torch()
        dev = f"cuda:{self.device}"
        bufs = [torch.empty((surv_cap, 4), dtype=torch.int32, device=dev) for _ in range(2)]
        chains = [torch.empty((chain_cap, 12), dtype=torch.int32, device=dev)]
        # one filter stream per instance: the caching allocator keeps the
        # blocks of earlier runs on it (a new stream would allocate afresh)
        if getattr(self, "_fstream", None) is None:
            self._fstream = torch.cuda.Stream(device=dev)
        fstream = self._fstream
        packed_q = queue.Queue(maxsize=2)
        work = queue.Queue(maxsize=2)
        tot = {"steps": 0, "q": 0, "survivors": 0, "chains": 0, "primes": 0}
        lines, err = [], []
        seen = set() if dedup_p0 else None

        def prover():
            while True:
                item = work.get()
                if item is None:
                    return
                segs, surv = item
                try:
                    if not err:
                        if surv.shape[0] > chains[0].shape[0]:
                            chains[0] = torch.empty((surv.shape[0], 12), dtype=torch.int32, device=dev)
                        c, pr = self.prove(segs, surv, out=chains[0])
                        tot["chains"] += c.shape[0]
                        tot["primes"] += pr
                        lines.extend(self.hit_lines(segs, c, min_report_len, pool_primes, seen))
                except Exception as ex:                   # reported to the caller below
                    err.append(ex)

        def filterer():
            group = {"segs": [], "surv": [], "steps": 0, "n": 0}

            def flush():
                if group["segs"] and not err:
                    # the group's survivors, segment indices into the
                    # concatenated segment list, back on the device (a copy
                    # from host memory: complete when it returns)
                    surv = torch.from_numpy(np.concatenate(group["surv"])).to(dev)
                    work.put((np.concatenate(group["segs"]), surv))
                group.update(segs=[], surv=[], steps=0, n=0)

            with torch.cuda.stream(fstream):
                i = 0
                while True:
                    packed = packed_q.get()
                    if packed is None:
                        break
                    if err:
                        continue                          # drain the queue
                    try:
                        s_ = self.filter(packed, out=bufs[i % 2], stream=fstream)
                        n_seg = self._nsegs(packed)
                        tot["steps"] += 1
                        tot["q"] += int(packed[:n_seg, 4].astype(np.int64).sum())
                        tot["survivors"] += s_.shape[0]
                        # survivors are few (tens per step): offset their
                        # segment indices on the host, so the pipeline runs
                        # copies only, no kernels of its own
                        base = sum(x.shape[0] for x in group["segs"])
                        s2 = s_.cpu().numpy()
                        if base:
                            s2[:, 1] += base
                        group["segs"].append(packed[:n_seg])
                        group["surv"].append(s2)
                        group["steps"] += 1
                        group["n"] += s_.shape[0]
                        i += 1
                        if group["steps"] >= prove_steps or group["n"] >= prove_survivors:
                            flush()
                    except Exception as ex:               # reported to the caller below
                        err.append(ex)
                try:
                    flush()
                except Exception as ex:
                    err.append(ex)
            work.put(None)

        th_p = threading.Thread(target=prover, daemon=True)
        th_f = threading.Thread(target=filterer, daemon=True)
        th_p.start()
        th_f.start()
        try:
            for segs in plan:
                if err:
                    break
                packed_q.put(self.pack(segs))
        finally:
            packed_q.put(None)
            th_f.join()
            th_p.join()
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


# ---------------------------------------------------------------------------
# campaign: Q walkers, checkpoint/resume, HIT log
# ---------------------------------------------------------------------------
QITER_CHECKPOINT_VERSION = "v16.0.3-drained-cursor"
_FNV_OFFSET, _FNV_PRIME, _M64 = 0xCBF29CE484222325, 0x100000001B3, (1 << 64) - 1


def fnv1a64(data):
    h = _FNV_OFFSET
    for b in data:
        h = ((h ^ b) * _FNV_PRIME) & _M64
    return h


def sieve_hash(primes):
    """FNV-1a 64 over the sieve list as little-endian u32 (v16:4080-4083)."""
    return fnv1a64(b"".join(int(q).to_bytes(4, "little") for q in primes))


def pool_hash(dv):
    """FNV-1a 64 over "D_dec," for every variant (v16:4087-4097)."""
    return fnv1a64(b"".join(str(int(d)).encode() + b"," for d in dv))


class QCampaign:
    """A q-iteration campaign: per-variant Q walkers over a bit band, the
    reference's round-robin variant choice, sequential cursors or random
    starts (--q-order), per-variant choice by window width
    (--q-band-mode exhaustive, --exhaustive-max-q-bits), its checkpoint file
    (v16:4108-4400: identity keys, FNV-1a hashes of the sieve list and the
    pool, sparse drained cursors) and its HIT log.

    The sieve list hashed is the reference's GPU list (primes 7..sieve_max
    outside the immune set); the engine may sieve more (509..1009), which
    the reference does on its CPU."""

    def __init__(self, qiter, bits_min=90, bits_max=127, q_order="random", q_band_mode="fixed",
                 exhaustive_max_q_bits=40, q_chunk=1 << 24, seed=1, immune=(2, 3, 5), sieve_max=503,
                 chunks_per_step=256, min_report_len=8, dedup_p0=True, checkpoint_path=None, resume=False,
                 out_path=None):
        if q_order not in ("random", "sequential") or q_band_mode not in ("fixed", "exhaustive"):
            raise ValueError("q_order: random | sequential; q_band_mode: fixed | exhaustive")
        self.qi = qiter
        self.bits_min, self.bits_max = bits_min, bits_max
        self.q_order, self.q_band_mode = q_order, q_band_mode
        self.xbits = exhaustive_max_q_bits
        self.q_chunk, self.seed = int(q_chunk), seed
        self.immune = tuple(immune)
        self.D = 1
        for q in self.immune:
            self.D *= q
        self.sieve_max = sieve_max
        self.gpu_list = qiter_sieve_primes(self.immune, sieve_max, ext=False)
        self.chunks_per_step = chunks_per_step
        self.min_report_len = min_report_len
        self.seen = set() if dedup_p0 else None
        self.ck_path, self.out_path = checkpoint_path, out_path
        from .campaign import XorShift64
        self.rng = XorShift64(seed)
        self.win = qiter.windows(bits_min, bits_max)
        n = len(self.win)
        self.exhausted = [a > b for a, b in self.win]
        self.cursor = [a for a, _ in self.win]
        self.random = []
        for a, b in self.win:
            if q_band_mode == "exhaustive":
                self.random.append(a <= b and (b - a + 1).bit_length() > self.xbits)
            else:
                self.random.append(q_order == "random")
        self.cur_v = 0
        self.totals = {"steps": 0, "q": 0, "survivors": 0, "chains": 0, "primes": 0}
        self.lines = []
        if resume and checkpoint_path:
            import os
            if os.path.exists(checkpoint_path):
                self.load(checkpoint_path)
        assert len(self.cursor) == n

    # -- walkers (v16:5647-5700) -------------------------------------------
    def _next_chunk(self):
        n = len(self.win)
        for step in range(n):
            v = (self.cur_v + step) % n
            if self.exhausted[v]:
                continue
            qmn, qmx = self.win[v]
            if self.random[v]:
                span = qmx - qmn + 1
                this = min(self.q_chunk, span)
                r = ((self.rng.next() << 64) | self.rng.next()) % (span - this + 1)
                qb = qmn + r
            else:
                cur = self.cursor[v]
                if cur > qmx:
                    self.exhausted[v] = True
                    continue
                this = min(self.q_chunk, qmx - cur + 1)
                qb = cur
                self.cursor[v] = cur + this
            self.cur_v = (v + 1) % n
            return (qb, this, v)
        return None

    def next_step(self):
        segs = []
        while len(segs) < self.chunks_per_step:
            c = self._next_chunk()
            if c is None:
                break
            segs.append(c)
        return segs or None

    def run(self, max_steps=None):
        done = 0
        plan = []
        while max_steps is None or done < max_steps:
            segs = self.next_step()
            if segs is None:
                break
            plan.append(segs)
            done += 1
        if plan:
            tot, lines = self.qi.run(plan, self.min_report_len, dedup_p0=False)
            for k in tot:
                self.totals[k] += tot[k]
            if self.seen is not None:
                kept = []
                for ln in lines:                              # dedup across steps and runs
                    p0 = int(ln.rsplit("p_0=0x", 1)[1], 16)
                    if p0 in self.seen:
                        A = ln.split(" A=", 1)[1].split(" ", 1)[0]
                        L = ln.split(" len=", 1)[1].split(" ", 1)[0]
                        ln = f"HIT-DUP seed={self.qi.seed_name} len={L} A={A} p_0=0x{p0:x}"
                    else:
                        self.seen.add(p0)
                    kept.append(ln)
                lines = kept
            self.lines.extend(lines)
            if self.out_path and lines:
                with open(self.out_path, "a") as f:
                    f.write("".join(ln + "\n" for ln in lines))
        if self.ck_path:
            self.save(self.ck_path)
        return dict(self.totals)

    # -- checkpoint (v16:4108-4218, 4242-4390) --------------------------------
    def _identity(self):
        return {"version": QITER_CHECKPOINT_VERSION, "mode": "q-iter", "target_len": str(self.qi.target),
                "sieve_depth": str(self.qi.depth), "bits_min": str(self.bits_min),
                "bits_max": str(self.bits_max), "seed_name": self.qi.seed_name, "D_dec": str(self.D),
                "exp_start": str(self.qi.exp_start), "sieve_prime_max": str(self.sieve_max),
                "sieve_fnv1a64": f"0x{sieve_hash(self.gpu_list):016x}",
                "pool_seeds_count": str(len(self.qi.dv)),
                "pool_seeds_fnv1a64": f"0x{pool_hash(self.qi.dv):016x}", "q_order": self.q_order,
                "q_band_mode": self.q_band_mode}

    def save(self, path):
        import os
        idn = self._identity()
        out = [f"version={idn['version']}", "mode=q-iter", f"target_len={idn['target_len']}",
               f"sieve_depth={idn['sieve_depth']}", "target_bits=0", f"bits_min={self.bits_min}",
               f"bits_max={self.bits_max}", f"seed_name={self.qi.seed_name}", f"D_dec={self.D}",
               "D_primes=" + ",".join(str(q) for q in self.immune), f"exp_start={self.qi.exp_start}",
               f"sieve_prime_max={self.sieve_max}",
               "sieve_primes=" + ",".join(str(q) for q in self.gpu_list if q > 53),
               f"sieve_fnv1a64={idn['sieve_fnv1a64']}", f"pool_seeds_count={idn['pool_seeds_count']}",
               f"pool_seeds_fnv1a64={idn['pool_seeds_fnv1a64']}", f"q_order={self.q_order}"]
        if self.q_order == "random":
            out.append(f"q_seed={self.seed}")
        out.append(f"q_chunk={self.q_chunk}")
        out.append(f"q_band_mode={self.q_band_mode}")
        if self.q_band_mode == "exhaustive":
            out.append(f"exhaustive_max_q_bits={self.xbits}")
        for v, (cur, (qmn, _)) in enumerate(zip(self.cursor, self.win)):
            if cur > qmn:
                out.append(f"v_cursor_drained[{v}]={cur}")
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            f.write("\n".join(out) + "\n")
        os.replace(tmp, path)

    def load(self, path):
        kv, cursors = {}, {}
        with open(path) as f:
            for ln in f:
                if "=" not in ln:
                    continue
                k, val = ln.rstrip("\n").split("=", 1)
                if k.startswith("v_cursor_drained["):
                    cursors[int(k[17:].split("]", 1)[0])] = int(val)
                else:
                    kv[k] = val
        if kv.get("mode") != "q-iter":
            raise ValueError("checkpoint is not a q-iter checkpoint")
        idn = self._identity()
        for k in ("version", "seed_name", "D_dec", "target_len", "sieve_depth", "exp_start", "bits_min",
                  "bits_max", "sieve_prime_max", "pool_seeds_count", "q_order"):
            if kv.get(k) != idn[k]:
                raise ValueError(f"checkpoint {k}={kv.get(k)} does not match current {idn[k]}")
        for k in ("sieve_fnv1a64", "pool_seeds_fnv1a64"):
            if int(kv.get(k, "0"), 0) != int(idn[k], 0):
                raise ValueError(f"checkpoint {k} does not match")
        if kv.get("q_band_mode", self.q_band_mode) != self.q_band_mode:
            raise ValueError("checkpoint q_band_mode does not match")
        if self.q_band_mode == "exhaustive" and int(kv.get("exhaustive_max_q_bits", self.xbits)) != self.xbits:
            raise ValueError("checkpoint exhaustive_max_q_bits does not match")
        for v, cur in cursors.items():
            if 0 <= v < len(self.cursor):
                self.cursor[v] = cur
                if cur > self.win[v][1]:
                    self.exhausted[v] = True
