"""B200 Cunningham-chain search engine: Python host side over the C ABI.

The compute path is libccs.so (hand-written sm_100a CUDA behind include/ccs.h);
this module only marshals arguments.  There is no CPU fallback: every compute
call raises when the shared library or a GPU is missing.

Names follow the reference (nmicic/cunningham-chain-search) where a
counterpart exists: compute_forbidden_residues (v13:771), Engine.bases
(generate_bases, v13:907), Engine.filter_range (one K1 batch, v13:1551 /
3764-3795), Engine.prove (K2 / prove_survivors_mt, v13:1462 / 1967),
format_chain_line (v13:2030-2033).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libccs.so")

# status codes (include/ccs.h)
OK, ERR_INVALID, ERR_CUDA, OVERFLOW, ERR_NOMEM, ERR_TIMEOUT, ERR_BUSY, ERR_NOT_FOUND, \
    ERR_CANCELLED, PENDING = range(10)
STATUS_NAMES = ["OK", "ERR_INVALID", "ERR_CUDA", "OVERFLOW", "ERR_NOMEM", "ERR_TIMEOUT",
                "ERR_BUSY", "ERR_NOT_FOUND", "ERR_CANCELLED", "PENDING"]

PRIME_MR, PRIME_BPSW, PRIME_V33 = 0, 1, 2
PROVE_ROOTS, PROVE_FULL = 0, 1
CHAIN_IS_ROOT, CHAIN_TARGET = 1, 2

# reference parameter set (src/cuda/cc18_filter_cuda_CpC_v13.cu:174-201)
REF_CRT = (5, 7, 11, 13, 17, 19)
REF_WHEEL = (23, 29, 31)
REF_L2 = (37, 41, 43, 47, 53, 59, 61)
REF_EXT = (67, 71, 73, 79, 83, 89, 97)
V13_WITNESSES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71)


def primes_in(lo, hi):
    """primes p with lo <= p < hi"""
    if hi <= 2:
        return []
    s = np.ones(hi, dtype=bool)
    s[:2] = False
    for p in range(2, int(hi ** 0.5) + 1):
        if s[p]:
            s[p * p::p] = False
    return [int(p) for p in np.nonzero(s)[0] if p >= lo]


REF_LINE = tuple(primes_in(101, 864))


def reference_stages():
    """L2 37..61 and ext-L2 67..97 from position 0, line sieve 101..863 from
    position 1 (v13:793-846)."""
    return [(REF_L2, 0), (REF_EXT, 0), (REF_LINE, 1)]


def compute_forbidden_residues(q, chain_len, pos_lo=0):
    """Residues n mod q that make some chain member p_i = 2^i (n+1) - 1,
    i in [pos_lo, min(chain_len, q)), divisible by q (v13:771-787)."""
    out = set()
    inv2 = (q + 1) // 2
    x = 1
    for i in range(min(chain_len, q)):
        if i >= pos_lo:
            out.add((x - 1) % q)
        x = x * inv2 % q
    return sorted(out)


class CCSError(RuntimeError):
    def __init__(self, status, msg):
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"{name}: {msg}")
        self.status = status


# ---------------------------------------------------------------------------
# ctypes structures (mirror include/ccs.h)
# ---------------------------------------------------------------------------
class _Stage(C.Structure):
    _fields_ = [("primes", C.POINTER(C.c_uint32)), ("n_primes", C.c_uint32),
                ("pos_lo", C.c_uint32)]


class _Params(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("target", C.c_uint32), ("depth", C.c_uint32),
                ("bits", C.c_uint32),
                ("crt_primes", C.POINTER(C.c_uint32)), ("n_crt", C.c_uint32),
                ("wheel_primes", C.POINTER(C.c_uint32)), ("n_wheel", C.c_uint32),
                ("stages", C.POINTER(_Stage)), ("n_stages", C.c_uint32),
                ("max_bases", C.c_uint32),
                ("witnesses", C.POINTER(C.c_uint64)), ("n_witnesses", C.c_uint32),
                ("primality", C.c_uint32), ("prove_mode", C.c_uint32), ("flags", C.c_uint32)]


class _Info(C.Structure):
    _fields_ = [("lattice_m", C.c_uint64), ("wheel_period", C.c_uint32), ("n_bases", C.c_uint32),
                ("n_lines", C.c_uint64), ("candidates_per_tile", C.c_uint64),
                ("target", C.c_uint32), ("depth", C.c_uint32), ("bits", C.c_uint32),
                ("n_filter_primes", C.c_uint32), ("expected_tests", C.c_double),
                ("pass_rate", C.c_double), ("launches", C.c_uint64)]


class _Range(C.Structure):
    _fields_ = [("tile_start_lo", C.c_uint64), ("tile_start_hi", C.c_uint64),
                ("n_tiles", C.c_uint64), ("profile", C.c_uint32), ("bits", C.c_uint32)]


class _RangeResult(C.Structure):
    _fields_ = [("n_survivors", C.c_uint64), ("n_chains", C.c_uint64), ("n_primes", C.c_uint64),
                ("candidates", C.c_uint64), ("surv_offset", C.c_uint64),
                ("chain_offset", C.c_uint64), ("status", C.c_uint32), ("_pad", C.c_uint32)]


class _ServerConfig(C.Structure):
    _fields_ = [("max_active", C.c_uint32), ("chunk_tiles", C.c_uint32), ("mem_cap_bytes", C.c_uint64),
                ("max_pending", C.c_uint32), ("_pad", C.c_uint32)]


class _RequestResult(C.Structure):
    _fields_ = [("n_survivors", C.c_uint64), ("n_chains", C.c_uint64), ("n_primes", C.c_uint64),
                ("candidates", C.c_uint64), ("submit_s", C.c_double), ("admit_s", C.c_double),
                ("done_s", C.c_double), ("status", C.c_uint32), ("ticks", C.c_uint32)]


class _Tuning(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("unit_words", C.c_uint32), ("split_prime", C.c_uint32),
                ("ext_min_words", C.c_uint32), ("table_primes", C.c_uint32)]


class _TunePoint(C.Structure):
    _fields_ = [("tuning", _Tuning), ("n_tiles", C.c_uint64), ("ms", C.c_float), ("_pad", C.c_uint32)]


TUNE_LATTICE, TUNE_STAGES, TUNE_UNITS, TUNE_SHAPE, TUNE_ALL = 1, 2, 4, 8, 15


class _BatchTuning(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("unit_words", C.c_uint32),
                ("_pad", C.c_uint32)]


# exported symbols of include/ccs.h, with their ctypes signatures
_vp = C.c_void_p
_u64 = C.c_uint64
class _QIterParams(C.Structure):
    _fields_ = [("n_variants", C.c_uint32), ("dv", C.POINTER(C.c_uint32)), ("exp_start", C.c_uint32),
                ("depth", C.c_uint32), ("target", C.c_uint32), ("n_primes", C.c_uint32),
                ("primes", C.POINTER(C.c_uint32)), ("primality", C.c_uint32), ("prove_mode", C.c_uint32),
                ("flags", C.c_uint32)]


class _RangePlan(C.Structure):
    _fields_ = [("extended", C.c_uint32), ("q0", C.c_uint32), ("n_lines", C.c_uint64),
                ("n_words", C.c_uint32), ("unit_words", C.c_uint32), ("units", C.c_uint64),
                ("grid", C.c_uint32), ("block_threads", C.c_uint32)]


class _QSeg(C.Structure):
    _fields_ = [("q_base", C.c_uint32 * 4), ("n_q", C.c_uint32), ("variant", C.c_uint32)]


_SIGS = {
    "ccs_describe": (C.c_int, [C.POINTER(_Params), C.POINTER(_Info), C.POINTER(_u64), C.c_uint32]),
    "ccs_create": (C.c_int, [C.POINTER(_Params), C.c_int, C.POINTER(_vp)]),
    "ccs_destroy": (C.c_int, [_vp]),
    "ccs_get_info": (C.c_int, [_vp, C.POINTER(_Info)]),
    "ccs_get_bases": (C.c_int, [_vp, C.POINTER(_u64), C.c_uint32]),
    "ccs_last_error": (C.c_char_p, []),
    "ccs_abi_version": (C.c_int, []),
    "ccs_filter_range": (C.c_int, [_vp, _u64, _u64, _u64, _vp, _u64, C.POINTER(_u64), _vp]),
    "ccs_filter_range_noalloc": (C.c_int, [_vp, _u64, _u64, _u64, _vp, _u64, C.POINTER(_u64), _vp]),
    "ccs_plan_range": (C.c_int, [_vp, _u64, _u64, _u64, C.POINTER(_RangePlan)]),
    "ccs_prove_stats": (C.c_int, [_vp, C.POINTER(_u64), C.c_int]),
    "ccs_prove": (C.c_int, [_vp, _vp, _u64, _u64, _u64, _vp, _u64, C.POINTER(_u64),
                            C.POINTER(_u64), _vp]),
    "ccs_set_bits": (C.c_int, [_vp, C.c_uint32]),
    "ccs_search_range_host": (C.c_int, [_vp, _u64, _u64, _u64, _vp, _u64, C.POINTER(_u64), _vp,
                                        _u64, C.POINTER(_u64), C.POINTER(_u64)]),
    "ccs_walk_numbers": (C.c_int, [_vp, _vp, _u64, C.c_uint32, _vp, _vp]),
    "ccs_batch_create": (C.c_int, [C.POINTER(_vp), C.c_uint32, C.c_uint32, _u64, _u64,
                                   C.POINTER(_vp)]),
    "ccs_batch_destroy": (C.c_int, [_vp]),
    "ccs_batch_run": (C.c_int, [_vp, C.POINTER(_Range), C.c_uint32, C.POINTER(_RangeResult),
                                _vp, _vp, _vp]),
    "ccs_batch_last_ms": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "ccs_get_tuning": (C.c_int, [_vp, C.POINTER(_Tuning)]),
    "ccs_server_create": (C.c_int, [C.POINTER(_vp), C.c_uint32, C.POINTER(_ServerConfig), C.POINTER(_vp)]),
    "ccs_server_destroy": (C.c_int, [_vp]),
    "ccs_submit": (C.c_int, [_vp, C.POINTER(_Range), C.POINTER(_u64)]),
    "ccs_poll": (C.c_int, [_vp, _u64, C.POINTER(_RequestResult), _vp, _u64, _vp, _u64]),
    "ccs_wait": (C.c_int, [_vp, _u64, C.c_uint32]),
    "ccs_cancel": (C.c_int, [_vp, _u64]),
    "ccs_server_stats": (C.c_int, [_vp, C.POINTER(_u64)]),
    "ccs_measure_int32_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "ccs_measure_imad_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "ccs_walk_modmuls": (C.c_int, [_vp, C.POINTER(_u64), C.c_int]),
    "ccs_walk_word_products": (C.c_int, [_vp, C.POINTER(_u64), C.POINTER(_u64), C.c_int]),
    "ccs_set_tuning": (C.c_int, [_vp, C.POINTER(_Tuning)]),
    "ccs_autotune": (C.c_int, [_vp, _u64, _u64, _u64, C.c_uint32, C.POINTER(_TunePoint), C.c_uint32,
                               C.POINTER(C.c_uint32), C.POINTER(_Tuning)]),
    "ccs_batch_get_tuning": (C.c_int, [_vp, C.POINTER(_BatchTuning)]),
    "ccs_batch_launch": (C.c_int, [_vp, _vp, C.c_uint32]),
    "ccs_batch_wait": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ccs_server_memory": (C.c_int, [_vp, C.POINTER(_u64), C.POINTER(_u64)]),
    "ccs_server_set_batch_tuning": (C.c_int, [_vp, C.POINTER(_BatchTuning)]),
    "ccs_batch_set_tuning": (C.c_int, [_vp, C.POINTER(_BatchTuning)]),
    "ccs_batch_autotune": (C.c_int, [_vp, _vp, C.c_uint32, C.POINTER(_TunePoint), C.c_uint32,
                                     C.POINTER(C.c_uint32), C.POINTER(_BatchTuning)]),
    "ccs_qiter_create": (C.c_int, [C.POINTER(_QIterParams), C.c_int, C.POINTER(_vp)]),
    "ccs_qiter_destroy": (C.c_int, [_vp]),
    "ccs_qiter_filter": (C.c_int, [_vp, C.POINTER(_QSeg), C.c_uint32, _vp, _u64, C.POINTER(_u64), _vp]),
    "ccs_qiter_prove": (C.c_int, [_vp, C.POINTER(_QSeg), C.c_uint32, _vp, _u64, _vp, _u64,
                                  C.POINTER(_u64), C.POINTER(_u64), _vp]),
    "ccs_qiter_forbidden_count": (C.c_int, [_vp, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32]),
}

_LIB = None


def load_library(path=LIB_PATH):
    """Loads libccs.so; raises when it is missing (no fallback)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(path):
            raise ImportError(f"libccs.so not built at {path}; run cunningham-chain-search_b200/build.py")
        lib = C.CDLL(path)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def exported_symbols():
    return sorted(_SIGS)


def _check(status, what=""):
    if status != OK:
        msg = load_library().ccs_last_error().decode(errors="replace")
        raise CCSError(status, f"{what}: {msg}" if what else msg)


def _split128(v):
    v = int(v)
    if v < 0 or v >= 1 << 128:
        raise ValueError("value must be a u128")
    return v & (2**64 - 1), v >> 64


def _u32arr(xs):
    a = (C.c_uint32 * max(len(xs), 1))(*[int(x) for x in xs])
    return a


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("a CUDA device is required: the engine has no CPU path")
    return torch


SURVIVOR_DTYPE = np.dtype([("base_idx", "<u4"), ("k_offset", "<u4"), ("tile_idx", "<u4"),
                           ("_pad", "<u4")])
CHAIN_DTYPE = np.dtype([("base_idx", "<u4"), ("k_offset", "<u4"), ("tile_idx", "<u4"),
                        ("chain_len", "<u4"), ("root", "<u4", (6,)), ("flags", "<u4"),
                        ("survivor", "<u4")])


def chain_root_int(rec):
    return sum(int(x) << (32 * i) for i, x in enumerate(rec["root"]))


KIND_FIRST, KIND_SECOND = 1, 2


def format_chain_line(chain_len, root, target, is_root=True):
    """Reference output line "[TARGET ][NON-ROOT ]CC<len> 0x<HEX> <bits>"
    (v13:2030-2033)."""
    tag = ("TARGET " if chain_len >= target else "") + ("" if is_root else "NON-ROOT ")
    return f"{tag}CC{chain_len} 0x{root:X} {root.bit_length()}"


FLAG_REVERSE_PROVE = 1     # CCS_FLAG_REVERSE_PROVE: v15 --prove-order reverse (roots mode)


def _make_params(target=18, depth=None, bits=89, crt=REF_CRT, wheel=REF_WHEEL, stages=None,
                 max_bases=0, witnesses=V13_WITNESSES, primality=PRIME_BPSW, prove_mode=PROVE_FULL,
                 reverse_prove=False, kind=1):
    """ccs_params plus the buffers it points to (keep both alive)."""
    if stages is None:
        stages = reference_stages()
    keep = []
    crt_a = _u32arr(crt)
    wheel_a = _u32arr(wheel)
    st = (_Stage * len(stages))()
    for i, (primes, pos_lo) in enumerate(stages):
        pa = _u32arr(primes)
        keep.append(pa)
        st[i].primes = C.cast(pa, C.POINTER(C.c_uint32))
        st[i].n_primes = len(primes)
        st[i].pos_lo = pos_lo
    wit = (C.c_uint64 * max(len(witnesses), 1))(*witnesses)
    keep += [crt_a, wheel_a, st, wit]
    p = _Params()
    p.kind = kind
    p.target = target
    p.depth = depth if depth is not None else target
    p.bits = bits
    p.crt_primes = C.cast(crt_a, C.POINTER(C.c_uint32))
    p.n_crt = len(crt)
    p.wheel_primes = C.cast(wheel_a, C.POINTER(C.c_uint32))
    p.n_wheel = len(wheel)
    p.stages = C.cast(st, C.POINTER(_Stage))
    p.n_stages = len(stages)
    p.max_bases = max_bases
    p.witnesses = C.cast(wit, C.POINTER(C.c_uint64))
    p.n_witnesses = len(witnesses)
    p.primality = primality
    p.prove_mode = prove_mode
    p.flags = FLAG_REVERSE_PROVE if reverse_prove else 0
    return p, keep


def describe(**kw):
    """Host-only lattice description (ccs_describe): info dict and base list.
    Needs no GPU."""
    lib = load_library()
    p, keep = _make_params(**kw)
    inf = _Info()
    cap = 1 << 16
    bases = (C.c_uint64 * cap)()
    _check(lib.ccs_describe(C.byref(p), C.byref(inf), bases, cap), "ccs_describe")
    info = {f: getattr(inf, f) for f, _ in _Info._fields_}
    return info, [int(bases[i]) for i in range(info["n_bases"])]


def reference_cpu_stages():
    """The reference CPU engine's filter stages on its own lattice: L2 primes
    37..61 and ext-L2 primes 67..97 at positions 0..depth-1, the line sieve
    101..863 at positions 1..depth-1 (v33 with --line-depth = target - 1)."""
    return [(primes_in(37, 62), 0), (primes_in(67, 98), 0), (primes_in(101, 864), 1)]


# configurations named by the workloads they describe
def config_cc16_scale():
    """CC18-style GPU filter scale: W = 31#, depth 16, stage primes
    37..2^10 / 2^10..2^14 / 2^14..2^17 at chain positions 0..15."""
    return dict(target=16, depth=16, bits=88,
                stages=[(primes_in(37, 1 << 10), 0), (primes_in(1 << 10, 1 << 14), 0),
                        (primes_in(1 << 14, 1 << 17), 0)])


def config_cpu_method():
    """The CPU-method lattice: W = 23#, depth 8, primes 29..1021 at positions 0..7."""
    return dict(target=8, depth=8, bits=64, wheel=(23,), stages=[(primes_in(29, 1022), 0)])


class Engine:
    """One lattice + filter + prover parameter set on one GPU (ccs_create)."""

    def __init__(self, target=18, depth=None, bits=89, crt=REF_CRT, wheel=REF_WHEEL, stages=None,
                 max_bases=0, witnesses=V13_WITNESSES, primality=PRIME_BPSW,
                 prove_mode=PROVE_FULL, device=0, reverse_prove=False, kind=1):
        lib = load_library()
        if stages is None:
            stages = reference_stages()
        p, self._keep = _make_params(target, depth, bits, crt, wheel, stages, max_bases, witnesses,
                                     primality, prove_mode, reverse_prove, kind)
        h = _vp()
        _check(lib.ccs_create(C.byref(p), device, C.byref(h)), "ccs_create")
        self.h = h
        self.device = device
        self.target = target
        self.bits = bits
        self.stages = stages
        inf = _Info()
        _check(lib.ccs_get_info(self.h, C.byref(inf)))
        self.info = {f: getattr(inf, f) for f, _ in _Info._fields_}

    def close(self):
        if getattr(self, "h", None):
            load_library().ccs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- lattice facts -----------------------------------------------------
    def bases(self):
        n = self.info["n_bases"]
        a = (C.c_uint64 * n)()
        _check(load_library().ccs_get_bases(self.h, a, n))
        return [int(x) for x in a]

    def set_bits(self, bits):
        """Prover bit-width gate for subsequent prove calls (--bits)."""
        _check(load_library().ccs_set_bits(self.h, int(bits)), "ccs_set_bits")
        self.bits = int(bits)

    def launches(self):
        inf = _Info()
        _check(load_library().ccs_get_info(self.h, C.byref(inf)))
        return inf.launches

    @property
    def candidates_per_tile(self):
        return self.info["candidates_per_tile"]

    def tuning(self):
        t = _Tuning()
        _check(load_library().ccs_get_tuning(self.h, C.byref(t)))
        return {f: getattr(t, f) for f, _ in _Tuning._fields_ if not f.startswith("_")}

    def set_tuning(self, **kw):
        t = _Tuning()
        _check(load_library().ccs_get_tuning(self.h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, v)
        _check(load_library().ccs_set_tuning(self.h, C.byref(t)), "ccs_set_tuning")

    def autotune(self, tile_start, n_tiles, what=TUNE_ALL, cap=256):
        """Project autotuner: times the filter on [tile_start, tile_start +
        n_tiles) under candidate tunings (stage splits, lattice threshold,
        positions per thread, block shape), keeps the fastest on the engine
        and returns (chosen tuning dict, [(tuning dict, n_tiles, ms), ...])."""
        pts = (_TunePoint * cap)()
        n = C.c_uint32(0)
        t = _Tuning()
        lo, hi = _split128(tile_start)
        _check(load_library().ccs_autotune(self.h, lo, hi, n_tiles, what, pts, cap, C.byref(n), C.byref(t)),
               "ccs_autotune")
        as_dict = lambda x: {f: getattr(x, f) for f, _ in _Tuning._fields_}
        return as_dict(t), [(as_dict(p.tuning), p.n_tiles, p.ms) for p in pts[:min(n.value, cap)]]

    # --- device path -------------------------------------------------------
    def filter_range(self, tile_start, n_tiles, cap=1 << 20, out=None, stream=None):
        """Survivors of tiles [tile_start, tile_start + n_tiles) as an int32
        CUDA tensor [n, 4] (reference Survivor records, uint32 bit patterns).
        Raises CCSError(OVERFLOW) when more than cap survive."""
        torch = _torch()
        if out is None:
            out = torch.empty((cap, 4), dtype=torch.int32, device=f"cuda:{self.device}")
        cap = out.shape[0]
        lo, hi = _split128(tile_start)
        n = _u64(0)
        s = stream.cuda_stream if stream is not None else None
        st = load_library().ccs_filter_range(self.h, lo, hi, int(n_tiles), out.data_ptr(), cap,
                                             C.byref(n), s)
        if st == OVERFLOW:
            raise CCSError(st, f"{n.value} survivors > cap {cap}")
        _check(st, "ccs_filter_range")
        return out[: n.value]

    def plan_range(self, tile_start, n_tiles):
        """How filter_range would sweep the range with the current tuning
        (ccs_plan_range): lattice, words, work units, launch shape."""
        lo, hi = _split128(tile_start)
        p = _RangePlan()
        _check(load_library().ccs_plan_range(self.h, lo, hi, int(n_tiles), C.byref(p)), "ccs_plan_range")
        return {f: getattr(p, f) for f, _ in _RangePlan._fields_}

    def filter_range_noalloc(self, tile_start, n_tiles, out, stream=None):
        """filter_range through the entry point that allocates no device
        memory (ccs_filter_range_noalloc); out is a caller-owned int32 CUDA
        tensor [cap, 4].  For callers that may not allocate device memory
        once running (a GPU footprint fixed at start-up, allocators that do
        not grow, memory quotas); synchronous; calls that overlap on one GPU
        race on its shared working array."""
        lo, hi = _split128(tile_start)
        n = _u64(0)
        s = stream.cuda_stream if stream is not None else None
        st = load_library().ccs_filter_range_noalloc(self.h, lo, hi, int(n_tiles), out.data_ptr(),
                                                     out.shape[0], C.byref(n), s)
        if st == OVERFLOW:
            raise CCSError(st, f"{n.value} survivors > cap {out.shape[0]}")
        _check(st, "ccs_filter_range_noalloc")
        return out[: n.value]

    def prove(self, survivors, tile_start, cap=1 << 16, out=None, stream=None):
        """Chain records [n, 12] (int32) for device survivors; also returns the
        count of survivors that tested prime."""
        torch = _torch()
        if out is None:
            out = torch.empty((cap, 12), dtype=torch.int32, device=f"cuda:{self.device}")
        cap = out.shape[0]
        lo, hi = _split128(tile_start)
        n = _u64(0)
        pr = _u64(0)
        s = stream.cuda_stream if stream is not None else None
        sv = survivors.contiguous()
        st = load_library().ccs_prove(self.h, sv.data_ptr() if sv.numel() else None, sv.shape[0],
                                      lo, hi, out.data_ptr(), cap, C.byref(n), C.byref(pr), s)
        if st == OVERFLOW:
            raise CCSError(st, f"{n.value} chains > cap {cap}")
        _check(st, "ccs_prove")
        return out[: n.value], pr.value

    def walk_numbers(self, numbers, limbs=6):
        """Forward chain length of every given int (0 when not prime)."""
        torch = _torch()
        arr = np.zeros((len(numbers), limbs), dtype=np.uint32)
        for i, v in enumerate(numbers):
            v = int(v)
            if v.bit_length() > 32 * limbs:
                raise ValueError("number wider than limbs")
            for w in range(limbs):
                arr[i, w] = (v >> (32 * w)) & 0xFFFFFFFF
        dev = torch.from_numpy(arr.view(np.int32)).to(f"cuda:{self.device}")
        out = torch.zeros(len(numbers), dtype=torch.int32, device=dev.device)
        _check(load_library().ccs_walk_numbers(self.h, dev.data_ptr(), len(numbers), limbs,
                                               out.data_ptr(), None), "ccs_walk_numbers")
        return out.cpu().numpy().astype(np.int64)

    def prove_stats(self, reset=True):
        """Staged-prove counters (ccs_prove_stats): survivors, primes n,
        predecessor tests, roots decided by a birth certificate."""
        out = (_u64 * 4)()
        _check(load_library().ccs_prove_stats(self.h, out, int(reset)), "ccs_prove_stats")
        return dict(zip(["survivors", "primes", "predecessor_tests", "certified_roots"], [int(x) for x in out]))

    def walk_modmuls(self, reset=True):
        """Montgomery products spent by walk launches since the last reset."""
        v = _u64(0)
        _check(load_library().ccs_walk_modmuls(self.h, C.byref(v), 1 if reset else 0))
        return v.value

    def walk_word_products(self, reset=True):
        """(Montgomery products, 32x32-bit word products) spent by walk
        launches since the last reset."""
        v, w = _u64(0), _u64(0)
        _check(load_library().ccs_walk_word_products(self.h, C.byref(v), C.byref(w), 1 if reset else 0))
        return v.value, w.value

    def walk_numbers_dev(self, numbers_dev, limbs, lengths_dev):
        _check(load_library().ccs_walk_numbers(self.h, numbers_dev.data_ptr(), numbers_dev.shape[0],
                                               limbs, lengths_dev.data_ptr(), None))

    # --- host path (reference boundary: host buffers, copies included) -----
    def search_range_host(self, tile_start, n_tiles, surv_cap=1 << 20, chain_cap=1 << 16):
        """Filter + prove through host buffers.  Returns (survivors, chains,
        primes) as numpy structured arrays."""
        lo, hi = _split128(tile_start)
        surv = np.zeros(surv_cap, dtype=SURVIVOR_DTYPE)
        ch = np.zeros(chain_cap, dtype=CHAIN_DTYPE)
        ns, nc, npr = _u64(0), _u64(0), _u64(0)
        st = load_library().ccs_search_range_host(
            self.h, lo, hi, int(n_tiles), surv.ctypes.data, surv_cap, C.byref(ns),
            ch.ctypes.data, chain_cap, C.byref(nc), C.byref(npr))
        _check(st, "ccs_search_range_host")
        return surv[: ns.value], ch[: nc.value], npr.value

    def reconstruct(self, tile_start, base_idx, k_offset, tile_idx, bases=None):
        """n = ((tile_start + tile_idx) * WP + k_offset) * M + base (v13:1479-1492)."""
        bases = bases if bases is not None else self.bases()
        return ((int(tile_start) + int(tile_idx)) * self.info["wheel_period"] + int(k_offset)) \
            * self.info["lattice_m"] + bases[int(base_idx)]


class Batch:
    """Many uneven ranges in one persistent filter launch + one prove launch,
    replayed from a CUDA graph (ccs_batch_*)."""

    def __init__(self, engines, max_ranges, surv_cap=1 << 20, chain_cap=1 << 18):
        lib = load_library()
        arr = (_vp * len(engines))(*[e.h for e in engines])
        h = _vp()
        _check(lib.ccs_batch_create(arr, len(engines), max_ranges, surv_cap, chain_cap, C.byref(h)),
               "ccs_batch_create")
        self.h = h
        self.engines = engines
        self.max_ranges = max_ranges
        self.surv_cap = surv_cap
        self.chain_cap = chain_cap

    def close(self):
        if getattr(self, "h", None):
            load_library().ccs_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, ranges, want_records=True):
        """ranges: list of (tile_start, n_tiles, profile, bits).  Returns
        (results list of dicts, survivors, chains); survivor records carry the
        range index in their last word."""
        lib = load_library()
        n = len(ranges)
        rr = (_Range * max(n, 1))()
        for i, (ts, nt, prof, bits) in enumerate(ranges):
            lo, hi = _split128(ts)
            rr[i].tile_start_lo, rr[i].tile_start_hi = lo, hi
            rr[i].n_tiles = nt
            rr[i].profile = prof
            rr[i].bits = bits
        res = (_RangeResult * max(n, 1))()
        surv = np.zeros(self.surv_cap if want_records else 0, dtype=SURVIVOR_DTYPE)
        ch = np.zeros(self.chain_cap if want_records else 0, dtype=CHAIN_DTYPE)
        st = lib.ccs_batch_run(self.h, rr, n, res, surv.ctypes.data if want_records else None,
                               ch.ctypes.data if want_records else None, None)
        _check(st, "ccs_batch_run")
        out = [{f: getattr(res[i], f) for f, _ in _RangeResult._fields_} for i in range(n)]
        ns = sum(o["n_survivors"] for o in out)
        nc = sum(o["n_chains"] for o in out)
        return out, surv[:ns], ch[:nc]

    def launch(self, ranges):
        """The first half of run(): stage the ranges and replay the graph
        without waiting (ccs_batch_launch); wait() collects."""
        self._pending = len(ranges)
        _check(load_library().ccs_batch_launch(self.h, self._ranges(ranges), len(ranges)), "ccs_batch_launch")

    def wait(self, want_records=True):
        """Waits for the launch in flight (ccs_batch_wait); returns what run()
        returns."""
        n = getattr(self, "_pending", 0)
        res = (_RangeResult * max(n, 1))()
        surv = np.zeros(self.surv_cap if want_records else 0, dtype=SURVIVOR_DTYPE)
        ch = np.zeros(self.chain_cap if want_records else 0, dtype=CHAIN_DTYPE)
        st = load_library().ccs_batch_wait(self.h, res, surv.ctypes.data if want_records else None,
                                           ch.ctypes.data if want_records else None)
        _check(st, "ccs_batch_wait")
        out = [{f: getattr(res[i], f) for f, _ in _RangeResult._fields_} for i in range(n)]
        ns = sum(o["n_survivors"] for o in out)
        nc = sum(o["n_chains"] for o in out)
        return out, surv[:ns], ch[:nc]

    def last_ms(self):
        ms = C.c_float(0)
        _check(load_library().ccs_batch_last_ms(self.h, C.byref(ms)))
        return ms.value

    @staticmethod
    def _ranges(ranges):
        rr = (_Range * max(len(ranges), 1))()
        for i, (ts, nt, prof, bits) in enumerate(ranges):
            lo, hi = _split128(ts)
            rr[i].tile_start_lo, rr[i].tile_start_hi = lo, hi
            rr[i].n_tiles = nt
            rr[i].profile = prof
            rr[i].bits = bits
        return rr

    def tuning(self):
        t = _BatchTuning()
        _check(load_library().ccs_batch_get_tuning(self.h, C.byref(t)))
        return {f: getattr(t, f) for f, _ in _BatchTuning._fields_ if not f.startswith("_")}

    def set_tuning(self, **kw):
        t = _BatchTuning()
        for k, v in kw.items():
            setattr(t, k, v)
        _check(load_library().ccs_batch_set_tuning(self.h, C.byref(t)), "ccs_batch_set_tuning")

    def autotune(self, ranges, cap=64):
        """Batch autotuner over a sample of ranges: block shape and unit
        length; returns (chosen dict, [(tuning dict, ms), ...])."""
        pts = (_TunePoint * cap)()
        n = C.c_uint32(0)
        t = _BatchTuning()
        _check(load_library().ccs_batch_autotune(self.h, self._ranges(ranges), len(ranges), pts, cap,
                                                 C.byref(n), C.byref(t)), "ccs_batch_autotune")
        pick = ("block_threads", "blocks_per_sm", "unit_words")
        return ({f: getattr(t, f) for f in pick},
                [({f: getattr(p.tuning, f) for f in pick}, p.ms) for p in pts[:min(n.value, cap)]])


# ---------------------------------------------------------------------------
# range planning (v13:411-518, 3480-3573): bit range, binary prefix, lanes
# ---------------------------------------------------------------------------
def parse_prefix(s):
    """'0b1...' -> (value, bits); same validation as v13 parse_prefix (v13:411-445)."""
    if not (s.startswith("0b") or s.startswith("0B")):
        raise ValueError("--prefix must be binary format (0b...)")
    d = s[2:]
    if not d:
        raise ValueError("--prefix has no digits after 0b")
    if d[0] != "1":
        raise ValueError("binary prefix must start with 1")
    if any(ch not in "01" for ch in d):
        raise ValueError("invalid character in binary prefix")
    if len(d) > 126:
        raise ValueError("prefix too long (max 126 bits)")
    return int(d, 2), len(d)


def bit_tile_range(bits, bases, M, WP):
    """Tiles whose candidates can have `bits` bits (v13:3480-3492):
    [k_min / WP, k_max / WP + 1)."""
    n_min, n_max = 1 << (bits - 1), (1 << bits) - 1
    k_min = (n_min - max(bases)) // M
    k_max = (n_max - min(bases)) // M
    return k_min // WP, k_max // WP + 1


def prefix_tile_range(bits, prefix_value, prefix_bits, bases, M, WP):
    """Tiles producing candidates with the given top bits (v13:464-518)."""
    shift = bits - prefix_bits
    cmin = prefix_value << shift
    cmax = ((prefix_value + 1) << shift) - 1
    vmin, vmax = 1 << (bits - 1), (1 << bits) - 1
    if cmax < vmin or cmin > vmax:
        raise ValueError("prefix does not overlap the bit range")
    cmin, cmax = max(cmin, vmin), min(cmax, vmax)
    k_min = -(-(cmin - max(bases)) // M) if cmin > max(bases) else 0
    k_max = (cmax - min(bases)) // M
    if k_min > k_max:
        raise ValueError("prefix produces empty k-range")
    return k_min // WP, k_max // WP + 1


def lane_range(tile_min, tile_max, lanes, lane_id):
    """Contiguous lane lane_id of lanes over [tile_min, tile_max); the
    remainder goes to the first lanes (v13:3533-3554).  Also the multi-GPU
    shard function: rank r of N takes lane r."""
    if not 0 <= lane_id < lanes:
        raise ValueError("lane id out of range")
    total = tile_max - tile_min
    size, rem = divmod(total, lanes)
    start = tile_min + lane_id * size + min(lane_id, rem)
    end = start + size + (1 if lane_id < rem else 0)
    return start, end


def measure_imad_peak(device=0):
    """Measured 32-bit multiply-add issue rate in tera-ops/s."""
    t = C.c_double(0)
    _check(load_library().ccs_measure_imad_peak(device, C.byref(t)), "ccs_measure_imad_peak")
    return t.value


def measure_int32_peak(device=0):
    """Measured INT32 ALU issue rate in tera-ops/s (ccs_measure_int32_peak)."""
    t = C.c_double(0)
    _check(load_library().ccs_measure_int32_peak(device, C.byref(t)), "ccs_measure_int32_peak")
    return t.value


class Server:
    """Continuous-batching request server (ccs_server_*): submit ranges at any
    time; admitted requests share every scheduling tick on the GPU."""

    def __init__(self, engines, max_active=256, chunk_tiles=1 << 20, mem_cap_bytes=120 << 30,
                 max_pending=1 << 20):
        lib = load_library()
        arr = (_vp * len(engines))(*[e.h for e in engines])
        cfg = _ServerConfig(max_active, chunk_tiles, mem_cap_bytes, max_pending, 0)
        h = _vp()
        _check(lib.ccs_server_create(arr, len(engines), C.byref(cfg), C.byref(h)), "ccs_server_create")
        self.h = h
        self.engines = engines

    def close(self):
        if getattr(self, "h", None):
            load_library().ccs_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, tile_start, n_tiles, profile=0, bits=None):
        lo, hi = _split128(tile_start)
        rg = _Range(lo, hi, int(n_tiles), profile, bits or self.engines[profile].bits)
        rid = _u64(0)
        _check(load_library().ccs_submit(self.h, C.byref(rg), C.byref(rid)), "ccs_submit")
        return rid.value

    def wait(self, rid, timeout_ms=600000):
        st = load_library().ccs_wait(self.h, rid, timeout_ms)
        _check(st, "ccs_wait")

    def poll(self, rid, surv_cap=1 << 20, chain_cap=1 << 16):
        """None while running, else (status, result dict, survivors, chains)."""
        res = _RequestResult()
        surv = np.zeros(surv_cap, dtype=SURVIVOR_DTYPE)
        ch = np.zeros(chain_cap, dtype=CHAIN_DTYPE)
        st = load_library().ccs_poll(self.h, rid, C.byref(res), surv.ctypes.data, surv_cap,
                                     ch.ctypes.data, chain_cap)
        if st == PENDING:
            return None
        if st not in (OK, OVERFLOW, ERR_CANCELLED):
            _check(st, "ccs_poll")
        r = {f: getattr(res, f) for f, _ in _RequestResult._fields_}
        return st, r, surv[: min(r["n_survivors"], surv_cap)], ch[: min(r["n_chains"], chain_cap)]

    def cancel(self, rid):
        _check(load_library().ccs_cancel(self.h, rid), "ccs_cancel")

    def set_batch_tuning(self, block_threads=0, blocks_per_sm=0, unit_words=0):
        """Tuning of the server's batch executor (from Batch.autotune),
        applied before its next tick."""
        t = _BatchTuning(block_threads, blocks_per_sm, unit_words, 0)
        _check(load_library().ccs_server_set_batch_tuning(self.h, C.byref(t)), "ccs_server_set_batch_tuning")

    def memory(self):
        """Device bytes reserved by admitted requests: (now, peak)."""
        a, b = _u64(0), _u64(0)
        _check(load_library().ccs_server_memory(self.h, C.byref(a), C.byref(b)), "ccs_server_memory")
        return a.value, b.value

    def stats(self):
        out = (_u64 * 6)()
        _check(load_library().ccs_server_stats(self.h, out))
        return dict(zip(["submitted", "admitted", "completed", "cancelled", "ticks", "pending"],
                        [int(x) for x in out]))


def config_depth_profile(depth):
    """One profile of the mixed-depth workloads: W = 31#, the given depth,
    stage primes 37..2^10 / 2^10..2^14 / 2^14..2^17 at positions [0, depth)."""
    return dict(target=depth, depth=depth, bits=89,
                stages=[(primes_in(37, 1 << 10), 0), (primes_in(1 << 10, 1 << 14), 0),
                        (primes_in(1 << 14, 1 << 17), 0)])


def mixed_ranges(engines, n, seed, min_log2=20, max_log2=34, width_lo=64, width_hi=110):
    """Seeded uneven ranges: length log-uniform in [2^min_log2, 2^max_log2]
    candidates, profile (depth) uniform over engines, root width uniform in
    [width_lo, width_hi], start drawn inside that width's tile range.
    Returns [(tile_start, n_tiles, profile, bits)]."""
    import random
    r = random.Random(seed)
    info = [(e.info["candidates_per_tile"], e.bases(), e.info["lattice_m"], e.info["wheel_period"])
            for e in engines]
    out = []
    for _ in range(n):
        p = r.randrange(len(engines))
        cpt, bases, M, WP = info[p]
        cands = 2.0 ** r.uniform(min_log2, max_log2)
        nt = max(1, int(round(cands / cpt)))
        bits = r.randint(width_lo, width_hi)
        t0, t1 = bit_tile_range(bits, bases, M, WP)
        ts = r.randint(t0, max(t0, t1 - nt - 1))
        out.append((ts, nt, p, bits))
    return out


from .qiter import (QIter, parse_pool, parse_pool_spec, parse_pool_specs, pool_from_text,  # noqa: E402
                    qiter_sieve_primes, q_window, V16_EXT_PRIMES, format_hit_line, synthetic_pool,
                    QCampaign, QITER_CHECKPOINT_VERSION, sieve_hash, pool_hash)
