"""ctypes bindings for the test oracle (oracle/liboracle.so) and the reference
harnesses built from the reference's own sources (oracle/_ref/).

Test infrastructure only: this module is the checker and is imported only by
tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

# Reference parameter set (src/cuda/cc18_filter_cuda_CpC_v13.cu:174-201)
CRT_PRIMES = [5, 7, 11, 13, 17, 19]
WHEEL_PRIMES = [23, 29, 31]
L2_PRIMES = [37, 41, 43, 47, 53, 59, 61]
EXT_PRIMES = [67, 71, 73, 79, 83, 89, 97]
CHAIN_SCREEN_PRIMES = [
    67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113, 127, 131, 137, 139, 149, 151,
    157, 163, 167, 173, 179, 181, 191, 193, 197, 199, 211, 223, 227, 229, 233, 239, 241,
    251, 257, 263, 269, 271, 277, 281, 283, 293, 307, 311, 313, 317, 331, 337, 347, 349,
    353, 359, 367, 373, 379, 383, 389, 397, 401, 409, 419, 421, 431, 433, 439, 443, 449,
    457, 461, 463, 467, 479, 487, 491, 499, 503, 509, 521, 523, 541, 547, 557, 563, 569,
    571, 577, 587, 593, 599, 601, 607, 613, 617, 619, 631, 641, 643, 647, 653, 659, 661,
    673, 677, 683, 691, 701, 709, 719, 727, 733, 739, 743, 751, 757, 761, 769, 773, 787,
    797, 809, 811, 821, 823, 827, 829, 839, 853, 857, 859, 863]
LINE_PRIMES = CHAIN_SCREEN_PRIMES[7:]
V13_WITNESSES = [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71]

PRIME_MR = 0
PRIME_BPSW = 1

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def _load_oracle():
    lib = C.CDLL(ORACLE_SO)
    vp = C.c_void_p
    lib.orc_lattice_create.restype = vp
    lib.orc_lattice_create.argtypes = [_u32p, C.c_int, _u32p, C.c_int, C.c_int, C.c_int]
    lib.orc_lattice_free.argtypes = [vp]
    lib.orc_num_bases.argtypes = [vp]
    lib.orc_base.argtypes = [vp, C.c_int]
    lib.orc_base.restype = C.c_uint64
    lib.orc_tkm6.argtypes = [vp, C.c_int]
    lib.orc_tkm6.restype = C.c_uint32
    lib.orc_bucket_size.argtypes = [vp, C.c_int, C.c_int]
    lib.orc_wheel_total.argtypes = [vp, C.c_int]
    lib.orc_bucket.argtypes = [vp, C.c_int, C.c_int, _u32p]
    lib.orc_add_stage.argtypes = [vp, _u32p, C.c_int, C.c_int, C.c_int]
    lib.orc_filter_range.restype = C.c_uint64
    lib.orc_filter_range.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint64, _u32p, C.c_uint64,
                                     _u64p]
    lib.orc_forbidden.argtypes = [C.c_uint32, C.c_int, C.c_int, _u32p]
    lib.orc_is_prime_mr.argtypes = [_u64p, C.c_int, _u64p, C.c_int]
    lib.orc_is_prime_bpsw.argtypes = [_u64p, C.c_int]
    lib.orc_strong_prp.argtypes = [_u64p, C.c_int, C.c_uint64]
    lib.orc_powmod.argtypes = [_u64p, _u64p, _u64p, C.c_int, _u64p]
    lib.orc_chain_from.argtypes = [_u64p, C.c_int, C.c_int, _u64p, C.c_int]
    lib.orc_prove_n.argtypes = [_u64p, C.c_int, C.c_int, C.c_int, C.c_int, _u64p, C.c_int, _u64p,
                                C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.orc_reconstruct.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32,
                                    C.c_uint32, _u64p]
    lib.orc_prove_v33.argtypes = [_u64p, C.c_int, C.c_int, C.c_int, _u64p, C.POINTER(C.c_int),
                                  C.POINTER(C.c_int)]
    lib.orc_chain_from_v33.argtypes = [_u64p, C.c_int, C.c_int, C.c_int]
    lib.orc_qiter_forbidden.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, C.c_int, C.c_int, _u32p]
    lib.orc_qiter_filter_seg.restype = C.c_uint64
    lib.orc_qiter_filter_seg.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64,
                                         C.c_int, C.c_int, _u32p, C.c_int, _u32p, C.c_uint64]
    lib.orc_qiter_prove.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, C.c_int,
                                    C.c_int, C.c_int, C.c_int, _u64p, C.c_int, _u64p,
                                    C.POINTER(C.c_int), C.POINTER(C.c_int)]
    return lib


_ORC = None


def oracle():
    global _ORC
    if _ORC is None:
        _ORC = _load_oracle()
    return _ORC


def int_to_words(n, nw=4):
    return np.array([(n >> (64 * i)) & (2**64 - 1) for i in range(nw)], dtype=np.uint64)


def words_to_int(w):
    return sum(int(x) << (64 * i) for i, x in enumerate(w))


class kind:
    """Context manager: run oracle calls for chain kind k (1 first, 2 second)."""

    def __init__(self, k):
        self.k = k

    def __enter__(self):
        oracle().orc_set_kind(self.k)

    def __exit__(self, *a):
        oracle().orc_set_kind(1)


def forbidden(q, L, pos_lo=0, kind_=1):
    out = np.zeros(64, dtype=np.uint32)
    with kind(kind_):
        n = oracle().orc_forbidden(q, L, pos_lo, out)
    return sorted(int(x) for x in out[:n])


def is_prime_mr(n, witnesses=V13_WITNESSES):
    w = np.array(witnesses, dtype=np.uint64)
    return bool(oracle().orc_is_prime_mr(int_to_words(n), 4, w, len(w)))


def is_prime_bpsw(n):
    return bool(oracle().orc_is_prime_bpsw(int_to_words(n), 4))


def strong_prp(n, a):
    return bool(oracle().orc_strong_prp(int_to_words(n), 4, a))


def powmod(b, e, m):
    out = np.zeros(4, dtype=np.uint64)
    oracle().orc_powmod(int_to_words(b), int_to_words(e), int_to_words(m), 4, out)
    return words_to_int(out)


def chain_from(n, primality=PRIME_BPSW, witnesses=V13_WITNESSES, kind_=1):
    w = np.array(witnesses, dtype=np.uint64)
    with kind(kind_):
        return oracle().orc_chain_from(int_to_words(n), 4, primality, w, len(w))


def prove_n(n, bits, mode=1, primality=PRIME_BPSW, witnesses=V13_WITNESSES, kind_=1):
    """Reference prove semantics for one candidate n.  mode 0 = GPU K2
    (roots only), mode 1 = CPU GMP prover (backward walk).  Returns None
    or (chain_len, root, is_root), plus whether n itself tested prime."""
    w = np.array(witnesses, dtype=np.uint64)
    root = np.zeros(4, dtype=np.uint64)
    flags = C.c_int(0)
    isp = C.c_int(0)
    with kind(kind_):
        r = oracle().orc_prove_n(int_to_words(n), 4, bits, mode, primality, w, len(w), root,
                                 C.byref(flags), C.byref(isp))
    if r < 0:
        return None, bool(isp.value)
    return (r, words_to_int(root), bool(flags.value & 1)), bool(isp.value)


def prove_v33(n, bits, target):
    """The reference CPU engine's proving semantics (CCS_PRIME_V33) for one
    candidate n: None or (chain_len, root, is_root), plus whether n passed
    its root test."""
    root = np.zeros(4, dtype=np.uint64)
    flags = C.c_int(0)
    isp = C.c_int(0)
    r = oracle().orc_prove_v33(int_to_words(n), 4, bits, target, root, C.byref(flags), C.byref(isp))
    if r < 0:
        return None, bool(isp.value)
    return (r, words_to_int(root), bool(flags.value & 1)), bool(isp.value)


def chain_from_v33(n, wide=False, cap_bits=127):
    """v33's walk of a given number: Baillie-PSW for it, then screened links."""
    return oracle().orc_chain_from_v33(int_to_words(n), 4, int(wide), cap_bits)


class Lattice:
    """Oracle lattice + filter stages.  stages: list of (primes, pos_lo)."""

    def __init__(self, crt=CRT_PRIMES, wheel=WHEEL_PRIMES, lattice_len=18, depth=18,
                 stages=None, max_bases=0, kind_=1):
        lib = oracle()
        lib.orc_set_kind(kind_)
        self.kind = kind_
        self.crt = list(crt)
        self.wheel = list(wheel)
        self.M = int(np.prod(self.crt, dtype=object))
        self.WP = int(np.prod(self.wheel, dtype=object))
        self.h = lib.orc_lattice_create(np.array(crt, dtype=np.uint32), len(crt),
                                        np.array(wheel, dtype=np.uint32), len(wheel),
                                        lattice_len, max_bases)
        if stages is None:
            stages = reference_stages()
        self.stages = stages
        for primes, pos_lo in stages:
            a = np.array(primes, dtype=np.uint32)
            lib.orc_add_stage(self.h, a, len(a), pos_lo, depth)
        self.n_bases = lib.orc_num_bases(self.h)
        lib.orc_set_kind(1)

    def __del__(self):
        try:
            oracle().orc_lattice_free(self.h)
        except Exception:
            pass

    def base(self, b):
        return int(oracle().orc_base(self.h, b))

    def bases(self):
        return [self.base(b) for b in range(self.n_bases)]

    def tkm6(self, b):
        return int(oracle().orc_tkm6(self.h, b))

    def bucket(self, b, m):
        n = oracle().orc_bucket_size(self.h, b, m)
        out = np.zeros(max(n, 1), dtype=np.uint32)
        oracle().orc_bucket(self.h, b, m, out)
        return out[:n].copy()

    def candidates_per_tile(self):
        return sum(oracle().orc_wheel_total(self.h, b) for b in range(self.n_bases)) // 6

    def filter_range(self, tile_start, n_tiles, cap=1 << 22, counters=False):
        out = np.zeros(4 * cap, dtype=np.uint32)
        sp = np.zeros(len(self.stages) + 1, dtype=np.uint64)
        n = oracle().orc_filter_range(self.h, tile_start & (2**64 - 1), tile_start >> 64,
                                      n_tiles, out, cap, sp)
        surv = out[: 4 * min(n, cap)].reshape(-1, 4).copy()
        if counters:
            return surv, int(n), [int(x) for x in sp]
        return surv

    def reconstruct(self, tile_start, base_idx, k, tile_idx):
        out = np.zeros(4, dtype=np.uint64)
        oracle().orc_reconstruct(self.h, tile_start & (2**64 - 1), tile_start >> 64, base_idx, k,
                                 tile_idx, out)
        return words_to_int(out)


def reference_stages():
    """Reference stage layout (v13:793-862): L2 mask 37..61 and ext-L2 67..97 at
    positions [0, L); line sieve 101..863 at positions [1, L)."""
    return [(L2_PRIMES, 0), (EXT_PRIMES, 0), (LINE_PRIMES, 1)]


def primes_between(lo, hi):
    """primes p with lo <= p < hi"""
    sieve = np.ones(hi, dtype=bool)
    sieve[:2] = False
    for p in range(2, int(hi ** 0.5) + 1):
        if sieve[p]:
            sieve[p * p::p] = False
    return [int(p) for p in np.nonzero(sieve)[0] if p >= lo]


def ref33():
    """The reference v33 engine harness (GMP), or None when not built."""
    path = os.path.join(REF_DIR, "libref33.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.ref33_base.restype = C.c_ulonglong
    lib.ref33_tkm6.restype = C.c_uint
    lib.ref33_bucket.argtypes = [C.c_int, C.c_int, _u32p]
    lib.ref33_l2_mask.restype = C.c_ulonglong
    lib.ref33_gmp_probab_prime.argtypes = [C.c_char_p, C.c_int]
    lib.ref33_gmp_powm.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p]
    lib.ref33_mr_mont.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_ulonglong]
    lib.ref33_is_prime_fast.argtypes = [C.c_char_p]
    lib.ref33_full_chain.argtypes = [C.c_char_p, C.c_char_p]
    lib.ref33_forward_chain.argtypes = [C.c_char_p]
    lib.ref33_is_root.argtypes = [C.c_char_p]
    lib.ref_gmp_forward_chain.argtypes = [C.c_char_p]
    lib.ref_gmp_forward_chain2.argtypes = [C.c_char_p]
    lib.ref33_follow_native.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_int]
    lib.ref33_root_native.argtypes = [C.c_ulonglong, C.c_ulonglong]
    lib.ref33_fermat2_native.argtypes = [C.c_ulonglong, C.c_ulonglong]
    lib.ref33_prove_native.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_int, C.c_char_p,
                                       C.POINTER(C.c_int)]
    return lib


def ref33_prove_native(lib, n, log_threshold=1):
    """The reference CPU engine's native proving path on one candidate (see
    oracle/ref/v33_harness.c): (code or chain length, root, is_root)."""
    buf = C.create_string_buffer(64)
    isr = C.c_int(0)
    r = lib.ref33_prove_native(n & (2**64 - 1), n >> 64, log_threshold, buf, C.byref(isr))
    root = int(buf.value, 16) if buf.value else 0
    return r, root, bool(isr.value)


def ref15():
    """The reference v15 engine harness (its K1 and K2 in either prove
    order), or None."""
    path = os.path.join(REF_DIR, "libref15.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.ref15_filter.restype = C.c_uint
    lib.ref15_filter.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_uint, C.c_int, _u32p, C.c_uint]
    lib.ref15_prove_gpu.restype = C.c_uint
    lib.ref15_prove_gpu.argtypes = [C.c_ulonglong, C.c_ulonglong, _u32p, C.c_uint, C.POINTER(C.c_uint)]
    return lib


def ref13b():
    """The reference second-kind engine v13b through the same harness, or None."""
    path = os.path.join(REF_DIR, "libref13b.so")
    if not os.path.exists(path):
        return None
    return _bind13(C.CDLL(path))


def ref13():
    """The reference v13 engine harness (GMP + its CUDA kernels), or None."""
    path = os.path.join(REF_DIR, "libref13.so")
    if not os.path.exists(path):
        return None
    return _bind13(C.CDLL(path))


def _bind13(lib):
    lib.ref13_base.restype = C.c_ulonglong
    lib.ref13_tkm6.restype = C.c_uint
    lib.ref13_bucket.argtypes = [C.c_int, C.c_int, _u32p]
    lib.ref13_l2_mask.restype = C.c_ulonglong
    lib.ref13_filter.restype = C.c_uint
    lib.ref13_filter.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_uint, C.c_int, _u32p, C.c_uint]
    lib.ref13_time_filter.restype = C.c_float
    lib.ref13_time_filter.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_uint, C.c_int, C.c_int]
    lib.ref13_prove_gpu.restype = C.c_uint
    lib.ref13_prove_gpu.argtypes = [C.c_ulonglong, C.c_ulonglong, _u32p, C.c_uint,
                                    C.POINTER(C.c_uint)]
    lib.ref13_prove_cpu.argtypes = [_u32p, C.c_int, C.c_ulonglong, C.c_ulonglong, C.c_int,
                                    C.c_int, C.c_char_p, C.POINTER(C.c_ulonglong),
                                    C.POINTER(C.c_ulonglong)]
    return lib


# ---------------------------------------------------------------------------
# fingerprint-pool Q iteration (v16)
# ---------------------------------------------------------------------------
M64 = 2**64 - 1


def qiter_forbidden(q, D, E, depth):
    """Forbidden residues of Q mod q, in first-appearance order ([] when q | D)."""
    out = np.zeros(max(depth, 1), dtype=np.uint32)
    n = oracle().orc_qiter_forbidden(q, D & M64, D >> 64, E, depth, out)
    return [int(x) for x in out[:n]]


def qiter_filter_seg(q_base, n_q, D, E, depth, primes, cap=1 << 22):
    """Survivor offsets of one segment, increasing."""
    pr = np.asarray(primes, dtype=np.uint32)
    out = np.zeros(max(cap, 1), dtype=np.uint32)
    n = oracle().orc_qiter_filter_seg(q_base & M64, q_base >> 64, n_q, D & M64, D >> 64, E, depth,
                                      pr, len(pr), out, cap)
    return [int(x) for x in out[: min(n, cap)]]


def qiter_prove(Q, D, E, target, reverse=True, mode=0, primality=PRIME_BPSW, witnesses=V13_WITNESSES):
    """(chain_len, root, is_root) or None, and whether p_0 tested prime."""
    wit = np.asarray(witnesses, dtype=np.uint64)
    root = np.zeros(4, dtype=np.uint64)
    fl, isp = C.c_int(0), C.c_int(0)
    L = oracle().orc_qiter_prove(Q & M64, Q >> 64, D & M64, D >> 64, E, target, 1 if reverse else 0, mode,
                                 primality, wit, len(wit), root, C.byref(fl), C.byref(isp))
    if L < 0:
        return None, bool(isp.value)
    return (L, words_to_int(root), bool(fl.value & 1)), bool(isp.value)


def ref16():
    """The reference v16 engine harness (its forbidden residues and its
    q-iteration kernel), or None."""
    path = os.path.join(REF_DIR, "libref16.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.ref16_forbidden.argtypes = [C.c_uint, C.c_ulonglong, C.c_ulonglong, C.c_int, C.c_int, _u32p, C.c_int]
    lib.ref16_qiter_filter.restype = C.c_uint
    lib.ref16_qiter_filter.argtypes = [_u32p, C.c_int, C.c_ulonglong, C.c_ulonglong, C.c_int, C.c_int,
                                       C.c_ulonglong, C.c_ulonglong, C.c_uint, _u32p, C.c_uint]
    ck = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, _u32p, C.c_int, C.c_int, C.c_uint,
          _u32p, C.c_int, C.c_int, C.c_ulonglong, C.c_uint, C.c_int, C.c_int, C.c_char_p, C.c_int]
    _u64p_ = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
    lib.ref16_ckpt_save.argtypes = ck + [_u64p_, _u64p_, _u64p_, _u64p_]
    lib.ref16_ckpt_load.argtypes = ck + [_u64p_, _u64p_]
    lib.ref16_qiter_time.restype = C.c_float
    lib.ref16_qiter_time.argtypes = [_u32p, C.c_int, C.c_ulonglong, C.c_ulonglong, C.c_int, C.c_int,
                                     C.c_ulonglong, C.c_ulonglong, C.c_uint, C.c_int, C.POINTER(C.c_uint)]
    return lib
