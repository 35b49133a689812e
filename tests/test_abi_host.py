"""CPU-side checks of the product: the C-ABI library loads and exports every
symbol include/ccs.h declares, and its host lattice builder (ccs_describe)
agrees with the oracle.  No compute call touches a GPU."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "ccs.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ccs_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(ccs):
    lib = ccs.load_library()
    declared = header_functions()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(ccs.exported_symbols())
    assert lib.ccs_abi_version() == 1


def test_describe_reference_lattice(ccs, ob):
    info, bases = ccs.describe()
    lat = ob.Lattice()
    assert info["n_bases"] == 36 and bases == lat.bases()
    assert info["n_lines"] == 123552
    assert info["candidates_per_tile"] == 20592
    assert abs(info["expected_tests"] - 2.46) < 0.01
    assert abs(info["pass_rate"] - 1.15e-5) / 1.15e-5 < 0.01


def test_describe_cc16_scale(ccs, ob):
    cfg = ccs.config_cc16_scale()
    info, bases = ccs.describe(**cfg)
    lat = ob.Lattice(lattice_len=16, depth=16, stages=[(ob.L2_PRIMES, 0)])
    assert bases == lat.bases() and len(bases) == 108
    assert info["n_lines"] == 438048 and info["candidates_per_tile"] == 73008
    assert abs(info["expected_tests"] - 2.84) < 0.01
    assert abs(info["pass_rate"] - 4.43e-9) / 4.43e-9 < 0.01
    assert info["n_filter_primes"] == 161 + 1728 + 10351


def test_describe_cpu_method_lattice(ccs, ob):
    info, bases = ccs.describe(**ccs.config_cpu_method())
    lat = ob.Lattice(wheel=[23], lattice_len=8, depth=8, stages=[(ob.primes_between(29, 1022), 0)])
    assert bases == lat.bases()
    assert info["n_lines"] == 89100 and info["lattice_m"] * info["wheel_period"] * 6 == 223092870
    assert abs(info["expected_tests"] - 6.89) < 0.01


def test_describe_v13_base_cap(ccs, ob):
    info, bases = ccs.describe(target=16, max_bases=64)
    assert info["n_bases"] == 64
    assert bases == ob.Lattice(lattice_len=16, depth=16)[:0] if False else bases == ob.Lattice(
        lattice_len=16, depth=16).bases()[:64]


@pytest.mark.parametrize("bad", [
    dict(crt=(5, 7, 9)),                                 # 9 is not prime
    dict(stages=[((37, 23), 0)]),                        # 23 divides the lattice modulus
    dict(stages=[((37,), 2)]),                           # pos_lo must be 0 or 1
    dict(stages=[((37,), 0)] * 5),                       # at most 4 stages
    dict(target=0x100),                                  # target > 64
    dict(bits=10),                                       # bits < 21
])
def test_describe_rejects_bad_params(ccs, bad):
    with pytest.raises(ccs.CCSError) as e:
        ccs.describe(**bad)
    assert e.value.status == ccs.ERR_INVALID


def test_depth_clamped_to_target(ccs):
    info, _ = ccs.describe(target=12, depth=30)
    assert info["depth"] == 12


def test_forbidden_residue_helper(ccs, ob):
    for q in (37, 101, 1031, 16411):
        for L in (8, 16, 18):
            for lo in (0, 1):
                assert ccs.compute_forbidden_residues(q, L, lo) == ob.forbidden(q, L, lo)


def test_range_planner(ccs):
    bases = ccs.describe()[1]
    M, WP = 1616615, 20677
    t0, t1 = ccs.bit_tile_range(89, bases, M, WP)
    # v13 main: k_min = (2^88 - max_base)/M, k_max = (2^89 - 1 - min_base)/M
    assert t0 == ((1 << 88) - max(bases)) // M // WP
    assert t1 == ((1 << 89) - 1 - min(bases)) // M // WP + 1
    v, nb = ccs.parse_prefix("0b101")
    assert (v, nb) == (5, 3)
    p0, p1 = ccs.prefix_tile_range(89, v, nb, bases, M, WP)
    assert t0 <= p0 < p1 <= t1
    # complementary prefixes tile the bit range (v13:2388-2508)
    a = ccs.prefix_tile_range(89, 2, 2, bases, M, WP)
    b = ccs.prefix_tile_range(89, 3, 2, bases, M, WP)
    assert a[1] >= b[0] - 1 and a[0] <= b[0]
    for bad in ("101", "0b", "0b0101", "0b12"):
        with pytest.raises(ValueError):
            ccs.parse_prefix(bad)
    # lanes are disjoint, contiguous and cover the range
    for lanes in (1, 2, 3, 7, 8):
        got = [ccs.lane_range(p0, p1, lanes, i) for i in range(lanes)]
        assert got[0][0] == p0 and got[-1][1] == p1
        for (s0, e0), (s1, e1) in zip(got, got[1:]):
            assert e0 == s1
        sizes = [e - s for s, e in got]
        assert max(sizes) - min(sizes) <= 1


def test_chain_line_format(ccs):
    assert ccs.format_chain_line(18, 0xABC, 18, True) == "TARGET CC18 0xABC 12"
    assert ccs.format_chain_line(9, 0xF, 18, False) == "NON-ROOT CC9 0xF 4"
