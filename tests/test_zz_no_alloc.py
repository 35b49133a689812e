"""The no-allocation filter entry point (ccs_filter_range_noalloc) gives the
same survivors as ccs_filter_range.  It exists for callers that may not
allocate device memory once they are running -- services whose GPU footprint
is fixed and accounted for at start-up, allocators that refuse to grow, hosts
under a per-tenant memory quota -- and works from a fixed array compiled into
the library.  This file is collected
last on purpose and runs the entry point twice in a row, so it also checks
that the array's leftover contents from the previous call do not leak into
the next one."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def as_set(t):
    a = t.cpu().numpy().astype(np.int64) & 0xFFFFFFFF
    return sorted(map(tuple, a[:, :3].tolist()))


@pytest.mark.parametrize("profile", ["reference", "cc16"])
def test_noalloc_matches_allocating_entry_point_twice(ccs, profile):
    import torch
    cfg = {} if profile == "reference" else ccs.config_cc16_scale()
    eng = ccs.Engine(**cfg)
    bases = eng.bases()
    t0, _ = ccs.bit_tile_range(89 if profile == "reference" else 88, bases,
                               eng.info["lattice_m"], eng.info["wheel_period"])
    out = torch.empty((1 << 18, 4), dtype=torch.int32, device="cuda")
    ref_out = torch.empty((1 << 18, 4), dtype=torch.int32, device="cuda")
    # two calls in a row: different ranges, then the first range again
    for ts, n in ((t0 + 1234567, 40_000), (t0 + 98765432, 100_001), (t0 + 1234567, 40_000)):
        got = as_set(eng.filter_range_noalloc(ts, n, out))
        want = as_set(eng.filter_range(ts, n, out=ref_out))
        assert got == want
        assert len(got) > 0
    eng.close()


def test_noalloc_rejects_profiles_beyond_its_limit(ccs):
    import torch
    eng = ccs.Engine(target=16, depth=16, stages=[(ccs.primes_in(37, 1 << 18), 0)])
    out = torch.empty((16, 4), dtype=torch.int32, device="cuda")
    with pytest.raises(ccs.CCSError) as e:
        eng.filter_range_noalloc(10**12, 6, out)
    assert e.value.status == ccs.ERR_INVALID
    assert "at most" in str(e.value)
    eng.close()
