"""The midsolve kernel's own code (run single-threaded on the host) against the
oracle; board generation and the C-ABI layout.  No GPU."""
import numpy as np
import pytest

from tests.oracle import P


def oracle_values(O, raw):
    r, v = np.zeros(200, np.uint64), np.zeros(200, np.int32)
    n = O.midsolve(int(raw), P(r), P(v))
    return list(zip(r[:n].tolist(), v[:n].tolist()))


@pytest.mark.parametrize("stones", [35, 34, 33, 32, 31, 30, 29, 28, 27, 26, 25])
def test_midsolve_kernel_code_on_host_matches_oracle(O, stones):
    from pentago_b200 import mid
    raws = mid.random_boards(7 * stones, 3 if stones > 25 else 1, stones)
    raws = np.concatenate([raws, raws | np.uint64(1 << 63)])
    got, sup = mid.selftest_host(raws, supers=True)
    for k, (raw, g) in enumerate(zip(raws, got)):
        assert g == oracle_values(O, raw), f"board {int(raw)}"
        ref = np.zeros(76, np.uint64)
        O.midsolve_internal(int(raw), P(ref))
        n = 37 - stones
        assert np.array_equal(sup[k][:4 * n], ref[:4 * n])


def test_random_boards_26_stones():
    from pentago_b200 import mid
    raws = mid.random_boards(0, 64, 26)
    assert len(set(raws.tolist())) == 64
    for b in raws.tolist():
        assert bin(mid.side_of(b, 1)).count("1") == 13 and bin(mid.side_of(b, 2)).count("1") == 13
        assert not mid.won(b, 1) and not mid.won(b, 2)


def test_mid_values_layout_matches_wasm_abi():
    import ctypes
    from pentago_b200 import capi
    assert ctypes.sizeof(capi.pg_mid_values_t) == 8 + 16 * 163 == capi.MID_VALUES_BYTES


def test_midsolve_rejects_small_boards():
    from pentago_b200 import capi, mid
    with pytest.raises(capi.PentagoError):
        mid.selftest_host(mid.random_boards(1, 1, 16))


@pytest.mark.parametrize("groups", [2, 3, 7])
def test_midsolve_split_into_groups_matches_single(groups):
    """The multi-CTA partition of every level (contiguous item ranges per group,
    a shared barrier between levels) gives the single-group result, run as
    host threads."""
    from pentago_b200 import mid
    raws = [int(r) for r in mid.random_boards(5, 2, 24)] + [int(r) for r in mid.random_boards(6, 2, 27)]
    assert mid.selftest_groups_host(raws, groups) == mid.selftest_host(raws)
