"""hs_dot_noalloc: the allocation-free dot product, for callers that cannot call
cudaMalloc (a host application that owns the device-memory budget, or a path
that must not take the allocator's locks).

It keeps its partial sums in a static device array instead of allocated
scratch, so it must return exactly what the allocating hs_dot returns (both
use the library's fixed reduction order; the dot parity tests compare bit for
bit), on consecutive calls that reuse the same array, up to the largest grid
the array serves (N = 321), and reject the first grid past it (N = 322)
before launching anything.  The file is named to be collected last.
"""
import numpy as np
import pytest

from mnhack8_b200 import _lib
from tests.helpers import Dev, random_field, random_nodes

RT, KF = 256, 2                     # flat partition: blocks of 512 nodes
ARRAY_DOUBLES = 2 * 65536           # the static array: two quantities per block
N_MAX = 321


def _nflat(N):
    return -(-((N + 1) ** 3) // (RT * KF))


def test_scratch_formula_covers_every_accepted_grid():
    """k_reduce writes partials[q*nflat + block] for q = 0, 1: every accepted
    grid must fit 2*nflat doubles, and the first rejected one must not."""
    assert all(2 * _nflat(N) <= ARRAY_DOUBLES for N in range(1, N_MAX + 1))
    assert 2 * _nflat(N_MAX + 1) > ARRAY_DOUBLES


def test_bound_is_checked_before_any_device_call():
    """On a host without a GPU the size check answers HS_ERR_ARG past the limit
    and HS_ERR_CUDA (no device) within it: the check runs first."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("passes placeholder pointers: run only where no device can be reached")
    for N in (1, 255, 256, N_MAX):
        with pytest.raises(_lib.HeatError) as e:
            _lib.dot_noalloc(N, 1, 1, 1)
        assert e.value.status == 4, N
    for N in (N_MAX + 1, 400, 1200):
        with pytest.raises(_lib.HeatError) as e:
            _lib.dot_noalloc(N, 1, 1, 1)
        assert e.value.status == 1, N


@pytest.mark.gpu
@pytest.mark.parametrize("N", [33, 128, 256, N_MAX])
def test_dot_noalloc_matches_hs_dot(N):
    dev = Dev()
    torch = dev.torch
    k, r = random_field(N, 5)
    g = _lib.Solver(N, 1e-3, k, r, kernel="wht", scatter="colored")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for call in range(2):                       # two calls in a row share the static scratch
        x = dev.put(random_nodes(N, 10 + call))
        y = dev.put(random_nodes(N, 20 + call))
        want = g.dot_ptr(x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        _lib.dot_noalloc(N, x.data_ptr(), y.data_ptr(), out.data_ptr())
        got = dev.get(out)[0]                   # synchronises the device first
        assert np.float64(got).view(np.uint64) == np.float64(want).view(np.uint64), (call, got, want)
        del x, y
    g.close()


@pytest.mark.gpu
def test_dot_noalloc_rejects_oversized_grid():
    Dev()
    with pytest.raises(_lib.HeatError) as e:
        _lib.dot_noalloc(N_MAX + 1, 1, 1, 1)    # 2*nflat exceeds the static array; nothing is launched
    assert e.value.status == 1
