"""hs_dot_noalloc: the allocation-free dot product, for callers that cannot call
cudaMalloc (a host application that owns the device-memory budget, or a path
that must not take the allocator's locks).

It keeps its partial sums in a static device array instead of allocated
scratch, so it must return exactly what the allocating hs_dot returns (both
use the library's fixed reduction order; the dot parity tests compare bit for
bit), on consecutive calls that reuse the same array, and reject grids larger
than the array serves.  The file is named to be collected last.
"""
import numpy as np
import pytest

from mnhack8_b200 import _lib
from tests.helpers import Dev, random_field, random_nodes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [33, 128])
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
    g.close()


def test_dot_noalloc_rejects_oversized_grid():
    with pytest.raises(_lib.HeatError) as e:
        _lib.dot_noalloc(322, 1, 1, 1)          # (323)^3 nodes exceed the static scratch; nothing is launched
    assert e.value.status == 1
