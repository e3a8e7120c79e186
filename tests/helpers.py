"""Shared helpers of the test-suite (fields, device buffers)."""
import numpy as np

from mnhack8_b200.fields import FieldSpec, make_field


def field(n, model="lognormal", **kw):
    k, r, _ = make_field(FieldSpec(n=n, model=model, **kw))
    return k.ravel(), r.ravel()


def random_field(n, seed, contrast=3.0):
    rng = np.random.default_rng(seed)
    k = np.exp(rng.uniform(-contrast, contrast, n ** 3))
    r = np.exp(rng.uniform(-1.0, 1.0, n ** 3))
    return k, r


def random_nodes(n, seed, boundary=True):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n + 1) ** 3)
    if not boundary:
        nn = n + 1
        idx = np.arange(nn ** 3)
        ix, iy, iz = idx // (nn * nn), (idx // nn) % nn, idx % nn
        b = (ix == 0) | (ix == n) | (iy == 0) | (iy == n) | (iz == 0) | (iz == n)
        x[b] = 0.0
    return x


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


class Dev:
    """Device buffers via torch (plumbing only) with explicit synchronisation."""

    def __init__(self):
        import torch
        self.torch = torch
        assert torch.cuda.is_available(), "GPU tests need a CUDA device"

    def put(self, a):
        t = self.torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
        self.torch.cuda.synchronize()
        return t

    def zeros(self, n):
        t = self.torch.zeros(n, dtype=self.torch.float64, device="cuda")
        self.torch.cuda.synchronize()
        return t

    def get(self, t):
        self.torch.cuda.synchronize()
        return t.cpu().numpy()
