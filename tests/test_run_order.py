"""The two canonical orders of the PCG vector dots, restated in plain Python
and checked bit for bit against the oracle (which the GPU parity tests pin
the library to).

FLAT: blocks of 512 consecutive nodes, thread t of block b summing nodes
b*512 + 2t and b*512 + 2t + 1 in order; each block's 256 sums go through the
block tree (a 32-lane xor butterfly per warp, then an 8-way butterfly over
the warp sums); the block partials are combined by 256 strided sequential
sums and the same tree.

RUN (the PCG update's b.b, r.z, r.r): the same blocks dealt to
G = min(blocks, 740) runs, run c taking blocks c, c+G, ...; thread t carries
one sum through its two nodes of each of the run's blocks; one tree per run;
the run sums combined like block partials.  Below 740 blocks (N < 89) the
two orders coincide.

The dots are taken against a vector of ones, so every term is added exactly
as a Python float addition (fma(a, 1, s) = s + a rounded once).
"""
import numpy as np
import pytest

from oracle import oracle as orc

RT, KF, SLOTS = 256, 2, 740


def tree(v):
    ws = []
    for w in range(8):
        a = list(v[w * 32:(w + 1) * 32])
        off = 16
        while off >= 1:
            a = [a[l] + a[l ^ off] for l in range(32)]
            off >>= 1
        ws.append(a[0])
    off = 4
    while off >= 1:
        ws = [ws[l] + ws[l ^ off] for l in range(8)]
        off >>= 1
    return ws[0]


def combine(P):
    return tree([sum_seq(P[l::RT]) for l in range(RT)])


def sum_seq(xs):
    acc = 0.0
    for x in xs:
        acc = acc + x
    return acc


def flat(a):
    nb = -(-len(a) // (RT * KF))
    P = []
    for b in range(nb):
        v = [sum_seq(a[b * RT * KF + l * KF: b * RT * KF + l * KF + KF]) for l in range(RT)]
        P.append(tree(v))
    return combine(P)


def run(a):
    nb = -(-len(a) // (RT * KF))
    G = min(nb, SLOTS)
    U = []
    for c in range(G):
        v = []
        for l in range(RT):
            acc = 0.0
            for b in range(c, nb, G):
                for x in a[b * RT * KF + l * KF: b * RT * KF + l * KF + KF]:
                    acc = acc + x
            v.append(acc)
        U.append(tree(v))
    return combine(U)


@pytest.mark.parametrize("N", [12, 90])
def test_orders_bitwise(N):
    NN = N + 1
    rng = np.random.default_rng(N)
    a = rng.normal(0.0, 1.0, NN ** 3) * np.exp(rng.normal(0.0, 6.0, NN ** 3))
    ones = np.ones(NN ** 3)
    o = orc.Oracle(N, 1e-4, np.ones(N ** 3), np.ones(N ** 3))
    al = a.tolist()
    f, u = flat(al), run(al)
    assert o.dot(a, ones) == f
    assert o.udot(a, ones) == u
    nb = -(-NN ** 3 // (RT * KF))
    if nb <= SLOTS:
        assert f == u
