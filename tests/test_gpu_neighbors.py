"""The device neighbor build against the oracle's pair sets and MDIR's own
bit counts (test/Runtime/neighbors-groups-gpu.mlir:508-630): the lists hold
exactly the oracle's set of (pair, image) bits, bit for bit."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.test_oracle import GROUPS_KAT, lcg_case

pytestmark = pytest.mark.gpu


def device_pairs(x, L, R, ex, allow_nan=False):
    from mdir_b200 import NonbondedTerm
    n = len(x)
    t = NonbondedTerm(n)
    t.set_interaction(cutoff=min(R, 0.49 * L), reach=R, beta=0.0)
    if ex is not None:
        t.set_exclusions(rows=ex)
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    sizes = t.build(xd, [L, L, L], allow_nan=allow_nan)
    pairs = t.pair_set(sizes)
    return t, sizes, pairs


def canon(p):
    p = np.asarray(p, dtype=np.int64)
    return p[np.lexsort((p[:, 2], p[:, 1], p[:, 0]))]


@pytest.mark.parametrize("L,R,deg,poison,n,bits", GROUPS_KAT)
def test_lists_are_the_oracle_set(cuda, L, R, deg, poison, n, bits):
    x, ex = lcg_case(L, R, deg, poison, n)
    t, sizes, pairs = device_pairs(x, L, R, ex, allow_nan=poison)
    assert len(pairs) == bits
    count, ref = O.pairset(x, [L, L, L], R, ex)
    assert count == bits
    np.testing.assert_array_equal(canon(pairs), canon(ref))
    assert sizes[4] == (1 if poison else 0)
    t.close()


def test_build_is_deterministic(cuda):
    x, _ = lcg_case(7.0, 1.0, 0, False, 2000)
    from mdir_b200 import _lib as L
    t1, s1, p1 = device_pairs(x, 7.0, 1.0, None)
    e1 = t1.buffer(L.SLOT_ENTRIES, np.int32, 2).copy()
    o1 = t1.buffer(L.SLOT_ORDER, np.int32).copy()
    c1 = t1.buffer(L.SLOT_COUNTS, np.int32).copy()
    t2, s2, p2 = device_pairs(x, 7.0, 1.0, None)
    e2 = t2.buffer(L.SLOT_ENTRIES, np.int32, 2)
    o2 = t2.buffer(L.SLOT_ORDER, np.int32)
    c2 = t2.buffer(L.SLOT_COUNTS, np.int32)
    np.testing.assert_array_equal(o1, o2)
    G = s1[6]
    cap = t1.info()["list_capacity"]
    assert cap == t2.info()["list_capacity"]
    np.testing.assert_array_equal(c1[:G], c2[:G])
    # every list entry for entry (the slab past a list's end is not written)
    for g in range(G):
        np.testing.assert_array_equal(e1[g * cap: g * cap + c1[g]], e2[g * cap: g * cap + c2[g]])


def test_capacity_grows_and_retries(cuda):
    # a reach of 0.975 of the edge needs lists far longer than the first
    # estimate: the build grows and completes with every bit (D331 growth)
    x, ex = lcg_case(4.0, 3.9, 0, False, 320)
    t, sizes, pairs = device_pairs(x, 4.0, 3.9, ex)
    assert len(pairs) == 198183
    assert t.info()["list_capacity"] >= sizes[1]


def test_reach_beyond_edge_is_refused(cuda):
    from mdir_b200 import NonbondedTerm, _lib
    x, _ = lcg_case(4.0, 1.0, 0, False, 320)
    t = NonbondedTerm(320)
    t.set_interaction(cutoff=1.0, reach=3.999, beta=0.0)
    with pytest.raises(_lib.NativeError) as e:
        t.build(torch.tensor(x, device="cuda"), [4.0, 4.0, 4.0])
    assert e.value.status == _lib.INVALID_BOX


@pytest.mark.parametrize("case", [0, 4, 5, 6, 8, 11])
def test_lists_staged_in_chunks_are_the_same(cuda, case):
    """With a dual list the search stages its entries in chunks of the inner
    slab (from the second build on): the outer lists must be the oracle's
    set and, entry for entry, the lists of the shared-memory staging."""
    from mdir_b200 import NonbondedTerm
    from mdir_b200 import _lib as Lb
    L, R, deg, poison, n, bits = GROUPS_KAT[case]
    x, ex = lcg_case(L, R, deg, poison, n)
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    lists = []
    for dual in (False, True):
        t = NonbondedTerm(len(x))
        t.set_interaction(cutoff=0.5 * R, reach=R, beta=0.0)
        if ex is not None:
            t.set_exclusions(rows=ex)
        if dual:
            t.set_pruned_reach(0.75 * R)
        t.build(xd, [L, L, L], allow_nan=poison)
        sizes = t.build(xd, [L, L, L], allow_nan=poison)  # the second build stages in chunks
        pairs = t.pair_set(sizes)
        assert len(pairs) == bits
        G = sizes[6]
        cap = t.info()["list_capacity"]
        e = t.buffer(Lb.SLOT_ENTRIES, np.int32, 2)[: G * cap].copy()
        c = t.buffer(Lb.SLOT_COUNTS, np.int32)[:G].copy()
        lists.append((canon(pairs), e, c, cap))
        t.close()
    (p1, e1, c1, cap1), (p2, e2, c2, cap2) = lists
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(c1, c2)
    assert cap1 == cap2
    for g in range(len(c1)):
        np.testing.assert_array_equal(e1[g * cap1: g * cap1 + c1[g]], e2[g * cap2: g * cap2 + c2[g]])
