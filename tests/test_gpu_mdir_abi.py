"""MDIR's own runtime names through ctypes, with MLIR's memref descriptors
built in Python: the groups registry (runtime/mdrt_cuda.c:3087-3330, the
slot table of include/mdir/Runtime/GroupsABI.h:10-44), the export of this
library's lists into it, and the f32 cuFFT entries including the
Gaussian backward transform (mdrt_cuda.c:2942-2990,
runtime/pme_callback.cu:5-21)."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O
from mdir_b200 import NonbondedTerm, systems
from mdir_b200 import _lib as L
from mdir_b200.term import _cudart, _dp

pytestmark = pytest.mark.gpu


def host(ptr, count, dtype):
    out = np.empty(count, dtype=dtype)
    torch.cuda.synchronize()
    assert _cudart().cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(ptr),
                                ctypes.c_size_t(out.nbytes), 2) == 0
    return out


def buffer(handle, slot):
    d = L.MemRef1D()
    L.lib()._mlir_ciface_mdrtGroupsBuffer(ctypes.byref(d), handle, slot)
    return d


def test_registry_shapes_growth_and_errors(cuda):
    lib = L.lib()
    assert lib.mdrtGroupsLastStatus() == L.OK
    h = lib.mdrtGroupsCreate(100, 3)  # places round up to 112 (7 groups)
    assert h != 0
    want = {L.GROUPS_ORDER: 112, L.GROUPS_COUNTS: 7, L.GROUPS_ENTRIES: 192, L.GROUPS_MASKS: 192,
            L.GROUPS_UNIT_GROUPS: 3, L.GROUPS_UNIT_ORDINALS: 3, L.GROUPS_SHIFTS: 112,
            L.GROUPS_INNER_COUNTS: 3, L.GROUPS_BLOCK_OF: 1, L.GROUPS_ACTIVE_COUNT: 1, 13: 1, 14: 1,
            L.GROUPS_PLACED: 336, 16: 7, 23: 2}
    for slot, size in want.items():
        d = buffer(h, slot)
        assert d.size == size and d.stride == 1 and d.offset == 0, slot
        assert d.aligned and d.allocated == d.aligned
    assert buffer(h, L.GROUPS_ORDER).aligned == buffer(h, L.GROUPS_ORDER).aligned  # the same buffer again
    p = L.MemRef2D()
    lib._mlir_ciface_mdrtGroupsPlaced(ctypes.byref(p), h)
    assert list(p.sizes) == [112, 3] and list(p.strides) == [3, 1]
    assert p.aligned == buffer(h, L.GROUPS_PLACED).aligned
    # growth: a quarter more than asked, only when asked for more
    lib.mdrtGroupsGrow(h, 100, 3)
    assert buffer(h, L.GROUPS_ENTRIES).size == 192
    assert lib.mdrtGroupsBuilt(h) == 0  # built now; no growth before
    lib.mdrtGroupsGrow(h, 200, 10)
    assert buffer(h, L.GROUPS_ORDER).size == (200 + 50 + 15) // 16 * 16
    assert buffer(h, L.GROUPS_ENTRIES).size == 64 * 12
    assert lib.mdrtGroupsBuilt(h) == 1  # one growth of the lists after the build
    assert lib.mdrtGroupsBuilt(h) == 0
    lib.mdrtGroupsGrow(h, 500, 10)  # places only: not a growth of the lists
    assert lib.mdrtGroupsBuilt(h) == 0
    lib.mdrtGroupsReserveBlockOf(h, 40)
    assert buffer(h, L.GROUPS_BLOCK_OF).size == 50
    lib.mdrtGroupsReserveBlockOf(h, 45)
    assert buffer(h, L.GROUPS_BLOCK_OF).size == 50
    # where MDIR aborts: an empty descriptor and a status
    d = buffer(h, 24)
    assert d.size == 0 and not d.aligned
    assert lib.mdrtGroupsLastStatus() == L.INVALID_ARGUMENT
    assert lib.mdrtGroupsLastStatus() == L.OK
    assert lib.mdrtGroupsDestroy(h) == L.OK


def test_export_holds_the_lists_of_the_build(cuda):
    s = systems.tip3p(waters=600, seed=13)
    n = len(s["charges"])
    t = NonbondedTerm(n)
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], 1.2, s["beta"])
    t.set_pruned_reach(1.0)
    x = torch.tensor(s["positions"], device=cuda)
    sizes = t.build(x, s["box"])
    t.prune(x, s["box"])
    lib = L.lib()
    h = lib.mdrtGroupsCreate(16, 1)  # too small: the export grows it
    L.check(lib.mdrtNbGroupsExport(t._h, h, None), "mdrtNbGroupsExport")
    G = int(sizes[L.SIZE_GROUPS])
    B = int(sizes[L.SIZE_UNITS])
    order = host(buffer(h, L.GROUPS_ORDER).aligned, 16 * G, np.int32)
    np.testing.assert_array_equal(order, t.buffer(L.SLOT_ORDER, np.int32)[:16 * G])
    counts = host(buffer(h, L.GROUPS_COUNTS).aligned, G, np.int32)
    np.testing.assert_array_equal(counts, t.buffer(L.SLOT_COUNTS, np.int32)[:G])
    shifts = host(buffer(h, L.GROUPS_SHIFTS).aligned, 16 * G, np.int32).view(np.int8).reshape(-1, 4)
    np.testing.assert_array_equal(shifts, t.buffer(L.SLOT_SHIFTS, np.int8, 4)[:16 * G])
    p = L.MemRef2D()
    lib._mlir_ciface_mdrtGroupsPlaced(ctypes.byref(p), h)
    placed = host(p.aligned, 3 * 16 * G, np.float32).reshape(-1, 3)
    np.testing.assert_array_equal(placed, t.buffer(L.SLOT_PLACED, np.float32, 4)[:16 * G, :3])

    def bits_of(entries, masks, groups):
        # (member place, partner place, image code) of every bit of the blocks
        blk, k = np.nonzero(entries >= 0)
        q, m = entries[blk, k], masks[blk, k].astype(np.uint32)
        out = []
        for u in range(16):
            on = (m >> u) & 1 == 1
            out.append(np.stack([16 * groups[blk[on]] + u, q[on], (m[on] >> 16) & 0x7FFF], 1))
        a = np.concatenate(out).astype(np.int64)
        return a[np.lexsort((a[:, 2], a[:, 1], a[:, 0]))]

    # the outer lists: every bit of the blocks is a bit of the build, and
    # the pair set they name is the oracle's
    ent = host(buffer(h, L.GROUPS_ENTRIES).aligned, 64 * B, np.int32).reshape(B, 64)
    msk = host(buffer(h, L.GROUPS_MASKS).aligned, 64 * B, np.int32).reshape(B, 64)
    grp = host(buffer(h, L.GROUPS_UNIT_GROUPS).aligned, B, np.int32)
    ordn = host(buffer(h, L.GROUPS_UNIT_ORDINALS).aligned, B, np.int32)
    assert np.all(ordn * 64 < counts[grp])
    assert int((ent >= 0).sum()) == int(counts.sum())
    mine = bits_of(ent, msk, grp)
    count, ref = O.pairset(s["positions"], s["box"], 1.2, O.rows_from_pairs(n, s["excluded_pairs"]))
    assert len(mine) == count == len(t.pair_set(sizes))
    # the pruned lists by blocks: the entries of the pruned lists, each block
    # with its count, every block active
    cnt_in = t.buffer(L.SLOT_INNER_COUNTS, np.int32)[:G]
    active = host(buffer(h, L.GROUPS_ACTIVE_COUNT).aligned, 1, np.int32)[0]
    assert active == int(np.sum((cnt_in + 63) // 64))
    ic = host(buffer(h, L.GROUPS_INNER_COUNTS).aligned, active, np.int32)
    assert int(ic.sum()) == int(cnt_in.sum()) and np.all(ic > 0)
    np.testing.assert_array_equal(host(buffer(h, L.GROUPS_ACTIVE_UNITS).aligned, active, np.int32),
                                  np.arange(active))
    ie = host(buffer(h, L.GROUPS_INNER_ENTRIES).aligned, 64 * active, np.int32).reshape(active, 64)
    assert int((ie >= 0).sum()) == int(cnt_in.sum())
    assert lib.mdrtGroupsDestroy(h) == L.OK
    t.close()


def test_fft_entries_with_descriptors(cuda):
    lib = L.lib()
    k1, k2, k3 = 24, 20, 18
    rng = np.random.default_rng(3)
    g = rng.normal(size=(k1, k2, k3)).astype(np.float32)
    real = torch.tensor(g, device=cuda)
    spec = torch.zeros((k1, k2, k3 // 2 + 1, 2), dtype=torch.float32, device=cuda)

    def desc(tensor):
        return L.MemRef1D(tensor.data_ptr(), tensor.data_ptr(), 0, tensor.numel(), 1)

    dr, ds = desc(real), desc(spec)
    lib.mdrtNbSetAbiStream(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    lib._mlir_ciface_mdrtCudaFFTForward3DF32(ctypes.byref(dr), ctypes.byref(ds), k1, k2, k3)
    want = np.fft.rfftn(g.astype(np.float64))
    got = spec.cpu().numpy()
    np.testing.assert_allclose(got[..., 0] + 1j * got[..., 1], want, atol=2e-4 * np.abs(want).max())
    # the Gaussian influence from per-axis tables, then the backward transform
    tables, ms = [], []
    for k in (k1, k2, k3):
        m = np.where(np.arange(k) <= k // 2, np.arange(k), np.arange(k) - k) / 1.7
        f = np.exp(-0.3 * m * m) * (1.0 + 0.1 * np.cos(np.arange(k)))
        tables.append(np.concatenate([m, m * m, f]).astype(np.float32))
        ms.append((m, f))
    tab = torch.tensor(np.concatenate(tables), device=cuda)
    dt_ = desc(tab)
    out = torch.zeros_like(real)
    do = desc(out)
    lib._mlir_ciface_mdrtCudaFFTGaussianBackwardF32(ctypes.byref(ds), ctypes.byref(do), ctypes.byref(dt_),
                                                     k1, k2, k3)
    (mx, fx), (my, fy), (mz, fz) = ms
    hz = k3 // 2 + 1
    sq = mx[:, None, None] ** 2 + my[None, :, None] ** 2 + mz[None, None, :hz] ** 2
    prod = fx[:, None, None] * fy[None, :, None] * fz[None, None, :hz]
    factor = np.where(sq == 0, 0.0, prod / np.where(sq == 0, 1.0, sq))
    ref = np.fft.irfftn(want * factor, s=(k1, k2, k3), axes=(0, 1, 2)) * (k1 * k2 * k3)  # not normalized
    np.testing.assert_allclose(out.cpu().numpy(), ref, atol=3e-4 * np.abs(ref).max())
    # the plain backward transform, not normalized, gives the grid back
    spec2 = torch.zeros_like(spec)
    ds2 = desc(spec2)
    lib._mlir_ciface_mdrtCudaFFTForward3DF32(ctypes.byref(dr), ctypes.byref(ds2), k1, k2, k3)
    back = torch.zeros_like(real)
    db = desc(back)
    lib._mlir_ciface_mdrtCudaFFTBackward3DF32(ctypes.byref(ds2), ctypes.byref(db), k1, k2, k3)
    np.testing.assert_allclose(back.cpu().numpy() / (k1 * k2 * k3), g, atol=2e-5 * np.abs(g).max())
    lib.mdrtNbSetAbiStream(None)
    assert lib.mdrtGroupsLastStatus() == L.OK
