"""Engine.batch(max_nodes=...) on the CPU: the Python binding's split of a
batch into calls of a bounded voxel count, driven against a stand-in for the
library's femh_homogenize_batch (no GPU).  The split returns what one call
returns: C in cell order, one info per cell, the gradients in cell order."""
import ctypes

import numpy as np

from fem_b200 import femh as F


class _FakeLib:
    """femh_homogenize_batch writing C_cell = (index of the cell's first voxel
    value) * I and dL/drho = rho * trace(dL/dC); records the call sizes."""

    def __init__(self, avail=1e12):
        self.calls = []
        self.avail = avail

    def femh_batch_memory(self, h, n, cells, need, avail):
        """1000 bytes per voxel; self.avail bytes available."""
        need._obj.value = sum(1000.0 * cells._obj.nx * cells._obj.ny * cells._obj.nz for _ in range(n))
        if avail is not None:
            avail._obj.value = self.avail
        return 0

    def femh_homogenize_batch(self, h, n, cells, Cp, dp, gp, infos):
        self.calls.append(sum(cells[i].nx * cells[i].ny * cells[i].nz for i in range(n)))
        off = 0
        for i in range(n):
            c = cells[i]
            vox = c.nx * c.ny * c.nz
            for k in range(6):
                Cp[36 * i + 7 * k] = c.rho[0]
            if gp.value:
                g = ctypes.cast(gp, ctypes.POINTER(ctypes.c_double))
                d = ctypes.cast(dp, ctypes.POINTER(ctypes.c_double))
                tr = sum(d[36 * i + 7 * k] for k in range(6))
                for v in range(vox):
                    g[off + v] = c.rho[v] * tr
            off += vox
            infos[i].status = 0
            infos[i].iterations[0] = 10 + i
        return 0


def _engine(avail=1e12):
    e = F.Engine.__new__(F.Engine)
    e.lib = _FakeLib(avail)
    e.h = ctypes.c_void_p(1)
    e.shape = None
    e._ncells = 0
    return e


def test_split_batch_equals_one_call():
    rng = np.random.default_rng(0)
    rhos = [rng.random((n, n, n)) for n in (4, 6, 4, 8, 4)]
    dLdC = np.stack([np.eye(6) * (k + 1) for k in range(5)])
    one = _engine()
    C1, i1, g1 = one.batch(rhos, dLdC=dLdC)
    split = _engine()
    C2, i2, g2 = split.batch(rhos, dLdC=dLdC, max_nodes=300)
    # 64 + 216 | 64 | 512 (over the budget, alone) | 64
    assert one.lib.calls == [920] and split.lib.calls == [280, 64, 512, 64]
    assert np.array_equal(C1, C2)
    assert [i["iterations"][0] for i in i2] == [10, 11, 10, 10, 10]
    assert all(np.array_equal(a, b) for a, b in zip(g1, g2))
    assert split._ncells == 0 and one._ncells == 5


def test_default_split_by_device_memory():
    """With no max_nodes the cells go in calls that fit 92% of the memory the
    engine reports available (femh_batch_memory): here 0.92 x 400 kB against
    1000 bytes a voxel = 368 voxels a call."""
    rng = np.random.default_rng(1)
    rhos = [rng.random((n, n, n)) for n in (4, 6, 4, 8, 4)]
    e = _engine(avail=400e3)
    C, infos, _ = e.batch(rhos)
    assert e.lib.calls == [344, 512, 64]   # 64 + 216 + 64 | 512 (over the budget, alone) | 64
    ref = _engine()
    C1, _, _ = ref.batch(rhos)
    assert ref.lib.calls == [920] and np.array_equal(C, C1)
