"""The reference-shaped field views of the lattice classes on CPU (the device
side stood in by NumPy): python-scope element writes as the reference's
drivers use them (``lattice.CT[i, j, k] = ...``, ``lattice.vel[i, j, k][0] =
u``) reach the host mirror, are pushed once at flush, and reads are served
from the mirror until the device side changes."""
import numpy as np
import pytest

from lbdem_taichi_b200.lbm3d.lattice import LatticeField


class _Owner:
    def __init__(self):
        self.dirty = []

    def _host_dirty(self, name):
        self.dirty.append(name)


def _field(shape, writable=True):
    dev = {"a": np.arange(np.prod(shape), dtype=np.float64).reshape(shape), "pulls": 0, "pushes": []}

    def pull():
        dev["pulls"] += 1
        return dev["a"].copy()

    def push(h):
        dev["pushes"].append(h.copy())
        dev["a"] = h.copy()

    owner = _Owner()
    return LatticeField(owner, "vel", shape, np.float64, pull, push if writable else None), dev, owner


def test_element_and_component_writes_reach_the_device_at_flush():
    f, dev, owner = _field((4, 3, 2, 3))
    f[1, 2, 0] = [7.0, 8.0, 9.0]
    f[0, 0, 1][2] = -5.0                      # component write through the cell vector
    assert owner.dirty == ["vel", "vel"]
    assert not dev["pushes"]
    f.flush()
    assert len(dev["pushes"]) == 1
    a = dev["a"]
    np.testing.assert_array_equal(a[1, 2, 0], [7.0, 8.0, 9.0])
    assert a[0, 0, 1, 2] == -5.0
    f.flush()                                 # nothing pending: no second push
    assert len(dev["pushes"]) == 1


def test_reads_are_served_from_the_mirror_until_invalidated():
    f, dev, _ = _field((2, 2, 2))
    assert f[1, 1, 1] == 7.0 and f.to_numpy().sum() == 28.0
    assert dev["pulls"] == 1
    dev["a"] = dev["a"] + 1.0                 # the device changed the field
    assert f[1, 1, 1] == 7.0                  # still the mirror
    f.invalidate()
    assert f[1, 1, 1] == 8.0 and dev["pulls"] == 2


def test_pending_writes_survive_invalidation():
    f, dev, _ = _field((2, 2, 2))
    f[0, 0, 0] = 42.0
    f.invalidate()                            # a kernel ran, but the write is not pushed yet
    assert f[0, 0, 0] == 42.0
    f.flush()
    assert dev["a"][0, 0, 0] == 42.0


def test_from_numpy_fill_and_shape():
    f, dev, _ = _field((3, 2, 2))
    assert f.shape == (3, 2, 2)
    f.from_numpy(np.ones(12))
    f.flush()
    np.testing.assert_array_equal(dev["a"], np.ones((3, 2, 2)))
    f.fill(2.5)
    f.flush()
    assert (dev["a"] == 2.5).all()


def test_read_only_fields_refuse_writes():
    f, _, _ = _field((2, 2, 2), writable=False)
    with pytest.raises(AttributeError):
        f[0, 0, 0] = 1.0
    with pytest.raises(AttributeError):
        f.from_numpy(np.zeros(8))
