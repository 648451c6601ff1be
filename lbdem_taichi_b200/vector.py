"""Small FP64 vector type standing in for ``ti.types.vector(3, float)``.

The reference's configuration objects carry Taichi vectors (``config.gravity.x``,
``Vector3(xmin, ymin, zmin)`` passed to ``init_particle_fields``); this numpy
subclass offers the same construction and ``.x/.y/.z`` access.
"""
import numpy as np


class Vec(np.ndarray):
    @property
    def x(self):
        return float(self[0])

    @property
    def y(self):
        return float(self[1])

    @property
    def z(self):
        return float(self[2])


def Vector3(*args):
    vals = list(args[0]) if len(args) == 1 and np.ndim(args[0]) == 1 else list(args)
    if len(vals) != 3:
        raise ValueError("Vector3 takes 3 components")
    return np.array(vals, dtype=np.float64).view(Vec)


def Vector4(*args):
    vals = list(args[0]) if len(args) == 1 and np.ndim(args[0]) == 1 else list(args)
    return np.array(vals, dtype=np.float64).view(Vec)
