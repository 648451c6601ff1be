"""Helpers shared by the golden-fixture tests."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def relmax(a, b, floor=1e-30):
    """max |a-b| / max |b| (scale-normalised error)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), floor))


def dem_params(g, model):
    """Parameters of the DEM golden scenarios (make_golden.py:_scen_dem)."""
    kw = dict(dt=float(g["dt"]), gravity=g["gravity"], domain=g["domain"],
              periodic=tuple(bool(v) for v in g["periodic"]), model=model,
              E=float(g["E"]), nu=float(g["nu"]), wall_E=float(g["wall_E"]), wall_nu=float(g["wall_nu"]),
              max_coord=int(g["max_coord"]), omega=g["gomega"], pp_mu=0.3, pw_mu=0.4)
    if model == "hertz":
        kw.update(pp_e=0.9, pw_e=0.8)
    else:
        kw.update(kn=200.0, ks=100.0, dpn=0.2)
    return kw
