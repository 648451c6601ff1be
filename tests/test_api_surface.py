"""The drop-in Python surface against the reference's, recorded from its
source by tests/golden/make_api_surface.py (tests/golden/api_surface.json):

- constructors take the reference's positional parameters in its order (the
  options this package adds all have defaults);
- every method the reference's LBM-DEM, LBM and DEM example drivers call on a
  lattice or a DEM solver exists on PSCLattice3D / BasicLattice3D / DEMSolver
  (the reference's other lattice and solver methods are Taichi kernels that
  the fused CUDA kernels replace);
- the configuration classes, UnitConverter and CellType have every public
  method and field of the reference's, CellType with the same values;
- the lattice class attributes (D, Q, c, w, qinv, the reflection tables,
  cssq, velmax, SmagorinskyConstant) exist, the scalar ones with the same
  values.
"""
import dataclasses
import inspect
import json
import os

import pytest

SURFACE = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "api_surface.json")))
REF = SURFACE["classes"]


def _ours():
    from lbdem_taichi_b200.dem3d.demconfig import (DEMSolverConfig, DomainBounds, HertzContactConfig,
                                                   LinearContactConfig)
    from lbdem_taichi_b200.dem3d.demsolver import DEMSolver
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    from lbdem_taichi_b200.lbm3d.lattice import BasicLattice3D, ForcedLattice3D
    from lbdem_taichi_b200.lbm3d.lbmutils import CellType, UnitConverter
    return {"PSCLattice3D": PSCLattice3D, "BasicLattice3D": BasicLattice3D, "ForcedLattice3D": ForcedLattice3D,
            "DEMSolver": DEMSolver, "DEMSolverConfig": DEMSolverConfig, "DomainBounds": DomainBounds,
            "HertzContactConfig": HertzContactConfig, "LinearContactConfig": LinearContactConfig,
            "UnitConverter": UnitConverter, "CellType": CellType}


def test_surface_covers_the_classes():
    assert set(REF) == set(_ours())
    assert "collide" in SURFACE["driver_calls"]["lattice"] and "run_simulation" in SURFACE["driver_calls"]["dem"]


@pytest.mark.parametrize("name", sorted(n for n, v in REF.items() if v["init"] is not None))
def test_constructor_parameters(name):
    params = list(inspect.signature(_ours()[name].__init__).parameters.values())[1:]
    ref = REF[name]["init"]
    assert [p.name for p in params[:len(ref)]] == ref
    assert all(p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD) for p in params[:len(ref)])
    assert all(p.default is not p.empty or p.kind in (p.VAR_POSITIONAL, p.VAR_KEYWORD) for p in params[len(ref):])


@pytest.mark.parametrize("name", ["PSCLattice3D", "BasicLattice3D"])
def test_driver_lattice_calls(name):
    cls = _ours()[name]
    missing = [m for m in SURFACE["driver_calls"]["lattice"] if not callable(getattr(cls, m, None))]
    assert not missing, missing


def test_driver_dem_calls():
    cls = _ours()["DEMSolver"]
    missing = [m for m in SURFACE["driver_calls"]["dem"] if not callable(getattr(cls, m, None))]
    assert not missing, missing


@pytest.mark.parametrize("name", ["DEMSolverConfig", "DomainBounds", "HertzContactConfig", "LinearContactConfig",
                                  "UnitConverter", "CellType"])
def test_helper_classes(name):
    cls = _ours()[name]
    assert not [m for m in REF[name]["public"] if not callable(getattr(cls, m, None))]
    fields = {f.name for f in dataclasses.fields(cls)} if dataclasses.is_dataclass(cls) else set()
    assert not [f for f in REF[name]["fields"] if f not in fields and not hasattr(cls, f)]
    for k, v in REF[name]["constants"].items():
        assert getattr(cls, k) == v, k


def test_lattice_class_attributes():
    cls = _ours()["BasicLattice3D"]
    ref = REF["BasicLattice3D"]
    assert not [f for f in ref["fields"] if not hasattr(cls, f)]
    for k, v in ref["constants"].items():
        assert getattr(cls, k) == v, k
