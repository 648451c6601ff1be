"""B200 (sm_100a) resolved LBM-DEM step with the API of dasfadwqd/LBDEM-Taichi's
``src`` package: PSCLattice3D, BasicLattice3D, ForcedLattice3D, DEMSolver and
its configuration classes.  Compute runs in liblbdem.so (hand-written CUDA);
there is no CPU fallback."""
from .vector import Vector3, Vector4
from .lbm3d.lbmutils import CellType, UnitConverter

__all__ = ["Vector3", "Vector4", "CellType", "UnitConverter", "PSCLattice3D", "BasicLattice3D",
           "ForcedLattice3D", "DEMSolver", "DEMSolverConfig", "DomainBounds", "HertzContactConfig",
           "LinearContactConfig"]


def __getattr__(name):
    # lazy imports keep `import lbdem_taichi_b200` torch-free until a solver is used
    if name == "PSCLattice3D":
        from .lbdem.psclattice3d import PSCLattice3D
        return PSCLattice3D
    if name in ("BasicLattice3D", "ForcedLattice3D"):
        from .lbm3d import lattice
        return getattr(lattice, name)
    if name == "DEMSolver":
        from .dem3d.demsolver import DEMSolver
        return DEMSolver
    if name in ("DEMSolverConfig", "DomainBounds", "HertzContactConfig", "LinearContactConfig"):
        from .dem3d import demconfig
        return getattr(demconfig, name)
    raise AttributeError(name)
