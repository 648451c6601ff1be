from .lbmutils import CellType, UnitConverter

__all__ = ["CellType", "UnitConverter"]
