"""Unit conversion and cell-type flags (API of src/lbm3d/lbmutils.py:14-97)."""


class UnitConverter:
    """Physical <-> lattice units for spacing dx, time step dt, density rho."""

    def __init__(self, dx: float, dt: float, rho: float):
        self.dx = dx
        self.dt = dt
        self.rho = rho

    def getLbLength(self, v): return v / self.dx
    def getLbTime(self, v): return v / self.dt
    def getLbVel(self, v): return v * self.dt / self.dx
    def getLbAccel(self, v): return v * (self.dt ** 2) / self.dx
    def getLbStrainRate(self, v): return v * self.dt
    def getLbRho(self, v): return v / self.rho
    def getLbNu(self, v): return v * self.dt / (self.dx ** 2)
    def getLbSigma(self, v): return v * (self.dt ** 2) / (self.rho * (self.dx ** 2))
    def getLbForce(self, v): return v * (self.dt ** 2) / (self.rho * (self.dx ** 4))
    def getPhysLength(self, v): return v * self.dx
    def getPhysTime(self, v): return v * self.dt
    def getPhysVel(self, v): return v * self.dx / self.dt
    def getPhysAccell(self, v): return v * self.dx / (self.dt ** 2)
    def getPhysStrainRate(self, v): return v / self.dt
    def getPhysRho(self, v): return v * self.rho
    def getPhysNu(self, v): return v * (self.dx ** 2) / self.dt
    def getPhysSigma(self, v): return v * (self.rho * (self.dx ** 2)) / (self.dt ** 2)
    def getPhysForce(self, v): return v * (self.rho * (self.dx ** 4)) / (self.dt ** 2)


class CellType:
    """Bit flags of lattice cells; values are part of the reference API."""
    FLUID = 1
    INTERFACE = 2
    GAS = 4
    OBSTACLE = 8
    FREE_SLIP = 16
    VEL_LADD = 32
    VEL_ZOUHE = 64
    VEL_EXIT = 128
    Pre_ZOUHE = 256
    VEL_INLET_LADD = 262144
    NO_FLUID_NEIGH = 512
    TO_FLUID = 1024
    TO_GAS = 2048
    RIGHT = 4096
    LEFT = 8192
    TOP = 16384
    BOTTOM = 32768
    FRONT = 65536
    BACK = 131072
