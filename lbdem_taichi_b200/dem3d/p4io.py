"""p4p / p4c particle and contact files (DEMSolver.save_single and
init_particle_fields, demsolver.py:59-177): plain-text frames, single-space
separated, 1-based particle IDs.

    p4p:  TIMESTEP  PARTICLES / "<t> <n>" / ID  GROUP  RAD  MASS  PX  PY  PZ  VX  VY  VZ / n rows
    p4c:  TIMESTEP  CONTACTS  / "<t> <m>" / P1  P2  CX  CY  CZ  FX  FY  FZ               / m rows
"""
from __future__ import annotations

import math

import numpy as np

P4P_FMT = "%d %d %.6e %.6e %.6e %.6e %.6e %.6e %.6e %.6e"
P4C_FMT = "%d %d %.6e %.6e %.6e %.6e %.6e %.6e"


def read_p4p(file_name: str) -> dict:
    """The first frame of a p4p file: ID, group, radius, mass, pos (n, 3),
    vel (n, 3), indexed by ID - 1, and the material density implied by the
    last row (demsolver.py:130-177 reads it the same way)."""
    with open(file_name, encoding="UTF-8") as fp:
        fp.readline()
        n = int(fp.readline().removesuffix("\n").split(" ")[1])
        fp.readline()
        rows = []
        for _ in range(n):
            line = fp.readline()
            if line == "":
                break
            rows.append(line.split(" "))
    ID = np.zeros(n, np.int64)
    group = np.zeros(n, np.int64)
    radius = np.zeros(n)
    mass = np.zeros(n)
    pos = np.zeros((n, 3))
    vel = np.zeros((n, 3))
    density = 0.0
    for tok in rows:
        i = int(tok[0]) - 1
        ID[i] = int(tok[0])
        group[i] = int(tok[1])
        radius[i] = float(tok[2])
        mass[i] = float(tok[3])
        pos[i] = [float(tok[4]), float(tok[5]), float(tok[6])]
        vel[i] = [float(tok[7]), float(tok[8]), float(tok[9])]
        density = 3 * mass[i] / (4 * math.pi * radius[i] ** 3)
    return {"ID": ID, "group": group, "radius": radius, "mass": mass, "pos": pos, "vel": vel, "density": density}


def write_p4p(fh, t: float, ID, group, radius, mass, pos, vel) -> None:
    """Append one particle frame."""
    pos, vel = np.asarray(pos), np.asarray(vel)
    fh.write("TIMESTEP  PARTICLES\n")
    fh.write(f"{t} {len(ID)}\n")
    fh.write("ID  GROUP  RAD  MASS  PX  PY  PZ  VX  VY  VZ\n")
    data = np.column_stack([ID, group, radius, mass, pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1],
                            vel[:, 2]])
    np.savetxt(fh, data, fmt=P4P_FMT)


def write_p4c(fh, t: float, rows) -> None:
    """Append one contact frame; rows are (P1 ID, P2 ID, CX, CY, CZ, FX, FY, FZ)."""
    fh.write("TIMESTEP  CONTACTS\n")
    fh.write(f"{t} {len(rows)}\n")
    fh.write("P1  P2  CX  CY  CZ  FX  FY  FZ\n")
    if len(rows):
        np.savetxt(fh, np.asarray(rows, dtype=np.float64), fmt=P4C_FMT)
