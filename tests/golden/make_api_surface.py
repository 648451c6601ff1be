"""Record the reference's driver-facing Python surface (constructor
parameters, the methods its LBM-DEM example drivers call, config fields,
CellType values, UnitConverter methods, lattice class attributes) by parsing
its source with `ast` -- nothing of the reference is executed -- into
tests/golden/api_surface.json, which tests/test_api_surface.py checks this
package against.

    python tests/golden/make_api_surface.py <reference checkout>     (or LBDEM_REFERENCE=<checkout>)
"""
import ast
import glob
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LBDEM_REFERENCE")
if not REF or not os.path.isdir(os.path.join(REF, "src")):
    sys.exit(f"usage: python {os.path.relpath(__file__)} <reference checkout> (or set LBDEM_REFERENCE); "
             "the checkout must hold the reference's src/ package")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "api_surface.json")

CLASSES = ("PSCLattice3D", "BasicLattice3D", "ForcedLattice3D", "DEMSolver", "DEMSolverConfig", "DomainBounds",
           "HertzContactConfig", "LinearContactConfig", "UnitConverter", "CellType")
# the resolved-coupling and pure-LBM/DEM drivers (the unresolved and hybrid ones use other lattices)
DRIVERS = ("example/lbdem", "example/lbm3d", "example/dem3d")
OBJECTS = {"lattice": "lattice", "lbm": "lattice", "demsolver": "dem", "solver": "dem", "dem": "dem"}


def classes():
    out = {}
    for f in sorted(glob.glob(os.path.join(REF, "src", "**", "*.py"), recursive=True)):
        tree = ast.parse(open(f).read())
        for n in ast.walk(tree):
            if not (isinstance(n, ast.ClassDef) and n.name in CLASSES):
                continue
            init = next((m for m in n.body if isinstance(m, ast.FunctionDef) and m.name == "__init__"), None)
            fields, consts = [], {}
            for m in n.body:
                if isinstance(m, ast.AnnAssign) and isinstance(m.target, ast.Name):
                    fields.append(m.target.id)
                elif isinstance(m, ast.Assign):
                    for t in m.targets:
                        if isinstance(t, ast.Name):
                            fields.append(t.id)
                            if isinstance(m.value, ast.Constant) and isinstance(m.value.value, (int, float)):
                                consts[t.id] = m.value.value
            out[n.name] = {
                "file": os.path.relpath(f, REF),
                "init": [a.arg for a in init.args.args[1:]] if init else None,
                "public": [m.name for m in n.body if isinstance(m, ast.FunctionDef) and not m.name.startswith("_")],
                "fields": fields,
                "constants": consts,
            }
    return out


def driver_calls():
    calls = {"lattice": set(), "dem": set()}
    pat = re.compile(r"\b(" + "|".join(OBJECTS) + r")\.([A-Za-z_]\w*)\(")
    for d in DRIVERS:
        for f in glob.glob(os.path.join(REF, d, "**", "*.py"), recursive=True):
            for obj, meth in pat.findall(open(f).read()):
                calls[OBJECTS[obj]].add(meth)
    return {k: sorted(v) for k, v in calls.items()}


if __name__ == "__main__":
    surface = {"classes": classes(), "driver_calls": driver_calls()}
    with open(OUT, "w") as fh:
        json.dump(surface, fh, indent=1, sort_keys=True)
    print(OUT, {k: len(v) for k, v in surface["driver_calls"].items()})
