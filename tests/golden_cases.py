"""Cases built from the committed golden fixtures (tests/golden)."""
import json
import os

import numpy as np

from dugks_b200 import case as cs
from dugks_b200 import meshgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def demo_cavity(flatten=True, geometry=None) -> cs.Case:
    """The reference cavity demo (demo/cavity: 60x60x1 hexes from blockMesh,
    28x28 half-range Gauss-Hermite DVs, Kn 0.075, lid 50 m/s)."""
    z = np.load(os.path.join(GOLDEN, "demo_cavity.npz"))
    patches = [{"name": str(n), "type": str(t), "startFace": int(s), "nFaces": int(k)}
               for n, t, s, k in zip(z["patch_names"], z["patch_types"], z["patch_start"], z["patch_size"])]
    owner = z["owner"].astype(np.int64)
    nei = z["neighbour"].astype(np.int64)
    pm = meshgen.PolyMesh(points=z["points"], face_offsets=z["face_offsets"].astype(np.int64),
                          face_points=z["face_points"].astype(np.int64), owner=owner, neighbour=nei,
                          n_cells=int(max(owner.max(), nei.max())) + 1, patches=patches, n_solution_dims=2)
    pU = json.loads(str(z["patch_U"]))
    pT = json.loads(str(z["patch_T"]))
    spec = []
    for p, rt, u, t in zip(patches, z["rho_bc_types"], pU, pT):
        if str(rt) == "empty":
            spec.append(cs.Patch(p["name"], "empty"))
        else:
            kind = {"calculatedMaxwell": "maxwellWall", "farField": "farField"}[str(rt)]
            spec.append(cs.Patch(p["name"], kind, tuple(u) if u else (0.0, 0.0, 0.0), t[0] if t else 273.0))
    R, omega, Tref, mu, Pr = (float(v) for v in z["gas"])
    gas = {"R": R, "omega": omega, "Tref": Tref, "muRef": mu, "Pr": Pr, "K": 0}
    c = cs.Case("demo_cavity60", pm, 2, gas, z["xis"], z["weights"], float(z["xi_max"]), spec,
                z["rho0"].copy(), z["U0"].reshape(-1, 3).copy(), z["T0"].copy())
    return c.flatten(geometry) if flatten else c


def setdv_quadrature() -> dict:
    with open(os.path.join(GOLDEN, "quadrature_setdv.json")) as f:
        return json.load(f)
