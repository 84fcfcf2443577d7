"""Generate the golden fixtures of tests/golden from the reference checkout.

Run where the reference checkout is readable, giving its root as REF (the
argument, or the environment variable DUGKS_REFERENCE; there is no
default):
    python tests/golden/gen_golden.py REF

* quadrature_setdv.json -- nodes and weights produced by the reference's own
  generator functions dvGH / dvNC (src/scripts/setDV.py:83-138).  The script
  is Python 2; only the text of those two functions is executed here (they
  run unchanged under Python 3 given an integer type whose `/` floors, as
  Python 2's does).
* para_golden.json -- the case parameters of the reference demos' own
  setup scripts (demo/cavity/para.py, demo/ball/para.py): gas constant,
  density from Kn, dimensionless viscosity and muRef, for their own Kn and
  for the Kn values of the benchmark configurations.  The scripts are
  Python 2; their statements up to the first print are executed with Kn
  (and L) substituted.
* demo_cavity.npz -- the reference cavity demo's inputs
  (demo/cavity/constant/polyMesh, constant/Xis, constant/weights,
  constant/DVMProperties, 0/rho, 0/U, 0/T), so that the GPU tests can run
  that exact case without the reference present.
"""
import json
import math
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "psp-vst_b200", "python"))

from dugks_b200 import foamio, meshgen  # noqa: E402


class _Py2Int(int):
    """int whose true division floors, as in Python 2."""

    def __truediv__(self, o):
        return _Py2Int(int(self) // o) if isinstance(o, int) else int(self) / o

    def __sub__(self, o):
        return _Py2Int(int(self) - o) if isinstance(o, int) else int(self) - o


def reference_quadrature(ref):
    src = open(os.path.join(ref, "src/scripts/setDV.py")).read()
    body = re.search(r"^def dvGH.*?(?=^if __name__)", src, re.S | re.M).group(0)
    ns = {"np": np, "LA": np.linalg}
    exec(body, ns)
    R, T = 208.244343891, 273.0
    C = math.sqrt(2 * R * T)
    out = {"C": C, "GH": {}, "NC": {}}
    for n in (6, 8, 16, 20, 28, 32):
        x, w = ns["dvGH"](C, _Py2Int(n))
        out["GH"][str(n)] = {"xis": [float(v) for v in x], "weights": [float(v) for v in w]}
    for xm, n in ((1600.0, 9), (1600.0, 41)):
        x, w = ns["dvNC"](xm, _Py2Int(n))
        out["NC"][f"{xm}_{n}"] = {"xis": [float(v) for v in x], "weights": [float(v) for v in w]}
    return out


def reference_para(ref):
    out = {}
    for demo in ("cavity", "ball"):
        src = open(os.path.join(ref, "demo", demo, "para.py")).read()
        body = src.split("print")[0]
        runs = {}
        for kn in (None, 0.01, 0.075, 0.1, 1.0):
            code = body if kn is None else re.sub(r"^Kn = .*$", f"Kn = {kn!r}", body, flags=re.M)
            ns = {}
            exec("from numpy import *\n" + code, ns)
            runs["own" if kn is None else repr(kn)] = {k: float(ns[k]) for k in ("Kn", "R", "rho", "muBar", "mu", "C", "T",
                                                                              "L", "omega_HS", "omega_VHS")}
        out[demo] = runs
    return out


def demo_cavity(ref):
    d = os.path.join(ref, "demo/cavity")
    pm = meshgen.read_polymesh(d)
    props = foamio.read_dict(os.path.join(d, "constant/DVMProperties"))
    gp, fp = props["gasProperties"], props["fvDVMparas"]
    val = lambda v: float(v[-1]) if isinstance(v, list) else float(v)
    sizes = {p["name"]: p["nFaces"] for p in pm.patches}
    rho = foamio.read_vol_field(os.path.join(d, "0/rho"), pm.n_cells, sizes)
    U = foamio.read_vol_field(os.path.join(d, "0/U"), pm.n_cells, sizes)
    T = foamio.read_vol_field(os.path.join(d, "0/T"), pm.n_cells, sizes)
    patch_names = [p["name"] for p in pm.patches]
    # constraint-type (empty) patches need no field entry
    ptypes = [rho["patches"][n]["type"] if n in rho["patches"] else p["type"]
              for n, p in zip(patch_names, pm.patches)]
    pU = [np.asarray(U["patches"].get(n, {}).get("value", np.zeros((0, 3))))[:1].reshape(-1).tolist()
          for n in patch_names]
    pT = [np.asarray(T["patches"].get(n, {}).get("value", np.zeros(0)))[:1].tolist() for n in patch_names]
    np.savez_compressed(
        os.path.join(HERE, "demo_cavity.npz"),
        points=pm.points, face_offsets=pm.face_offsets.astype(np.int32), face_points=pm.face_points.astype(np.int32),
        owner=pm.owner.astype(np.int32), neighbour=pm.neighbour.astype(np.int32),
        patch_names=np.array(patch_names), patch_types=np.array([p["type"] for p in pm.patches]),
        patch_start=np.array([p["startFace"] for p in pm.patches]), patch_size=np.array([p["nFaces"] for p in pm.patches]),
        rho_bc_types=np.array(ptypes), patch_U=np.array(json.dumps(pU)), patch_T=np.array(json.dumps(pT)),
        xis=foamio.read_scalar_list(os.path.join(d, "constant/Xis")),
        weights=foamio.read_scalar_list(os.path.join(d, "constant/weights")),
        gas=np.array([val(gp["R"]), val(gp["omega"]), val(gp["Tref"]), val(gp["muRef"]), val(gp["Pr"])]),
        xi_max=val(fp["xiMax"]), rho0=rho["internal"], U0=U["internal"], T0=T["internal"])


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DUGKS_REFERENCE", "")
    if not ref or not os.path.isdir(ref):
        sys.exit("usage: gen_golden.py REF  (the reference checkout's root; or set DUGKS_REFERENCE)")
    with open(os.path.join(HERE, "quadrature_setdv.json"), "w") as f:
        json.dump(reference_quadrature(ref), f, indent=0)
    with open(os.path.join(HERE, "para_golden.json"), "w") as f:
        json.dump(reference_para(ref), f, indent=1)
    demo_cavity(ref)
    print("written:", sorted(os.listdir(HERE)))
