"""Cases for the DUGKS step: mesh + DV set + gas + boundary conditions +
initial state, flattened to the arrays the C ABI takes.

Physical parameters follow the reference demos' generator scripts
(demo/cavity/para.py, demo/ball/para.py): argon (k = 1.38066e-23,
m = 6.63e-26 kg, d = 4.17e-10 m), density from the Knudsen number,
rho = m / (Kn L sqrt(2) pi d^2), viscosity mu = rho C L muBar with
muBar = 5 (a+1)(a+2) sqrt(pi) Kn / (4 a (5 - 2 w)(7 - 2 w)), a = 1,
C = sqrt(2 R T).  mu does not depend on Kn or L.

Workloads (synthetic; the reference ships no mesh for them):
* ``cavity_case``      2-D lid-driven cavity (the demo/cavity setup,
  demo/cavity/constant/DVMProperties, 0/rho, 0/U, 0/T), n x n cells.
* ``demo_cavity_case`` the demo's own 60 x 60 polyMesh read from a case directory.
* ``cube_case``        3-D lid-driven cube, n^3 cells.
* ``ball_case``        flow past a sphere on a cubed-sphere mesh, far field
  at Mach Ma along +x, isothermal diffuse wall.
* ``channel_case``     2-D channel whose four sides take any patch kind
  (inlet/outlet/walls/symmetry), for the boundary types of
  discreteVelocity::setBCtype.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import meshgen, quadrature

K_BOLTZMANN = 1.38066e-23
M_ARGON = 6.63e-26
D_ARGON = 4.17e-10
R_DEMO = 208.244343891          # demo/cavity/constant/DVMProperties
MU_DEMO = 1.60281882485e-05     # demo/cavity/constant/DVMProperties (Kn 0.075 cavity, T 273)
RHO_DEMO = 1.14423514927e-06    # demo/cavity/0/rho
PR_DEMO = 0.666666666666667
OMEGA_VHS = 0.81


def rho_from_kn(kn: float, L: float) -> float:
    return M_ARGON / (kn * L * math.sqrt(2.0) * math.pi * D_ARGON * D_ARGON)


def mu_bar(kn: float, omega: float) -> float:
    a = 1.0
    return 5.0 * (a + 1.0) * (a + 2.0) * math.sqrt(math.pi) * kn / (4.0 * a * (5.0 - 2 * omega) * (7.0 - 2.0 * omega))


# patch kind (the g/h surface type discreteVelocity::setBCtype picks from
# the rho patch type, discreteVelocity.C:188-195) -> dugks_patch_type
PATCH_TYPES = {"maxwellWall": 1, "farField": 2, "zeroGradient": 3, "mixed": 4, "symmetryPlane": 5,
               "DVMsymmetry": 6, "pressureIn": 7, "pressureOut": 8}
# rho patch type in a case's 0/rho -> patch kind
RHO_PATCH_KINDS = {"calculatedMaxwell": "maxwellWall", "farField": "farField", "zeroGradient": "zeroGradient",
                   "fixedValue": "mixed", "symmetryPlane": "symmetryPlane", "symmetryMod": "DVMsymmetry",
                   "pressureIn": "pressureIn", "pressureOut": "pressureOut"}


@dataclass
class Patch:
    name: str
    kind: str                       # a PATCH_TYPES key or "empty"
    U: tuple = (0.0, 0.0, 0.0)
    T: float = 273.0
    rho: float = 0.0                # farField / mixed patch density
    p: float = 0.0                  # pressureIn / pressureOut value


@dataclass
class Case:
    name: str
    mesh: meshgen.PolyMesh
    D: int
    gas: dict
    xis: np.ndarray
    weights: np.ndarray
    xi_max: float
    patches: list
    rho0: np.ndarray
    U0: np.ndarray
    T0: np.ndarray
    dt: float = 0.0
    macro_flux: bool = False        # fvDVMparas macroFlux yes
    # a DV list instead of the tensor product of xis (the unstructured
    # velocity mesh: xi = vMesh cell centres [n, 3], w = their volumes [n])
    dv_xi: np.ndarray | None = None
    dv_w: np.ndarray | None = None
    vmesh: object = None            # the velocity PolyMesh they came from
    flat: dict = field(default_factory=dict)
    geometry: dict = field(default_factory=dict)

    @property
    def n_cells(self) -> int:
        return self.mesh.n_cells

    @property
    def n_dv(self) -> int:
        if self.dv_w is not None:
            return len(self.dv_w)
        return len(self.xis) ** self.D

    def flatten(self, geometry: dict | None = None) -> "Case":
        """Geometry (OpenFOAM primitiveMesh algorithm) and fv addressing:
        internal faces, then the faces of the non-empty patches."""
        pm = self.mesh
        if geometry is None:
            from . import lib
            geometry = lib.mesh_geometry(pm)
        self.geometry = geometry
        nIF = pm.n_internal_faces
        by_name = {p.name: p for p in self.patches}
        sel = [np.arange(nIF)]
        ptype, pstart = [], [0]
        rho_b, U_b, T_b, p_b = [], [], [], []
        for p in pm.patches:
            spec = by_name.get(p["name"])
            if spec is None:
                raise KeyError(f"no boundary condition for patch {p['name']}")
            if spec.kind == "empty":
                if p["nFaces"] and pm.n_solution_dims == 3:
                    raise ValueError("empty patch on a 3-D mesh")
                continue
            faces = np.arange(p["startFace"], p["startFace"] + p["nFaces"])
            sel.append(faces)
            if spec.kind not in PATCH_TYPES:
                raise ValueError(f"unknown patch kind {spec.kind}")
            ptype.append(PATCH_TYPES[spec.kind])
            pstart.append(pstart[-1] + len(faces))
            # pressureIn/Out and symmetryMod rho patches start at one: their
            # dictionary constructors assign pTraits::one and read no value
            # (pressureInFvPatchField.C:72-75, symmetryModFvPatchField.C:72)
            starts_at_one = spec.kind in ("pressureIn", "pressureOut", "DVMsymmetry")
            rho_b.append(np.full(len(faces), 1.0 if starts_at_one else spec.rho))
            p_b.append(np.full(len(faces), spec.p))
            U_b.append(np.tile(np.asarray(spec.U, dtype=np.float64), (len(faces), 1)))
            T_b.append(np.full(len(faces), spec.T))
        idx = np.concatenate(sel)
        cat = lambda lst, shape: np.concatenate(lst) if lst else np.zeros(shape)
        self.flat = {
            "n_internal": nIF,
            "n_boundary": len(idx) - nIF,
            "owner": pm.owner[idx].astype(np.int64),
            "neighbour": pm.neighbour.astype(np.int64),
            "C": geometry["C"], "V": geometry["V"],
            "Cf": geometry["Cf"][idx], "Sf": geometry["Sf"][idx],
            "patch_type": np.array(ptype, dtype=np.int32),
            "patch_start": np.array(pstart, dtype=np.int32),
            "rho_b": cat(rho_b, (0,)), "U_b": cat(U_b, (0, 3)), "T_b": cat(T_b, (0,)), "p_b": cat(p_b, (0,)),
        }
        if self.dt == 0.0:
            self.dt = cfl_dt(self, 0.5)
        return self

    def dv_set(self) -> tuple[np.ndarray, np.ndarray]:
        if self.dv_w is not None:
            xi = np.array(self.dv_xi, dtype=np.float64).reshape(-1, 3)
            if self.D == 2:
                xi[:, 2] = 0.0
            return xi, np.asarray(self.dv_w, dtype=np.float64)
        return quadrature.tensor_product(self.xis, self.weights, self.D)

    def use_velocity_mesh(self, vmesh, geometry: dict | None = None) -> "Case":
        """DVs from an unstructured velocity mesh (the reference's VMESH
        build, fvDVM.C:166-196): xi = cell centres, weights = cell volumes,
        xiMax = max |xi|."""
        if geometry is None:
            from . import lib
            geometry = lib.mesh_geometry(vmesh)
        xi = np.array(geometry["C"], dtype=np.float64)
        if self.D == 2:
            xi[:, 2] = 0.0
        self.dv_xi = xi
        self.dv_w = np.array(geometry["V"], dtype=np.float64)
        self.vmesh = vmesh
        self.xi_max = float(np.max(np.linalg.norm(xi, axis=1)))
        return self


def cfl_dt(case: Case, co: float) -> float:
    """Time step with Courant number ``co`` for the initial face velocity:
    fvDVM::getCoNum uses deltaCoeffs (|U_f| + sqrt(D) xiMax) (fvDVM.C:2180-2183)."""
    fl = case.flat
    own, nei = fl["owner"][: fl["n_internal"]], fl["neighbour"]
    C = fl["C"]
    d = C[nei] - C[own]
    dc = 1.0 / np.linalg.norm(d, axis=1)
    U = case.U0
    # OpenFOAM linear interpolation weights
    Sf, Cf = fl["Sf"][: fl["n_internal"]], fl["Cf"][: fl["n_internal"]]
    so = np.abs(np.einsum("ij,ij->i", Sf, Cf - C[own]))
    sn = np.abs(np.einsum("ij,ij->i", Sf, C[nei] - Cf))
    w = sn / (so + sn)
    Uf = w[:, None] * (U[own] - U[nei]) + U[nei]
    ubydx = dc * (np.linalg.norm(Uf, axis=1) + math.sqrt(case.D) * case.xi_max)
    return co / ubydx.max()


def _gh_set(n_dv: int, T: float, R: float):
    C = math.sqrt(2.0 * R * T)
    xis, w = quadrature.gauss_hermite_half_range(C, n_dv)
    return xis, w, float(np.max(np.abs(xis)))


def cavity_case(n: int = 61, n_dv: int = 28, kn: float = 0.075, u_lid: float = 50.0, T_wall: float = 273.0,
                T0: float = 273.0, flatten: bool = True, geometry=None) -> Case:
    """2-D lid-driven cavity as demo/cavity (Argon, omega 0.81, Pr 2/3),
    density scaled from the demo's Kn = 0.075 value."""
    mesh = meshgen.cavity(n)
    xis, w, xmax = _gh_set(n_dv, 273.0, R_DEMO)
    gas = {"R": R_DEMO, "omega": OMEGA_VHS, "Tref": 273.0, "muRef": MU_DEMO, "Pr": PR_DEMO, "K": 0}
    rho = RHO_DEMO * 0.075 / kn
    nc = mesh.n_cells
    c = Case(f"cavity{n}x{n}_dv{n_dv}", mesh, 2, gas, xis, w, xmax,
             [Patch("movingWall", "maxwellWall", (u_lid, 0.0, 0.0), T_wall),
              Patch("fixedWalls", "maxwellWall", (0.0, 0.0, 0.0), T_wall),
              Patch("frontAndBack", "empty")],
             np.full(nc, rho), np.zeros((nc, 3)), np.full(nc, T0))
    return c.flatten(geometry) if flatten else c


def refined_cavity_case(n: int = 8, n_dv: int = 8, kn: float = 0.075, u_lid: float = 50.0, T_wall: float = 273.0,
                        T0: float = 273.0, flatten: bool = True, geometry=None) -> Case:
    """The cavity of cavity_case on meshgen.refined_cavity(n): 2:1 refined
    squares beside octagons with eight internal faces."""
    c = cavity_case(2, n_dv, kn=kn, u_lid=u_lid, T_wall=T_wall, T0=T0, flatten=False)
    c.mesh = meshgen.refined_cavity(n)
    nc = c.mesh.n_cells
    c.name = f"refined_cavity{n}x{n}_dv{n_dv}"
    c.rho0 = np.full(nc, float(c.rho0[0]))
    c.U0 = np.zeros((nc, 3))
    c.T0 = np.full(nc, float(c.T0[0]))
    return c.flatten(geometry) if flatten else c


def channel_case(nx: int = 24, ny: int = 12, n_dv: int = 16, sides: dict | None = None, kn: float = 0.1,
                 T0: float = 273.0, U0: tuple = (0.0, 0.0, 0.0), flatten: bool = True, geometry=None) -> Case:
    """2-D channel [0, 2] x [0, 1] of argon at rest (or U0); ``sides`` maps
    inlet / outlet / bottom / top to Patch arguments (kind, U, T, rho, p),
    by default diffuse walls all round."""
    mesh = meshgen.channel(nx, ny)
    xis, w, xmax = _gh_set(n_dv, 273.0, R_DEMO)
    gas = {"R": R_DEMO, "omega": OMEGA_VHS, "Tref": 273.0, "muRef": MU_DEMO, "Pr": PR_DEMO, "K": 0}
    rho = RHO_DEMO * 0.075 / kn
    sides = dict(sides or {})
    patches = []
    for name in ("inlet", "outlet", "bottom", "top"):
        spec = dict(sides.get(name, {"kind": "maxwellWall"}))
        kind = spec.pop("kind")
        patches.append(Patch(name, kind, **spec))
    patches.append(Patch("frontAndBack", "empty"))
    nc = mesh.n_cells
    c = Case(f"channel{nx}x{ny}_dv{n_dv}", mesh, 2, gas, xis, w, xmax, patches, np.full(nc, rho),
             np.tile(np.asarray(U0, dtype=np.float64), (nc, 1)), np.full(nc, T0))
    return c.flatten(geometry) if flatten else c


def demo_cavity_case(case_dir: str, flatten: bool = True, geometry=None, vmesh: bool = False) -> Case:
    """The reference demo cavity read from its case files (polyMesh, Xis,
    weights, DVMProperties, 0/rho, 0/U, 0/T); vmesh: the DVs from
    constant/vMesh instead of Xis and weights."""
    from . import foamio
    mesh = meshgen.read_polymesh(case_dir)
    xis = foamio.read_scalar_list(f"{case_dir}/constant/Xis")
    w = foamio.read_scalar_list(f"{case_dir}/constant/weights")
    props = foamio.read_dict(f"{case_dir}/constant/DVMProperties")
    gp, fp = props["gasProperties"], props["fvDVMparas"]

    def val(v):
        return float(v[-1]) if isinstance(v, list) else float(v)

    gas = {"R": val(gp["R"]), "omega": val(gp["omega"]), "Tref": val(gp["Tref"]), "muRef": val(gp["muRef"]),
           "Pr": val(gp["Pr"]), "K": int(val(gp.get("KInner", 0)))}
    sizes = {p["name"]: p["nFaces"] for p in mesh.patches}
    rho = foamio.read_vol_field(f"{case_dir}/0/rho", mesh.n_cells, sizes)
    U = foamio.read_vol_field(f"{case_dir}/0/U", mesh.n_cells, sizes)
    T = foamio.read_vol_field(f"{case_dir}/0/T", mesh.n_cells, sizes)
    patches = []
    for p in mesh.patches:
        # constraint-type (empty) patches need no field entry
        rtype = rho["patches"][p["name"]]["type"] if p["name"] in rho["patches"] else p["type"]
        if rtype == "empty":
            patches.append(Patch(p["name"], "empty"))
            continue
        uv = U["patches"][p["name"]].get("value")
        tv = T["patches"][p["name"]].get("value")
        rv = rho["patches"][p["name"]].get("value")
        if rtype not in RHO_PATCH_KINDS:
            raise ValueError(f"unsupported rho patch type {rtype}")
        kind = RHO_PATCH_KINDS[rtype]
        pval = rho["patches"][p["name"]].get(kind, 0.0) if kind in ("pressureIn", "pressureOut") else 0.0
        patches.append(Patch(p["name"], kind, tuple(uv[0]) if uv is not None and len(uv) else (0, 0, 0),
                             float(tv[0]) if tv is not None and len(tv) else 273.0,
                             float(rv[0]) if rv is not None and len(rv) else 0.0, float(pval)))
    c = Case("demo_cavity60", mesh, mesh.n_solution_dims, gas, xis, w, val(fp["xiMax"]), patches,
             rho["internal"], U["internal"], T["internal"])
    c.macro_flux = str(fp.get("macroFlux", "no")) == "yes"
    if vmesh:
        c.use_velocity_mesh(meshgen.read_polymesh(case_dir, 3, mesh="vMesh"))
    return c.flatten(geometry) if flatten else c


def cube_case(n: int = 64, n_dv: int = 20, kn: float = 0.1, u_lid: float = 50.0, T_wall: float = 273.0,
              flatten: bool = True, geometry=None) -> Case:
    mesh = meshgen.cube(n)
    xis, w, xmax = _gh_set(n_dv, 273.0, R_DEMO)
    gas = {"R": R_DEMO, "omega": OMEGA_VHS, "Tref": 273.0, "muRef": MU_DEMO, "Pr": PR_DEMO, "K": 0}
    rho = rho_from_kn(kn, 1.0)
    nc = mesh.n_cells
    c = Case(f"cube{n}_dv{n_dv}_kn{kn}", mesh, 3, gas, xis, w, xmax,
             [Patch("movingWall", "maxwellWall", (u_lid, 0.0, 0.0), T_wall),
              Patch("fixedWalls", "maxwellWall", (0.0, 0.0, 0.0), T_wall)],
             np.full(nc, rho), np.zeros((nc, 3)), np.full(nc, T_wall))
    return c.flatten(geometry) if flatten else c


def ball_case(m: int = 24, nr: int = 32, stretch: float = 1.12, n_dv: int = 16, kn: float = 0.1, mach: float = 0.5,
              T_inf: float = 273.0, flatten: bool = True, geometry=None) -> Case:
    """Sphere of radius 1 in a far field of radius 10 (demo/ball shape),
    Kn on the diameter; farField rho/T at the free stream, wall at T_inf."""
    mesh = meshgen.cubed_sphere(m, nr, stretch, 1.0, 10.0)
    R = K_BOLTZMANN / M_ARGON
    xis, w, xmax = _gh_set(n_dv, T_inf, R)
    Cm = math.sqrt(2.0 * R * T_inf)
    rho_inf = rho_from_kn(kn, 2.0)
    mu = rho_inf * Cm * 2.0 * mu_bar(kn, OMEGA_VHS)   # demo/ball/para.py viscosity
    gas = {"R": R, "omega": OMEGA_VHS, "Tref": T_inf, "muRef": mu, "Pr": 2.0 / 3.0, "K": 0}
    u_inf = mach * math.sqrt(5.0 / 3.0 * R * T_inf)
    nc = mesh.n_cells
    U0 = np.zeros((nc, 3))
    U0[:, 0] = u_inf
    c = Case(f"ball{m}x{m}x{nr}_dv{n_dv}", mesh, 3, gas, xis, w, xmax,
             [Patch("wall", "maxwellWall", (0.0, 0.0, 0.0), T_inf),
              Patch("farField", "farField", (u_inf, 0.0, 0.0), T_inf, rho_inf)],
             np.full(nc, rho_inf), U0, np.full(nc, T_inf))
    return c.flatten(geometry) if flatten else c
