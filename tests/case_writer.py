"""Writes a dugksFoam case directory (the files a reference case holds:
constant/polyMesh/{points,faces,owner,neighbour,boundary}, constant/Xis,
constant/weights, constant/DVMProperties, 0/rho, 0/U, 0/T, and optionally
system/controlDict) from a dugks_b200 Case, for tests of the C++ host
driver.  Numbers are written with 17 significant digits so that a reader
gets the same doubles back."""
import os

import numpy as np

_HEADER = "FoamFile\n{{\n    version     2.0;\n    format      ascii;\n    class       {cls};\n    object      {obj};\n}}\n\n"


def _num(x) -> str:
    return repr(float(x))


def _write(path, cls, obj, body):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        f.write(_HEADER.format(cls=cls, obj=obj))
        f.write(body)


def _list(vals) -> str:
    return f"{len(vals)}\n(\n" + "\n".join(vals) + "\n)\n"


def _write_polymesh(pm, mesh):
    _write(os.path.join(mesh, "points"), "vectorField", "points",
           _list(["(%s %s %s)" % tuple(_num(v) for v in p) for p in pm.points]))
    faces = []
    for k in range(pm.n_faces):
        lab = pm.face_points[pm.face_offsets[k]:pm.face_offsets[k + 1]]
        faces.append(f"{len(lab)}(" + " ".join(str(int(v)) for v in lab) + ")")
    _write(os.path.join(mesh, "faces"), "faceList", "faces", _list(faces))
    _write(os.path.join(mesh, "owner"), "labelList", "owner", _list([str(int(v)) for v in pm.owner]))
    _write(os.path.join(mesh, "neighbour"), "labelList", "neighbour", _list([str(int(v)) for v in pm.neighbour]))
    bnd = []
    for p in pm.patches:
        bnd.append(f"{p['name']}\n{{\n    type {p['type']};\n    nFaces {p['nFaces']};\n    startFace {p['startFace']};\n}}")
    _write(os.path.join(mesh, "boundary"), "polyBoundaryMesh", "boundary", _list(bnd))


def write_case(case, directory, control: dict | None = None, rho_patch_type: dict | None = None):
    pm = case.mesh
    if getattr(case, "vmesh", None) is not None:
        _write_polymesh(case.vmesh, os.path.join(directory, "constant", "vMesh"))
    mesh = os.path.join(directory, "constant", "polyMesh")
    _write(os.path.join(mesh, "points"), "vectorField", "points",
           _list(["(%s %s %s)" % tuple(_num(v) for v in p) for p in pm.points]))
    faces = []
    for k in range(pm.n_faces):
        lab = pm.face_points[pm.face_offsets[k]:pm.face_offsets[k + 1]]
        faces.append(f"{len(lab)}(" + " ".join(str(int(v)) for v in lab) + ")")
    _write(os.path.join(mesh, "faces"), "faceList", "faces", _list(faces))
    _write(os.path.join(mesh, "owner"), "labelList", "owner", _list([str(int(v)) for v in pm.owner]))
    _write(os.path.join(mesh, "neighbour"), "labelList", "neighbour", _list([str(int(v)) for v in pm.neighbour]))
    bnd = []
    for p in pm.patches:
        bnd.append(f"{p['name']}\n{{\n    type {p['type']};\n    nFaces {p['nFaces']};\n    startFace {p['startFace']};\n}}")
    _write(os.path.join(mesh, "boundary"), "polyBoundaryMesh", "boundary", _list(bnd))

    const = os.path.join(directory, "constant")
    _write(os.path.join(const, "Xis"), "scalarList", "Xis", _list([_num(v) for v in case.xis]))
    _write(os.path.join(const, "weights"), "scalarList", "weights", _list([_num(v) for v in case.weights]))
    g = case.gas
    props = (
        "fvDVMparas\n{\n"
        f"    xiMax   xiMax [0 1 -1 0 0 0 0] {_num(case.xi_max)};\n"
        f"    xiMin   xiMin [0 1 -1 0 0 0 0] {_num(-case.xi_max)};\n"
        f"    nDV     {len(case.xis)};\n"
        f"    macroFlux {'yes' if getattr(case, 'macro_flux', False) else 'no'};\n}}\n\n"
        "gasProperties\n{\n"
        f"    R       R [0 2 -2 -1 0 0 0] {_num(g['R'])};\n"
        f"    omega   {_num(g['omega'])};\n"
        f"    Tref    Tref [0 0 0 1 0 0 0] {_num(g['Tref'])};\n"
        f"    muRef   muRef [1 -1 -1 0 0 0 0] {_num(g['muRef'])};\n"
        f"    Pr      {_num(g['Pr'])};\n"
        f"    KInner  {int(g.get('K', 0))};\n}}\n")
    _write(os.path.join(const, "DVMProperties"), "dictionary", "DVMProperties", props)

    by_name = {p.name: p for p in case.patches}
    rtypes = rho_patch_type or {}

    def field(name, cls, internal, dims, entry):
        vec = cls == "volVectorField"
        t = "vector" if vec else "scalar"
        vals = ["(%s %s %s)" % tuple(_num(x) for x in v) for v in internal] if vec else [_num(v) for v in internal]
        body = f"dimensions      {dims};\n\ninternalField   nonuniform List<{t}>\n" + _list(vals) + ";\n\nboundaryField\n{\n"
        for p in pm.patches:
            body += f"    {p['name']}\n    {{\n{entry(by_name[p['name']], p)}    }}\n"
        body += "}\n"
        _write(os.path.join(directory, "0", name), cls, name, body)

    rho_types = {"maxwellWall": "calculatedMaxwell", "farField": "farField", "zeroGradient": "zeroGradient",
                 "mixed": "fixedValue", "symmetryPlane": "symmetryPlane", "DVMsymmetry": "symmetryMod",
                 "pressureIn": "pressureIn", "pressureOut": "pressureOut"}

    def rho_entry(s, p):
        if s.kind == "empty":
            return "        type            empty;\n"
        t = rtypes.get(p['name'], rho_types[s.kind])
        if s.kind in ("farField", "mixed"):
            return f"        type            {t};\n        value           uniform {_num(s.rho)};\n"
        if s.kind in ("pressureIn", "pressureOut"):
            return f"        type            {t};\n        {s.kind}      {_num(s.p)};\n"
        if s.kind in ("zeroGradient", "symmetryPlane", "DVMsymmetry"):
            return f"        type            {t};\n"
        return f"        type            {t};\n        value           uniform {_num(case.rho0[0])};\n"

    def u_entry(s, p):
        if s.kind == "empty":
            return "        type            empty;\n"
        return "        type            fixedValue;\n        value           uniform (%s %s %s);\n" % tuple(
            _num(v) for v in s.U)

    def t_entry(s, p):
        if s.kind == "empty":
            return "        type            empty;\n"
        return f"        type            fixedValue;\n        value           uniform {_num(s.T)};\n"

    field("rho", "volScalarField", case.rho0, "[1 -3 0 0 0 0 0]", rho_entry)
    field("U", "volVectorField", np.asarray(case.U0).reshape(-1, 3), "[0 1 -1 0 0 0 0]", u_entry)
    field("T", "volScalarField", case.T0, "[0 0 0 1 0 0 0]", t_entry)
    if control:
        body = "".join(f"{k} {_num(v) if isinstance(v, float) else v};\n" for k, v in control.items())
        _write(os.path.join(directory, "system", "controlDict"), "dictionary", "controlDict", body)
    return directory
