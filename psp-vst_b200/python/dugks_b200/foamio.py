"""Minimal reader/writer for the OpenFOAM ASCII files a dugksFoam case uses.

Read: dictionaries (``constant/DVMProperties``, ``system/controlDict``,
``constant/polyMesh/boundary``), scalar lists (``constant/Xis``,
``constant/weights``, ``polyMesh/owner``/``neighbour``), point and face
lists (``polyMesh/points``, ``polyMesh/faces``) and volume fields
(``0/rho``, ``0/U``, ``0/T``).  Write: volume fields in the same layout
``runTime.write()`` produces for the AUTO_WRITE macro fields
(src/dugksFoam.C:83; fields declared in src/createFields.H:1-38 and
src/fvDVM/fvDVM/fvDVM.C:2016-2105).

This is host I/O only; OpenFOAM itself is not needed.
"""
from __future__ import annotations

import os
import re

import numpy as np

_TOKEN = re.compile(r'"[^"]*"|[(){}\[\];]|[^\s(){}\[\];"]+')


def _strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    return text


def tokenize(text: str) -> list[str]:
    return _TOKEN.findall(_strip_comments(text))


def _is_number(tok: str) -> bool:
    try:
        float(tok)
        return True
    except ValueError:
        return False


class _Parser:
    def __init__(self, toks: list[str]):
        self.t = toks
        self.i = 0

    def peek(self, k: int = 0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else None

    def next(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def expect(self, tok: str):
        got = self.next()
        if got != tok:
            raise ValueError(f"expected {tok!r}, got {got!r} at token {self.i}")

    def parse_dict_body(self, end: str | None = "}") -> dict:
        out: dict = {}
        while True:
            tok = self.peek()
            if tok is None:
                if end is None:
                    return out
                raise ValueError("unterminated dictionary")
            if tok == end:
                self.next()
                return out
            key = self.next().strip('"')
            if self.peek() == "{":
                self.next()
                out[key] = self.parse_dict_body("}")
                continue
            vals = []
            while self.peek() != ";":
                vals.append(self.parse_value())
            self.next()
            out[key] = vals[0] if len(vals) == 1 else vals
        return out

    def parse_value(self):
        tok = self.peek()
        if tok == "(":
            return self.parse_list_body()
        if tok == "[":
            self.next()
            dims = []
            while self.peek() != "]":
                dims.append(float(self.next()))
            self.next()
            return ("dims", dims)
        if tok == "{":
            self.next()
            return self.parse_dict_body("}")
        self.next()
        if _is_number(tok) and self.peek() == "(":
            # counted list "N ( ... )"
            return self.parse_list_body()
        if _is_number(tok) and self.peek() == "{":
            # uniform list "N{value}"
            self.next()
            v = self.parse_value()
            self.expect("}")
            return [v] * int(tok)
        if _is_number(tok):
            return float(tok) if any(c in tok for c in ".eE") else int(tok)
        return tok

    def parse_list_body(self):
        self.expect("(")
        items = []
        while self.peek() != ")":
            items.append(self.parse_value())
        self.next()
        return items


def read_dict(path: str) -> dict:
    with open(path) as f:
        p = _Parser(tokenize(f.read()))
    d = p.parse_dict_body(end=None)
    d.pop("FoamFile", None)
    return d


def _read_body_tokens(path: str) -> list[str]:
    with open(path) as f:
        toks = tokenize(f.read())
    # drop the FoamFile header block
    if toks and toks[0] == "FoamFile":
        depth = 0
        for k, tok in enumerate(toks):
            if tok == "{":
                depth += 1
            elif tok == "}":
                depth -= 1
                if depth == 0:
                    return toks[k + 1:]
    return toks


def read_scalar_list(path: str) -> np.ndarray:
    """A counted scalar/label list (Xis, weights, owner, neighbour)."""
    toks = _read_body_tokens(path)
    n = int(toks[0])
    if toks[1] == "{":
        return np.full(n, float(toks[2]))
    assert toks[1] == "(", path
    vals = toks[2:2 + n]
    assert toks[2 + n] == ")", path
    return np.array([float(v) for v in vals])


def read_label_list(path: str) -> np.ndarray:
    return read_scalar_list(path).astype(np.int64)


def read_points(path: str) -> np.ndarray:
    toks = _read_body_tokens(path)
    n = int(toks[0])
    body = [t for t in toks[1:] if t not in ("(", ")")]
    arr = np.array([float(v) for v in body[: 3 * n]]).reshape(n, 3)
    return arr


def read_faces(path: str) -> tuple[np.ndarray, np.ndarray]:
    """faceList -> (offsets [nFaces+1], point labels)."""
    toks = _read_body_tokens(path)
    n = int(toks[0])
    assert toks[1] == "("
    k = 2
    offsets = [0]
    labels: list[int] = []
    for _ in range(n):
        m = int(toks[k])
        assert toks[k + 1] == "("
        labels.extend(int(v) for v in toks[k + 2:k + 2 + m])
        assert toks[k + 2 + m] == ")"
        k += m + 3
        offsets.append(len(labels))
    return np.array(offsets, dtype=np.int64), np.array(labels, dtype=np.int64)


def read_boundary(path: str) -> list[dict]:
    toks = _read_body_tokens(path)
    p = _Parser(toks)
    p.next()  # count
    lst = p.parse_list_body()
    patches = []
    # list body parses as alternating name, dict
    for k in range(0, len(lst), 2):
        d = dict(lst[k + 1])
        d["name"] = lst[k]
        d["nFaces"] = int(d["nFaces"])
        d["startFace"] = int(d["startFace"])
        patches.append(d)
    return patches


def _field_value(v, ncomp: int, n: int) -> np.ndarray:
    """Decode 'uniform x' / 'nonuniform List<T> N(...)' entries."""
    if isinstance(v, list) and v and v[0] == "uniform":
        x = v[1]
        arr = np.array(x if isinstance(x, list) else [x], dtype=np.float64)
        return np.tile(arr, (n, 1)) if ncomp > 1 else np.full(n, float(arr[0]))
    if isinstance(v, list) and v and v[0] == "nonuniform":
        data = v[-1]
        arr = np.array(data, dtype=np.float64)
        return arr.reshape(-1, ncomp) if ncomp > 1 else arr.reshape(-1)
    raise ValueError(f"unsupported field value {v!r}")


def read_vol_field(path: str, n_cells: int, patch_sizes: dict[str, int]) -> dict:
    """Read a volScalarField/volVectorField: returns
    {'internal': array, 'patches': {name: {'type': str, 'value': array|None, ...}}}."""
    d = read_dict(path)
    with open(path) as f:
        head = f.read(2000)
    ncomp = 3 if "volVectorField" in head else 1
    internal = _field_value(d["internalField"], ncomp, n_cells)
    patches = {}
    for name, pd in d.get("boundaryField", {}).items():
        entry = {k: v for k, v in pd.items()}
        size = patch_sizes.get(name.strip('"'), 0)
        if "value" in pd:
            entry["value"] = _field_value(pd["value"], ncomp, size)
        patches[name.strip('"')] = entry
    return {"internal": internal, "patches": patches, "ncomp": ncomp}


def write_vol_field(path: str, name: str, internal: np.ndarray, patches: list[tuple[str, str, np.ndarray | None]],
                    dims: str, location: str) -> None:
    """Write a vol field; ``patches`` = [(name, type, values-or-None)]."""
    vec = internal.ndim == 2
    cls = "volVectorField" if vec else "volScalarField"

    def fmt(v):
        if vec:
            return "(%.12g %.12g %.12g)" % tuple(v)
        return "%.12g" % v

    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        f.write("FoamFile\n{\n    version     2.0;\n    format      ascii;\n"
                f"    class       {cls};\n    location    \"{location}\";\n    object      {name};\n}}\n\n")
        f.write(f"dimensions      {dims};\n\n")
        f.write(f"internalField   nonuniform List<{'vector' if vec else 'scalar'}>\n{len(internal)}\n(\n")
        for v in internal:
            f.write(fmt(v) + "\n")
        f.write(")\n;\n\nboundaryField\n{\n")
        for pname, ptype, vals in patches:
            f.write(f"    {pname}\n    {{\n        type            {ptype};\n")
            if vals is not None and len(vals) > 0:
                f.write(f"        value           nonuniform List<{'vector' if vec else 'scalar'}> {len(vals)}(")
                f.write(" ".join(fmt(v) for v in vals))
                f.write(");\n")
            f.write("    }\n")
        f.write("}\n")
