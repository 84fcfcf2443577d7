"""Synthetic OpenFOAM-style polyMesh generators for the DUGKS workloads.

A mesh is returned as a :class:`PolyMesh` holding what ``constant/polyMesh``
holds: points, faces (CSR), owner (all faces), neighbour (internal faces)
and the boundary patch list.  Internal faces are in OpenFOAM's
upper-triangular order (owner ascending, then neighbour ascending,
owner < neighbour); boundary faces follow, grouped by patch.  Every face is
oriented so that its right-hand normal points out of its owner cell.

Workloads:
* ``cavity(n)``    -- n x n x 1 hexes on [0,1]^2 x [0,0.1] (the reference
  cavity demo's domain, demo/cavity/constant/polyMesh/blockMeshDict:17-47),
  patches movingWall (y = 1), fixedWalls, frontAndBack (empty).
* ``cube(n)``      -- n^3 hexes on [0,1]^3, lid (y = 1) + fixed walls.
* ``cubed_sphere(m, nr, stretch, r0, r1)`` -- 6 patches x m x m x nr hexes
  between spheres of radius r0 and r1, equiangular cube-face mapping and
  geometric radial stretching; patches ``wall`` (r = r0) and ``farField``
  (r = r1).
* ``refined_cavity(n)`` -- the cavity's domain as n x n squares of which
  every other one (checkerboard) is split into 2 x 2: the unsplit squares
  are octagons with a hanging node on every side, so an interior one has
  eight internal faces (ten with front and back), as a 2:1 refined
  OpenFOAM mesh has.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# outward-oriented faces of an OpenFOAM hex (vertices 0-3 at the low third
# coordinate, 4-7 at the high one)
_HEX_FACES = np.array([
    [0, 4, 7, 3],  # -x
    [1, 2, 6, 5],  # +x
    [0, 1, 5, 4],  # -y
    [3, 7, 6, 2],  # +y
    [0, 3, 2, 1],  # -z
    [4, 5, 6, 7],  # +z
], dtype=np.int64)


@dataclass
class PolyMesh:
    points: np.ndarray                 # [nPoints, 3]
    face_offsets: np.ndarray           # [nFaces + 1]
    face_points: np.ndarray            # point labels
    owner: np.ndarray                  # [nFaces]
    neighbour: np.ndarray              # [nInternalFaces]
    n_cells: int
    patches: list = field(default_factory=list)   # dicts: name, type, startFace, nFaces
    n_solution_dims: int = 3

    @property
    def n_faces(self) -> int:
        return len(self.owner)

    @property
    def n_internal_faces(self) -> int:
        return len(self.neighbour)

    def patch(self, name: str) -> dict:
        for p in self.patches:
            if p["name"] == name:
                return p
        raise KeyError(name)


def _signed_volumes(pts: np.ndarray, cells: np.ndarray) -> np.ndarray:
    """Approximate signed volume of each hex (from the diagonal triple product)."""
    p = pts[cells]
    a = p[:, 1] - p[:, 0]
    b = p[:, 3] - p[:, 0]
    c = p[:, 4] - p[:, 0]
    return np.einsum("ij,ij->i", np.cross(a, b), c)


def hexes_to_polymesh(points: np.ndarray, cells: np.ndarray, classify, patch_defs: list[tuple[str, str]],
                      n_solution_dims: int = 3) -> PolyMesh:
    """Build a polyMesh from hex cells.

    ``classify(face_centres) -> patch index`` assigns boundary faces to the
    patches of ``patch_defs`` = [(name, type)], in that order.
    """
    cells = np.asarray(cells, dtype=np.int64)
    vol = _signed_volumes(points, cells)
    flip = vol < 0
    if np.any(flip):
        c = cells[flip].copy()
        cells[flip] = c[:, [0, 3, 2, 1, 4, 7, 6, 5]]
    nc = len(cells)
    fverts = cells[:, _HEX_FACES]            # [nc, 6, 4]
    fverts = fverts.reshape(-1, 4)
    fcell = np.repeat(np.arange(nc, dtype=np.int64), 6)
    key = np.sort(fverts, axis=1)
    order = np.lexsort(key.T[::-1])
    key_s = key[order]
    same = np.all(key_s[1:] == key_s[:-1], axis=1)
    # pairs: positions i where key_s[i] == key_s[i+1]
    pair_i = np.nonzero(same)[0]
    is_paired = np.zeros(len(order), dtype=bool)
    is_paired[pair_i] = True
    is_paired[pair_i + 1] = True
    a = order[pair_i]
    b = order[pair_i + 1]
    ca, cb = fcell[a], fcell[b]
    own = np.minimum(ca, cb)
    nei = np.maximum(ca, cb)
    # face orientation: as seen from the owner (outward from owner)
    fv_int = np.where((ca <= cb)[:, None], fverts[a], fverts[b])
    o = np.lexsort((nei, own))
    own, nei, fv_int = own[o], nei[o], fv_int[o]
    # boundary faces
    bidx = order[~is_paired]
    bcell = fcell[bidx]
    bverts = fverts[bidx]
    bcent = points[bverts].mean(axis=1)
    pid = np.asarray(classify(bcent), dtype=np.int64)
    patches = []
    blocks_v, blocks_o = [], []
    start = len(own)
    for k, (name, ptype) in enumerate(patch_defs):
        sel = np.nonzero(pid == k)[0]
        sel = sel[np.lexsort((bidx[sel], bcell[sel]))]
        blocks_v.append(bverts[sel])
        blocks_o.append(bcell[sel])
        patches.append({"name": name, "type": ptype, "startFace": start, "nFaces": len(sel)})
        start += len(sel)
    if np.any((pid < 0) | (pid >= len(patch_defs))):
        raise ValueError("unclassified boundary faces")
    allv = np.concatenate([fv_int] + blocks_v)
    owner = np.concatenate([own] + blocks_o)
    offs = np.arange(0, 4 * len(allv) + 1, 4, dtype=np.int64)
    return PolyMesh(points=np.ascontiguousarray(points, dtype=np.float64), face_offsets=offs,
                    face_points=allv.reshape(-1).astype(np.int64), owner=owner.astype(np.int64),
                    neighbour=nei.astype(np.int64), n_cells=nc, patches=patches,
                    n_solution_dims=n_solution_dims)


def polygons_to_polymesh(points2d: np.ndarray, cells: list, classify, patch_defs: list[tuple[str, str]],
                         thickness: float = 0.1) -> PolyMesh:
    """Build a one-cell-thick 2-D polyMesh from polygon cells.

    ``cells[c]`` lists cell c's vertices (indices into ``points2d``)
    counter-clockwise; neighbouring cells must share whole edges.  Every
    edge becomes a quad face extruded to ``thickness``; each cell also gets
    a front (z = 0) and a back (z = thickness) face, both classified like
    the edge faces: ``classify(face_centres) -> patch index`` of
    ``patch_defs``.
    """
    pts2 = np.asarray(points2d, dtype=np.float64)
    npt = len(pts2)
    points = np.concatenate([np.column_stack([pts2, np.zeros(npt)]),
                             np.column_stack([pts2, np.full(npt, thickness)])])
    edge_cell = {}
    internal, boundary = [], []
    for c, poly in enumerate(cells):
        for k in range(len(poly)):
            a, b = int(poly[k]), int(poly[(k + 1) % len(poly)])
            if (b, a) in edge_cell:
                o = edge_cell.pop((b, a))
                # the owner is the lower cell; the face keeps the owner's
                # counter-clockwise edge direction, so its normal leaves the owner
                if o[0] < c:
                    internal.append((o[0], c, o[1], o[2]))
                else:
                    internal.append((c, o[0], a, b))
            else:
                edge_cell[(a, b)] = (c, a, b)
    for (a, b), (c, _, _) in edge_cell.items():
        boundary.append((c, [a, b, b + npt, a + npt]))
    for c, poly in enumerate(cells):
        boundary.append((c, [int(v) for v in poly[::-1]]))          # front, normal -z
        boundary.append((c, [int(v) + npt for v in poly]))          # back, normal +z
    internal.sort(key=lambda f: (f[0], f[1]))
    faces = [[a, b, b + npt, a + npt] for (_, _, a, b) in internal]
    owner = [f[0] for f in internal]
    neighbour = [f[1] for f in internal]
    bcent = np.array([points[fv].mean(axis=0) for _, fv in boundary])
    pid = np.asarray(classify(bcent), dtype=np.int64)
    if np.any((pid < 0) | (pid >= len(patch_defs))):
        raise ValueError("unclassified boundary faces")
    patches = []
    for k, (name, ptype) in enumerate(patch_defs):
        sel = sorted(np.nonzero(pid == k)[0], key=lambda i: boundary[i][0])
        patches.append({"name": name, "type": ptype, "startFace": len(faces), "nFaces": len(sel)})
        for i in sel:
            owner.append(boundary[i][0])
            faces.append(boundary[i][1])
    offs = np.concatenate([[0], np.cumsum([len(f) for f in faces])]).astype(np.int64)
    return PolyMesh(points=np.ascontiguousarray(points), face_offsets=offs,
                    face_points=np.concatenate(faces).astype(np.int64), owner=np.asarray(owner, dtype=np.int64),
                    neighbour=np.asarray(neighbour, dtype=np.int64), n_cells=len(cells), patches=patches,
                    n_solution_dims=2)


def refined_cavity(n: int, thickness: float = 0.1) -> PolyMesh:
    """[0,1]^2 x [0, thickness] as n x n squares, those with i + j even split
    into 2 x 2; the others are octagons through the midpoints of their
    sides.  Patches as ``cavity``: movingWall (y = 1), fixedWalls,
    frontAndBack (empty)."""
    m = 2 * n + 1                                   # lattice of half squares

    def pid(i, j):
        return j * m + i

    X, Y = np.meshgrid(np.linspace(0.0, 1.0, m), np.linspace(0.0, 1.0, m))
    pts = np.column_stack([X.ravel(), Y.ravel()])
    cells = []
    for j in range(n):
        for i in range(n):
            I, J = 2 * i, 2 * j
            if (i + j) % 2 == 0:
                for dj in (0, 1):
                    for di in (0, 1):
                        a, b = I + di, J + dj
                        cells.append([pid(a, b), pid(a + 1, b), pid(a + 1, b + 1), pid(a, b + 1)])
            else:
                cells.append([pid(I, J), pid(I + 1, J), pid(I + 2, J), pid(I + 2, J + 1), pid(I + 2, J + 2),
                              pid(I + 1, J + 2), pid(I, J + 2), pid(I, J + 1)])
    tol = 1e-9

    def classify(c):
        out = np.full(len(c), 1, dtype=np.int64)       # fixedWalls
        out[np.abs(c[:, 1] - 1.0) < tol] = 0           # movingWall
        out[(np.abs(c[:, 2]) < tol) | (np.abs(c[:, 2] - thickness) < tol)] = 2
        return out

    return polygons_to_polymesh(pts, cells, classify,
                                [("movingWall", "wall"), ("fixedWalls", "wall"), ("frontAndBack", "empty")],
                                thickness)


def _box_hexes(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float):
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    zs = np.linspace(0.0, lz, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    def pid(i, j, k):
        return (k * (ny + 1) + j) * (nx + 1) + i

    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    cells = np.stack([pid(i, j, k), pid(i + 1, j, k), pid(i + 1, j + 1, k), pid(i, j + 1, k),
                      pid(i, j, k + 1), pid(i + 1, j, k + 1), pid(i + 1, j + 1, k + 1), pid(i, j + 1, k + 1)], axis=1)
    return pts, cells


def cavity(n: int, thickness: float = 0.1) -> PolyMesh:
    pts, cells = _box_hexes(n, n, 1, 1.0, 1.0, thickness)
    tol = 1e-9

    def classify(c):
        out = np.full(len(c), 1, dtype=np.int64)       # fixedWalls
        out[np.abs(c[:, 1] - 1.0) < tol] = 0           # movingWall
        out[(np.abs(c[:, 2]) < tol) | (np.abs(c[:, 2] - thickness) < tol)] = 2
        return out

    return hexes_to_polymesh(pts, cells, classify,
                             [("movingWall", "wall"), ("fixedWalls", "wall"), ("frontAndBack", "empty")],
                             n_solution_dims=2)


def channel(nx: int, ny: int, lx: float = 2.0, ly: float = 1.0, thickness: float = 0.1) -> PolyMesh:
    """2-D channel [0, lx] x [0, ly]: patches inlet (x = 0), outlet (x = lx),
    bottom (y = 0), top (y = ly), frontAndBack (empty)."""
    pts, cells = _box_hexes(nx, ny, 1, lx, ly, thickness)
    tol = 1e-9

    def classify(c):
        out = np.full(len(c), -1, dtype=np.int64)
        out[np.abs(c[:, 0]) < tol] = 0
        out[np.abs(c[:, 0] - lx) < tol] = 1
        out[np.abs(c[:, 1]) < tol] = 2
        out[np.abs(c[:, 1] - ly) < tol] = 3
        out[(np.abs(c[:, 2]) < tol) | (np.abs(c[:, 2] - thickness) < tol)] = 4
        return out

    return hexes_to_polymesh(pts, cells, classify,
                             [("inlet", "patch"), ("outlet", "patch"), ("bottom", "wall"), ("top", "wall"),
                              ("frontAndBack", "empty")], n_solution_dims=2)


def velocity_box(n: int, half_width: float, D: int, jitter: float = 0.0, seed: int = 7,
                 thickness: float = 1.0) -> PolyMesh:
    """An unstructured-looking velocity mesh: the box [-L, L]^D in n cells per
    direction (2-D: one cell of ``thickness`` in z, whose volume is the DV
    weight), interior points moved by up to ``jitter`` of a cell width so
    that the cell centres are no tensor product."""
    nz = n if D == 3 else 1
    lz = 2.0 * half_width if D == 3 else thickness
    pts, cells = _box_hexes(n, n, nz, 2.0 * half_width, 2.0 * half_width, lz)
    pts = pts.copy()
    pts[:, 0] -= half_width
    pts[:, 1] -= half_width
    if D == 3:
        pts[:, 2] -= half_width
    if jitter > 0:
        rng = np.random.default_rng(seed)
        h = 2.0 * half_width / n
        inner = np.all(np.abs(pts[:, :D]) < half_width - 1e-9 * half_width, axis=1)
        pts[inner, :D] += rng.uniform(-jitter * h, jitter * h, size=(int(inner.sum()), D))
    tol = 1e-9 * half_width

    def classify(c):
        return np.zeros(len(c), dtype=np.int64)

    return hexes_to_polymesh(pts, cells, classify, [("outside", "patch")], n_solution_dims=D)


def cube(n: int) -> PolyMesh:
    pts, cells = _box_hexes(n, n, n, 1.0, 1.0, 1.0)
    tol = 1e-9

    def classify(c):
        out = np.full(len(c), 1, dtype=np.int64)
        out[np.abs(c[:, 1] - 1.0) < tol] = 0
        return out

    return hexes_to_polymesh(pts, cells, classify, [("movingWall", "wall"), ("fixedWalls", "wall")],
                             n_solution_dims=3)


def radial_stations(nr: int, stretch: float, r0: float, r1: float) -> np.ndarray:
    """nr+1 radii from r0 to r1 with cell sizes growing by ``stretch``."""
    g = stretch ** np.arange(nr + 1) - 1.0
    return r0 + (r1 - r0) * g / g[-1]


def cubed_sphere(m: int = 24, nr: int = 32, stretch: float = 1.12, r0: float = 1.0, r1: float = 10.0) -> PolyMesh:
    if m % 2:
        raise ValueError("m must be even")
    h = m // 2
    # equiangular coordinate per lattice index, exact +-1 at the cube edges
    lat = np.tan(np.pi / 4.0 * np.arange(-h, h + 1) / h)
    lat[0], lat[h], lat[-1] = -1.0, 0.0, 1.0
    # unique lattice points on the cube surface
    idx = np.arange(-h, h + 1)
    I, J, K = np.meshgrid(idx, idx, idx, indexing="ij")
    surf = (np.abs(I) == h) | (np.abs(J) == h) | (np.abs(K) == h)
    I, J, K = I[surf], J[surf], K[surf]
    n_surf = len(I)
    lookup = -np.ones((m + 1, m + 1, m + 1), dtype=np.int64)
    lookup[I + h, J + h, K + h] = np.arange(n_surf)
    d = np.stack([lat[I + h], lat[J + h], lat[K + h]], axis=1)
    d /= np.linalg.norm(d, axis=1)[:, None]
    radii = radial_stations(nr, stretch, r0, r1)
    pts = (radii[:, None, None] * d[None, :, :]).reshape(-1, 3)

    def pidx(surf_id, kr):
        return kr * n_surf + surf_id

    cells = []
    a, b = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    a, b = a.ravel(), b.ravel()
    faces = [(0, +1), (0, -1), (1, +1), (1, -1), (2, +1), (2, -1)]
    for axis, sign in faces:
        others = [ax for ax in range(3) if ax != axis]

        def sid(u, v):
            c = [None, None, None]
            c[axis] = np.full_like(u, h * sign + h)
            c[others[0]] = u
            c[others[1]] = v
            return lookup[c[0], c[1], c[2]]

        s00, s10, s11, s01 = sid(a, b), sid(a + 1, b), sid(a + 1, b + 1), sid(a, b + 1)
        for kr in range(nr):
            cells.append(np.stack([pidx(s00, kr), pidx(s10, kr), pidx(s11, kr), pidx(s01, kr),
                                   pidx(s00, kr + 1), pidx(s10, kr + 1), pidx(s11, kr + 1), pidx(s01, kr + 1)],
                                  axis=1))
    cells = np.concatenate(cells)
    rmid = 0.5 * (r0 + r1)

    def classify(c):
        r = np.linalg.norm(c, axis=1)
        return np.where(r < rmid, 0, 1)

    return hexes_to_polymesh(pts, cells, classify, [("wall", "wall"), ("farField", "patch")], n_solution_dims=3)


def read_polymesh(case_dir: str, n_solution_dims: int | None = None, mesh: str = "polyMesh") -> PolyMesh:
    """Read ``constant/<mesh>`` of an OpenFOAM case (polyMesh, or vMesh for
    the velocity mesh)."""
    from . import foamio
    base = f"{case_dir}/constant/{mesh}"
    pts = foamio.read_points(f"{base}/points")
    offs, labels = foamio.read_faces(f"{base}/faces")
    owner = foamio.read_label_list(f"{base}/owner")
    nei = foamio.read_label_list(f"{base}/neighbour")
    patches = foamio.read_boundary(f"{base}/boundary")
    n_cells = int(max(owner.max(), nei.max() if len(nei) else 0)) + 1
    if n_solution_dims is None:
        n_solution_dims = 3 - sum(1 for p in patches if p["type"] == "empty" and p["nFaces"] > 0)
    return PolyMesh(points=pts, face_offsets=offs, face_points=labels, owner=owner, neighbour=nei,
                    n_cells=n_cells, patches=patches, n_solution_dims=n_solution_dims)
