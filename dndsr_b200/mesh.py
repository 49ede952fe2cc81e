"""Synthetic unstructured meshes in the structure-of-arrays layout the C-ABI takes.

The reference reads CGNS meshes and builds face/ghost connectivity
(src/Geom/Mesh/Mesh.hpp, Mesh_Serial_ReadFromCGNS.cpp).  Here the meshes are
generated directly, with the same topological conventions the reference relies
on:

* every cell row lists its faces (``cell2face``, the reference's
  ``mesh->cell2face``) and every face lists its two cells (``face2cell``;
  side 1 is ``-1`` on a boundary face, like ``UnInitIndex``);
* a face's node order makes its normal point out of ``face2cell[f, 0]``
  (the reference asserts this in FiniteVolume.cpp ConstructFaceMeanNorm);
* periodic meshes carry, per face, the translation that maps a point seen from
  cell 0 into the frame of cell 1 (``face_pshift``).  Pure translation
  periodicity is all the reference's IV/TGV/box cases use
  (Geom/PeriodicInfo.hpp TransCoord with an identity rotation).

Geometry is stored as node coordinates plus per cell-vertex (and face-vertex)
image offsets, so that each cell is geometrically contiguous even when its
nodes wrap around a periodic boundary, and derivatives with respect to node
coordinates still land on the shared node.
"""
from __future__ import annotations

import dataclasses
import numpy as np

# element kinds; the integer values are the C-ABI's DNDSB_ELEM_* codes
TRI3, QUAD4, TET4, HEX8 = 1, 2, 3, 4

# local faces, ordered so that each face normal points out of the cell
_LOCAL_FACES = {
    TRI3: [(0, 1), (1, 2), (2, 0)],
    QUAD4: [(0, 1), (1, 2), (2, 3), (3, 0)],
    TET4: [(0, 2, 1), (0, 1, 3), (0, 3, 2), (1, 2, 3)],
    HEX8: [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)],
}
_DIM = {TRI3: 2, QUAD4: 2, TET4: 3, HEX8: 3}

# boundary zone codes: 0 is an interior (or periodic) face; >0 indexes the BC table
ZONE_INTERIOR = 0


@dataclasses.dataclass
class Mesh:
    dim: int
    cell_type: int
    coords: np.ndarray        # (nNode, 3) float64
    cell2node: np.ndarray     # (nCell, nv) int64
    cell_shift: np.ndarray    # (nCell, nv, 3) float64, image offset of each cell vertex
    face2node: np.ndarray     # (nFace, nfv) int64, in face2cell[f,0]'s orientation
    face_shift: np.ndarray    # (nFace, nfv, 3) float64, image offsets in cell 0's frame
    face2cell: np.ndarray     # (nFace, 2) int64, -1 on boundary side 1
    face_zone: np.ndarray     # (nFace,) int32, 0 interior/periodic, >0 boundary zone id
    face_pshift: np.ndarray   # (nFace, 3) float64, cell-0 frame -> cell-1 frame translation
    cell2face: np.ndarray     # (nCell, nf) int64
    face_type: int            # element kind of the faces (line=0, TRI3, QUAD4)

    @property
    def n_cell(self):
        return self.cell2node.shape[0]

    @property
    def n_face(self):
        return self.face2node.shape[0]

    @property
    def n_node(self):
        return self.coords.shape[0]

    def cell_coords(self):
        """(nCell, nv, 3) vertex coordinates of each cell in its own frame."""
        return self.coords[self.cell2node] + self.cell_shift

    def face_coords(self):
        """(nFace, nfv, 3) vertex coordinates of each face in cell 0's frame."""
        return self.coords[self.face2node] + self.face_shift

    def arrays(self):
        """Contiguous arrays in the order the C-ABI mesh constructor takes them."""
        c = np.ascontiguousarray
        return dict(
            coords=c(self.coords, dtype=np.float64),
            cell2node=c(self.cell2node, dtype=np.int64),
            cell_shift=c(self.cell_shift, dtype=np.float64),
            face2node=c(self.face2node, dtype=np.int64),
            face_shift=c(self.face_shift, dtype=np.float64),
            face2cell=c(self.face2cell, dtype=np.int64),
            face_zone=c(self.face_zone, dtype=np.int32),
            face_pshift=c(self.face_pshift, dtype=np.float64),
            cell2face=c(self.cell2face, dtype=np.int64),
        )


def _build_faces(cell_type, cell2node, cell_shift, zone_of_face_key=None):
    """Derive faces from cell rows.  The first cell that lists a face owns it (side 0)."""
    lf = np.array(_LOCAL_FACES[cell_type], dtype=np.int64)  # (nf, nfv)
    n_cell = cell2node.shape[0]
    nf, nfv = lf.shape
    fnodes = cell2node[:, lf].reshape(n_cell * nf, nfv)              # per (cell, local face)
    fshift = cell_shift[:, lf, :].reshape(n_cell * nf, nfv, 3)
    key = np.sort(fnodes, axis=1)
    _, first, inverse, counts = np.unique(key, axis=0, return_index=True,
                                          return_inverse=True, return_counts=True)
    inverse = inverse.reshape(-1)
    if counts.max() > 2:
        raise ValueError("a face is shared by more than two cells")
    n_face = first.shape[0]
    # order faces by first appearance so numbering follows cell order
    order = np.argsort(first, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(n_face)
    face_of_row = rank[inverse]
    owner_row = first[order]
    face2node = fnodes[owner_row]
    face_shift = fshift[owner_row]
    face2cell = np.full((n_face, 2), -1, dtype=np.int64)
    face2cell[:, 0] = owner_row // nf
    rows = np.arange(n_cell * nf)
    other = rows[rows != first[inverse]]
    face2cell[face_of_row[other], 1] = other // nf
    # periodic translation: compare the image offset of the smallest node id on both sides
    face_pshift = np.zeros((n_face, 3))
    if other.size:
        amin = np.argmin(fnodes, axis=1)
        shift_min = fshift[rows, amin]                 # (rows, 3)
        f_o = face_of_row[other]
        face_pshift[f_o] = shift_min[other] - shift_min[owner_row[f_o]]
    cell2face = face_of_row.reshape(n_cell, nf)
    face_zone = np.zeros(n_face, dtype=np.int32)
    return face2node, face_shift, face2cell, face_pshift, cell2face, face_zone


def _face_type(cell_type):
    return {TRI3: 0, QUAD4: 0, TET4: TRI3, HEX8: QUAD4}[cell_type]


def _jitter(rng, shape, amp):
    return rng.uniform(-amp, amp, size=shape)


def periodic_quad_2d(n, L=10.0, jitter=0.0, seed=0x1234, split_tri=False):
    """Periodic [0,L]^2 grid of n x n quads (optionally each split into 2 triangles).

    All nodes are jittered by a uniform fraction ``jitter`` of h = L/n in x and y.
    """
    h = L / n
    rng = np.random.default_rng(seed)
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    nid = lambda i, j: (i % n) + n * (j % n)
    coords = np.zeros((n * n, 3))
    coords[nid(ii, jj).ravel(), 0] = (ii * h).ravel()
    coords[nid(ii, jj).ravel(), 1] = (jj * h).ravel()
    if jitter:
        coords[:, :2] += _jitter(rng, (n * n, 2), jitter * h)
    ci, cj = ii.ravel(), jj.ravel()
    corners = [(0, 0), (1, 0), (1, 1), (0, 1)]
    qn = np.stack([nid(ci + a, cj + b) for a, b in corners], axis=1)
    qs = np.zeros((ci.size, 4, 3))
    for k, (a, b) in enumerate(corners):
        qs[:, k, 0] = np.where(ci + a >= n, L, 0.0)
        qs[:, k, 1] = np.where(cj + b >= n, L, 0.0)
    if split_tri:
        # diagonal from corner 0 to corner 2; both triangles counter-clockwise
        t1 = [0, 1, 2]
        t2 = [0, 2, 3]
        c2n = np.empty((2 * ci.size, 3), dtype=np.int64)
        csh = np.empty((2 * ci.size, 3, 3))
        c2n[0::2], c2n[1::2] = qn[:, t1], qn[:, t2]
        csh[0::2], csh[1::2] = qs[:, t1], qs[:, t2]
        ct = TRI3
    else:
        c2n, csh, ct = qn.astype(np.int64), qs, QUAD4
    f2n, fsh, f2c, fps, c2f, fz = _build_faces(ct, c2n, csh)
    return Mesh(2, ct, coords, c2n, csh, f2n, fsh, f2c, fz, fps, c2f, _face_type(ct))


def periodic_hex_3d(n, L=2 * np.pi, jitter=0.0, seed=0x1234):
    """Periodic [0,L]^3 grid of n^3 hexahedra, all nodes jittered by ``jitter`` x h."""
    h = L / n
    rng = np.random.default_rng(seed)
    ii, jj, kk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    nid = lambda i, j, k: (i % n) + n * ((j % n) + n * (k % n))
    coords = np.zeros((n ** 3, 3))
    ids = nid(ii, jj, kk).ravel()
    coords[ids, 0] = (ii * h).ravel()
    coords[ids, 1] = (jj * h).ravel()
    coords[ids, 2] = (kk * h).ravel()
    if jitter:
        coords += _jitter(rng, (n ** 3, 3), jitter * h)
    # cells ordered x fastest, matching a lexicographic i + n(j + n k) numbering
    kk2, jj2, ii2 = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ci, cj, ck = ii2.ravel(), jj2.ravel(), kk2.ravel()
    corners = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    c2n = np.stack([nid(ci + a, cj + b, ck + c) for a, b, c in corners], axis=1).astype(np.int64)
    csh = np.zeros((ci.size, 8, 3))
    for q, (a, b, c) in enumerate(corners):
        csh[:, q, 0] = np.where(ci + a >= n, L, 0.0)
        csh[:, q, 1] = np.where(cj + b >= n, L, 0.0)
        csh[:, q, 2] = np.where(ck + c >= n, L, 0.0)
    f2n, fsh, f2c, fps, c2f, fz = _build_faces(HEX8, c2n, csh)
    return Mesh(3, HEX8, coords, c2n, csh, f2n, fsh, f2c, fz, fps, c2f, QUAD4)


def iv_mesh(n=64, seed=0x1234, jitter=0.1):
    """Isentropic-vortex mesh: periodic [0,10]^2, n x n quads split into triangles."""
    return periodic_quad_2d(n, L=10.0, jitter=jitter, seed=seed, split_tri=True)


def tgv_mesh(n=64, seed=0x1234, jitter=0.05):
    """Taylor-Green mesh: periodic [0,2 pi]^3, n^3 hexahedra."""
    return periodic_hex_3d(n, L=2 * np.pi, jitter=jitter, seed=seed)


# boundary zones of the bump channel and their EulerBC.hpp types (BCFar 1, BCWallInvis 3, BCSym 9)
BUMP_ZONES = {"inflow": 1, "outflow": 2, "bump": 3, "top": 4, "side0": 5, "side1": 6}
BUMP_BC_TYPES = {1: 1, 2: 1, 3: 3, 4: 3, 5: 9, 6: 9}


def bump_height(x, amp=0.05, width=25.0):
    return amp * np.exp(-width * x * x)


def _kuhn_offsets():
    """Vertex offsets of the 6 tetrahedra of a unit hexahedron split along its main diagonal."""
    out = []
    for perm in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
        off = np.zeros((4, 3), dtype=np.int64)
        off[1, perm[0]] = 1
        off[2] = off[1]
        off[2, perm[1]] = 1
        off[3] = 1
        out.append(off)
    return out


def bump_channel_tet(nx=160, ny=80, nz=26, jitter=0.05, seed=0x1234, amp=0.05, L=(4.0, 1.0, 0.5), periodic_z=False):
    """Channel [-2,2] x [0,1] x [0,0.5] over the bump y = amp exp(-25 x^2), in tetrahedra.

    A structured nx x ny x nz hexahedral grid whose vertical lines follow the bump
    (y = h(x) + eta (1 - h(x))) is split into 6 tetrahedra per hexahedron along its
    main diagonal (Kuhn split); interior nodes are jittered by a uniform fraction
    ``jitter`` of the grid step in every parametric direction.  Boundary faces carry
    the zones of ``BUMP_ZONES``; with ``periodic_z`` the two side planes are joined
    periodically instead (translation Lz) and carry no zone.  Cells: 6 nx ny nz.
    """
    rng = np.random.default_rng(seed)
    Lx, Ly, Lz = L
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    xi, eta, zeta = i / nx, j / ny, k / nz
    kin = (k > 0) & (k < nz) if not periodic_z else (k < nz)
    interior = (i > 0) & (i < nx) & (j > 0) & (j < ny) & kin
    if jitter:
        for a, n in ((xi, nx), (eta, ny), (zeta, nz)):
            a += np.where(interior, rng.uniform(-jitter / n, jitter / n, size=a.shape), 0.0)
    if periodic_z:  # the k = nz plane is the image of k = 0
        for a in (xi, eta, zeta):
            a[:, :, nz] = a[:, :, 0]
        zeta[:, :, nz] += 1.0
    x = -Lx / 2 + Lx * xi
    h = bump_height(x, amp)
    y = h + eta * (Ly - h)
    z = Lz * zeta
    nz_id = nz if periodic_z else nz + 1
    nid = lambda a, b, c: (a * (ny + 1) + b) * nz_id + (c % nz_id)
    sel = np.s_[:, :, :nz_id]
    coords = np.stack([x[sel].ravel(), y[sel].ravel(), z[sel].ravel()], axis=1)
    ci, cj, ck = [a.ravel() for a in np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")]
    tets = [np.stack([nid(ci + o[0], cj + o[1], ck + o[2]) for o in off], axis=1) for off in _kuhn_offsets()]
    c2n = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int64)  # 6 tets of one hexahedron are consecutive
    csh = np.zeros((c2n.shape[0], 4, 3))
    if periodic_z:  # vertices on the k = nz plane are images of k = 0, shifted by Lz
        kk = np.stack([np.stack([ck + o[2] for o in off6], axis=1) for off6 in _kuhn_offsets()], axis=1).reshape(-1, 4)
        csh[:, :, 2] = np.where(kk >= nz, Lz, 0.0)
    X = coords[c2n] + csh
    vol6 = np.einsum("ij,ij->i", np.cross(X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]), X[:, 3] - X[:, 0])
    neg = vol6 < 0
    c2n[neg, 1], c2n[neg, 2] = c2n[neg, 2].copy(), c2n[neg, 1].copy()
    csh[neg, 1], csh[neg, 2] = csh[neg, 2].copy(), csh[neg, 1].copy()
    f2n, fsh, f2c, fps, c2f, fz = _build_faces(TET4, c2n, csh)
    bnd = f2c[:, 1] < 0
    I, J, K = i[sel].ravel(), j[sel].ravel(), k[sel].ravel()
    fn = f2n[bnd]
    zone = np.zeros(fn.shape[0], dtype=np.int32)
    tests = [("inflow", I == 0), ("outflow", I == nx), ("bump", J == 0), ("top", J == ny)]
    if not periodic_z:
        tests += [("side0", K == 0), ("side1", K == nz)]
    for nm, test in tests:
        zone[np.all(test[fn], axis=1)] = BUMP_ZONES[nm]
    if np.any(zone == 0):
        raise RuntimeError("unclassified boundary face")
    fz[bnd] = zone
    return Mesh(3, TET4, coords, c2n, csh, f2n, fsh, f2c, fz, fps, c2f, TRI3)


def freestream(mach, gamma=1.4, rho=1.0, p=1.0, direction=(1.0, 0.0, 0.0)):
    """Conservative state [rho, rho u, rho v, rho w, E] of a uniform flow at Mach ``mach``."""
    a = np.sqrt(gamma * p / rho)
    v = mach * a * np.asarray(direction, dtype=np.float64) / np.linalg.norm(direction)
    return np.array([rho, rho * v[0], rho * v[1], rho * v[2], p / (gamma - 1) + 0.5 * rho * v @ v])


# boundary zones of the flat-plate mesh and their EulerBC.hpp types (BCFar 1, BCWall 2, BCSym 9); the top is a
# symmetry plane: a far-field face there has u.n = 0, where the characteristic switch is decided by rounding
PLATE_ZONES = {"inflow": 1, "outflow": 2, "plate": 3, "upstream": 4, "top": 5}
PLATE_BC_TYPES = {1: 1, 2: 1, 3: 2, 4: 9, 5: 9}


def flat_plate_hex(nx=120, ny=80, nz=4, x0=-0.25, length=1.0, y1=5e-6, growth=1.1, lz=0.05, jitter=0.02, seed=0x1234, nx_up=None):
    """Stretched hexahedral boundary-layer mesh over a flat plate on y = 0, 0 <= x <= length.

    x in [x0, length] (``nx_up`` cells upstream of the leading edge, the rest on the plate), y from
    0 with first spacing ``y1`` and geometric ``growth`` (ny cells), z periodic over ``lz``
    (nz cells).  Interior nodes are jittered tangentially (x and z) by a uniform fraction
    ``jitter`` of the local spacing.  Zones: ``PLATE_ZONES``.  Cells: nx ny nz.
    """
    if nz < 3:
        raise ValueError("the periodic z direction needs nz >= 3 cells")
    rng = np.random.default_rng(seed)
    nx_up = max(1, int(round(nx * (-x0) / (length - x0)))) if nx_up is None else nx_up
    xs = np.concatenate([np.linspace(x0, 0.0, nx_up + 1)[:-1], np.linspace(0.0, length, nx - nx_up + 1)])
    ys = np.concatenate([[0.0], y1 * np.cumsum(growth ** np.arange(ny))])
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz), indexing="ij")
    x, y, z = xs[i].astype(float), ys[j].astype(float), (k * lz / nz).astype(float)
    if jitter:
        interior = (i > 0) & (i < nx) & (j > 0) & (j < ny)
        hx = np.diff(xs).min()
        x += np.where(interior, rng.uniform(-jitter, jitter, size=x.shape) * hx, 0.0)
        z += np.where(j > 0, rng.uniform(-jitter, jitter, size=z.shape) * lz / nz, 0.0) * (j < ny)
    nid = lambda a, b, c: (a * (ny + 1) + b) * nz + (c % nz)
    coords = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    ci, cj, ck = [a.ravel() for a in np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")]
    corners = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    c2n = np.stack([nid(ci + a, cj + b, ck + c) for a, b, c in corners], axis=1).astype(np.int64)
    csh = np.zeros((ci.size, 8, 3))
    for q, (a, b, c) in enumerate(corners):
        csh[:, q, 2] = np.where(ck + c >= nz, lz, 0.0)
    f2n, fsh, f2c, fps, c2f, fz = _build_faces(HEX8, c2n, csh)
    bnd = f2c[:, 1] < 0
    I, J = i.ravel(), j.ravel()
    fn = f2n[bnd]
    zone = np.zeros(fn.shape[0], dtype=np.int32)
    onx = np.all(J[fn] == 0, axis=1)
    upstream = np.all(I[fn] <= nx_up, axis=1)
    for nm, test in (("inflow", np.all(I[fn] == 0, axis=1)), ("outflow", np.all(I[fn] == nx, axis=1)), ("plate", onx & ~upstream),
                     ("upstream", onx & upstream), ("top", np.all(J[fn] == ny, axis=1))):
        zone[test] = PLATE_ZONES[nm]
    if np.any(zone == 0):
        raise RuntimeError("unclassified boundary face")
    fz[bnd] = zone
    return Mesh(3, HEX8, coords, c2n, csh, f2n, fsh, f2c, fz, fps, c2f, QUAD4)


def plate_wall_distance(points):
    """Distance to the plate segment {0 <= x, y = 0}: y over the plate, the distance to the leading
    edge upstream of it.  ``points`` is (..., 3)."""
    x, y = points[..., 0], points[..., 1]
    return np.where(x >= 0, np.abs(y), np.sqrt(x * x + y * y))


def greedy_colors(mesh):
    """First-fit colouring of the cell adjacency graph in cell order."""
    nbr = np.where(mesh.face2cell[mesh.cell2face, 0] == np.arange(mesh.n_cell)[:, None],
                   mesh.face2cell[mesh.cell2face, 1], mesh.face2cell[mesh.cell2face, 0])
    col = np.full(mesh.n_cell, -1, dtype=np.int64)
    for c in range(mesh.n_cell):
        used = {int(col[o]) for o in nbr[c] if o >= 0 and o != c and col[o] >= 0}
        k = 0
        while k in used:
            k += 1
        col[c] = k
    return col


def renumber_cells(mesh, perm_new2old):
    """Relabel cells: new cell i is old cell perm_new2old[i]. Faces keep their order and orientation."""
    perm = np.asarray(perm_new2old, dtype=np.int64)
    old2new = np.empty_like(perm)
    old2new[perm] = np.arange(perm.size)
    f2c = mesh.face2cell.copy()
    f2c[:, 0] = old2new[f2c[:, 0]]
    has1 = f2c[:, 1] >= 0
    f2c[has1, 1] = old2new[f2c[has1, 1]]
    return dataclasses.replace(mesh, cell2node=mesh.cell2node[perm], cell_shift=mesh.cell_shift[perm],
                               face2cell=f2c, cell2face=mesh.cell2face[perm])


def renumber_by_color(mesh):
    """Number cells colour by colour (first-fit colouring), so that a colour-ordered
    Gauss-Seidel sweep visits cells exactly as the sequential sweep in index order."""
    col = greedy_colors(mesh)
    return renumber_cells(mesh, np.argsort(col, kind="stable"))
