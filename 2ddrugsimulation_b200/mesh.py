"""Mesh files of the reference and a VTK writer (host side).

`read_inp` / `write_inp` follow the reference's mesh reader
(Cmesh::loadInp, mesh.cpp:59-186): a header up to a line starting "CML",
then "all_nodes all_elements target0 target1 target2" (targets 1-based), a
"*NODE" block of "id, x, y, z" lines, a "**HWCOLOR" line, an
"*ELEMENT, TYPE=..." line and "id, n1, ..., nk" lines (1-based nodes), then
either "CELLTYPE" with one integer per node and "eof", or "eof". Element
types: S2/T3D2 (line), S3 (triangle), S4 (quadrilateral), C3D4 (tetrahedron),
C3D8I (hexahedron).

`write_vtk` writes legacy ASCII VTK unstructured grids with point data, as
the reference's VTK writers do (heart.cpp:743-963, bspm.cpp:31-58).

`box_tets` builds a tetrahedral mesh of a box (each cube cut into six
tetrahedra around its main diagonal, all positively oriented) for tests and
examples.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

NODES_PER = {"S2": 2, "T3D2": 2, "S3": 3, "S4": 4, "C3D4": 4, "C3D8I": 8}
VTK_CELL = {2: 3, 3: 5, 4: 10, 8: 12}  # line, triangle, tetra, hexahedron (S4 quads: 9)


@dataclass
class Mesh:
    xyz: np.ndarray                 # [n, 3]
    elements: np.ndarray            # [e, k], 0-based
    etype: str                      # C3D4, C3D8I, S4, S3, S2, T3D2
    targets: tuple = (0, 0, 0)      # 0-based monitoring nodes
    celltype: np.ndarray | None = field(default=None)


def read_inp(path) -> Mesh:
    with open(path) as fh:
        lines = fh.read().splitlines()
    k = 0
    while not lines[k].startswith("CML"):
        k += 1
    n, ne, t0, t1, t2 = (int(x) for x in lines[k + 1].split()[:5])
    while not lines[k].startswith("*NODE"):
        k += 1
    xyz = np.array([[float(v) for v in lines[k + 1 + i].split(",")[1:4]] for i in range(n)])
    k += 1 + n
    k += 1  # **HWCOLOR
    etype = lines[k].split(",")[1].strip().split("=")[1].strip()
    nn = NODES_PER[etype]
    elements = np.array([[int(v) - 1 for v in lines[k + 1 + i].split(",")[1:1 + nn]] for i in range(ne)], np.int32)
    k += 1 + ne
    celltype = None
    if lines[k].startswith("CELLTYPE"):
        celltype = np.array([int(lines[k + 1 + i]) for i in range(n)], np.int32)
        k += 1 + n
    if not lines[k].startswith("eof"):
        raise ValueError(f"{path}: no eof after the elements / CELLTYPE block")
    return Mesh(xyz, elements, etype, (t0 - 1, t1 - 1, t2 - 1), celltype)


def write_inp(path, mesh: Mesh) -> None:
    t = [x + 1 for x in mesh.targets]
    with open(path, "w") as fh:
        fh.write("** cep-b200 mesh\nCML\n")
        fh.write(f"{len(mesh.xyz)} {len(mesh.elements)} {t[0]} {t[1]} {t[2]}\n")
        fh.write("*NODE\n")
        for i, (x, y, z) in enumerate(mesh.xyz):
            fh.write(f"{i + 1}, {float(x)!r}, {float(y)!r}, {float(z)!r}\n")
        fh.write("**HWCOLOR COMP 1 1\n")
        fh.write(f"*ELEMENT, TYPE={mesh.etype}, ELSET=heart\n")
        for i, el in enumerate(mesh.elements):
            fh.write(f"{i + 1}, " + ", ".join(str(int(v) + 1) for v in el) + "\n")
        if mesh.celltype is not None:
            fh.write("CELLTYPE\n")
            for c in mesh.celltype:
                fh.write(f"{int(c)}\n")
        fh.write("eof\n")


def write_vtk(path, mesh: Mesh, point_data: dict) -> None:
    """Legacy ASCII VTK of the mesh with named point arrays (e.g. Voltage)."""
    nn = mesh.elements.shape[1]
    ctype = 9 if mesh.etype == "S4" else VTK_CELL[nn]
    with open(path, "w") as fh:
        fh.write("# vtk DataFile Version 3.0\nvtk output\nASCII\nDATASET UNSTRUCTURED_GRID\n")
        fh.write(f"POINTS {len(mesh.xyz)} float\n")
        for x, y, z in mesh.xyz:
            fh.write(f"{x:.9g} {y:.9g} {z:.9g}\n")
        fh.write(f"CELLS {len(mesh.elements)} {len(mesh.elements) * (nn + 1)}\n")
        for el in mesh.elements:
            fh.write(f"{nn} " + " ".join(str(int(v)) for v in el) + "\n")
        fh.write(f"CELL_TYPES {len(mesh.elements)}\n")
        fh.write("".join(f"{ctype}\n" for _ in range(len(mesh.elements))))
        fh.write(f"POINT_DATA {len(mesh.xyz)}\n")
        for name, vals in point_data.items():
            fh.write(f"SCALARS {name} float\nLOOKUP_TABLE default\n")
            fh.write("".join(f"{float(v):.9g}\n" for v in np.asarray(vals).ravel()))


def grid_mesh(dim: int, nx: int, ny: int, nz: int, h: float) -> Mesh:
    """The structured grid of cep_fem_create_grid as a Mesh (node
    i + nx*(j + ny*k) at (i h, j h, k h); S4 quads in 2D, C3D8I hexahedra in
    3D, corners in VTK order), so a grid tissue's V can go to write_vtk."""
    if dim == 2:
        nz = 1
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    xyz = np.stack([ii.transpose(2, 1, 0).ravel(), jj.transpose(2, 1, 0).ravel(), kk.transpose(2, 1, 0).ravel()],
                   1).astype(np.float64) * h
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), indexing="xy")
    i, j = i.ravel(), j.ravel()
    if dim == 2:
        n0 = i + nx * j
        els = np.stack([n0, n0 + 1, n0 + 1 + nx, n0 + nx], 1)
        return Mesh(xyz, els.astype(np.int32), "S4")
    els = []
    plane = nx * ny
    for k in range(nz - 1):
        n0 = i + nx * j + plane * k
        quad = np.stack([n0, n0 + 1, n0 + 1 + nx, n0 + nx], 1)
        els.append(np.concatenate([quad, quad + plane], 1))
    return Mesh(xyz, np.concatenate(els).astype(np.int32), "C3D8I")


def box_tets(nx: int, ny: int, nz: int, h: float) -> Mesh:
    """Tetrahedral mesh of an (nx-1) x (ny-1) x (nz-1) box of cubes of edge h,
    node (i, j, k) = i + nx*(j + ny*k) at (i h, j h, k h)."""
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    xyz = np.stack([ii.transpose(2, 1, 0).ravel(), jj.transpose(2, 1, 0).ravel(), kk.transpose(2, 1, 0).ravel()], 1) * h
    nid = lambda i, j, k: i + nx * (j + ny * k)  # noqa: E731
    # six tetrahedra around the cube's diagonal (corner 0 -> corner 7), each a
    # path 0 -> a -> b -> 7 through the cube's edges
    paths = [(1, 3), (1, 5), (2, 3), (2, 6), (4, 5), (4, 6)]
    corner = lambda c: ((c >> 0) & 1, (c >> 1) & 1, (c >> 2) & 1)  # noqa: E731
    els = []
    for k in range(nz - 1):
        for j in range(ny - 1):
            for i in range(nx - 1):
                for a, b in paths:
                    tet = [(i, j, k)] + [tuple(np.add((i, j, k), corner(c))) for c in (a, b, 7)]
                    ids = [nid(*p) for p in tet]
                    p0, p1, p2, p3 = (xyz[q] for q in ids)
                    if np.dot(np.cross(p1 - p0, p2 - p0), p3 - p0) < 0:
                        ids[1], ids[2] = ids[2], ids[1]
                    els.append(ids)
    return Mesh(xyz.astype(np.float64), np.array(els, np.int32), "C3D4")


def write_output(path, time: float, states: np.ndarray) -> None:
    """A tissue snapshot in the reference's output.<rank> format
    (heart.cpp:943-963): the time ("%f \\n"), then one line per node with
    its states ("%f " each). Six decimals, as the reference writes them."""
    st = np.asarray(states, np.float64)
    with open(path, "w") as f:
        f.write("%f \n" % time)
        for row in st:
            f.write("".join("%f " % x for x in row) + "\n")


def read_output(path, n_states: int) -> tuple[float, np.ndarray]:
    """An output.<rank> snapshot as heart.cpp:595-616 reads it (fscanf
    "%lf " throughout): the time, then n_states values per node."""
    vals = np.array(Path(path).read_text().split(), dtype=np.float64)
    if len(vals) < 1 or (len(vals) - 1) % n_states:
        raise ValueError(f"{path}: {len(vals) - 1} state values is not a multiple of {n_states}")
    return float(vals[0]), vals[1:].reshape(-1, n_states)


def write_states(path, y) -> None:
    """One cell's states, one "%lf" per line (drug_sim_full.cpp:318), the
    file the single-cell benches read back as output_orudy.dat."""
    with open(path, "w") as f:
        for x in np.asarray(y, np.float64).reshape(-1):
            f.write("%f\n" % x)


def read_states(path) -> np.ndarray:
    """A single-cell states file as cipa_drug_bench.cpp:104-111 reads it
    (strtod per line)."""
    return np.array([float(ln.split()[0]) for ln in Path(path).read_text().splitlines() if ln.split()])
