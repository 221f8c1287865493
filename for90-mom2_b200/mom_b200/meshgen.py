"""Synthetic surface meshes for the PMCHWT workloads, written as Gmsh 2.2 ASCII.

The reference solver reads Gmsh 2.1/2.2 files through ``load_mesh_gmsh``
(mesh.f90:610-736): ``$Nodes`` with 1-based node numbers and ``$Elements``
whose triangles (type 2) carry the physical id as their first tag.  These
generators build the inputs of the benchmark workloads from seeded
constructions (no external dataset is involved):

* icosphere: a regular icosahedron subdivided ``s`` times and projected to a
  sphere (V = 10*4**s + 2, F = 20*4**s, E = 30*4**s), faces oriented outward;
* triaxial ellipsoid: the unit icosphere scaled by three semi-axes;
* perturbed sphere: the icosphere with radius r(theta, phi) = r0 (1 + sum of
  real spherical harmonics Y_lm, l <= lmax, coefficients ~ N(0, sigma^2));
* core-shell: two concentric icospheres with physical ids 1 (inner) and 2.

Coordinates are written in nanometres; the ``mesh`` command's scale factor
(1e-9) converts them to metres, as in the reference's own inputs.
"""
from __future__ import annotations

import math
import os

import numpy as np


def icosphere(subdiv: int, radius: float = 1.0):
    """Return (nodes[V,3], faces[F,3] 0-based) of an outward-oriented icosphere."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
             (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in verts]
    for _ in range(subdiv):
        cache = {}
        nf = []

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]

        for (a, b, c) in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    nodes = np.array(v) * radius
    faces = np.array(faces, dtype=np.int64)
    # Orient outward: the normal (p2-p1)x(p3-p1) must point away from the origin.
    p1, p2, p3 = nodes[faces[:, 0]], nodes[faces[:, 1]], nodes[faces[:, 2]]
    nrm = np.cross(p2 - p1, p3 - p1)
    inward = np.einsum("ij,ij->i", nrm, (p1 + p2 + p3)) < 0
    faces[inward] = faces[inward][:, ::-1]
    return nodes, faces


def octasphere(subdiv: int, radius: float = 1.0):
    """(nodes, faces) of an outward-oriented sphere from the subdivided octahedron:
    no face crosses a coordinate plane, so the mesh has the three mirror symmetries
    x -> -x, y -> -y, z -> -z exactly (nodes on a plane stay on it)."""
    v = [np.array(p, dtype=np.float64) for p in
         ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))]
    faces = [(0, 2, 4), (2, 1, 4), (1, 3, 4), (3, 0, 4), (2, 0, 5), (1, 2, 5), (3, 1, 5), (0, 3, 5)]
    for _ in range(subdiv):
        cache = {}
        nf = []

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]

        for (a, b, c) in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    nodes = np.array(v) * radius
    faces = np.array(faces, dtype=np.int64)
    p1, p2, p3 = nodes[faces[:, 0]], nodes[faces[:, 1]], nodes[faces[:, 2]]
    nrm = np.cross(p2 - p1, p3 - p1)
    inward = np.einsum("ij,ij->i", nrm, (p1 + p2 + p3)) < 0
    faces[inward] = faces[inward][:, ::-1]
    return nodes, faces


def symmetry_fragment(nodes, faces, planes):
    """The part of a mirror-symmetric mesh on the positive side of each plane in
    `planes` (0 = x, 1 = y, 2 = z): (nodes, faces, lines), where lines[plane] lists
    the fragment's edges (node pairs) that lie on that plane, the boundary edges a
    reference script marks with `sbnd <id> xplane` (yplane, zplane)."""
    nodes = np.asarray(nodes, dtype=np.float64)
    faces = np.asarray(faces)
    keep = np.ones(len(faces), bool)
    cen = nodes[faces].mean(axis=1)
    for ax in planes:
        keep &= cen[:, ax] > 0
    sub = faces[keep]
    used = np.unique(sub)
    remap = -np.ones(len(nodes), np.int64)
    remap[used] = np.arange(len(used))
    fn = nodes[used]
    ff = remap[sub]
    lines = {}
    scale = np.abs(fn).max()
    for ax in planes:
        on = np.abs(fn[:, ax]) <= 1e-12 * scale
        pairs = set()
        for f in ff:
            for k in range(3):
                a, b = int(f[k]), int(f[(k + 1) % 3])
                if on[a] and on[b]:
                    pairs.add((min(a, b), max(a, b)))
        lines[ax] = sorted(pairs)
    return fn, ff, lines


def ellipsoid(subdiv: int, axes):
    nodes, faces = icosphere(subdiv, 1.0)
    return nodes * np.asarray(axes, dtype=np.float64)[None, :], faces


def real_sph_harm(l: int, m: int, theta, phi):
    """Real spherical harmonic Y_lm (orthonormal) at polar angle theta, azimuth phi."""
    from scipy.special import sph_harm_y
    y = sph_harm_y(l, abs(m), theta, phi)
    if m > 0:
        return math.sqrt(2.0) * (-1) ** m * y.real
    if m < 0:
        return math.sqrt(2.0) * (-1) ** m * y.imag
    return y.real


def perturbed_sphere(subdiv: int, radius: float, lmax: int = 4, sigma: float = 0.03, seed: int = 4):
    """Icosphere with r = radius * (1 + sum_{l<=lmax, |m|<=l} c_lm Y_lm), c_lm ~ N(0, sigma^2)."""
    nodes, faces = icosphere(subdiv, 1.0)
    rng = np.random.default_rng(seed)
    coef = {(l, m): rng.normal(0.0, sigma) for l in range(lmax + 1) for m in range(-l, l + 1)}
    theta = np.arccos(np.clip(nodes[:, 2], -1.0, 1.0))
    phi = np.arctan2(nodes[:, 1], nodes[:, 0])
    pert = np.zeros(len(nodes))
    for (l, m), c in coef.items():
        pert += c * real_sph_harm(l, m, theta, phi)
    return nodes * (radius * (1.0 + pert))[:, None], faces


def write_gmsh22(path: str, nodes, faces, face_ids) -> None:
    """Write nodes/triangles as a Gmsh 2.2 ASCII file (1-based numbering)."""
    nodes = np.asarray(nodes, dtype=np.float64)
    faces = np.asarray(faces)
    face_ids = np.broadcast_to(np.asarray(face_ids), (len(faces),))
    with open(path, "w") as fh:
        fh.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(nodes))
        for i, p in enumerate(nodes):
            fh.write("%d %.17g %.17g %.17g\n" % (i + 1, p[0], p[1], p[2]))
        fh.write("$EndNodes\n$Elements\n%d\n" % len(faces))
        for i, (f, pid) in enumerate(zip(faces, face_ids)):
            fh.write("%d 2 2 %d %d %d %d %d\n" % (i + 1, pid, pid, f[0] + 1, f[1] + 1, f[2] + 1))
        fh.write("$EndElements\n")


def read_gmsh(path: str):
    """Minimal Gmsh 2.1/2.2 ASCII reader: (nodes[V,3], faces[F,3] 0-based, ids[F])."""
    with open(path) as fh:
        lines = [ln.strip() for ln in fh]
    i = 0
    nodes = faces = ids = None
    while i < len(lines):
        tag = lines[i]
        if tag == "$MeshFormat":
            ver = lines[i + 1][:3]
            if ver not in ("2.1", "2.2"):
                raise ValueError("Mesh version is unsupported!")
            i += 3
        elif tag == "$Nodes":
            n = int(lines[i + 1])
            nodes = np.zeros((n, 3))
            for j in range(n):
                parts = lines[i + 2 + j].split()
                nodes[int(parts[0]) - 1] = [float(x) for x in parts[1:4]]
            i += n + 3
        elif tag == "$Elements":
            n = int(lines[i + 1])
            fl, il = [], []
            for j in range(n):
                parts = [int(x) for x in lines[i + 2 + j].split()]
                if parts[1] == 2:
                    nt = parts[2]
                    il.append(parts[3])
                    fl.append([parts[3 + nt] - 1, parts[4 + nt] - 1, parts[5 + nt] - 1])
            faces = np.array(fl, dtype=np.int64)
            ids = np.array(il, dtype=np.int64)
            i += n + 3
        else:
            i += 1
    return nodes, faces, ids


def sphere_msh(path: str, subdiv: int, radius_nm: float, pid: int = 1) -> str:
    nodes, faces = icosphere(subdiv, radius_nm)
    write_gmsh22(path, nodes, faces, pid)
    return path


def core_shell_msh(path: str, subdiv: int, r_core: float, r_shell: float) -> str:
    n1, f1 = icosphere(subdiv, r_core)
    n2, f2 = icosphere(subdiv, r_shell)
    nodes = np.vstack([n1, n2])
    faces = np.vstack([f1, f2 + len(n1)])
    ids = np.concatenate([np.full(len(f1), 1), np.full(len(f2), 2)])
    write_gmsh22(path, nodes, faces, ids)
    return path


def workload_dir() -> str:
    d = os.environ.get("MOM_B200_MESHDIR") or os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "_meshes")
    os.makedirs(d, exist_ok=True)
    return d
