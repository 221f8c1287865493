"""Python front end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the CPU legs of bench.py use
this module, and only as the checker.  It loads ``_build/libmomoracle.so``
(a plain-C FP64 restatement of the reference's hot path, see mom_oracle.c)
and adds the LAPACK step of ``solve_multi_linsys`` (linalg.f90:159-180):
ZGETRF + ZGETRS, here from the OpenBLAS that ships with scipy.  The
reference links Intel MKL (CMakeLists.txt:27) with no version pinned, so the
LU step is pinned by backward error instead of bitwise factors.

Parity status: unpinned against reference outputs (no Fortran compiler
exists to run the reference, and it ships no golden vectors).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

PI_F = float(np.float32(3.141592653589))  # constants.f90:10 (single-precision literal)
EPS0 = 8.8541878176e-12
MU0 = 4 * PI_F * 1e-7
C0 = 2.997924580003e8
ETA0 = 3.767303134622e2
DEGTORAD = PI_F / 180.0


def load_mesh_gmsh(path: str):
    """load_mesh_gmsh (mesh.f90:610-705): Gmsh 2.1 / 2.2 ASCII.  Returns
    (nodes [V][3], faces [F][3] 0-based, physical ids [F]) of the triangle
    elements (type 2); the physical id is the first tag and the node indices
    follow the ntags tags, as element_data(4) and element_data(4+ntags:6+ntags)."""
    with open(path) as fh:
        tok = [ln.split() for ln in fh]
    nodes = faces = ids = None
    i = 0
    while i < len(tok):
        head = tok[i][0] if tok[i] else ""
        if head == "$MeshFormat":
            if tok[i + 1][0][:3] not in ("2.1", "2.2"):
                raise ValueError("Mesh version is unsupported!")
            if tok[i + 2][0] != "$EndMeshFormat":
                raise ValueError("Could not find $MeshFormatNodes specifier!")
            i += 3
        elif head == "$Nodes":
            nn = int(tok[i + 1][0])
            nodes = np.zeros((nn, 3))
            for r in tok[i + 2:i + 2 + nn]:
                nodes[int(r[0]) - 1] = [float(v) for v in r[1:4]]
            if tok[i + 2 + nn][0] != "$EndNodes":
                raise ValueError("Could not find $EndNodes specifier!")
            i += nn + 3
        elif head == "$Elements":
            ne = int(tok[i + 1][0])
            fl, il = [], []
            for r in tok[i + 2:i + 2 + ne]:
                d = [int(v) for v in r]
                if d[1] == 2:
                    nt = d[2]
                    il.append(d[3])
                    fl.append([d[3 + nt] - 1, d[4 + nt] - 1, d[5 + nt] - 1])
            if tok[i + 2 + ne][0] != "$EndElements":
                raise ValueError("Could not find $EndElements specifier!")
            faces = np.array(fl, dtype=np.int32)
            ids = np.array(il, dtype=np.int32)
            i += ne + 3
        else:
            i += 1
    return nodes, faces, ids


def get_refind(path: str, wl: float) -> complex:
    """get_refind (aux.f90:100-167): linear interpolation in a (wl, n, k) table
    with linterp (aux.f90:58-63); CMPLX without a kind rounds to single
    precision; wavelengths outside the table give 1."""
    rows = []
    with open(path) as fh:
        for ln in fh:
            p = ln.split()
            if len(p) >= 3:
                rows.append([float(v.replace("d", "e").replace("D", "e")) for v in p[:3]])
    f32 = np.float32
    wl1, nr1, ni1 = rows[0]
    if wl < wl1:
        return 1.0 + 0j
    for wl2, nr2, ni2 in rows[1:]:
        if wl1 <= wl <= wl2 and wl1 != wl2:
            t = (wl - wl1) / (wl2 - wl1)
            return complex(float(f32(nr1 + t * (nr2 - nr1))), float(f32(ni1 + t * (ni2 - ni1))))
        if wl == wl1:
            return complex(float(f32(nr1)), float(f32(ni1)))
        if wl == wl2:
            return complex(float(f32(nr2)), float(f32(ni2)))
        if wl1 > wl2:
            raise ValueError("Refractive index data disordered!")
        wl1, nr1, ni1 = wl2, nr2, ni2
    return 1.0 + 0j


def omega_of(wl: float) -> float:
    """Angular frequency as solve_batch computes it (solver.f90:77)."""
    return 2.0 * PI_F * C0 / wl


def build() -> str:
    path = os.path.join(_HERE, "_build", "libmomoracle.so")
    src = os.path.join(_HERE, "mom_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return path


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        L = _LIB
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        L.oracle_problem_create.argtypes = [C.c_int, dp, C.c_int, ip, ip, C.c_double, C.c_int, ip, ip,
                                            C.c_char_p, C.POINTER(C.c_void_p)]
        L.oracle_problem_free.argtypes = [C.c_void_p]
        L.oracle_problem_sizes.argtypes = [C.c_void_p, ip]
        L.oracle_problem_export.argtypes = [C.c_void_p, C.c_int, dp, ip, ip, ip, ip, ip, ip, dp]
        L.oracle_sysmat.argtypes = [C.c_void_p, C.c_double, dp, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int]
        L.oracle_sysmat_sample.argtypes = [C.c_void_p, C.c_double, dp, C.c_int, C.c_int, C.c_int]
        L.oracle_sysmat_sample.restype = C.c_double
        L.oracle_operator.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, dp, C.c_void_p]
        L.oracle_srcvec.argtypes = [C.c_void_p, C.c_int, C.c_double, dp, C.c_void_p, C.c_void_p]
        L.oracle_cs.argtypes = [C.c_void_p, C.c_int, C.c_double, dp, C.c_void_p, C.c_void_p, dp, dp]
        L.oracle_rcs.argtypes = [C.c_void_p, C.c_int, C.c_double, dp, C.c_void_p, C.c_int, C.c_int, dp, C.c_int]
        L.oracle_srcint.argtypes = [C.c_void_p, C.c_int, C.c_int, dp, C.c_int, C.c_int, dp, C.c_int, C.c_void_p]
        L.oracle_static_integrals.argtypes = [C.c_void_p, C.c_int, dp, C.c_int, C.c_int, dp]
        L.oracle_face_geometry.argtypes = [C.c_void_p, C.c_int, C.c_int, dp, dp, ip, dp, dp]
        L.oracle_tri_rule.argtypes = [C.c_char_p, ip, dp, dp]
        L.oracle_problem_set_symmetry.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_char_p)]
        L.oracle_group_info.argtypes = [C.c_void_p, dp, dp, C.c_void_p]
        L.oracle_problem_classify_edges.argtypes = [C.c_void_p, C.c_int, ip, C.c_int]
        L.oracle_edge_bc.argtypes = [C.c_void_p, C.c_int, ip, C.c_void_p]
        L.oracle_sysmat_sym.argtypes = [C.c_void_p, C.c_double, dp, C.c_void_p, C.c_int]
        L.oracle_sysmat_sym_dom.argtypes = [C.c_void_p, C.c_double, dp, C.c_void_p, C.c_int, C.c_int]
        L.oracle_srcvec_sym.argtypes = [C.c_void_p, C.c_double, dp, C.c_void_p, C.c_void_p]
        L.oracle_cs_sym.argtypes = [C.c_void_p, C.c_int, C.c_double, dp, C.c_void_p, C.c_void_p, dp, dp]
        L.oracle_scat_fields.argtypes = [C.c_void_p, C.c_int, C.c_double, dp, C.c_int, C.c_void_p, C.c_int64,
                                         C.c_void_p, C.c_int, C.c_int, dp, C.c_void_p, C.c_void_p]
        L.oracle_pi.restype = C.c_double
    return _LIB


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class OSrc(C.Structure):
    _fields_ = [("type", C.c_int), ("theta", C.c_double), ("phi", C.c_double), ("psi", C.c_double),
                ("phase_re", C.c_double), ("phase_im", C.c_double)]


def make_src(src: dict) -> OSrc:
    """src: {'type': 'pw', 'theta', 'phi', 'psi'} or {'type': 'pw_elliptic', 'theta', 'phi', 'phase'},
    angles in radians (``ssrc`` converts degrees with the float-rounded pi, interface.f90:486-515);
    {'type': 'none'}: no incident field (type 0, the second-harmonic cross sections)."""
    if src["type"] == "none":
        return OSrc(0, 0.0, 0.0, 0.0, 0.0, 0.0)
    if src["type"] == "pw":
        return OSrc(1, src["theta"], src["phi"], src["psi"], 0.0, 0.0)
    ph = complex(src["phase"])
    return OSrc(10, src["theta"], src["phi"], 0.0, ph.real, ph.imag)


def tri_rule(name: str = "tri_gl13"):
    nq = C.c_int()
    w = np.zeros(13)
    nd = np.zeros((13, 3))
    if lib().oracle_tri_rule(name.encode(), C.byref(nq), _dp(w), _dp(nd)):
        raise ValueError("Unrecognized quadrature type " + name)
    return w[: nq.value].copy(), nd[: nq.value].copy()


class OracleProblem:
    """Master mesh + domain submeshes after ``mesh``/``sdom``/``fdom``."""

    def __init__(self, nodes, faces, face_ids, scale, domains, quad="tri_gl13"):
        L = lib()
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        faces = np.ascontiguousarray(faces, dtype=np.int32)
        ids = np.ascontiguousarray(face_ids, dtype=np.int32)
        nsurf = np.array([len(d) for d in domains], dtype=np.int32)
        dids = np.array([i for d in domains for i in d], dtype=np.int32)
        h = C.c_void_p()
        rc = L.oracle_problem_create(len(nodes), _dp(nodes), len(faces), _ip(faces), _ip(ids), scale,
                                     len(domains), _ip(nsurf), _ip(dids), quad.encode(), C.byref(h))
        if rc:
            raise RuntimeError("oracle problem setup failed (%d)" % rc)
        self.h = h
        self.ndom = len(domains)
        sz = np.zeros(3 + 3 * self.ndom, dtype=np.int32)
        L.oracle_problem_sizes(h, _ip(sz))
        self.N = int(sz[0])
        self.master_sizes = (int(sz[1]), int(sz[2]), int(sz[0]))
        self.dom_sizes = [tuple(int(v) for v in sz[3 + 3 * d: 6 + 3 * d]) for d in range(self.ndom)]

    @classmethod
    def from_msh(cls, path, scale, domains, quad="tri_gl13"):
        nodes, faces, ids = load_mesh_gmsh(path)
        return cls(nodes, faces, ids, scale, domains, quad)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_problem_free(self.h)
            self.h = None

    def export(self, d: int) -> dict:
        nn, nf, ne = self.master_sizes if d < 0 else self.dom_sizes[d]
        out = dict(nodes=np.zeros((nn, 3)), face_node=np.zeros((nf, 3), np.int32),
                   face_edge=np.zeros((nf, 3), np.int32), edge_node=np.zeros((ne, 2), np.int32),
                   edge_face=np.zeros((ne, 2), np.int32), edge_bnode=np.zeros((ne, 2), np.int32),
                   edge_parent=np.zeros(ne, np.int32))
        av = C.c_double()
        lib().oracle_problem_export(self.h, d, _dp(out["nodes"]), _ip(out["face_node"]), _ip(out["face_edge"]),
                                    _ip(out["edge_node"]), _ip(out["edge_face"]), _ip(out["edge_bnode"]),
                                    _ip(out["edge_parent"]), C.byref(av))
        out["avelen"] = av.value
        return out

    def sysmat(self, omega, ri, mlo=0, mhi=-1, nthreads=0):
        """sysmat_pmchwt (sysmat.f90:18-105): the 2N x 2N PMCHWT matrix, Fortran order."""
        A = np.zeros((2 * self.N, 2 * self.N), dtype=np.complex128, order="F")
        rr = np.array([[complex(v).real, complex(v).imag] for v in ri], dtype=np.float64)
        lib().oracle_sysmat(self.h, omega, _dp(rr), A.ctypes.data, 2 * self.N, mlo, mhi, nthreads)
        return A

    def sysmat_sample(self, omega, ri, mlo, mhi, nthreads=0):
        """Timing sample: the sysmat work of test faces [mlo, mhi) of every domain (no matrix)."""
        rr = np.array([[complex(v).real, complex(v).imag] for v in ri], dtype=np.float64)
        return lib().oracle_sysmat_sample(self.h, omega, _dp(rr), mlo, mhi, nthreads)

    def operator(self, d, op, omega, ri):
        """One domain operator: op 0 = D, 1 = H, 2 = K (computeD/H/K)."""
        nd = self.dom_sizes[d][2]
        M = np.zeros((nd, nd), dtype=np.complex128, order="F")
        rr = np.array([complex(ri).real, complex(ri).imag])
        lib().oracle_operator(self.h, d, op, omega, _dp(rr), M.ctypes.data)
        return M

    def srcvec(self, omega, ri, src, d=0):
        q = np.zeros(2 * self.N, dtype=np.complex128)
        rr = np.array([complex(ri).real, complex(ri).imag])
        s = make_src(src)
        lib().oracle_srcvec(self.h, d, omega, _dp(rr), C.byref(s), q.ctypes.data)
        return q

    def cs(self, omega, ri, x, src, d=0):
        """cs_prtsrf (cs.f90:14-104): returns (csca, cabs)."""
        x = np.ascontiguousarray(x, dtype=np.complex128)
        rr = np.array([complex(ri).real, complex(ri).imag])
        s = make_src(src)
        a, b = C.c_double(), C.c_double()
        lib().oracle_cs(self.h, d, omega, _dp(rr), x.ctypes.data, C.byref(s), C.byref(a), C.byref(b))
        return a.value, b.value

    def rcs(self, omega, ri, x, ntheta, nphi, d=0, nthreads=0):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        rr = np.array([complex(ri).real, complex(ri).imag])
        out = np.zeros((ntheta, nphi), order="F")
        lib().oracle_rcs(self.h, d, omega, _dp(rr), x.ctypes.data, ntheta, nphi, _dp(out), nthreads)
        return out

    # ---- symmetry groups (read_symm, sbnd; mirror planes) ----
    BND = {"xplane": 2, "yplane": 3, "zplane": 4}

    def set_symmetry(self, names):
        """read_symm (interface.f90:160-210): product of the named groups ("id", "mxp",
        "myp", "mzp"); returns the group order."""
        arr = (C.c_char_p * max(1, len(names)))(*[n.encode() for n in names])
        n = lib().oracle_problem_set_symmetry(self.h, len(names), arr)
        if n < 0:
            raise ValueError("unsupported symmetry group %r" % (names,))
        self.nga = n
        return n

    def group_info(self):
        n = getattr(self, "nga", 1)
        j = np.zeros((n, 9))
        detj = np.zeros(n)
        ef = np.zeros((n, n), dtype=np.complex128)
        lib().oracle_group_info(self.h, _dp(j), _dp(detj), ef.ctypes.data)
        return j.reshape(n, 3, 3), detj, ef

    def classify_edges(self, lines, bnd):
        """sbnd / classify_edges (mesh.f90:155-175): lines = master node pairs (0-based)."""
        ln = np.ascontiguousarray(np.asarray(lines, dtype=np.int32).reshape(-1, 2))
        return lib().oracle_problem_classify_edges(self.h, len(ln), _ip(ln), self.BND.get(bnd, bnd))

    def edge_bc(self, nr):
        idv = np.zeros(2 * self.N, dtype=np.int32)
        ph = np.zeros(2 * self.N, dtype=np.complex128)
        lib().oracle_edge_bc(self.h, nr, _ip(idv), ph.ctypes.data)
        return idv, ph

    def sysmat_sym(self, omega, ri, nthreads=0):
        """sysmat_pmchwt with the group: A[nga][2N][2N]."""
        rr = np.array([[complex(v).real, complex(v).imag] for v in ri]).ravel()
        n = getattr(self, "nga", 1)
        A = np.zeros((n, 2 * self.N, 2 * self.N), dtype=np.complex128)  # [nf] column-major blocks
        lib().oracle_sysmat_sym(self.h, omega, _dp(rr), A.ctypes.data, nthreads)
        return np.ascontiguousarray(A.transpose(0, 2, 1))

    def sysmat_sym_dom(self, omega, ri, d, nthreads=0):
        """The blocks of domain d alone in every representation (sysmat_pmchwt_nls's
        per-domain terms, sysmat.f90:112-229): A[nga][2N][2N]."""
        rr = np.array([[complex(v).real, complex(v).imag] for v in ri]).ravel()
        n = getattr(self, "nga", 1)
        A = np.zeros((n, 2 * self.N, 2 * self.N), dtype=np.complex128)
        lib().oracle_sysmat_sym_dom(self.h, omega, _dp(rr), A.ctypes.data, nthreads, d)
        return np.ascontiguousarray(A.transpose(0, 2, 1))

    def srcvec_sym(self, omega, ri, src):
        n = getattr(self, "nga", 1)
        q = np.zeros((n, 2 * self.N), dtype=np.complex128)
        rr = np.array([complex(ri).real, complex(ri).imag])
        s = make_src(src)
        lib().oracle_srcvec_sym(self.h, omega, _dp(rr), C.byref(s), q.ctypes.data)
        return q

    def solve_sym(self, A, q):
        """solve_systems (solver.f90:325-357): per representation the boundary
        conditions of edge_bc (bc.f90:28-117), reduce_system, solve, expand_solution."""
        x = np.zeros_like(q)
        for r in range(A.shape[0]):
            idv, ph = self.edge_bc(r)
            Ar, br = A[r].copy(), q[r][:, None].copy()
            for n in np.nonzero(idv > 0)[0]:  # resolve_system_dependencies (coupled edges)
                Ar[:, n] += Ar[:, idv[n] - 1] * ph[n]
            for n in np.nonzero(idv > 0)[0]:
                Ar[n, :] += Ar[idv[n] - 1, :] * np.conj(ph[n])
                br[n, :] += br[idv[n] - 1, :] * np.conj(ph[n])
            keep = np.nonzero(idv != -1)[0]
            xr = solve(Ar[np.ix_(keep, keep)], br[keep])[:, 0]
            full = np.zeros(2 * self.N, dtype=np.complex128)
            full[keep] = xr
            for n in np.nonzero(idv > 0)[0]:
                full[idv[n] - 1] = full[n] * ph[n]
            x[r] = full
        return x

    def cs_sym(self, omega, ri, x, src, d=0):
        """cs_prtsrf with the group: x[nga][2N] for one source; (csca, cabs)."""
        x = np.ascontiguousarray(x, dtype=np.complex128)
        rr = np.array([complex(ri).real, complex(ri).imag])
        s = make_src(src)
        a, b = C.c_double(), C.c_double()
        lib().oracle_cs_sym(self.h, d, omega, _dp(rr), x.ctypes.data, C.byref(s), C.byref(a), C.byref(b))
        return a.value, b.value

    def scat_fields(self, omega, ri, x, pts, srcs=None, d=0):
        """scat_fields (nfields.f90:29-197) of domain d at pts[npts][3]; x[2N, nsrc]
        (columns = sources).  With srcs the incident fields are added, as
        field_plane (nfpost.f90:316-374) does in the exterior domain.
        Returns (e, h), each [nsrc][npts][3] complex."""
        x = np.asarray(x, dtype=np.complex128)
        if x.ndim == 1:
            x = x[:, None]
        xs = np.ascontiguousarray(x.T)
        nsrc = xs.shape[0]
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        rr = np.array([complex(ri).real, complex(ri).imag])
        e = np.zeros((nsrc, len(pts), 3), dtype=np.complex128)
        h = np.zeros_like(e)
        arr = (OSrc * max(1, nsrc))(*([make_src(s) for s in srcs] if srcs else [OSrc()]))
        lib().oracle_scat_fields(self.h, d, omega, _dp(rr), nsrc, xs.ctypes.data, xs.shape[1], arr,
                                 1 if srcs else 0, len(pts), _dp(pts), e.ctypes.data, h.ctypes.data)
        return e, h

    def srcint(self, d, which, r, f, tface, k, near):
        r = np.ascontiguousarray(r, dtype=np.float64)
        kk = np.array([complex(k).real, complex(k).imag])
        res = np.zeros(3 if which == 1 else 9, dtype=np.complex128)
        lib().oracle_srcint(self.h, d, which, _dp(r), f, tface, _dp(kk), int(near), res.ctypes.data)
        return res if which == 1 else res.reshape(3, 3)

    def static_integrals(self, d, r, f, e):
        r = np.ascontiguousarray(r, dtype=np.float64)
        out = np.zeros(14)
        lib().oracle_static_integrals(self.h, d, _dp(r), f, e, _dp(out))
        return dict(K2m1=out[0:3], K21=out[3:6], K4m1=out[6:9], K41=out[9:12], K1m1=out[12], K11=out[13])

    def face_geometry(self, d, f):
        nodes = np.zeros((3, 3))
        area = C.c_double()
        sign = np.zeros(3, np.int32)
        ln = np.zeros(3)
        bn = np.zeros((3, 3))
        lib().oracle_face_geometry(self.h, d, f, _dp(nodes), C.byref(area), _ip(sign), _dp(ln), _dp(bn))
        return dict(nodes=nodes, area=area.value, sign=sign, length=ln, bnode=bn)


def field_mesh(P, d, omega, ri, x, group=None):
    """field_mesh (nfpost.f90:167-262): the fields at the centroid of every face
    of domain d's submesh (and of its images under the group), from the
    currents x (2N, nga) alone: E = sum_r ef_g(r) sum_q (beta_q f' + n div f_q
    alpha_q / (i w eps)), H likewise with -alpha, beta and det J, where f' = J
    (n0 x f_q(cp)) and n = J n0.  group: (j[nga][3][3], detj[nga],
    ef[nga][nga]) as group_info returns, default the identity.  Returns
    (e, h), each [nga * F][3]."""
    m = P.export(d)
    nodes, fn_, fe, ef_, eb = m["nodes"], m["face_node"], m["face_edge"], m["edge_face"], m["edge_bnode"]
    par = m["edge_parent"]
    N = P.N
    x = np.asarray(x, dtype=np.complex128).reshape(2 * N, -1)
    if group is None:
        J, detj, ef = np.eye(3)[None], np.ones(1), np.ones((1, 1))
    else:
        J, detj, ef = group
    nga = len(detj)
    eps = ri * ri * EPS0
    F = len(fn_)
    e = np.zeros((nga * F, 3), dtype=np.complex128)
    h = np.zeros_like(e)
    for f in range(F):
        p = nodes[fn_[f]]
        cp = p.mean(axis=0)
        cr = np.cross(p[1] - p[0], p[2] - p[0])
        n0 = cr / np.linalg.norm(cr)
        A = 0.5 * np.linalg.norm(np.cross(-(p[0] - p[2]), p[2] - p[1]))
        for g in range(nga):
            nor = J[g] @ n0
            et = np.zeros(3, complex)
            ht = np.zeros(3, complex)
            en = hn = 0j
            for r in range(nga):
                gae = ef[g, r]
                for q in range(3):
                    ed = fe[f, q]
                    sign = 1.0 if ef_[ed, 0] == f else -1.0
                    free = nodes[eb[ed, 0] if sign > 0 else eb[ed, 1]]
                    L = np.linalg.norm(nodes[m["edge_node"][ed, 0]] - nodes[m["edge_node"][ed, 1]])
                    fr = sign * L / (2 * A) * (cp - free)
                    fn = J[g] @ np.cross(n0, fr)
                    div = sign * L / A
                    al, be = x[par[ed], r], x[par[ed] + N, r]
                    ht -= fn * al * gae * detj[g]
                    hn += div * be * gae * detj[g]
                    et += fn * be * gae
                    en += div * al * gae
            en /= 1j * omega * eps
            hn /= 1j * omega * MU0
            e[g * F + f] = et + nor * en
            h[g * F + f] = ht + nor * hn
    return e, h


# ---- second-harmonic generation from a centrosymmetric surface nonlinearity ----

def _domain_geometry(P, d, qd):
    """Per face of domain d: vertices, centroid, normal, area, quadrature points;
    per (face, local edge): domain edge index, sign, length, free vertex."""
    m = P.export(d)
    nodes, fnode, fedge = m["nodes"], m["face_node"], m["face_edge"]
    w, qn = qd
    F = len(fnode)
    g = dict(m=m, F=F, w=w)
    p = nodes[fnode]  # [F][3][3]
    g["n"] = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    g["n"] /= np.linalg.norm(g["n"], axis=1)[:, None]
    g["A"] = 0.5 * np.linalg.norm(np.cross(-(p[:, 0] - p[:, 2]), p[:, 2] - p[:, 1]), axis=1)
    # quad_tri_points (quad.f90:352-367): qn[2] p1 + qn[0] p2 + qn[1] p3
    g["qp"] = (qn[None, :, 2, None] * p[:, None, 0] + qn[None, :, 0, None] * p[:, None, 1]
               + qn[None, :, 1, None] * p[:, None, 2])
    g["edge"] = fedge
    sign = np.where(m["edge_face"][fedge, 0] == np.arange(F)[:, None], 1.0, -1.0)
    g["sign"] = sign
    en = m["edge_node"][fedge]
    g["len"] = np.linalg.norm(nodes[en[..., 0]] - nodes[en[..., 1]], axis=-1)
    g["free"] = nodes[np.where(sign > 0, m["edge_bnode"][fedge, 0], m["edge_bnode"][fedge, 1])]
    return g


def _rwg(g, f, q, r):
    """rwg (rwgf.f90:13-49) of local edge q of face f at points r [..., 3]."""
    return g["sign"][f, q] * g["len"][f, q] / (2 * g["A"][f]) * (r - g["free"][f, q])


def rwg_moments(g):
    """rwg_moments (rwgf.f90:148-221): the Gram matrix <f_m, f_n> of the domain's
    RWG functions (diagonal over both faces of an edge; off-diagonal over the
    first common face)."""
    Nd = len(g["m"]["edge_node"])
    Fm = np.zeros((Nd, Nd))
    for f in range(g["F"]):
        for q in range(3):
            for p_ in range(3):
                a = _rwg(g, f, q, g["qp"][f])
                b = _rwg(g, f, p_, g["qp"][f])
                Fm[g["edge"][f, q], g["edge"][f, p_]] += g["A"][f] * np.sum(g["w"] * np.einsum("ri,ri->r", a, b))
    return Fm


def nlsurf_coef(P, d, qd, omega_ff, ri_ff, epsp, xff, chi2):
    """nlsurf_coef (nlsurf.f90:137-338, identity group, the expansion method):
    the surface polarisation P = eps0 (chi_nnn En^2 + chi_ntt Et.Et) n
    + 2 eps0 chi_ttn Et En of the fundamental surface field (efield,
    nlsurf.f90:22-51), projected on the domain's RWG functions and expanded
    through the Gram matrix.  Returns (src_coef (cM, cJ), src_vec (E0, H0)),
    each 2 Nd in the domain's edge numbering."""
    g = _domain_geometry(P, d, qd)
    m = g["m"]
    N, Nd = P.N, len(m["edge_node"])
    par = m["edge_parent"]
    chi_nnn, chi_ntt, chi_ttn = chi2
    omega_sh = 2.0 * omega_ff
    eps = ri_ff ** 2 * EPS0
    coef = np.zeros(Nd, complex)
    sc = np.zeros(2 * Nd, complex)
    sv = np.zeros(2 * Nd, complex)
    for f in range(g["F"]):
        nor = g["n"][f]
        qp = g["qp"][f]
        # efield at the quadrature points
        divj = sum(xff[par[g["edge"][f, q]]] * g["sign"][f, q] * g["len"][f, q] / g["A"][f] for q in range(3))
        ms = sum(xff[N + par[g["edge"][f, q]]] * _rwg(g, f, q, qp) for q in range(3))
        en_ = divj / (1j * omega_ff * eps)
        e = np.cross(nor, ms) + nor[None, :] * en_
        en = e @ nor
        et = e - en[:, None] * nor[None, :]
        Pn_ = EPS0 * (chi_nnn * en ** 2 + chi_ntt * np.sum(et * et, axis=1))
        Pt_ = 2.0 * EPS0 * chi_ttn * et * en[:, None]
        Pfull = Pt_ + Pn_[:, None] * nor[None, :]
        Pn = Pfull @ nor
        Pt = Pfull - Pn[:, None] * nor[None, :]
        for q in range(3):
            fmdiv = g["sign"][f, q] * g["len"][f, q] / g["A"][f]
            fm = _rwg(g, f, q, qp)
            int1 = -np.sum(g["w"] * fmdiv * Pn)
            int2 = np.sum(g["w"] * np.sum(fm * np.cross(Pt, nor[None, :]), axis=1))
            int3 = np.sum(g["w"] * np.sum(fm * Pt, axis=1))
            idx = g["edge"][f, q]
            coef[idx] += int1 * g["A"][f] / epsp[f]
            sc[idx + Nd] += int3 * g["A"][f]
            sv[idx + Nd] += int2 * g["A"][f]
    sc[Nd:] = -sc[Nd:] * 1j * omega_sh
    sv[:Nd] = 0.5 * coef
    sv[Nd:] = 0.5 * 1j * omega_sh * sv[Nd:]
    Fm = rwg_moments(g)
    sol = np.linalg.solve(Fm, np.stack([coef, sc[Nd:]], axis=1))
    coef = sol[:, 0]
    sc[Nd:] = sol[:, 1]
    cm = np.zeros(Nd, complex)
    for f in range(g["F"]):
        nor = g["n"][f]
        qp = g["qp"][f]
        ex = sum(_rwg(g, f, q, qp) * coef[g["edge"][f, q]] for q in range(3))
        ncr = np.cross(nor[None, :], ex)
        for q in range(3):
            cm[g["edge"][f, q]] += g["A"][f] * np.sum(g["w"] * np.sum(_rwg(g, f, q, qp) * ncr, axis=1))
    sc[:Nd] = np.linalg.solve(Fm, cm)
    return sc, sv


def nlsurf_coef_sym(P, d, qd, omega_ff, ri_ff, epsp, xff, chi2, nf, group, keep_e, keep_h):
    """nlsurf_coef (nlsurf.f90:137-338) in representation nf of a symmetry group:
    the polarisation of Pnls_frag (nlsurf.f90:106-125) from the fundamental
    solutions of every representation (efield_invmap / Pnls_invmap,
    nlsurf.f90:54-103: the field of the image J_n r from sum_m conj(ef_n(m))
    J_n^T E_m(r), the normal J_n^T n), and the Gram systems under the
    representation's boundary conditions (edge_bc on the domain mesh: the
    E-type unknowns keep_e for coef and cJ, the H-type keep_h for cM; removed
    unknowns are zero, as reduce_system / expand_solution leave them).
    xff: [nga][2N]; group: (J[nga][3][3], detj[nga], ef[nga][nga])."""
    g = _domain_geometry(P, d, qd)
    m = g["m"]
    N, Nd = P.N, len(m["edge_node"])
    par = m["edge_parent"]
    Jg, detj, efg = group
    nga = len(detj)
    chi_nnn, chi_ntt, chi_ttn = chi2
    omega_sh = 2.0 * omega_ff
    eps = ri_ff ** 2 * EPS0
    coef = np.zeros(Nd, complex)
    sc = np.zeros(2 * Nd, complex)
    sv = np.zeros(2 * Nd, complex)
    for f in range(g["F"]):
        nor = g["n"][f]
        qp = g["qp"][f]
        # the fields of every representation at the quadrature points (efield)
        Em = []
        for mm in range(nga):
            x = xff[mm]
            divj = sum(x[par[g["edge"][f, q]]] * g["sign"][f, q] * g["len"][f, q] / g["A"][f] for q in range(3))
            ms = sum(x[N + par[g["edge"][f, q]]] * _rwg(g, f, q, qp) for q in range(3))
            en_ = divj / (1j * omega_ff * eps)
            Em.append(np.cross(nor, ms) + nor[None, :] * en_)
        Pf = np.zeros((len(qp), 3), complex)
        for n in range(nga):
            e = sum(np.conj(efg[n][mm]) * (Em[mm] @ Jg[n]) for mm in range(nga))  # J^T E, row vectors
            nn = Jg[n].T @ nor
            en = e @ nn
            et = e - en[:, None] * nn[None, :]
            Pn_ = EPS0 * (chi_nnn * en ** 2 + chi_ntt * np.sum(et * et, axis=1))
            Pt_ = 2.0 * EPS0 * chi_ttn * et * en[:, None]
            Pv = Pt_ + Pn_[:, None] * nn[None, :]
            Pf += efg[n][nf] * (Pv @ Jg[n].T)  # J P, row vectors
        Pf /= nga
        Pn = Pf @ nor
        Pt = Pf - Pn[:, None] * nor[None, :]
        for q in range(3):
            fmdiv = g["sign"][f, q] * g["len"][f, q] / g["A"][f]
            fm = _rwg(g, f, q, qp)
            int1 = -np.sum(g["w"] * fmdiv * Pn)
            int2 = np.sum(g["w"] * np.sum(fm * np.cross(Pt, nor[None, :]), axis=1))
            int3 = np.sum(g["w"] * np.sum(fm * Pt, axis=1))
            idx = g["edge"][f, q]
            coef[idx] += int1 * g["A"][f] / epsp[f]
            sc[idx + Nd] += int3 * g["A"][f]
            sv[idx + Nd] += int2 * g["A"][f]
    sc[Nd:] = -sc[Nd:] * 1j * omega_sh
    sv[:Nd] = 0.5 * coef
    sv[Nd:] = 0.5 * 1j * omega_sh * sv[Nd:]
    Fm = rwg_moments(g)
    ke = np.nonzero(keep_e)[0]
    sol = np.zeros((Nd, 2), complex)
    sol[ke] = np.linalg.solve(Fm[np.ix_(ke, ke)], np.stack([coef, sc[Nd:]], axis=1)[ke])
    coef = sol[:, 0]
    sc[Nd:] = sol[:, 1]
    cm = np.zeros(Nd, complex)
    for f in range(g["F"]):
        nor = g["n"][f]
        qp = g["qp"][f]
        ex = sum(_rwg(g, f, q, qp) * coef[g["edge"][f, q]] for q in range(3))
        ncr = np.cross(nor[None, :], ex)
        for q in range(3):
            cm[g["edge"][f, q]] += g["A"][f] * np.sum(g["w"] * np.sum(_rwg(g, f, q, qp) * ncr, axis=1))
    kh = np.nonzero(keep_h)[0]
    sc[:Nd] = 0
    sc[kh] = np.linalg.solve(Fm[np.ix_(kh, kh)], cm[kh])
    return sc, sv


def shg_solve_sym(P, omega, ri, shri, nls, x, qd_name="tri_gl13", coef_out=None):
    """The nonlinear branch of solve_batch with the problem's symmetry group
    (solver.f90:143-217): per representation nf the source terms of every
    nonlinear domain (nlsurf_coef_sym, and -A_{d,nf} c_{d,nf} with the domain's
    blocks, sysmat.f90:112-229), the matrices at 2 omega with the SH indices
    and solve_sym.  x: fundamental solutions [nga][2N] for one source.  Returns
    nlx [nga][2N]."""
    qd = tri_rule(qd_name)
    N = P.N
    J, detj, ef = P.group_info()
    nga = len(detj)
    x = np.asarray(x, dtype=np.complex128).reshape(nga, 2 * N)
    nlx = np.zeros((nga, 2 * N), complex)
    for d in range(P.ndom):
        if nls[d] is None:
            continue
        m = P.export(d)
        par = m["edge_parent"]
        Nd = len(par)
        epsp = epsp_of(P, d, ri)
        Ad = P.sysmat_sym_dom(2.0 * omega, [complex(v) for v in shri], d)
        for nf in range(nga):
            idv, _ = P.edge_bc(nf)
            keep_e = idv[par] != -1
            keep_h = idv[N + par] != -1
            sc, sv = nlsurf_coef_sym(P, d, qd, omega, complex(ri[d]), epsp, x, nls[d], nf, (J, detj, ef), keep_e,
                                     keep_h)
            nlx[nf, par] += sv[:Nd]
            nlx[nf, par + N] += sv[Nd:]
            c = np.zeros(2 * N, complex)
            c[par] = sc[Nd:]
            c[par + N] = sc[:Nd]
            nlx[nf] -= Ad[nf] @ c
            if coef_out is not None:
                coef_out.setdefault(d, np.zeros((nga, 2 * N), complex))[nf] = c
    A = P.sysmat_sym(2.0 * omega, [complex(v) for v in shri])
    return P.solve_sym(A, nlx)


def epsp_of(P, d, ri):
    """determine_epsp (solver.f90:393-433): per face of domain d, eps0 ri^2 of the
    first other domain that contains the same face."""
    md = P.export(d)
    key = lambda nodes, fn: [tuple(sorted(map(tuple, np.round(nodes[f], 20)))) for f in fn]
    mine = key(md["nodes"], md["face_node"])
    out = np.zeros(len(mine), complex)
    found = np.zeros(len(mine), bool)
    for d2 in range(P.ndom):
        if d2 == d:
            continue
        m2 = P.export(d2)
        other = set(key(m2["nodes"], m2["face_node"]))
        for i, k in enumerate(mine):
            if not found[i] and k in other:
                out[i] = complex(ri[d2]) ** 2 * EPS0
                found[i] = True
    if not found.all():
        raise RuntimeError("Could not find epsp!")
    return out


def domain_matrix(P, d, omega, ri_d):
    """The PMCHWT blocks of domain d alone (sysmat.f90:70-99 for one domain,
    identity group), 2N x 2N."""
    m = P.export(d)
    par = m["edge_parent"]
    N = P.N
    S = P.operator(d, 0, omega, ri_d) + P.operator(d, 1, omega, ri_d)
    K = P.operator(d, 2, omega, ri_d)
    Zsi = ri_d ** 2 / ETA0 ** 2
    A = np.zeros((2 * N, 2 * N), complex)
    ix = np.ix_(par, par)
    A[ix] += S
    A[np.ix_(par + N, par + N)] += Zsi * S
    A[np.ix_(par + N, par)] += K
    A[np.ix_(par, par + N)] -= K
    return A


def shg_solve(P, omega, ri, shri, nls, x, qd_name="tri_gl13", coef_out=None):
    """The nonlinear branch of solve_batch for a centrosymmetric surface
    nonlinearity (solver.f90:143-217, identity group): for every domain d with
    nls[d] = (chi_nnn, chi_ntt, chi_ttn) the source coefficients of
    nlsurf_coef, the source vector E0, H0 and the matrix terms of
    sysmat_pmchwt_nls (sysmat.f90:112-229) at 2 omega with the SH refractive
    indices, then the SH solve.  x: fundamental solutions [2N][nsrc].
    Returns nlx [2N][nsrc]; coef_out (a dict), if given, receives per
    nonlinear domain the source coefficients on the global unknowns (cJ in
    rows [0, N), cM in rows [N, 2N)), [2N][nsrc]."""
    qd = tri_rule(qd_name)
    N = P.N
    x = np.asarray(x, dtype=np.complex128).reshape(2 * N, -1)
    nsrc = x.shape[1]
    nlx = np.zeros((2 * N, nsrc), complex)
    for d in range(P.ndom):
        if nls[d] is None:
            continue
        m = P.export(d)
        par = m["edge_parent"]
        Nd = len(par)
        epsp = epsp_of(P, d, ri)
        Ad = domain_matrix(P, d, 2.0 * omega, complex(shri[d]))
        if coef_out is not None:
            coef_out[d] = np.zeros((2 * N, nsrc), complex)
        for s in range(nsrc):
            sc, sv = nlsurf_coef(P, d, qd, omega, complex(ri[d]), epsp, x[:, s], nls[d])
            nlx[par, s] += sv[:Nd]
            nlx[par + N, s] += sv[Nd:]
            c = np.zeros(2 * N, complex)
            c[par] = sc[Nd:]      # cJ on the J columns
            c[par + N] = sc[:Nd]  # cM on the M columns
            nlx[:, s] -= Ad @ c
            if coef_out is not None:
                coef_out[d][:, s] = c
    A = P.sysmat(2.0 * omega, [complex(v) for v in shri])
    return solve(A, nlx)


def solve(A, q):
    """solve_multi_linsys (linalg.f90:159-180): ZGETRF + ZGETRS('N'), STOP on INFO /= 0."""
    from scipy.linalg import lapack
    lu, piv, info = lapack.zgetrf(A, overwrite_a=False)
    if info != 0:
        raise RuntimeError("Matrix factorization failed!")
    x, info = lapack.zgetrs(lu, piv, q)
    if info != 0:
        raise RuntimeError("Solving of system failed!")
    return x
