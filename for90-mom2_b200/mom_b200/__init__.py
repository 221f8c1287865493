"""Python front end of the B200 PMCHWT library (``lib/libmomgpu.so``).

A thin ctypes layer over the C ABI in ``include/mom_gpu.h``, with names that
mirror the reference's Fortran entry points for the linear scattering path:

    sysmat_pmchwt  (sysmat.f90:18)      -> Solver.sysmat
    srcvec         (source.f90:136)     -> Solver.srcvec
    solve_systems  (solver.f90:325)     -> Solver.solve
    cs_prtsrf      (cs.f90:14)          -> Solver.cross_sections
    rcs            (ffields.f90:252)    -> Solver.rcs
    solve_batch    (solver.f90:17)      -> Solver.solve_wavelength (one wavelength)

and the problem set-up commands ``mesh`` / ``ndom`` / ``sdom`` / ``fdom``
(interface.f90:32-123, 357-366) -> Problem.  All computation runs in the
CUDA library; there is no CPU fallback: importing this module on a machine
where the library cannot be loaded raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# MOM_GPU_LIB selects another build of the same library (e.g. for A/B timing).
LIB_PATH = os.environ.get("MOM_GPU_LIB") or os.path.join(os.path.dirname(_HERE), "lib", "libmomgpu.so")

MOM_OK = 0
MOM_ERR_ARG, MOM_ERR_ALLOC, MOM_ERR_CUDA, MOM_ERR_SINGULAR, MOM_ERR_TIMEOUT = 1, 2, 3, 4, 5
MOM_ERR_STATE, MOM_ERR_MESH, MOM_ERR_NOCONV, MOM_ERR_IO = 6, 7, 8, 9
FP64, MIXED = 0, 1
SRC_NONE, SRC_PW, SRC_PW_ELLIPTIC = 0, 1, 10

# constants.f90:8-14 (pi is a single-precision literal in the reference)
PI_F = float(np.float32(3.141592653589))
C0 = 2.997924580003e8
DEGTORAD = PI_F / 180.0

# Every entry point the C ABI header declares (checked by the tests).
EXPORTS = [
    "mom_gpu_create", "mom_gpu_destroy", "mom_gpu_strerror", "mom_gpu_last_error", "mom_gpu_set_problem",
    "mom_gpu_sysmat", "mom_gpu_srcvec", "mom_gpu_solve", "mom_gpu_solve_wavelength", "mom_gpu_cross_sections",
    "mom_gpu_rcs", "mom_gpu_cross_sections_noalloc", "mom_gpu_device_matrix", "mom_gpu_device_solution", "mom_gpu_synchronize",
    "mom_gpu_launch_count", "mom_gpu_stream", "mom_gpu_library_calls", "mom_gpu_tensor_flops", "mom_gpu_profile", "mom_gpu_profile_read",
    "mom_gpu_selftest_cgemm", "mom_problem_create", "mom_problem_destroy", "mom_problem_load_gmsh",
    "mom_problem_set_mesh", "mom_problem_set_ndom", "mom_problem_set_domain", "mom_problem_finalize",
    "mom_problem_nedges", "mom_problem_ndom", "mom_problem_domain", "mom_tri_rule", "mom_problem_upload",
    "mom_gpu_adjoint", "mom_gpu_adjoint_mean_eps", "mom_gpu_domain_nodes", "mom_problem_node_parent",
    "mom_gpu_sweep", "mom_gpu_sweep_many", "mom_gpu_autotune_result", "mom_gpu_autotune_placement", "mom_gpu_scat_fields",
    "mom_gpu_set_matrix", "mom_gpu_set_wait_limits", "mom_gpu_set_symmetry", "mom_gpu_group_order",
    "mom_problem_set_lines", "mom_problem_classify_edges", "mom_problem_edge_bnd",
    "mom_gpu_surface_fields", "mom_gpu_group_action", "mom_gpu_shg_solve",
    "mom_gpu_shg_source_coef",
]

# Boundary types of mesh edges (sbnd; mesh.f90:16-25).
BND_NONE, BND_XPLANE, BND_YPLANE, BND_ZPLANE = 1, 2, 3, 4
BND_NAMES = {"xplane": BND_XPLANE, "yplane": BND_YPLANE, "zplane": BND_ZPLANE}


class MomError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d)" % (msg, status))
        self.status = status


class MomMesh(C.Structure):
    _fields_ = [("nnodes", C.c_int32), ("nfaces", C.c_int32), ("nedges", C.c_int32),
                ("nodes", C.POINTER(C.c_double)), ("face_nodes", C.POINTER(C.c_int32)),
                ("face_edges", C.POINTER(C.c_int32)), ("edge_nodes", C.POINTER(C.c_int32)),
                ("edge_faces", C.POINTER(C.c_int32)), ("edge_bnodes", C.POINTER(C.c_int32)),
                ("edge_parent", C.POINTER(C.c_int32))]


class MomSrc(C.Structure):
    _fields_ = [("type", C.c_int32), ("theta", C.c_double), ("phi", C.c_double), ("psi", C.c_double),
                ("phase_re", C.c_double), ("phase_im", C.c_double)]


class MomNls(C.Structure):
    _fields_ = [("active", C.c_int32), ("chi_nnn", C.c_double * 2), ("chi_ntt", C.c_double * 2),
                ("chi_ttn", C.c_double * 2)]


_lib = None


def lib():
    """Load the CUDA library (raises if it is missing: no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libmomgpu.so not built; run __graft_entry__.build() (for90-mom2_b200/mom_build.py)")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
    L.mom_gpu_create.argtypes = [C.c_int32, C.POINTER(vp)]
    L.mom_gpu_destroy.argtypes = [vp]
    L.mom_gpu_destroy.restype = None
    L.mom_gpu_strerror.argtypes = [C.c_int32]
    L.mom_gpu_strerror.restype = C.c_char_p
    L.mom_gpu_last_error.argtypes = [vp]
    L.mom_gpu_last_error.restype = C.c_char_p
    L.mom_gpu_set_problem.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(MomMesh), C.c_int32, dp, dp]
    L.mom_gpu_sysmat.argtypes = [vp, C.c_double, dp, C.c_int32, vp, C.c_int64]
    L.mom_gpu_srcvec.argtypes = [vp, C.c_double, dp, C.c_int32, C.POINTER(MomSrc), vp, C.c_int64]
    L.mom_gpu_solve.argtypes = [vp, C.c_int32, C.c_double, C.c_int32, vp, C.c_int64, ip]
    L.mom_gpu_solve_wavelength.argtypes = [vp, C.c_double, dp, C.c_int32, C.POINTER(MomSrc), C.c_int32, C.c_double,
                                           C.c_int32, vp, C.c_int64, ip]
    L.mom_gpu_cross_sections.argtypes = [vp, C.c_int32, C.c_double, dp, C.c_int32, C.POINTER(MomSrc), vp, C.c_int64,
                                         dp, dp]
    L.mom_gpu_rcs.argtypes = [vp, C.c_int32, C.c_double, dp, C.c_int32, vp, C.c_int64, C.c_int32, C.c_int32, dp]
    L.mom_gpu_scat_fields.argtypes = [vp, C.c_int32, C.c_double, dp, C.c_int32, C.POINTER(MomSrc), vp, C.c_int64,
                                      C.c_int32, dp, dp, dp]
    L.mom_gpu_cross_sections_noalloc.argtypes = [vp, C.c_int32, C.c_double, dp, C.c_int32, C.POINTER(MomSrc), vp,
                                                 C.c_int64, dp, dp]
    L.mom_gpu_adjoint.argtypes = [vp, C.c_int32, C.c_double, dp, C.c_int32, C.POINTER(MomSrc), C.c_int32, C.c_double,
                                  C.c_int32, vp, vp, ip]
    L.mom_gpu_adjoint_mean_eps.argtypes = [vp, C.c_int32, C.c_double, dp, C.c_int32, C.POINTER(MomSrc), C.c_int32,
                                           C.c_double, C.c_int32, dp, ip]
    L.mom_gpu_domain_nodes.argtypes = [vp, C.c_int32]
    L.mom_gpu_sweep.argtypes = [vp, C.c_int32, dp, dp, C.c_int32, C.POINTER(MomSrc), C.c_int32, C.c_double,
                                C.c_int32, dp, dp, ip]
    L.mom_gpu_sweep_many.argtypes = [C.c_int32, C.POINTER(vp), ip, C.POINTER(dp), C.POINTER(dp), C.c_int32,
                                     C.POINTER(MomSrc), C.c_int32, C.c_double, C.c_int32, C.POINTER(dp),
                                     C.POINTER(dp), ip]
    L.mom_gpu_autotune_result.argtypes = [vp, C.c_int32, C.c_int32, ip, C.POINTER(C.c_int64), ip, dp, dp]
    L.mom_gpu_autotune_placement.argtypes = [vp, C.c_int32, C.c_int32, ip, ip, dp]
    L.mom_problem_node_parent.argtypes = [vp, C.c_int32, ip]
    L.mom_gpu_device_matrix.argtypes = [vp, C.POINTER(vp), C.POINTER(C.c_int64)]
    L.mom_gpu_set_matrix.argtypes = [vp, C.c_int32, vp, C.c_int64]
    L.mom_gpu_set_wait_limits.argtypes = [vp, C.c_int64, C.c_int64, C.c_int64]
    L.mom_gpu_set_symmetry.argtypes = [vp, C.c_int32, C.POINTER(C.c_char_p), ip]
    L.mom_gpu_group_order.argtypes = [vp]
    L.mom_problem_set_lines.argtypes = [vp, C.c_int32, ip, ip]
    L.mom_problem_classify_edges.argtypes = [vp, C.c_int32, C.c_int32, ip]
    L.mom_problem_edge_bnd.argtypes = [vp, ip]
    L.mom_gpu_surface_fields.argtypes = [vp, C.c_int32, C.c_double, dp, C.c_int32, vp, C.c_int64, dp, dp]
    L.mom_gpu_group_action.argtypes = [vp, C.c_int32, dp, dp]
    L.mom_gpu_shg_solve.argtypes = [vp, C.c_double, dp, dp, C.POINTER(MomNls), C.c_int32, C.c_double, C.c_int32,
                                    vp, C.c_int64, ip]
    L.mom_gpu_shg_source_coef.argtypes = [vp, C.c_int32, vp, C.c_int64]
    L.mom_gpu_device_solution.argtypes = [vp, C.POINTER(vp), C.POINTER(C.c_int64), ip]
    L.mom_gpu_synchronize.argtypes = [vp]
    L.mom_gpu_launch_count.argtypes = [vp]
    L.mom_gpu_launch_count.restype = C.c_int64
    L.mom_gpu_stream.argtypes = [vp]
    L.mom_gpu_stream.restype = C.c_void_p
    L.mom_gpu_library_calls.argtypes = [vp]
    L.mom_gpu_library_calls.restype = C.c_int64
    L.mom_gpu_tensor_flops.argtypes = [vp]
    L.mom_gpu_tensor_flops.restype = C.c_double
    L.mom_gpu_profile.argtypes = [vp, C.c_int32]
    L.mom_gpu_profile_read.argtypes = [vp, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    fp = C.POINTER(C.c_float)
    L.mom_gpu_selftest_cgemm.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, fp, fp, fp]
    L.mom_problem_create.argtypes = [C.POINTER(vp)]
    L.mom_problem_destroy.argtypes = [vp]
    L.mom_problem_destroy.restype = None
    L.mom_problem_load_gmsh.argtypes = [vp, C.c_char_p, C.c_double]
    L.mom_problem_set_mesh.argtypes = [vp, C.c_int32, dp, C.c_int32, ip, ip, C.c_double]
    L.mom_problem_set_ndom.argtypes = [vp, C.c_int32]
    L.mom_problem_set_domain.argtypes = [vp, C.c_int32, C.c_int32, ip]
    L.mom_problem_finalize.argtypes = [vp]
    L.mom_problem_nedges.argtypes = [vp]
    L.mom_problem_ndom.argtypes = [vp]
    L.mom_problem_domain.argtypes = [vp, C.c_int32, C.POINTER(MomMesh)]
    L.mom_tri_rule.argtypes = [C.c_char_p, dp, dp]
    L.mom_problem_upload.argtypes = [vp, vp, C.c_char_p]
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _check(status, ctx=None, what=""):
    if status != MOM_OK:
        msg = lib().mom_gpu_strerror(status).decode()
        if ctx is not None:
            detail = lib().mom_gpu_last_error(ctx).decode()
            if detail:
                msg = detail
        raise MomError(status, (what + ": " if what else "") + msg)


def tri_rule(name: str = "tri_gl13"):
    """Triangle quadrature of quad.f90 (weights[nq], nodes[nq, 3])."""
    w = np.zeros(13)
    nd = np.zeros((13, 3))
    nq = lib().mom_tri_rule(name.encode(), _dp(w), _dp(nd))
    if nq < 0:
        raise MomError(MOM_ERR_ARG, "Unrecognized quadrature type " + name)
    return w[:nq].copy(), nd[:nq].copy()


def omega_of(wl: float) -> float:
    """omega = 2 pi c0 / wl with the reference's float-rounded pi (solver.f90:77)."""
    return 2.0 * PI_F * C0 / wl


def src_pw(theta_deg: float, phi_deg: float, psi_deg: float) -> dict:
    """``ssrc i 'pw' theta phi psi`` (interface.f90:500-505): degrees -> radians."""
    return dict(type="pw", theta=theta_deg * DEGTORAD, phi=phi_deg * DEGTORAD, psi=psi_deg * DEGTORAD)


def src_pw_elliptic(theta_deg: float, phi_deg: float, phase: complex) -> dict:
    return dict(type="pw_elliptic", theta=theta_deg * DEGTORAD, phi=phi_deg * DEGTORAD, phase=complex(phase))


def src_none() -> dict:
    """No incident field (nlsrc%type = 0): the cross sections of second-harmonic solutions."""
    return dict(type="none")


def _srcs(srcs):
    if isinstance(srcs, dict):
        srcs = [srcs]
    arr = (MomSrc * len(srcs))()
    for i, s in enumerate(srcs):
        if s["type"] == "none":
            arr[i] = MomSrc(SRC_NONE, 0.0, 0.0, 0.0, 0.0, 0.0)
        elif s["type"] == "pw":
            arr[i] = MomSrc(SRC_PW, s["theta"], s["phi"], s["psi"], 0.0, 0.0)
        else:
            ph = complex(s["phase"])
            arr[i] = MomSrc(SRC_PW_ELLIPTIC, s["theta"], s["phi"], 0.0, ph.real, ph.imag)
    return arr, len(srcs)


def _ri(ri):
    vals = [complex(v) for v in (ri if np.ndim(ri) else [ri])]
    return np.array([[v.real, v.imag] for v in vals], dtype=np.float64).ravel()


class Problem:
    """Master mesh and domain submeshes (mesh / ndom / sdom / fdom commands)."""

    def __init__(self):
        h = C.c_void_p()
        _check(lib().mom_problem_create(C.byref(h)), what="mom_problem_create")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            lib().mom_problem_destroy(self.h)
            self.h = None

    @classmethod
    def from_gmsh(cls, path, scale, domains):
        p = cls()
        _check(lib().mom_problem_load_gmsh(p.h, path.encode(), scale), what="load " + path)
        p.set_domains(domains)
        return p

    @classmethod
    def from_arrays(cls, nodes, faces, face_ids, scale, domains):
        p = cls()
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        faces = np.ascontiguousarray(faces, dtype=np.int32)
        ids = np.ascontiguousarray(face_ids, dtype=np.int32)
        _check(lib().mom_problem_set_mesh(p.h, len(nodes), _dp(nodes), len(faces), _ip(faces), _ip(ids), scale),
               what="mesh")
        p.set_domains(domains)
        return p

    def set_lines(self, line_nodes, line_ids):
        """Line elements of the master mesh (0-based node pairs and physical ids)."""
        ln = np.ascontiguousarray(np.asarray(line_nodes, dtype=np.int32).reshape(-1, 2))
        li = np.ascontiguousarray(np.broadcast_to(np.asarray(line_ids, dtype=np.int32), (len(ln),)))
        _check(lib().mom_problem_set_lines(self.h, len(ln), _ip(ln), _ip(li)), what="lines")

    def classify_edges(self, line_id, bnd):
        """sbnd: master edges on the lines of physical id line_id get boundary type
        bnd ("xplane", "yplane", "zplane" or a BND_* value); returns the match count."""
        b = BND_NAMES.get(bnd, bnd)
        cnt = C.c_int32()
        _check(lib().mom_problem_classify_edges(self.h, line_id, b, C.byref(cnt)), what="sbnd")
        return cnt.value

    def edge_bnd(self):
        out = np.zeros(self.nedges, dtype=np.int32)
        _check(lib().mom_problem_edge_bnd(self.h, _ip(out)), what="edge_bnd")
        return out

    def set_domains(self, domains):
        L = lib()
        _check(L.mom_problem_set_ndom(self.h, len(domains)), what="ndom")
        for d, ids in enumerate(domains):
            a = np.ascontiguousarray(ids, dtype=np.int32)
            _check(L.mom_problem_set_domain(self.h, d, len(a), _ip(a)), what="sdom %d" % (d + 1))
        _check(L.mom_problem_finalize(self.h), what="fdom")

    @property
    def nedges(self):
        return lib().mom_problem_nedges(self.h)

    @property
    def ndom(self):
        return lib().mom_problem_ndom(self.h)

    def domain(self, d):
        """Copy of the flattened topology of domain d (d = -1: master mesh)."""
        m = MomMesh()
        _check(lib().mom_problem_domain(self.h, d, C.byref(m)), what="domain")

        def arr(ptr, n, k, dt):
            return np.ctypeslib.as_array(ptr, shape=(n * k,)).reshape(n, k).astype(dt).copy() if n else None

        return dict(nodes=arr(m.nodes, m.nnodes, 3, np.float64), face_node=arr(m.face_nodes, m.nfaces, 3, np.int32),
                    face_edge=arr(m.face_edges, m.nfaces, 3, np.int32),
                    edge_node=arr(m.edge_nodes, m.nedges, 2, np.int32),
                    edge_face=arr(m.edge_faces, m.nedges, 2, np.int32),
                    edge_bnode=arr(m.edge_bnodes, m.nedges, 2, np.int32),
                    edge_parent=arr(m.edge_parent, m.nedges, 1, np.int32).ravel())


    def node_parent(self, d):
        """Master-mesh node index of each submesh node of domain d."""
        n = self.domain(d)["nodes"].shape[0]
        out = np.zeros(n, dtype=np.int32)
        _check(lib().mom_problem_node_parent(self.h, d, out.ctypes.data_as(C.POINTER(C.c_int32))),
               what="node_parent")
        return out

    def master_nodes(self):
        return self.domain(-1)["nodes"].shape[0]


def sweep_many(solvers, omegas, ri_per_wl, srcs, precision=MIXED, tol=1e-12, maxit=30):
    """Sweeps of several problems concurrently (one host thread per solver inside
    the library).  omegas[i], ri_per_wl[i]: wavelengths of solver i.  Returns a list
    of (csca, cabs)."""
    arr, ns = _srcs(srcs)
    k = len(solvers)
    hs = (C.c_void_p * k)(*[s.h for s in solvers])
    oms = [np.ascontiguousarray(o, dtype=np.float64) for o in omegas]
    ris = [np.ascontiguousarray(np.asarray(r, dtype=np.complex128).reshape(len(o), s.ndom)).view(np.float64).ravel()
           for r, o, s in zip(ri_per_wl, oms, solvers)]
    outs = [(np.zeros((len(o), ns)), np.zeros((len(o), ns))) for o in oms]
    nwl = np.array([len(o) for o in oms], dtype=np.int32)
    dpp = C.POINTER(C.c_double)
    po = (dpp * k)(*[_dp(o) for o in oms])
    pr = (dpp * k)(*[_dp(r) for r in ris])
    pa = (dpp * k)(*[_dp(o[0]) for o in outs])
    pb = (dpp * k)(*[_dp(o[1]) for o in outs])
    st = np.zeros(k, dtype=np.int32)
    rc = lib().mom_gpu_sweep_many(k, hs, nwl.ctypes.data_as(C.POINTER(C.c_int32)), po, pr, ns, arr, precision, tol,
                                  maxit, pa, pb, st.ctypes.data_as(C.POINTER(C.c_int32)))
    if rc != MOM_OK:
        bad = int(np.nonzero(st)[0][0]) if np.any(st) else 0
        _check(rc, solvers[bad].h, "sweep_many")
    return outs


class Solver:
    """One CUDA context of the PMCHWT library on ``device``."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = lib().mom_gpu_create(device, C.byref(h))
        if st != MOM_OK:
            raise MomError(st, "mom_gpu_create failed: " + lib().mom_gpu_strerror(st).decode())
        self.h = h
        self.N = None
        self.ndom = None
        self.nga = 1

    def close(self):
        if getattr(self, "h", None):
            lib().mom_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _ck(self, st, what):
        _check(st, self.h, what)

    def set_problem(self, problem: Problem, quad: str = "tri_gl13"):
        self._ck(lib().mom_problem_upload(problem.h, self.h, quad.encode()), "set_problem")
        self.N = problem.nedges
        self.ndom = problem.ndom
        self.nga = 1
        self._dom_faces = [problem.domain(d)["face_node"].shape[0] for d in range(problem.ndom)]

    def domain_faces(self, dom):
        return self._dom_faces[dom]

    def set_symmetry(self, names, problem: Problem):
        """read_symm: the product of the named groups ("id", "mxp", "myp", "mzp") with the
        boundary types of the problem's master edges (sbnd); returns the group order."""
        arr = (C.c_char_p * max(1, len(names)))(*[n.encode() for n in names])
        bnd = problem.edge_bnd()
        self._ck(lib().mom_gpu_set_symmetry(self.h, len(names), arr, _ip(bnd)), "set_symmetry")
        self.nga = lib().mom_gpu_group_order(self.h)
        return self.nga

    def _cols(self, ns):
        """Host array of solutions or right-hand sides: (2N, ns), or (2N, nga, ns) with a group."""
        shape = (2 * self.N, ns) if self.nga == 1 else (2 * self.N, self.nga, ns)
        return np.zeros(shape, dtype=np.complex128, order="F")

    def sysmat(self, omega, ri, precision=FP64, want_host=False):
        """sysmat_pmchwt: build the 2N x 2N matrix (one per representation) on the
        device, optionally copied back: (2N, 2N), or (nga, 2N, 2N) with a group."""
        r = _ri(ri)
        if len(r) != 2 * self.ndom:
            raise ValueError("one refractive index per domain")
        A = np.zeros((2 * self.N, 2 * self.N, self.nga), dtype=np.complex128, order="F") if want_host else None
        self._ck(lib().mom_gpu_sysmat(self.h, omega, _dp(r), precision, A.ctypes.data if A is not None else None,
                                      2 * self.N), "sysmat")
        if A is None:
            return None
        return A[:, :, 0] if self.nga == 1 else np.moveaxis(A, 2, 0)

    def set_matrix(self, A, precision=FP64):
        """A caller's 2N x 2N system matrix in place of sysmat (mom_gpu_set_matrix)."""
        A = np.asfortranarray(np.asarray(A, dtype=np.complex128))
        if A.shape != (2 * self.N, 2 * self.N):
            raise ValueError("the matrix must be 2N x 2N")
        self._ck(lib().mom_gpu_set_matrix(self.h, precision, A.ctypes.data, 2 * self.N), "set_matrix")

    def set_wait_limits(self, panel=0, gemm=0, solve=0):
        """Polls before the bounded device waits give up (0: the defaults)."""
        self._ck(lib().mom_gpu_set_wait_limits(self.h, panel, gemm, solve), "set_wait_limits")

    def srcvec(self, omega, ri1, srcs, want_host=False):
        arr, ns = _srcs(srcs)
        r = _ri(ri1)
        q = self._cols(ns) if want_host else None
        self._ck(lib().mom_gpu_srcvec(self.h, omega, _dp(r), ns, arr, q.ctypes.data if q is not None else None,
                                      2 * self.N), "srcvec")
        self.nsrc = ns
        return q

    def solve(self, precision=FP64, tol=1e-12, maxit=30, want_host=True):
        x = self._cols(self.nsrc) if want_host else None
        it = C.c_int32()
        self._ck(lib().mom_gpu_solve(self.h, precision, tol, maxit, x.ctypes.data if x is not None else None,
                                     2 * self.N, C.byref(it)), "solve")
        self.iters = it.value
        return x

    def solve_wavelength(self, omega, ri, srcs, precision=FP64, tol=1e-12, maxit=30, want_host=True):
        arr, ns = _srcs(srcs)
        r = _ri(ri)
        x = self._cols(ns) if want_host else None
        it = C.c_int32()
        self._ck(lib().mom_gpu_solve_wavelength(self.h, omega, _dp(r), ns, arr, precision, tol, maxit,
                                                x.ctypes.data if x is not None else None, 2 * self.N, C.byref(it)),
                 "solve_wavelength")
        self.nsrc = ns
        self.iters = it.value
        return x

    def shg_solve(self, omega, ri, shri, nls, precision=FP64, tol=1e-12, maxit=30, want_host=True):
        """The second-harmonic solve after solve_wavelength at the fundamental
        frequency omega (solver.f90:143-217): nls[d] is None for a linear domain or
        (chi_nnn, chi_ntt, chi_ttn) of its surface nonlinearity (``smed m nlsurf
        value ...``); ri / shri are the fundamental and second-harmonic refractive
        indices per domain.  Returns nlx (2N x nsrc, or 2N x nga x nsrc with a
        mirror group: the polarisation projected on each representation);
        afterwards the device solutions are the second harmonic's (cross sections
        with src_none() at 2 omega and shri)."""
        if len(nls) != self.ndom:
            raise ValueError("nls needs one entry per domain")
        arr = (MomNls * self.ndom)()
        for d, v in enumerate(nls):
            if v is None:
                arr[d] = MomNls(0, (0.0, 0.0), (0.0, 0.0), (0.0, 0.0))
            else:
                c = [complex(t) for t in v]
                arr[d] = MomNls(1, (c[0].real, c[0].imag), (c[1].real, c[1].imag), (c[2].real, c[2].imag))
        r, rs = _ri(ri), _ri(shri)
        x = self._cols(self.nsrc) if want_host else None
        it = C.c_int32()
        self._ck(lib().mom_gpu_shg_solve(self.h, omega, _dp(r), _dp(rs), arr, precision, tol, maxit,
                                         x.ctypes.data if x is not None else None, 2 * self.N, C.byref(it)),
                 "shg_solve")
        self.iters = it.value
        return x

    def shg_source_coef(self, dom):
        """The source coefficients (cJ on rows [0, N), cM on [N, 2N)) of nonlinear
        domain dom from the last shg_solve, 2N x nsrc (2N x nga x nsrc with a group)."""
        x = self._cols(self.nsrc)
        self._ck(lib().mom_gpu_shg_source_coef(self.h, dom, x.ctypes.data, 2 * self.N), "shg_source_coef")
        return x

    def cross_sections(self, omega, ri, srcs, x=None, dom=0):
        """cs_prtsrf: (csca[nsrc], cabs[nsrc]) from x (2N x nsrc) or the device solutions."""
        arr, ns = _srcs(srcs)
        r = _ri(ri)
        csca = np.zeros(ns)
        cabs = np.zeros(ns)
        xp = None
        if x is not None:
            x = np.asfortranarray(np.asarray(x, dtype=np.complex128).reshape(2 * self.N, -1, order="F"))
            xp = x.ctypes.data
        self._ck(lib().mom_gpu_cross_sections(self.h, dom, omega, _dp(r), ns, arr, xp, 2 * self.N, _dp(csca),
                                              _dp(cabs)), "cross_sections")
        return csca, cabs

    def adjoint(self, omega, ri, srcs, precision, eps_dom=None, nodes=False, tol=1e-12, maxit=30):
        """Adjoint gradients of sigma_ext and sigma_abs for the sources of the last solve.

        Returns a dict: ``deps`` [nsrc][2 (ext, abs)][2 (d/dRe eps, d/dIm eps)] of interior
        domain eps_dom, and with nodes=True ``dnodes``: a list over domains of
        [nsrc][2][nnodes_d][3] arrays (d sigma / d node coordinates, per metre)."""
        arr, ns = _srcs(srcs)
        r = _ri(ri)
        deps = np.zeros((ns, 2, 2)) if eps_dom is not None else None
        counts = [lib().mom_gpu_domain_nodes(self.h, d) for d in range(self.ndom)]
        total = sum(counts)
        dn = np.zeros((ns, 2, total, 3)) if nodes else None
        it = C.c_int32()
        self._ck(lib().mom_gpu_adjoint(self.h, precision, omega, _dp(r), ns, arr,
                                       -1 if eps_dom is None else eps_dom, 1e-12 if tol is None else tol, maxit,
                                       deps.ctypes.data if deps is not None else None,
                                       dn.ctypes.data if dn is not None else None, C.byref(it)), "adjoint")
        out = {"iters": it.value}
        if deps is not None:
            out["deps"] = deps
        if dn is not None:
            offs = np.cumsum([0] + counts)
            out["dnodes"] = [dn[:, :, offs[d]:offs[d + 1], :] for d in range(self.ndom)]
        return out

    def sweep(self, omegas, ri_per_wl, srcs, precision=MIXED, tol=1e-12, maxit=30):
        """solve_batch over wavelengths: (csca[nwl][nsrc], cabs[nwl][nsrc], iters[nwl])."""
        arr, ns = _srcs(srcs)
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        nwl = len(om)
        r = np.ascontiguousarray(np.asarray(ri_per_wl, dtype=np.complex128).reshape(nwl, self.ndom)).view(np.float64)
        csca = np.zeros((nwl, ns))
        cabs = np.zeros((nwl, ns))
        it = np.zeros(nwl, dtype=np.int32)
        self._ck(lib().mom_gpu_sweep(self.h, nwl, _dp(om), _dp(r.ravel()), ns, arr, precision, tol, maxit, _dp(csca),
                                     _dp(cabs), it.ctypes.data_as(C.POINTER(C.c_int32))), "sweep")
        return csca, cabs, it

    def autotune_result(self, precision):
        """The LU autotuner's table for the current order: dict(heights, ctas, us_per_column, tune_ms)."""
        k = 32
        nent = C.c_int32()
        hs = np.zeros(k, dtype=np.int64)
        ps = np.zeros(k, dtype=np.int32)
        us = np.zeros(k)
        ms = C.c_double()
        self._ck(lib().mom_gpu_autotune_result(self.h, precision, k, C.byref(nent), hs.ctypes.data_as(C.POINTER(C.c_int64)),
                                               ps.ctypes.data_as(C.POINTER(C.c_int32)), _dp(us), C.byref(ms)),
                 "autotune_result")
        m = min(k, nent.value)
        nx = C.c_int32()
        xs = C.c_int32()
        xus = np.zeros(k)
        self._ck(lib().mom_gpu_autotune_placement(self.h, precision, k, C.byref(nx), C.byref(xs), _dp(xus)),
                 "autotune_placement")
        return dict(heights=hs[:m].tolist(), ctas=ps[:m].tolist(), us_per_column=us[:m].round(3).tolist(),
                    tune_ms=ms.value, placement=xs.value, placement_us_per_column=xus[:min(k, nx.value)].round(3).tolist())

    def adjoint_mean_eps(self, omega, ri, srcs, precision, eps_dom, tol=1e-12, maxit=30):
        """d(mean sigma_ext, mean sigma_abs) / d(Re eps, Im eps) of domain eps_dom: [2][2]."""
        arr, ns = _srcs(srcs)
        r = _ri(ri)
        out = np.zeros((2, 2))
        it = C.c_int32()
        self._ck(lib().mom_gpu_adjoint_mean_eps(self.h, precision, omega, _dp(r), ns, arr, eps_dom, tol, maxit,
                                                _dp(out), C.byref(it)), "adjoint_mean_eps")
        return out

    def cross_sections_noalloc(self, omega, ri, srcs, x_dev, ldx, dom=0):
        """Cross sections through the allocation-free entry point: x_dev is a device
        pointer (int) to the 2N x nsrc solutions with leading dimension ldx."""
        arr, ns = _srcs(srcs)
        r = _ri(ri)
        csca = np.zeros(ns)
        cabs = np.zeros(ns)
        self._ck(lib().mom_gpu_cross_sections_noalloc(self.h, dom, omega, _dp(r), ns, arr, C.c_void_p(x_dev), ldx,
                                                      _dp(csca), _dp(cabs)), "cross_sections_noalloc")
        return csca, cabs

    def selftest_cgemm(self, L, U, Cmat):
        """Cmat - L U (complex64) computed by the library's tensor-core LU-update kernel."""
        L = np.asfortranarray(L, dtype=np.complex64)
        U = np.asfortranarray(U, dtype=np.complex64)
        Cc = np.asfortranarray(Cmat, dtype=np.complex64).copy(order="F")
        m, k = L.shape
        nc = U.shape[1]
        fp = C.POINTER(C.c_float)
        self._ck(lib().mom_gpu_selftest_cgemm(self.h, m, nc, k, L.ctypes.data_as(fp), U.ctypes.data_as(fp),
                                              Cc.ctypes.data_as(fp)), "selftest_cgemm")
        return Cc

    def device_solution(self):
        """(device pointer, leading dimension, number of sources) of the solutions."""
        p = C.c_void_p()
        ld = C.c_int64()
        ns = C.c_int32()
        self._ck(lib().mom_gpu_device_solution(self.h, C.byref(p), C.byref(ld), C.byref(ns)), "device_solution")
        return p.value, ld.value, ns.value

    def scat_fields(self, omega, ri, pts, x=None, nsrc=None, srcs=None, dom=0):
        """scat_fields (nfields.f90:29-197) at pts[npts][3] (metres) from the currents of
        domain dom with that domain's refractive index ri: (e, h), each [nsrc][npts][3]
        complex.  x: 2N x nsrc host solutions, or None for the first nsrc device
        solutions.  srcs: add each source's incident field (the exterior-domain
        total field of field_plane)."""
        r = _ri(ri)
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        xp = None
        if x is not None:
            x = np.asfortranarray(np.asarray(x, dtype=np.complex128).reshape(2 * self.N, -1, order="F"))
            xp = x.ctypes.data
            ns = x.shape[1]
        else:
            ns = nsrc if nsrc is not None else (len(srcs) if srcs else 1)
        arr = None
        if srcs:
            arr, nss = _srcs(srcs)
            if nss != ns:
                raise ValueError("one source per solution column")
        e = np.zeros((ns, len(pts), 3), dtype=np.complex128)
        h = np.zeros_like(e)
        self._ck(lib().mom_gpu_scat_fields(self.h, dom, omega, _dp(r), ns, arr, xp, 2 * self.N, len(pts), _dp(pts),
                                           e.ctypes.data_as(C.POINTER(C.c_double)),
                                           h.ctypes.data_as(C.POINTER(C.c_double))), "scat_fields")
        return e, h

    def surface_fields(self, omega, ri, isrc=0, x=None, dom=0):
        """field_mesh: (e, h), each [nga * nfaces_dom][3] complex, the fields at the
        centroids of the domain's faces and of their symmetry images (face g F + f is
        the image of face f under group element g)."""
        r = _ri(ri)
        nf = self.domain_faces(dom) * self.nga
        e = np.zeros((nf, 3), dtype=np.complex128)
        h = np.zeros_like(e)
        xp = None
        if x is not None:
            x = np.asfortranarray(np.asarray(x, dtype=np.complex128).reshape(2 * self.N, -1, order="F"))
            xp = x.ctypes.data
        self._ck(lib().mom_gpu_surface_fields(self.h, dom, omega, _dp(r), isrc, xp, 2 * self.N, e.ctypes.data_as(
            C.POINTER(C.c_double)), h.ctypes.data_as(C.POINTER(C.c_double))), "surface_fields")
        return e, h

    def group_action(self, g):
        """(J [3][3], det J) of group element g."""
        j = np.zeros(9)
        d = C.c_double()
        self._ck(lib().mom_gpu_group_action(self.h, g, _dp(j), C.byref(d)), "group_action")
        return j.reshape(3, 3), d.value

    def rcs(self, omega, ri, ntheta, nphi, isrc=0, x=None, dom=0):
        r = _ri(ri)
        out = np.zeros((ntheta, nphi), order="F")
        xp = None
        if x is not None:
            x = np.asfortranarray(np.asarray(x, dtype=np.complex128).reshape(2 * self.N, -1, order="F"))
            xp = x.ctypes.data
        self._ck(lib().mom_gpu_rcs(self.h, dom, omega, _dp(r), isrc, xp, 2 * self.N, ntheta, nphi, _dp(out)), "rcs")
        return out

    def synchronize(self):
        self._ck(lib().mom_gpu_synchronize(self.h), "synchronize")

    @property
    def stream(self):
        """The library's cudaStream_t as an integer handle."""
        return lib().mom_gpu_stream(self.h)

    @property
    def launch_count(self):
        """Kernel launches of this library (its own kernels) since creation."""
        return lib().mom_gpu_launch_count(self.h)

    @property
    def library_calls(self):
        """cuBLAS GEMM calls since creation."""
        return lib().mom_gpu_library_calls(self.h)

    PROF_CATEGORIES = ("pair", "near", "gather", "panel", "gemm", "trsv", "residual", "post", "pivot_aux", "tc_gemm",
                       "diag_inv", "lu")

    @property
    def tensor_flops(self):
        """FLOP executed by the tensor-core LU update kernel since creation."""
        return lib().mom_gpu_tensor_flops(self.h)

    def profile(self, enable=True):
        """Turn the per-category kernel timers on (and reset them) or off."""
        self._ck(lib().mom_gpu_profile(self.h, 1 if enable else 0), "profile")

    def profile_read(self):
        """{category: (ms_total, launches)} of the kernel timers."""
        out = {}
        for i, name in enumerate(self.PROF_CATEGORIES):
            ms = C.c_double()
            n = C.c_int64()
            self._ck(lib().mom_gpu_profile_read(self.h, i, C.byref(ms), C.byref(n)), "profile_read")
            out[name] = (ms.value, n.value)
        return out

    def device_matrix(self):
        p = C.c_void_p()
        ld = C.c_int64()
        self._ck(lib().mom_gpu_device_matrix(self.h, C.byref(p), C.byref(ld)), "device_matrix")
        return p.value, ld.value


# Reference-named wrappers ----------------------------------------------------

def sysmat_pmchwt(solver: Solver, omega, ri, precision=FP64):
    return solver.sysmat(omega, ri, precision, want_host=True)


def srcvec(solver: Solver, omega, ri1, srcs):
    return solver.srcvec(omega, ri1, srcs, want_host=True)


def solve_systems(solver: Solver, precision=FP64, tol=1e-12, maxit=30):
    return solver.solve(precision, tol, maxit)


def cs_prtsrf(solver: Solver, omega, ri, x, src, dom=0):
    csca, cabs = solver.cross_sections(omega, ri, [src], x=x, dom=dom)
    return float(csca[0]), float(cabs[0])


def rcs(solver: Solver, omega, ri, x, ntheta, nphi, dom=0):
    return solver.rcs(omega, ri, ntheta, nphi, x=x, dom=dom)
