/*
 * mom_gpu.h -- C ABI of the B200 PMCHWT solver (drop-in for the linear
 * scattering hot path of for90-mom2).
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (MOM_OK on success) and is thread safe per context (an internal mutex
 * serialises calls on one context; the reference calls cs_prtsrf from
 * OpenMP threads, interface.f90:1411-1432).  Matrices and vectors are
 * column-major complex(dp) with interleaved re/im, exactly the Fortran
 * COMPLEX(KIND=dp) layout; "double *" arguments that hold complex data point
 * at 2*count doubles.  Indices in the mesh structures are 0-based.
 *
 * The reference's Fortran caller would bind these through ISO_C_BINDING;
 * each declaration names the reference routine it replaces.
 */
#ifndef MOM_GPU_H
#define MOM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference prints and STOPs on these conditions. */
#define MOM_OK 0
#define MOM_ERR_ARG 1      /* invalid argument (size, index, pointer) */
#define MOM_ERR_ALLOC 2    /* device or host allocation failed */
#define MOM_ERR_CUDA 3     /* CUDA runtime / cuBLAS error */
#define MOM_ERR_SINGULAR 4 /* zero pivot: ZGETRF INFO > 0 (linalg.f90:170-173) */
#define MOM_ERR_TIMEOUT 5  /* a bounded device wait ran out */
#define MOM_ERR_STATE 6    /* call order violated (e.g. solve before sysmat) */
#define MOM_ERR_MESH 7     /* inconsistent mesh (mesh.f90:415-418, 1366-1367) */
#define MOM_ERR_NOCONV 8   /* iterative refinement did not reach the tolerance */
#define MOM_ERR_IO 9       /* mesh file could not be read (mesh.f90:622-626) */

/* Arithmetic of sysmat / solve. */
#define MOM_PREC_FP64 0  /* FP64 assembly and FP64 LU (the reference's arithmetic) */
#define MOM_PREC_MIXED 1 /* FP32 far pairs + FP64 near pairs; FP32 LU with TF32
                            tensor-core trailing updates; FP64 refinement */

/* Boundary types of mesh edges (mesh.f90:16-25): the symmetry planes. */
#define MOM_BND_NONE 1
#define MOM_BND_XPLANE 2
#define MOM_BND_YPLANE 3
#define MOM_BND_ZPLANE 4

/* Largest symmetry group (three mirror planes). */
#define MOM_MAX_GROUP 8

/* Source types (source.f90:20-30).  MOM_SRC_NONE has no incident field: the
 * reference's cross sections of second-harmonic solutions use it
 * (nlsrc%type = 0, interface.f90:1441-1458). */
#define MOM_SRC_NONE 0
#define MOM_SRC_PW 1
#define MOM_SRC_PW_ELLIPTIC 10

typedef struct mom_ctx mom_ctx;

/* One domain's boundary submesh after the reference's sdom/fdom commands
 * (mesh_container, mesh.f90:27-83, flattened to structure-of-arrays).
 * Orientation (orient_basis, mesh.f90:454-558) is already applied:
 * edge_faces[2e] is the "+" face and edge_bnodes[2e] its free vertex. */
typedef struct mom_mesh {
  int32_t nnodes, nfaces, nedges;
  const double *nodes;        /* [nnodes][3], metres */
  const int32_t *face_nodes;  /* [nfaces][3] */
  const int32_t *face_edges;  /* [nfaces][3]: local edge k = (node k, node k+1) */
  const int32_t *edge_nodes;  /* [nedges][2] */
  const int32_t *edge_faces;  /* [nedges][2]: (+face, -face) */
  const int32_t *edge_bnodes; /* [nedges][2]: free vertex of the + / - face */
  const int32_t *edge_parent; /* [nedges]: global (master) edge index */
} mom_mesh;

/* Excitation (srcdata, source.f90:36-58); angles in radians. */
typedef struct mom_src {
  int32_t type;           /* MOM_SRC_PW, MOM_SRC_PW_ELLIPTIC or MOM_SRC_NONE */
  double theta, phi, psi; /* psi unused for pw_elliptic */
  double phase_re, phase_im; /* pw_elliptic Ex/Ey phase factor */
} mom_src;

/* Surface second-order nonlinearity of a domain's medium (medium_nls,
 * nlsurf.f90:14-18; `smed m nlsurf value chi_nnn chi_ntt chi_ttn`).  The
 * susceptibilities are complex (re, im); active = 0 marks a linear medium. */
typedef struct mom_nls {
  int32_t active;
  double chi_nnn[2], chi_ntt[2], chi_ttn[2];
} mom_nls;

/* Context on one CUDA device.  Owns a stream, cuBLAS handle and the device
 * copies of the problem, the system matrix, its LU factors and solutions. */
int mom_gpu_create(int32_t device, mom_ctx **out);
void mom_gpu_destroy(mom_ctx *ctx);
const char *mom_gpu_strerror(int32_t status);
/* Text of the last error on this context (empty if none). */
const char *mom_gpu_last_error(mom_ctx *ctx);

/* Upload the domain submeshes and the triangle rule (b%domains(:)%mesh and
 * b%qd_tri of the batch type, common.f90:71-108).  nedges_total is the
 * master mesh edge count N (2N unknowns).  qw[nq], qnodes[nq][3] follow
 * quad_data (quad.f90:269-274): point = qn[2] p1 + qn[0] p2 + qn[1] p3.
 * Geometry (normals, areas, edge lengths, average edge length) is derived
 * as compute_basis_data does (mesh.f90:1265-1322).  nq <= 13. */
int mom_gpu_set_problem(mom_ctx *ctx, int32_t nedges_total, int32_t ndom, const mom_mesh *doms, int32_t nq,
                        const double *qw, const double *qnodes);

/* Symmetry group of the problem (read_symm, interface.f90:160-210, and the
 * sbnd boundary classification, mesh.f90:155-175): the product of the named
 * groups "id", "mxp", "myp", "mzp" (mirror planes x = 0, y = 0, z = 0;
 * symmetry.f90:45-103, 178-241), nga = 2^(number of mirrors) elements and
 * as many representations.  edge_bnd[N] holds the boundary type of every
 * master edge (MOM_BND_*, from mom_problem_edge_bnd), which decides the
 * symmetry-plane boundary conditions of each representation (edge_bc,
 * bc.f90:28-117) and which group actions act on interior domains
 * (admissible_ga, bc.f90:237-257).  Call after mom_gpu_set_problem (which
 * resets the group to the identity).  With nga > 1, every matrix, right-hand
 * side and solution exists once per representation: host arrays of
 * solutions and right-hand sides are 2N x nga x nsrc (x(2N, nga, nsrc) of
 * the reference, solver.f90:116), and sysmat's A_host receives nga
 * consecutive 2N x 2N blocks.  Rotation groups (rN) are not supported. */
int mom_gpu_set_symmetry(mom_ctx *ctx, int32_t nnames, const char *const *names, const int32_t *edge_bnd);
/* Number of group elements (and representations) of the context, 1 for the
 * identity, -1 without a problem. */
int32_t mom_gpu_group_order(mom_ctx *ctx);

/* Replaces sysmat_pmchwt (sysmat.f90:18-105): builds the 2N x 2N PMCHWT
 * matrix of every representation (one for the identity group) for angular
 * frequency omega and one refractive index per domain (ri[2*ndom], re/im).
 * The matrices stay on the device; if A_host is not NULL they are also
 * copied there (leading dimension lda >= 2N, representation r at
 * A_host + 2 r lda 2N doubles). */
int mom_gpu_sysmat(mom_ctx *ctx, double omega, const double *ri, int32_t precision, double *A_host, int64_t lda);

/* Replaces srcvec (source.f90:136-247) for nsrc sources on domain 1's
 * boundary with refractive index ri1 (re/im): the right-hand sides are kept
 * on the device; if q_host is not NULL they are also copied there as a
 * 2N x nsrc column-major block (leading dimension ldq >= 2N). */
int mom_gpu_srcvec(mom_ctx *ctx, double omega, const double *ri1, int32_t nsrc, const mom_src *src, double *q_host,
                   int64_t ldq);

/* Replaces solve_systems / solve_multi_linsys (solver.f90:325-357,
 * linalg.f90:159-180): LU-factors the device matrix with partial pivoting
 * and solves for the device right-hand sides.  MOM_PREC_MIXED factors in
 * FP32 and refines in FP64 until ||b - A x|| <= tol ||b|| (at most maxit
 * steps; iters_out may be NULL).  x_host (2N x nsrc, ldx) may be NULL. */
int mom_gpu_solve(mom_ctx *ctx, int32_t precision, double tol, int32_t maxit, double *x_host, int64_t ldx,
                  int32_t *iters_out);

/* One wavelength of solve_batch (solver.f90:76-142): sysmat + srcvec +
 * solve.  x_host (2N x nsrc, ldx) receives the solutions if not NULL. */
int mom_gpu_solve_wavelength(mom_ctx *ctx, double omega, const double *ri, int32_t nsrc, const mom_src *src,
                             int32_t precision, double tol, int32_t maxit, double *x_host, int64_t ldx,
                             int32_t *iters_out);

/* The second-harmonic branch of solve_batch for centrosymmetric surface
 * nonlinearities (solver.f90:143-217): after a solve at the fundamental
 * frequency omega (the device solutions of its nsrc sources), for every
 * domain with nls[d].active the source coefficients and source vector of
 * nlsurf_coef (nlsurf.f90:137-338: the surface polarisation of the
 * fundamental field inside domain d, expanded in the domain's RWG functions),
 * the system matrix at 2 omega with the second-harmonic refractive indices
 * shri [ndom][2] and its source terms (sysmat_pmchwt_nls, sysmat.f90:112-229),
 * then the solve.  ri [ndom][2] are the fundamental indices (the field
 * inside domain d and the selvedge permittivity of determine_epsp,
 * solver.f90:393-433).  Afterwards the device solutions, matrix and factors
 * are those of the second harmonic: cross sections with MOM_SRC_NONE
 * sources at 2 omega and shri give the reference's -sh.crs values.
 * With a symmetry group the polarisation is projected on every
 * representation (Pnls_frag, nlsurf.f90:106-125) and the Gram systems and
 * the SH solves keep the representations' boundary conditions; nlx_host is
 * then (2N, nga, nsrc).  nlx_host (ldx) may be NULL.  A domain face that no
 * other domain shares gives MOM_ERR_ARG ("Could not find epsp!"); a Gram
 * system that does not converge (NaN input) MOM_ERR_NOCONV. */
int mom_gpu_shg_solve(mom_ctx *ctx, double omega, const double *ri, const double *shri, const mom_nls *nls,
                      int32_t precision, double tol, int32_t maxit, double *nlx_host, int64_t ldx,
                      int32_t *iters_out);

/* The source coefficients of domain dom from the last mom_gpu_shg_solve
 * (src_coef(:, dom, :, :), nlsurf.f90:137-338) on the global unknowns: cJ on
 * the domain's edges in rows [0, N), cM in rows [N, 2N), zero elsewhere;
 * 2N x nsrc (2N x nga x nsrc with a symmetry group), ldc.  The fields inside a nonlinear domain come from nlx plus
 * these (read_nfem, interface.f90:1060-1078).  MOM_ERR_STATE if dom was not
 * nonlinear in that solve. */
int mom_gpu_shg_source_coef(mom_ctx *ctx, int32_t dom, double *coef_host, int64_t ldc);

/* Replaces cs_prtsrf (cs.f90:14-104) for nsrc sources: scattering and
 * absorption cross sections from the surface currents on domain dom
 * (0-based; the reference uses domain 1) with refractive index ri (re/im).
 * x_host (2N x nsrc, ldx) or, if NULL, the device solutions. */
int mom_gpu_cross_sections(mom_ctx *ctx, int32_t dom, double omega, const double *ri, int32_t nsrc,
                           const mom_src *src, const double *x_host, int64_t ldx, double *csca, double *cabs);

/* Replaces rcs / rcs_ext (ffields.f90:203-266, far_fields 16-122): the
 * bistatic |E_theta|^2 + |E_phi|^2 at r = 1 m on the endpoint-inclusive
 * ntheta x nphi grid (column-major, as rcsdata(1:ntheta,1:nphi)) for
 * source column isrc of x_host (2N x ?, ldx) or, if NULL, of the device
 * solutions. */
int mom_gpu_rcs(mom_ctx *ctx, int32_t dom, double omega, const double *ri, int32_t isrc, const double *x_host,
                int64_t ldx, int32_t ntheta, int32_t nphi, double *rcs);

/* Replaces scat_fields (nfields.f90:29-197, identity group) at npts points
 * pts[npts][3] (metres): the fields radiated by the surface currents of
 * domain dom (0-based) with that domain's refractive index ri (re/im), for
 * the nsrc solution columns of x_host (2N x nsrc, ldx) or, if NULL, the
 * device solutions.  e, h: [nsrc][npts][3] complex (2 doubles each).  If src
 * is not NULL the incident field of src[s] is added to column s (what
 * field_plane and field_domain do in the exterior domain, nfpost.f90:85-165,
 * 316-374).  Faces within three average edge lengths of a point use the
 * singularity-subtracted integrals (srcint.f90 intK2/3/4). */
int mom_gpu_scat_fields(mom_ctx *ctx, int32_t dom, double omega, const double *ri, int32_t nsrc, const mom_src *src,
                        const double *x_host, int64_t ldx, int32_t npts, const double *pts, double *e, double *h);

/* Replaces field_mesh (nfpost.f90:167-262, the nfms command): the fields
 * on the boundary of domain dom (0-based, refractive index ri) at the
 * centroid of every face of every image of the domain's submesh under the
 * symmetry group, from the surface currents alone: with n the image normal,
 * E = n x M + n (div J) / (i omega eps), H = -n x J + n (div M) / (i omega mu0)
 * (the group's field actions and det J applied as the reference does).
 * isrc: source column of x_host (2N x nga x nsrc, ldx) or, if NULL, of the
 * device solutions.  e, h: [nga * nfaces][3] complex; face g * nfaces + f is
 * the image of face f under group element g (mom_gpu_group_action). */
int mom_gpu_surface_fields(mom_ctx *ctx, int32_t dom, double omega, const double *ri, int32_t isrc,
                           const double *x_host, int64_t ldx, double *e, double *h);
/* Point action j[9] (row-major) and det J of group element g (symmetry.f90:24-40). */
int mom_gpu_group_action(mom_ctx *ctx, int32_t g, double *j, double *detj);

/* Allocation-free cross sections.  No counterpart in the reference.  For
 * callers that cannot allocate device memory at call time (their device
 * memory is reserved up front by another allocator, or they cannot accept
 * the implicit device-wide synchronisation of cudaMalloc / cudaFree): the
 * same results as mom_gpu_cross_sections, computed with a fixed scratch
 * array compiled into the library instead of allocated buffers.  x_dev is a
 * device pointer to the 2N x nsrc solutions (leading dimension ldx >= 2N,
 * e.g. from mom_gpu_device_solution); csca / cabs are host arrays.
 * Limits: 1 <= nsrc <= 64 and at most 65536 faces in domain dom; larger
 * requests return MOM_ERR_ARG.  With lazy module loading (the CUDA default)
 * the first call on a device may load the library's module, which allocates
 * the scratch array: callers that must not allocate at all make one warm-up
 * call at set-up.  Every call synchronises the context's stream, so none may
 * be made while a stream capture is open.  All calls on a device share the
 * scratch array: calls that overlap on the GPU (from different contexts)
 * race. */
int mom_gpu_cross_sections_noalloc(mom_ctx *ctx, int32_t dom, double omega, const double *ri, int32_t nsrc,
                                   const mom_src *src, const void *x_dev, int64_t ldx, double *csca,
                                   double *cabs);

/* ---- Wavelength sweeps ----
 * solve_batch (solver.f90:17-142) over nwl wavelengths of one problem:
 * sysmat, srcvec, LU and solve, then cs_prtsrf on domain 0 for every
 * wavelength; ri is [nwl][ndom] complex (interleaved), csca / cabs
 * [nwl][nsrc], iters [nwl] or NULL. */
int mom_gpu_sweep(mom_ctx *ctx, int32_t nwl, const double *omega, const double *ri, int32_t nsrc, const mom_src *src,
                  int32_t precision, double tol, int32_t maxit, double *csca, double *cabs, int32_t *iters);
/* Sweeps of several problems at once (no counterpart in the reference): one
 * host thread per context, each context on its own stream, so that the GPU
 * overlaps the problems' launches.  status[nctx] (or NULL) per context. */
int mom_gpu_sweep_many(int32_t nctx, mom_ctx **ctx, const int32_t *nwl, const double *const *omega,
                       const double *const *ri, int32_t nsrc, const mom_src *src, int32_t precision, double tol,
                       int32_t maxit, double *const *csca, double *const *cabs, int32_t *status);
/* Table of the LU autotuner for the current matrix order (no counterpart in
 * the reference): for panel heights heights[i] the CTA count ctas[i] chosen
 * and its time per panel column; up to max_entries entries, *nent = table
 * size, *tune_ms = time spent tuning.  MOM_ERR_STATE before the first
 * factorisation (or with MOM_AUTOTUNE=0 / MOM_PANEL_CTAS set). */
int mom_gpu_autotune_result(mom_ctx *ctx, int32_t precision, int32_t max_entries, int32_t *nent, int64_t *heights,
                            int32_t *ctas, double *us_per_column, double *tune_ms);
/* Placement of the panel exchange buffers chosen by the same autotuner (no
 * counterpart in the reference): *chosen = index of the placement in use;
 * us_per_column[i] = time per column of placement i at the tallest panel
 * height (up to max_entries, *nent = number probed; 0 when the tallest
 * panel runs on one thread-block cluster and has no global exchange). */
int mom_gpu_autotune_placement(mom_ctx *ctx, int32_t precision, int32_t max_entries, int32_t *nent, int32_t *chosen,
                               double *us_per_column);

/* ---- Adjoint gradients (no counterpart in the reference) ----
 * After mom_gpu_solve for the same sources (and the same omega and ri), the
 * factors of `precision` are reused for one transposed solve A^T lambda = G
 * per objective, G = d sigma / dx of cs_prtsrf on domain 0 (cs.f90:14-104).
 * Derivatives of the system matrix are recomputed face pair by face pair in
 * dual arithmetic and contracted with lambda and x (never stored).
 * Objectives per source s: o = 2 s (sigma_ext), 2 s + 1 (sigma_abs).
 *   deps   (or NULL) [2 nsrc][2]: d sigma_o / d Re(eps), d / d Im(eps) of the
 *          permittivity eps = ri[eps_dom]^2 of interior domain eps_dom;
 *   dnodes (or NULL) [2 nsrc][sum_d nnodes_d][3]: d sigma_o / d(node
 *          coordinates, metres) of each domain's submesh nodes, domains
 *          concatenated in order (mom_gpu_domain_nodes); a master-mesh
 *          vertex shared by several domains sums its entries
 *          (mom_problem_node_parent).
 * The near-pair classification stays that of the unperturbed mesh.  1 to 4
 * sources; tol / maxit drive the refinement of a mixed transposed solve. */
int mom_gpu_adjoint(mom_ctx *ctx, int32_t precision, double omega, const double *ri, int32_t nsrc, const mom_src *src,
                    int32_t eps_dom, double tol, int32_t maxit, double *deps, double *dnodes, int32_t *iters);
/* d(mean over the nsrc sources of sigma_ext, sigma_abs) / d(Re eps, Im eps)
 * of interior domain eps_dom: dmean[2][2]; any nsrc.  Uses an n x n complex
 * FP64 work matrix W = (1/nsrc) sum_s lambda_s x_s^T. */
int mom_gpu_adjoint_mean_eps(mom_ctx *ctx, int32_t precision, double omega, const double *ri, int32_t nsrc,
                             const mom_src *src, int32_t eps_dom, double tol, int32_t maxit, double *dmean,
                             int32_t *iters);
/* Number of submesh nodes of domain dom, -1 without a problem. */
int32_t mom_gpu_domain_nodes(mom_ctx *ctx, int32_t dom);

/* Diagnostics: C -= L U for host complex64 arrays (column-major; L m x k,
 * U k x nc, C m x nc; m a multiple of 64, k of 16) through the tensor-core
 * kernel that performs the trailing updates of the mixed-precision LU. */
int mom_gpu_selftest_cgemm(mom_ctx *ctx, int32_t m, int32_t nc, int32_t k, const float *L, const float *U, float *C);

/* Replaces the device system matrix by a caller's 2N x 2N matrix (host,
 * column-major, lda >= 2N), as if mom_gpu_sysmat had built it; the next
 * mom_gpu_solve factors and solves it.  The matrix argument of
 * solve_multi_linsys (linalg.f90:159-180) for callers that assemble A
 * themselves; a zero pivot returns MOM_ERR_SINGULAR as ZGETRF's INFO > 0
 * makes the reference STOP (linalg.f90:170-173). */
int mom_gpu_set_matrix(mom_ctx *ctx, int32_t precision, const double *A_host, int64_t lda);

/* Bounds of the device waits (no counterpart in the reference): polls
 * before the LU panel exchange, the tensor-core GEMM's mbarrier waits and
 * the triangular solve's hand-offs give up with MOM_ERR_TIMEOUT; 0 restores
 * each default (a few seconds).  A kernel that gives up records the error,
 * waits (bounded) for its own copies and tensor-core work, frees its tensor
 * memory and returns, so the context stays usable: the next call that
 * rebuilds the matrix (mom_gpu_sysmat or mom_gpu_set_matrix) starts clean. */
int mom_gpu_set_wait_limits(mom_ctx *ctx, int64_t panel_polls, int64_t gemm_polls, int64_t solve_polls);

/* Device views for callers that keep data resident (bench, tests). */
int mom_gpu_device_matrix(mom_ctx *ctx, void **A_dev, int64_t *lda);
int mom_gpu_device_solution(mom_ctx *ctx, void **x_dev, int64_t *ldx, int32_t *nsrc);
int mom_gpu_synchronize(mom_ctx *ctx);
/* Kernel launches issued by this context since creation (instrumentation). */
int64_t mom_gpu_launch_count(mom_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or
 * order their own work against the library's. */
void *mom_gpu_stream(mom_ctx *ctx);
/* cuBLAS GEMM calls issued by this context (library kernels). */
int64_t mom_gpu_library_calls(mom_ctx *ctx);
/* FLOP executed by the tensor-core LU update kernel since creation. */
double mom_gpu_tensor_flops(mom_ctx *ctx);
/* Optional kernel timers: enable (1) / disable (0) and reset; then read the
 * summed device time and launch count of a category: 0 pair (far-pair
 * assembly), 1 near pairs, 2 gather, 3 LU panel, 4 LU GEMMs, 5 triangular
 * solves, 6 refinement residual, 7 post-processing, 8 row interchanges of
 * the LU, 9 the tensor-core LU update kernel alone, 10 diagonal-block
 * inverses of the LU, 11 the whole LU factorisation (wall time on the
 * context stream; the categories inside it overlap under the look-ahead). */
int mom_gpu_profile(mom_ctx *ctx, int32_t enable);
int mom_gpu_profile_read(mom_ctx *ctx, int32_t category, double *ms_total, int64_t *launches);

/* ---- Host-side problem set-up (the reference's mesh/sdom/fdom commands) ---- */

typedef struct mom_problem mom_problem;

int mom_problem_create(mom_problem **out);
void mom_problem_destroy(mom_problem *p);
/* read_mesh (interface.f90:357-366): load_mesh_gmsh + build_mesh(scale). */
int mom_problem_load_gmsh(mom_problem *p, const char *path, double scale);
/* The same from arrays: faces[nfaces][3] 0-based, face_ids[nfaces]. */
int mom_problem_set_mesh(mom_problem *p, int32_t nnodes, const double *nodes, int32_t nfaces, const int32_t *faces,
                         const int32_t *face_ids, double scale);
/* read_ndom / read_sdom (interface.f90:32-105): signed surface ids; a
 * negative id inverts those faces (invert_faces, mesh.f90:278-288). */
int mom_problem_set_ndom(mom_problem *p, int32_t ndom);
int mom_problem_set_domain(mom_problem *p, int32_t dom, int32_t nsurf, const int32_t *surf_ids);
/* Line elements of the master mesh (node pairs, 0-based, and physical ids),
 * as load_mesh_gmsh keeps them for sbnd; set by mom_problem_load_gmsh from
 * the file's type-1 elements. */
int mom_problem_set_lines(mom_problem *p, int32_t nlines, const int32_t *line_nodes, const int32_t *line_ids);
/* read_sbnd / classify_edges (interface.f90:125-157, mesh.f90:155-175):
 * master edges that coincide with a line of physical id `id` get boundary
 * type bnd (MOM_BND_*); *nclassified (may be NULL) = number of matches. */
int mom_problem_classify_edges(mom_problem *p, int32_t id, int32_t bnd, int32_t *nclassified);
/* Boundary type of every master edge: bnd[N]. */
int mom_problem_edge_bnd(const mom_problem *p, int32_t *bnd);
/* read_fdom (interface.f90:107-123): submesh_edge_connectivity +
 * orient_basis. */
int mom_problem_finalize(mom_problem *p);
int32_t mom_problem_nedges(const mom_problem *p);
int32_t mom_problem_ndom(const mom_problem *p);
/* Flattened view of domain dom (valid until the problem is destroyed); dom
 * = -1 gives the master mesh, available from the mesh command on (before
 * fdom; its edge_parent is not set). */
int mom_problem_domain(const mom_problem *p, int32_t dom, mom_mesh *out);
/* Master-mesh node of each submesh node of domain dom: parent[nnodes]. */
int mom_problem_node_parent(const mom_problem *p, int32_t dom, int32_t *parent);
/* Named triangle rule of quad.f90 ("tri_gl1", "tri_gl3", "tri_gl4",
 * "tri_gl7", "tri_gl13"): qw[13], qnodes[13][3]; returns nq or < 0. */
int32_t mom_tri_rule(const char *name, double *qw, double *qnodes);
/* Convenience: mom_gpu_set_problem with all domains of p and a named rule. */
int mom_problem_upload(const mom_problem *p, mom_ctx *ctx, const char *quad_name);

#ifdef __cplusplus
}
#endif
#endif
