// Internal declarations of the B200 PMCHWT library (not part of the C ABI).
#pragma once

#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/mom_gpu.h"

namespace mom {

// Physical constants as the reference defines them (constants.f90:8-14):
// pi is the single-precision literal 3.141592653589 widened to double, and
// it leaks into mu0, 1/(4 pi) and every angle conversion.
constexpr double kPi = (double)3.141592653589f;
constexpr double kEps0 = 8.8541878176e-12;
constexpr double kMu0 = 4 * kPi * 1e-7;
constexpr double kC0 = 2.997924580003e8;
constexpr double kEta0 = 3.767303134622e2;

constexpr int kMaxQ = 13;
constexpr size_t kBlasWorkspace = 64u << 20;

constexpr int kMaxGroup = MOM_MAX_GROUP;

// One element of a symmetry group (group_action, symmetry.f90:24-40): point
// action J (row-major, j[3 i + k] = J(i, k)), det J, the special-action id
// (0 none, 1 identity, 2/3/4 the mirrors x/y/z, symmetry.f90:20-23), the
// generator bits and the field action per representation (+1 / -1 for the
// mirror groups, whose characters are real).
struct GroupAction {
  double j[9];
  double detj;
  int id;
  unsigned genbits;
  double ef[kMaxGroup];
};

// A non-identity group action g on one domain: the domain's test faces
// mapped by J^T.  The reference maps the source face by J; for an orthogonal
// J the pair (test r, source J r') equals (test J^T r, source r'), so the
// identity kernels run on the mapped test side: D_g, H_g from the mapped
// pair as they are, K_g = det J times the mapped pair's K.  Near pairs
// (|cp_m - J cp_n| < 3 avelen) and their closed-form integrals follow the
// mapped test faces.
struct ActDev {
  bool admissible = false;  // admissible_ga (bc.f90:237-257)
  double *qrel = nullptr;   // [F][nq][3] mapped test points minus the mapped centroid
  double *cp = nullptr;     // [F][3] mapped centroids
  double *mu = nullptr;     // [F][3][3] mapped free vertices minus the mapped centroid
  int64_t nnear = 0;
  int *near_m = nullptr, *near_n = nullptr;
  double *near_static = nullptr;  // [nnear][6][9]
};

// Per-domain device data (structure of arrays).  "Half-edge" h = 3*face +
// local edge identifies one RWG half (one face of an edge).
struct DomDev {
  int F = 0, Nd = 0;
  double avelen = 0;
  double *qrel = nullptr;  // [F][nq][3] quadrature points minus the face centroid
  double *qabs = nullptr;  // [F][nq][3] absolute quadrature points
  double *cp = nullptr;    // [F][3] centroid
  double *area = nullptr;  // [F]
  double *nrm = nullptr;   // [F][3] unit normal
  double *mu = nullptr;    // [F][3][3] free vertex of local edge e minus centroid
  double *sl = nullptr;    // [F][3] sign * edge length of local edge e
  int *hpar = nullptr;     // [F][3] global (parent) edge index of local edge e
  int *eh = nullptr;       // [Nd][2] half-edges (+, -) of domain edge e, -1 if none
  int *epar = nullptr;     // [Nd] global edge index of domain edge e
  // Near pairs (sysmat.f90:233-260), wavelength independent.
  int64_t nnear = 0;
  int *near_m = nullptr;   // [nnear] test face
  int *near_n = nullptr;   // [nnear] source face
  double *near_static = nullptr;  // [nnear][6][9] contracted closed-form terms
  // Host mirrors used at set-up.
  std::vector<double> h_cp, h_qrel, h_qabs, h_area, h_nrm, h_mu, h_sl;
  std::vector<double> h_fv, h_fs, h_fm, h_bn;  // [F][3][3]: vertices, s(:,e), m(:,e), free vertex of e
  std::vector<int> h_hpar, h_eh, h_epar;
  // Topology for the geometry derivatives of the adjoint (uploaded on first use).
  int nnodes = 0;
  std::vector<double> h_nodes;                   // [nnodes][3]
  std::vector<int> h_fnode, h_fea, h_feb, h_fbn;  // [F][3] face vertices; ends and free vertex of local edge e
  std::vector<double> h_fsign;                   // [F][3] +1 / -1
  bool adj_ready = false;
  double *nodes = nullptr, *fsign = nullptr;
  int *fnode = nullptr, *fea = nullptr, *feb = nullptr, *fbn = nullptr;
  unsigned *near_bits = nullptr;                 // [F*F] bits
  int ninc = 0;                                  // (vertex, face) incidences, by vertex
  int *inc_node = nullptr, *inc_face = nullptr;
  // Face geometry of the near-field kernel (uploaded on first use).
  void *nf_geo = nullptr;
  double *nf_bn = nullptr;
  // Symmetry group actions on this domain, [nga] (element 0 is the identity,
  // which uses the arrays above).
  std::vector<ActDev> act;
  // Second-harmonic sources (uploaded on first use): free vertex of each
  // local edge, the domain edge of each local edge, and the RWG Gram matrix
  // <f_m, f_n> as 5 entries per row (the diagonal first).
  double *shg_bn = nullptr;    // [F][3][3]
  int *shg_fedge = nullptr;    // [F][3]
  int *gram_col = nullptr;     // [Nd][5]
  double *gram_val = nullptr;  // [Nd][5]
};

struct Ctx {
  int device = 0;
  int nsm = 0;
  cudaStream_t stream = nullptr;
  cublasHandle_t blas = nullptr;
  void *blas_ws = nullptr;  // fixed cuBLAS workspace
  // Look-ahead of the LU: the next outer block is factored on a second stream
  // (with its own cuBLAS handle and workspace) while the trailing update of
  // the current one runs on `stream`.
  cudaStream_t stream2 = nullptr;
  cublasHandle_t blas2 = nullptr;
  void *blas_ws2 = nullptr;
  cudaEvent_t la_ev[3] = {nullptr, nullptr, nullptr};
  int lookahead = 1;       // MOM_LOOKAHEAD=0 turns it off
  // Defaults from a sweep on a B200 at n = 30,720 (the cap 32/48/64 and the
  // fraction 0.9/0.95/all within 3% of each other; these were the fastest).
  bool pair_sym = true;    // MOM_PAIR_SYM: far pairs once per unordered pair (identity action), both blocks written
  bool pair_e32 = false;   // MOM_PAIR_E32: FP32 block contraction in the FP32 far-pair kernel
  int pair_ctas = 3;       // MOM_PAIR_CTAS: resident CTAs per SM of the 13-point FP32 far-pair kernel (3 or 4)
  int la_ctas = 48;        // MOM_LA_CTAS: CTA cap of the look-ahead panels (0: the smallest that fits)
  double la_from = 1.0;    // MOM_LA_FROM: overlap blocks whose trailing height is below this fraction of n
  std::mutex mu;
  std::string last_error;
  int64_t launches = 0;

  // Problem
  int N = 0;  // master edges; 2N unknowns
  int ndom = 0;
  int nq = 0;
  double qw[kMaxQ] = {0};
  double qn[kMaxQ][3] = {{0}};
  std::vector<DomDev> dom;
  bool have_problem = false;

  // Symmetry group (identity unless mom_gpu_set_symmetry) and, per
  // representation, the unknowns its symmetry-plane boundary conditions
  // remove (edge_bc, bc.f90:28-117; rows and columns replaced by identity).
  int nga = 1;
  GroupAction ga[kMaxGroup];
  std::vector<int> edge_bnd;                 // [N] master-edge boundary types
  std::vector<std::vector<int>> removed;     // [nga]
  int *removed_dev = nullptr;                // concatenated lists
  std::vector<int> removed_off;              // [nga + 1]

  // System matrix and factors.  With a symmetry group there is one matrix
  // (and one set of factors) per representation: the *_all buffers hold
  // them all and A, A32, ipiv, perm, invd, inv32 point at the
  // representation being worked on (select_rep).
  double2 *A_all = nullptr, *invd_all = nullptr;
  float2 *A32_all = nullptr, *inv32_all = nullptr;
  int *ipiv_all = nullptr, *perm_all = nullptr;
  int64_t n = 0, lda = 0;  // n = 2N
  double2 *A = nullptr;    // FP64 matrix (LU in place in FP64 mode)
  float2 *A32 = nullptr;   // FP32 copy (LU in place in mixed mode)
  size_t A_bytes = 0, A32_bytes = 0;
  double2 *blk = nullptr;  // face-pair blocks [source F][test F][9][2] of the largest domain
  size_t blk_bytes = 0;    //   or, when blk_fused, of every domain at blk + blk_off[d]
  bool blk_fused = false;
  std::vector<size_t> blk_off;  // [ndom], in double2
  int *dmap = nullptr;     // [ndom][N]: domain edge of each global edge, -1 if none
  int *ipiv = nullptr;     // [n]
  int *perm = nullptr;     // [n] composed row permutation of the factorisation
  double2 *invd = nullptr; // inverses of diagonal blocks (L then U), FP64
  float2 *inv32 = nullptr; // FP32 copy of invd for the mixed-precision solves
  size_t invd_bytes = 0;
  int *dinfo = nullptr;    // device status words [0]=info, [1]=timeout
  void *ws = nullptr;      // general device workspace
  size_t ws_bytes = 0;
  void *ws2 = nullptr;     // workspace of the many-right-hand-side solve
  size_t ws2_bytes = 0;
  int assembled = 0;       // 0 none, 1 FP64 matrix present
  int factored = -1;       // precision of the factors in place, -1 none
  int nb = 64;             // panel width

  // Right-hand sides / solutions
  int nsrc = 0;
  bool solved = false;     // X holds the solutions of the current right-hand sides
  double2 *B = nullptr;    // [nsrc][n] right-hand sides
  double2 *X = nullptr;    // [nsrc][n] solutions
  size_t BX_cap = 0;
  double2 *Xh = nullptr;   // solutions uploaded from the host for post-processing
  size_t Xh_cap = 0;
  void *nf_buf = nullptr;   // near-field points, fields and source records
  size_t nf_cap = 0;
  std::vector<mom_src> srcs;
  double omega_rhs = 0;
  double ri1[2] = {1, 0};

  // Optional per-category kernel timers (CUDA events on the context stream).
  bool prof = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_ev[12];
  int64_t prof_launch[12] = {0};
  double prof_ms[12] = {0};  // time of scopes replayed inside graphs, resolved after each replay

  // The LU factorisation of each precision as one CUDA graph, replayed while
  // the matrix order, buffers and profiling state stay those it was captured with.
  struct LuGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<uintptr_t> key;
    std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> ev;  // timed scopes inside the graph
    int64_t launches = 0, blas_calls = 0;  // per replay
    double tc_flops = 0;
    void reset();
  };
  std::vector<LuGraph *> lu_graphs;  // by key (one per precision and representation)
  bool use_graph = true;   // MOM_LU_GRAPH=0 turns graph replay off (every launch issued eagerly)
  // Panel parallelism: CTAs per panel as a function of the panel's rows m,
  // autotuned per (matrix order, precision) at the first factorisation
  // (unless MOM_AUTOTUNE=0: one CTA per SM); MOM_PANEL_CTAS fixes a cap.
  int panel_cap_env = 0;
  // Short panels run on one thread-block cluster of up to panel_cluster CTAs
  // (the largest the device schedules; MOM_PANEL_CLUSTER caps it, 0 = off).
  int panel_cluster = 0;
  int outer_panels = 4;  // panels per outer block of the LU (MOM_LU_OUTER): trailing GEMMs have K = 64 * this
  int small_tc = 0;      // mixed path: K = 64 updates on the tensor cores too (MOM_SMALL_TC=1), else library FP32 GEMM
  // Look-ahead path: the block TRSMs of an outer block by block_trsm_kernel
  // instead of library CGEMMs: MOM_FUSED_TRSM=1 everywhere (measured slower
  // at 15,360 unknowns: 158.6 against 155.0 ms per solve), 2 only for the
  // narrow updates on the panels' critical path (the next block's columns and
  // the in-block updates), 0 (default) nowhere.
  int fused_trsm = 0;
  // Permittivity gradients by adj_eps_kernel (FP64 geometry, dual numbers in
  // k only); MOM_ADJ_EPS_PLAIN=0 selects the all-dual adj_pair_kernel.
  int adj_eps_plain = 1;
  // Vertex gradients by adj_vertex_kernel (the seeded face dual in shared
  // memory, plain partners); MOM_ADJ_VERTEX_PLAIN=0 selects adj_pair_kernel.
  int adj_vertex_plain = 1;
  bool autotune = true;
  struct Tuned {
    int64_t n;
    int precision;
    std::vector<int64_t> m;  // panel heights probed
    std::vector<int> P;      // fastest CTA count at each height
    std::vector<double> us;  // its time per panel column (microseconds)
    int xslot = 0;           // placement of the panel exchange buffers (kXSlotBytes apart)
    std::vector<double> xslot_us;  // per-column time of each placement at the tallest height
    double ms = 0;           // time spent tuning
  };
  std::vector<Tuned> tuned;
  const Tuned *tune = nullptr;  // table in use by the factorisation being issued
  bool capturing = false;  // a stream capture is open on the context stream
  std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> cap_ev;
  int64_t blas_calls = 0;  // cuBLAS GEMM calls (library kernels, not counted in launches)
  double tc_flops = 0;     // FLOP executed by the tensor-core LU updates since creation

  // Adjoint buffers: objective gradients, adjoint currents, forward currents,
  // block partial sums, and the dense objective matrix of the mean gradient.
  void *adj = nullptr;
  size_t adj_bytes = 0;
  void *adj_part = nullptr;
  size_t adj_part_bytes = 0;
  void *adjW = nullptr;
  size_t adjW_bytes = 0;

  // Second-harmonic solve: source coefficients of the nonlinear domains and
  // the scratch of their expansion.
  void *shg_c = nullptr;
  size_t shg_c_bytes = 0;
  std::vector<int> shg_slot;  // [ndom]: slot of the domain's coefficients in shg_c, -1 for a linear domain
  void *shg_ws = nullptr;
  size_t shg_ws_bytes = 0;

  // Host-side staging (pinned)
  double *pinned = nullptr;
  size_t pinned_bytes = 0;

  // Polls before a bounded device wait gives up (MOM_ERR_TIMEOUT), per kind:
  // 0 LU panel exchange, 1 tensor-core GEMM mbarriers, 2 triangular-solve
  // hand-offs; 0 selects the default (mom_gpu_set_wait_limits).
  int64_t wait_limit[3] = {0, 0, 0};
};

// Default bounds of the device waits (a few seconds each).
constexpr int64_t kDefaultWaitPolls[3] = {int64_t(1) << 26, int64_t(1) << 22, int64_t(1) << 26};
inline long long wait_polls(const Ctx *c, int kind) {
  return (long long)(c->wait_limit[kind] > 0 ? c->wait_limit[kind] : kDefaultWaitPolls[kind]);
}

// Kernel categories for the optional timers.
enum ProfCat {
  kProfPair = 0, kProfNear, kProfGather, kProfPanel, kProfGemm, kProfTrsv, kProfResidual, kProfPost, kProfPivotAux,
  kProfTc, kProfDiagInv, kProfLu,
  kProfCount
};

// Records start/end events around a launch when profiling is on (on the
// context stream, or on the stream given).
struct ProfScope {
  struct Ctx *c;
  int cat;
  cudaStream_t s;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(struct Ctx *c_, int cat_, cudaStream_t s_ = nullptr);
  ~ProfScope();
};

// Error helpers
int fail(Ctx *c, int code, const std::string &msg);
int cuda_fail(Ctx *c, cudaError_t e, const char *where);
#define MOM_CUDA(c, expr)                                      \
  do {                                                         \
    cudaError_t _e = (expr);                                   \
    if (_e != cudaSuccess) return ::mom::cuda_fail(c, _e, #expr); \
  } while (0)
#define MOM_BLAS(c, expr)                                                              \
  do {                                                                                 \
    cublasStatus_t _s = (expr);                                                        \
    if (_s != CUBLAS_STATUS_SUCCESS)                                                   \
      return ::mom::fail(c, MOM_ERR_CUDA, std::string("cuBLAS error ") + std::to_string((int)_s) + " in " #expr); \
  } while (0)
#define MOM_TRY(expr)        \
  do {                       \
    int _r = (expr);         \
    if (_r != MOM_OK) return _r; \
  } while (0)

int ensure_buffer(Ctx *c, void **p, size_t *cap, size_t bytes);

// Points A, A32, ipiv, perm, invd, inv32 at representation r's buffers.
inline void select_rep(Ctx *c, int r) {
  const size_t mat = (size_t)c->lda * c->n, vec = (size_t)c->n, inv = 2 * (size_t)c->nb * c->n;
  c->A = c->A_all ? c->A_all + r * mat : nullptr;
  c->A32 = c->A32_all ? c->A32_all + r * mat : nullptr;
  c->ipiv = c->ipiv_all ? c->ipiv_all + r * vec : nullptr;
  c->perm = c->perm_all ? c->perm_all + r * vec : nullptr;
  c->invd = c->invd_all ? c->invd_all + r * inv : nullptr;
  c->inv32 = c->inv32_all ? c->inv32_all + r * inv : nullptr;
}

// assemble.cu
int upload_quadrature(Ctx *c);
int near_precompute(Ctx *c, int d);
int assemble(Ctx *c, double omega, const double *ri, int precision);
// The steps of assemble(): clear (and pad) the matrices; add domain d's
// D, H and K blocks; boundary conditions, FP32 copy and state.
int assemble_begin(Ctx *c);
int assemble_domain(Ctx *c, int d, double omega, const double *ri, int precision);
int assemble_end(Ctx *c, int precision);
// The test faces of domain d mapped by group action g (J^T), their near
// pairs and closed-form integrals (set-up of a symmetry group).
int action_precompute(Ctx *c, int d, int g);
void free_actions(DomDev &D);
// group.cu: the symmetry-plane boundary conditions of representation r
int apply_bc_matrix(Ctx *c, int r);
int apply_bc_rhs(Ctx *c, int r, double2 *B, int ncol);
int alloc_representations(Ctx *c, int nga);
int load_matrix(Ctx *c, const double *A_host, int64_t ldh, int precision);

// lu.cu
int lu_init_kernels(Ctx *c);
int lu_factor(Ctx *c, int precision);
int lu_solve(Ctx *c, int precision, double tol, int maxit, int *iters);
int lu_solve_ex(Ctx *c, int precision, int trans, const double2 *B, double2 *X, int nrhs, double tol, int maxit,
                int *iters);
// Y[:, s] += sign * A X[:, s] with the FP64 matrix of the current
// representation (n rows, ld n columns for X and Y).
int matvec_acc(Ctx *c, const double2 *X, int nrhs, double2 *Y, double sign);

// shg.cu: the second-harmonic solve (mom_gpu_shg_solve)
int shg_solve(Ctx *c, double omega, const double *ri, const double *shri, const mom_nls *nls, int precision,
              double tol, int maxit, int *iters);
void free_shg(DomDev &D);

// tc_gemm.cu: C -= L U (complex FP32) on the tensor cores, 3xTF32
int tc_cgemm_update(Ctx *c, float2 *C, int64_t ldc, const float2 *L, int64_t ldl, const float2 *U, int64_t ldu, int m,
                    int nc, int k, float *work, int *err, int max_ctas = 0, bool reuse_a = false,
                    bool trans_l = false);
size_t tc_cgemm_work_bytes(int m, int nc, int k);
int tc_init_kernels(Ctx *c);

// post.cu
int rhs_build(Ctx *c, double omega, const double *ri1, int nsrc, const mom_src *src);
// With a symmetry group, the solution of representation r, source s is at
// xdev + r xrep + s ldx (xrep unused for the identity group).
int cross_sections(Ctx *c, int dom, double omega, const double *ri, int nsrc, const mom_src *src,
                   const double2 *xdev, int64_t ldx, double *csca, double *cabs, int64_t xrep = 0);
int far_field(Ctx *c, int dom, double omega, const double *ri, const double2 *xdev, int ntheta, int nphi,
              double *rcs, int64_t xrep = 0);
// Near fields (nfields.f90 scat_fields; csrc/nfields_impl.cuh): E, H
// [nsrc][npts][3] of the currents X ([nsrc][ldx], device) at device points.
int scat_fields(Ctx *c, int d, double omega, const double *ri, int nsrc, const double2 *X, int64_t ldx, int npts,
                const double *pts, double2 *E, double2 *H);
// Adds the incident plane-wave fields of the sources at the device points
// (field_plane's addsrc, nfpost.f90:342-348); srcbuf: device scratch of at
// least 128 bytes per source.
int add_incident_fields(Ctx *c, double omega, const double *ri, int nsrc, const mom_src *src, int npts,
                        const double *pts, double2 *E, double2 *H, void *srcbuf);
int surface_fields(Ctx *c, int dom, double omega, const double *ri, const double2 *xdev, int64_t xrep, double2 *E,
                   double2 *H);
int cs_gradient(Ctx *c, int dom, double omega, const double *ri, int nsrc, const mom_src *src, const double2 *xdev,
                int64_t ldx, double2 *G);
void src_geometry(const mom_src &s, double dir[3], double pol[3]);

// adjoint (assemble.cu): derivative contractions.  Objective o pairs the
// adjoint currents lam[o] with the forward currents xv[o] (n each); R = 0
// uses the dense W(r, c) = sum lam[r] x[c] instead.
// adjoint_eps: t'_o = lam_o^T (dA / d eps_d) x_o (complex) into out[o][2].
int adjoint_eps(Ctx *c, double omega, const double *ri, int d, int R, const double2 *lam, const double2 *xv,
                const double2 *W, double *out);
// adjoint_nodes: d sigma_o / d(node coordinates) of every domain, out
// [R][sum of the domains' nodes][3]; obj_src / obj_kind give the source and
// the cross section (0 ext, 1 abs) of each objective.
int adjoint_nodes(Ctx *c, double omega, const double *ri, int R, const double2 *lam, const double2 *xv,
                  const int *obj_src, const int *obj_kind, int nsrc, const mom_src *src, double *out);

}  // namespace mom
