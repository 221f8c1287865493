// C ABI of the B200 PMCHWT library: context, problem upload and the entry
// points that replace sysmat_pmchwt, srcvec, solve_systems, cs_prtsrf and
// rcs of the reference (declarations and citations in include/mom_gpu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "mom_internal.h"

namespace mom {

int fail(Ctx *c, int code, const std::string &msg) {
  if (c) c->last_error = msg;
  return code;
}

int cuda_fail(Ctx *c, cudaError_t e, const char *where) {
  return fail(c, MOM_ERR_CUDA, std::string(cudaGetErrorString(e)) + " in " + where);
}

ProfScope::ProfScope(Ctx *c_, int cat_, cudaStream_t s_) : c(c_), cat(cat_), s(s_ ? s_ : c_->stream) {
  if (!c->prof) return;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    cudaGetLastError();
    a = b = nullptr;
    return;
  }
  // Inside a capture the records become event nodes of the graph.
  if (c->capturing) cudaEventRecordWithFlags(a, s, cudaEventRecordExternal);
  else cudaEventRecord(a, s);
}

ProfScope::~ProfScope() {
  if (!a) return;
  if (c->capturing) {
    cudaEventRecordWithFlags(b, s, cudaEventRecordExternal);
    c->cap_ev.emplace_back(cat, a, b);
    return;
  }
  cudaEventRecord(b, s);
  c->prof_ev[cat].push_back({a, b});
  c->prof_launch[cat]++;
}

void Ctx::LuGraph::reset() {
  if (exec) cudaGraphExecDestroy(exec);
  exec = nullptr;
  for (auto &e : ev) {
    cudaEventDestroy(std::get<1>(e));
    cudaEventDestroy(std::get<2>(e));
  }
  ev.clear();
  key.clear();
  launches = blas_calls = 0;
  tc_flops = 0;
}

int ensure_buffer(Ctx *c, void **p, size_t *cap, size_t bytes) {
  if (*p && *cap >= bytes) return MOM_OK;
  if (*p) {
    MOM_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
  }
  const size_t want = std::max<size_t>(bytes, 1 << 20);
  if (cudaMalloc(p, want) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(c, MOM_ERR_ALLOC, "device allocation of " + std::to_string(want) + " bytes failed");
  }
  *cap = want;
  return MOM_OK;
}

namespace {

void free_domain(DomDev &D) {
  cudaFree(D.qrel);
  cudaFree(D.qabs);
  cudaFree(D.cp);
  cudaFree(D.area);
  cudaFree(D.nrm);
  cudaFree(D.mu);
  cudaFree(D.sl);
  cudaFree(D.hpar);
  cudaFree(D.eh);
  cudaFree(D.epar);
  cudaFree(D.near_m);
  cudaFree(D.near_n);
  cudaFree(D.near_static);
  cudaFree(D.nodes);
  cudaFree(D.fsign);
  cudaFree(D.fnode);
  cudaFree(D.fea);
  cudaFree(D.feb);
  cudaFree(D.fbn);
  cudaFree(D.near_bits);
  cudaFree(D.inc_node);
  cudaFree(D.inc_face);
  cudaFree(D.nf_geo);
  cudaFree(D.nf_bn);
  free_shg(D);
  D = DomDev();
}

void free_problem(Ctx *c) {
  for (auto &D : c->dom) {
    free_actions(D);
    free_domain(D);
  }
  c->dom.clear();
  cudaFree(c->A_all);
  cudaFree(c->A32_all);
  cudaFree(c->blk);
  cudaFree(c->dmap);
  c->dmap = nullptr;
  c->blk_fused = false;
  cudaFree(c->ipiv_all);
  cudaFree(c->perm_all);
  cudaFree(c->invd_all);
  cudaFree(c->inv32_all);
  cudaFree(c->B);
  cudaFree(c->X);
  cudaFree(c->removed_dev);
  c->A_all = c->A = nullptr;
  c->A32_all = c->A32 = nullptr;
  c->blk = nullptr;
  c->ipiv_all = c->ipiv = nullptr;
  c->perm_all = c->perm = nullptr;
  c->invd_all = c->invd = nullptr;
  c->inv32_all = c->inv32 = nullptr;
  c->removed_dev = nullptr;
  c->removed.clear();
  c->removed_off.assign(2, 0);
  c->nga = 1;
  c->B = c->X = nullptr;
  c->BX_cap = 0;
  c->nsrc = 0;
  c->solved = false;
  c->shg_slot.clear();
  c->have_problem = false;
  c->assembled = 0;
  c->factored = -1;
}

template <typename T>
int upload(Ctx *c, T **dst, const std::vector<T> &h) {
  MOM_CUDA(c, cudaMalloc(dst, sizeof(T) * std::max<size_t>(1, h.size())));
  if (!h.empty()) MOM_CUDA(c, cudaMemcpyAsync(*dst, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, c->stream));
  return MOM_OK;
}

inline void cross(const double *a, const double *b, double *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
inline double nrm(const double *v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

// Geometry of one domain as compute_basis_data / average_edge_length /
// quad_tri_points compute it (mesh.f90:138-153, 1265-1322; quad.f90:352-367).
int build_domain(Ctx *c, const mom_mesh &m, DomDev &D) {
  const int F = m.nfaces, Nd = m.nedges, nq = c->nq;
  if (F <= 0 || Nd <= 0 || m.nnodes <= 0 || !m.nodes || !m.face_nodes || !m.face_edges || !m.edge_nodes ||
      !m.edge_faces || !m.edge_bnodes || !m.edge_parent)
    return fail(c, MOM_ERR_ARG, "incomplete domain mesh");
  for (int i = 0; i < 3 * F; i++)
    if (m.face_nodes[i] < 0 || m.face_nodes[i] >= m.nnodes || m.face_edges[i] < 0 || m.face_edges[i] >= Nd)
      return fail(c, MOM_ERR_MESH, "face index out of range");
  for (int e = 0; e < Nd; e++) {
    if (m.edge_parent[e] < 0 || m.edge_parent[e] >= c->N) return fail(c, MOM_ERR_MESH, "edge parent out of range");
    for (int k = 0; k < 2; k++) {
      if (m.edge_faces[2 * e + k] >= F || m.edge_nodes[2 * e + k] < 0 || m.edge_nodes[2 * e + k] >= m.nnodes)
        return fail(c, MOM_ERR_MESH, "edge index out of range");
      if (m.edge_faces[2 * e + k] >= 0 && (m.edge_bnodes[2 * e + k] < 0 || m.edge_bnodes[2 * e + k] >= m.nnodes))
        return fail(c, MOM_ERR_MESH, "edge free vertex out of range");
    }
  }
  D.F = F;
  D.Nd = Nd;
  const double *P = m.nodes;
  D.nnodes = m.nnodes;
  D.h_nodes.assign(P, P + 3 * (size_t)m.nnodes);
  D.h_fnode.assign(m.face_nodes, m.face_nodes + 3 * (size_t)F);
  D.h_fea.resize(3 * (size_t)F);
  D.h_feb.resize(3 * (size_t)F);
  D.h_fbn.resize(3 * (size_t)F);
  D.h_fsign.resize(3 * (size_t)F);
  D.h_cp.resize(3 * (size_t)F);
  D.h_area.resize(F);
  D.h_nrm.resize(3 * (size_t)F);
  D.h_qrel.resize((size_t)F * nq * 3);
  D.h_qabs.resize((size_t)F * nq * 3);
  D.h_mu.resize(9 * (size_t)F);
  D.h_sl.resize(3 * (size_t)F);
  D.h_hpar.resize(3 * (size_t)F);
  D.h_fv.resize(9 * (size_t)F);
  D.h_fs.resize(9 * (size_t)F);
  D.h_fm.resize(9 * (size_t)F);
  D.h_bn.resize(9 * (size_t)F);
  std::vector<double> elen(Nd);
  double ave = 0.0;
  for (int e = 0; e < Nd; e++) {
    const double *a = P + 3 * m.edge_nodes[2 * e], *b = P + 3 * m.edge_nodes[2 * e + 1];
    double d[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
    elen[e] = nrm(d);
    ave = ave + elen[e];
  }
  D.avelen = ave / Nd;
  for (int f = 0; f < F; f++) {
    const double *p1 = P + 3 * m.face_nodes[3 * f], *p2 = P + 3 * m.face_nodes[3 * f + 1],
                 *p3 = P + 3 * m.face_nodes[3 * f + 2];
    double a[3], b[3], cc[3], p21[3], p32[3], p13[3];
    for (int i = 0; i < 3; i++) {
      a[i] = p2[i] - p1[i];
      cc[i] = p3[i] - p1[i];
      p21[i] = p2[i] - p1[i];
      p32[i] = p3[i] - p2[i];
      p13[i] = p1[i] - p3[i];
    }
    cross(a, cc, b);
    const double nb = nrm(b);
    double *n = &D.h_nrm[3 * (size_t)f];
    for (int i = 0; i < 3; i++) n[i] = b[i] / nb;
    double *s = &D.h_fs[9 * (size_t)f], *mm = &D.h_fm[9 * (size_t)f];
    const double l21 = nrm(p21), l32 = nrm(p32), l13 = nrm(p13);
    for (int i = 0; i < 3; i++) {
      s[i] = p21[i] / l21;
      s[3 + i] = p32[i] / l32;
      s[6 + i] = p13[i] / l13;
    }
    for (int e = 0; e < 3; e++) {
      cross(s + 3 * e, n, mm + 3 * e);
      const double l = nrm(mm + 3 * e);
      for (int i = 0; i < 3; i++) mm[3 * e + i] = mm[3 * e + i] / l;
    }
    double mp13[3] = {-p13[0], -p13[1], -p13[2]}, cr[3];
    cross(mp13, p32, cr);
    const double A = 0.5 * nrm(cr);
    D.h_area[f] = A;
    double *cp = &D.h_cp[3 * (size_t)f];
    for (int i = 0; i < 3; i++) cp[i] = (p1[i] + p2[i] + p3[i]) / 3.0;
    for (int i = 0; i < 3; i++) {
      D.h_fv[9 * (size_t)f + i] = p1[i];
      D.h_fv[9 * (size_t)f + 3 + i] = p2[i];
      D.h_fv[9 * (size_t)f + 6 + i] = p3[i];
    }
    for (int t = 0; t < nq; t++)
      for (int i = 0; i < 3; i++) {
        const double q = c->qn[t][2] * p1[i] + c->qn[t][0] * p2[i] + c->qn[t][1] * p3[i];
        D.h_qabs[((size_t)f * nq + t) * 3 + i] = q;
        D.h_qrel[((size_t)f * nq + t) * 3 + i] = q - cp[i];
      }
    for (int e = 0; e < 3; e++) {
      const int ge = m.face_edges[3 * f + e];
      double sign;
      int bn;
      if (m.edge_faces[2 * ge] == f) {
        sign = 1.0;
        bn = m.edge_bnodes[2 * ge];
      } else if (m.edge_faces[2 * ge + 1] == f) {
        sign = -1.0;
        bn = m.edge_bnodes[2 * ge + 1];
      } else {
        return fail(c, MOM_ERR_MESH,
                    "Error evaluating mesh face sign (this could imply corrupted mesh connectivity)!");
      }
      D.h_sl[3 * (size_t)f + e] = sign * elen[ge];
      D.h_fsign[3 * (size_t)f + e] = sign;
      D.h_fea[3 * (size_t)f + e] = m.edge_nodes[2 * ge];
      D.h_feb[3 * (size_t)f + e] = m.edge_nodes[2 * ge + 1];
      D.h_fbn[3 * (size_t)f + e] = bn;
      D.h_hpar[3 * (size_t)f + e] = m.edge_parent[ge];
      for (int i = 0; i < 3; i++) {
        D.h_bn[9 * (size_t)f + 3 * e + i] = P[3 * bn + i];
        D.h_mu[9 * (size_t)f + 3 * e + i] = P[3 * bn + i] - cp[i];
      }
    }
  }
  D.h_eh.assign(2 * (size_t)Nd, -1);
  D.h_epar.resize(Nd);
  for (int e = 0; e < Nd; e++) {
    D.h_epar[e] = m.edge_parent[e];
    for (int k = 0; k < 2; k++) {
      const int f = m.edge_faces[2 * e + k];
      if (f < 0) continue;
      for (int p = 0; p < 3; p++)
        if (m.face_edges[3 * f + p] == e) D.h_eh[2 * e + k] = 3 * f + p;
    }
  }
  MOM_TRY(upload(c, &D.qrel, D.h_qrel));
  MOM_TRY(upload(c, &D.qabs, D.h_qabs));
  MOM_TRY(upload(c, &D.cp, D.h_cp));
  MOM_TRY(upload(c, &D.area, D.h_area));
  MOM_TRY(upload(c, &D.nrm, D.h_nrm));
  MOM_TRY(upload(c, &D.mu, D.h_mu));
  MOM_TRY(upload(c, &D.sl, D.h_sl));
  MOM_TRY(upload(c, &D.hpar, D.h_hpar));
  MOM_TRY(upload(c, &D.eh, D.h_eh));
  MOM_TRY(upload(c, &D.epar, D.h_epar));
  return MOM_OK;
}

int ensure_rhs(Ctx *c, int nsrc) {
  const size_t need = sizeof(double2) * (size_t)c->n * nsrc;
  if (c->B && c->BX_cap >= need) return MOM_OK;
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  cudaFree(c->B);
  cudaFree(c->X);
  c->B = c->X = nullptr;
  c->BX_cap = 0;
  if (cudaMalloc(&c->B, need) != cudaSuccess || cudaMalloc(&c->X, need) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, MOM_ERR_ALLOC, "right-hand side allocation failed");
  }
  c->BX_cap = need;
  return MOM_OK;
}

int ensure_a32(Ctx *c) {
  if (c->A32_all) return MOM_OK;
  const size_t bytes = sizeof(float2) * (size_t)c->lda * c->n * c->nga;
  if (cudaMalloc(&c->A32_all, bytes) != cudaSuccess ||
      cudaMalloc(&c->inv32_all, sizeof(float2) * 2 * (size_t)c->nb * c->n * c->nga) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(c->A32_all);
    c->A32_all = nullptr;
    return fail(c, MOM_ERR_ALLOC, "FP32 matrix allocation failed");
  }
  c->A32_bytes = bytes;
  select_rep(c, 0);
  return MOM_OK;
}

// Copy the 2N x ncol column blocks of every representation (device: rep r,
// column s at dev + (r ncol + s) n) to the host layout (2N, nga, ncol) with
// leading dimension ld (column (r, s) at host + 2 (s nga + r) ld doubles).
int copy_block_to_host(Ctx *c, const double2 *dev, int64_t ncol, double *host, int64_t ld) {
  const int64_t rows = 2 * (int64_t)c->N;
  for (int r = 0; r < c->nga; r++)
    MOM_CUDA(c, cudaMemcpy2DAsync(host + 2 * (size_t)r * ld, sizeof(double2) * ld * c->nga,
                                  dev + (size_t)r * ncol * c->n, sizeof(double2) * c->n, sizeof(double2) * rows, ncol,
                                  cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  return MOM_OK;
}

// The host layout (2N, nga, ncol), ld, to the device layout of copy_block_to_host.
int copy_block_to_device(Ctx *c, const double *host, int64_t ld, int64_t ncol, double2 *dev) {
  const int64_t rows = 2 * (int64_t)c->N;
  for (int r = 0; r < c->nga; r++)
    MOM_CUDA(c, cudaMemcpy2DAsync(dev + (size_t)r * ncol * c->n, sizeof(double2) * c->n, host + 2 * (size_t)r * ld,
                                  sizeof(double2) * ld * c->nga, sizeof(double2) * rows, ncol, cudaMemcpyHostToDevice,
                                  c->stream));
  return MOM_OK;
}

int no_group(Ctx *c, const char *what) {
  if (c->nga > 1) return fail(c, MOM_ERR_ARG, std::string(what) + " is not available with a symmetry group");
  return MOM_OK;
}

int check_prec(Ctx *c, int p) {
  if (p != MOM_PREC_FP64 && p != MOM_PREC_MIXED) return fail(c, MOM_ERR_ARG, "unknown precision");
  return MOM_OK;
}

}  // namespace
}  // namespace mom

using namespace mom;

struct mom_ctx : public Ctx {};

extern "C" {

int mom_gpu_create(int32_t device, mom_ctx **out) {
  if (!out) return MOM_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return MOM_ERR_CUDA;
  }
  mom_ctx *c = new (std::nothrow) mom_ctx();
  if (!c) return MOM_ERR_ALLOC;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaMalloc(&c->dinfo, sizeof(int) * 16) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return MOM_ERR_CUDA;
  }
  if (cublasCreate(&c->blas) != CUBLAS_STATUS_SUCCESS || cublasSetStream(c->blas, c->stream) != CUBLAS_STATUS_SUCCESS) {
    cudaStreamDestroy(c->stream);
    delete c;
    return MOM_ERR_CUDA;
  }
  // A fixed cuBLAS workspace (no allocation inside the captured LU graph);
  // the look-ahead stream has its own handle and workspace.
  bool ok = cudaMalloc(&c->blas_ws, kBlasWorkspace) == cudaSuccess &&
            cublasSetWorkspace(c->blas, c->blas_ws, kBlasWorkspace) == CUBLAS_STATUS_SUCCESS &&
            cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking) == cudaSuccess &&
            cublasCreate(&c->blas2) == CUBLAS_STATUS_SUCCESS &&
            cublasSetStream(c->blas2, c->stream2) == CUBLAS_STATUS_SUCCESS &&
            cudaMalloc(&c->blas_ws2, kBlasWorkspace) == cudaSuccess &&
            cublasSetWorkspace(c->blas2, c->blas_ws2, kBlasWorkspace) == CUBLAS_STATUS_SUCCESS;
  for (int i = 0; ok && i < 3; i++) ok = cudaEventCreateWithFlags(&c->la_ev[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok || lu_init_kernels(c) != MOM_OK || tc_init_kernels(c) != MOM_OK) {
    cudaGetLastError();
    cublasDestroy(c->blas);
    if (c->blas2) cublasDestroy(c->blas2);
    cudaFree(c->blas_ws);
    cudaFree(c->blas_ws2);
    for (auto &e : c->la_ev)
      if (e) cudaEventDestroy(e);
    if (c->stream2) cudaStreamDestroy(c->stream2);
    cudaStreamDestroy(c->stream);
    delete c;
    return MOM_ERR_CUDA;
  }
  const char *eg = std::getenv("MOM_LU_GRAPH");
  c->use_graph = !(eg && eg[0] == '0');
  const char *ea = std::getenv("MOM_AUTOTUNE");
  c->autotune = !(ea && ea[0] == '0');
  const char *et = std::getenv("MOM_SMALL_TC");
  if (et) c->small_tc = et[0] != '0';
  const char *eo = std::getenv("MOM_LU_OUTER");
  if (eo) c->outer_panels = std::max(1, std::min(16, std::atoi(eo)));
  const char *ep = std::getenv("MOM_PANEL_CTAS");
  if (ep) c->panel_cap_env = std::max(0, std::atoi(ep));
  const char *el = std::getenv("MOM_LOOKAHEAD");
  if (el) c->lookahead = el[0] != '0';
  const char *es = std::getenv("MOM_PAIR_SYM");
  if (es) c->pair_sym = es[0] != '0';
  const char *ee = std::getenv("MOM_PAIR_E32");
  if (ee) c->pair_e32 = ee[0] != '0';
  const char *ep3 = std::getenv("MOM_PAIR_CTAS");
  if (ep3) c->pair_ctas = std::atoi(ep3) == 3 ? 3 : 4;
  const char *ec = std::getenv("MOM_LA_CTAS");
  if (ec) c->la_ctas = std::max(0, std::atoi(ec));
  const char *ef = std::getenv("MOM_LA_FROM");
  if (ef) c->la_from = std::atof(ef);
  const char *ae = std::getenv("MOM_ADJ_EPS_PLAIN");
  if (ae) c->adj_eps_plain = std::atoi(ae) != 0;
  const char *av = std::getenv("MOM_ADJ_VERTEX_PLAIN");
  if (av) c->adj_vertex_plain = std::atoi(av) != 0;
  const char *ft = std::getenv("MOM_FUSED_TRSM");
  if (ft) c->fused_trsm = std::max(0, std::min(2, std::atoi(ft)));
  *out = c;
  return MOM_OK;
}

void mom_gpu_destroy(mom_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  free_problem(c);
  cudaFree(c->ws);
  cudaFree(c->ws2);
  cudaFree(c->Xh);
  cudaFree(c->nf_buf);
  cudaFree(c->adj);
  cudaFree(c->adj_part);
  cudaFree(c->adjW);
  cudaFree(c->shg_c);
  cudaFree(c->shg_ws);
  cudaFree(c->dinfo);
  if (c->pinned) cudaFreeHost(c->pinned);
  for (auto *g : c->lu_graphs) {
    g->reset();
    delete g;
  }
  c->lu_graphs.clear();
  cublasDestroy(c->blas);
  cublasDestroy(c->blas2);
  cudaFree(c->blas_ws);
  cudaFree(c->blas_ws2);
  for (auto &e : c->la_ev) cudaEventDestroy(e);
  cudaStreamDestroy(c->stream2);
  cudaStreamDestroy(c->stream);
  delete c;
}

const char *mom_gpu_strerror(int32_t s) {
  switch (s) {
    case MOM_OK: return "success";
    case MOM_ERR_ARG: return "invalid argument";
    case MOM_ERR_ALLOC: return "allocation failed";
    case MOM_ERR_CUDA: return "CUDA error";
    case MOM_ERR_SINGULAR: return "Matrix factorization failed! (singular matrix)";
    case MOM_ERR_TIMEOUT: return "device wait timed out";
    case MOM_ERR_STATE: return "call order violated";
    case MOM_ERR_MESH: return "inconsistent mesh";
    case MOM_ERR_NOCONV: return "iterative refinement did not converge";
    case MOM_ERR_IO: return "could not read mesh file";
    default: return "unknown status";
  }
}

const char *mom_gpu_last_error(mom_ctx *c) { return c ? c->last_error.c_str() : ""; }

int mom_gpu_set_problem(mom_ctx *c, int32_t nedges_total, int32_t ndom, const mom_mesh *doms, int32_t nq,
                        const double *qw, const double *qnodes) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (nedges_total <= 0 || ndom <= 0 || !doms || nq <= 0 || nq > kMaxQ || !qw || !qnodes)
    return fail(c, MOM_ERR_ARG, "invalid problem description");
  if (nq != 1 && nq != 3 && nq != 4 && nq != 7 && nq != 13)
    return fail(c, MOM_ERR_ARG, "triangle rule must have 1, 3, 4, 7 or 13 points");
  MOM_CUDA(c, cudaSetDevice(c->device));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  free_problem(c);
  c->N = nedges_total;
  c->ndom = ndom;
  c->nq = nq;
  for (int i = 0; i < kMaxQ; i++) {
    c->qw[i] = i < nq ? qw[i] : 0.0;
    for (int k = 0; k < 3; k++) c->qn[i][k] = i < nq ? qnodes[3 * i + k] : 0.0;
  }
  MOM_TRY(upload_quadrature(c));
  c->dom.resize(ndom);
  size_t maxF = 0;
  for (int d = 0; d < ndom; d++) {
    MOM_TRY(build_domain(c, doms[d], c->dom[d]));
    maxF = std::max<size_t>(maxF, c->dom[d].F);
  }
  for (int d = 0; d < ndom; d++) MOM_TRY(near_precompute(c, d));
  const int64_t n2 = 2 * (int64_t)c->N;
  c->nb = 64;
  c->n = (n2 + c->nb - 1) / c->nb * c->nb;
  c->lda = c->n;
  c->blk_bytes = sizeof(double2) * 18 * maxF * maxF;
  // Face-pair blocks of all domains at once (one gather writes the matrix)
  // when they fit beside the matrices with room to spare.
  {
    size_t total = 0;
    c->blk_off.assign(ndom, 0);
    for (int d = 0; d < ndom; d++) {
      c->blk_off[d] = total / sizeof(double2);
      total += sizeof(double2) * 18 * (size_t)c->dom[d].F * c->dom[d].F;
    }
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    const size_t mats = (size_t)c->lda * c->n * (sizeof(double2) + sizeof(float2)) + (size_t(4) << 30);
    const char *fg = std::getenv("MOM_FUSED_GATHER");
    c->blk_fused = ndom <= 8 && fr > total + mats && !(fg && std::atoi(fg) == 0);
    if (c->blk_fused) {
      std::vector<int> dm((size_t)ndom * c->N, -1);
      for (int d = 0; d < ndom; d++)
        for (int e = 0; e < c->dom[d].Nd; e++) dm[(size_t)d * c->N + c->dom[d].h_epar[e]] = e;
      MOM_TRY(upload(c, &c->dmap, dm));
      c->blk_bytes = total;
    }
  }
  // the identity group: one element, one representation, nothing removed
  std::memset(c->ga, 0, sizeof c->ga);
  c->ga[0].j[0] = c->ga[0].j[4] = c->ga[0].j[8] = 1.0;
  c->ga[0].detj = 1.0;
  c->ga[0].id = 1;
  c->ga[0].genbits = 2u;
  c->ga[0].ef[0] = 1.0;
  c->nga = 1;
  c->removed.assign(1, {});
  c->removed_off.assign(2, 0);
  c->edge_bnd.assign(c->N, MOM_BND_NONE);
  if (cudaMalloc(&c->blk, c->blk_bytes) != cudaSuccess || alloc_representations(c, 1) != MOM_OK) {
    cudaGetLastError();
    free_problem(c);
    return fail(c, MOM_ERR_ALLOC, "device allocation for the system matrix failed");
  }
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  c->have_problem = true;
  return MOM_OK;
}

int mom_gpu_sysmat(mom_ctx *c, double omega, const double *ri, int32_t precision, double *A_host, int64_t lda) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem before sysmat");
  if (!ri || !(omega > 0)) return fail(c, MOM_ERR_ARG, "invalid omega or refractive indices");
  MOM_TRY(check_prec(c, precision));
  if (A_host && lda < 2 * (int64_t)c->N) return fail(c, MOM_ERR_ARG, "lda < 2N");
  MOM_CUDA(c, cudaSetDevice(c->device));
  if (precision == MOM_PREC_MIXED) MOM_TRY(ensure_a32(c));
  MOM_TRY(assemble(c, omega, ri, precision));
  for (int r = 0; A_host && r < c->nga; r++) {
    const int64_t rows = 2 * (int64_t)c->N;
    MOM_CUDA(c, cudaMemcpy2DAsync(A_host + 2 * (size_t)r * lda * rows, sizeof(double2) * lda,
                                  c->A_all + (size_t)r * c->lda * c->n, sizeof(double2) * c->lda,
                                  sizeof(double2) * rows, rows, cudaMemcpyDeviceToHost, c->stream));
  }
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  return MOM_OK;
}

int mom_gpu_srcvec(mom_ctx *c, double omega, const double *ri1, int32_t nsrc, const mom_src *src, double *q_host,
                   int64_t ldq) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem before srcvec");
  if (!ri1 || nsrc <= 0 || !src || !(omega > 0)) return fail(c, MOM_ERR_ARG, "invalid sources");
  if (q_host && ldq < 2 * (int64_t)c->N) return fail(c, MOM_ERR_ARG, "ldq < 2N");
  MOM_CUDA(c, cudaSetDevice(c->device));
  MOM_TRY(ensure_rhs(c, nsrc * c->nga));
  MOM_TRY(rhs_build(c, omega, ri1, nsrc, src));
  c->nsrc = nsrc;
  c->solved = false;
  c->srcs.assign(src, src + nsrc);
  c->omega_rhs = omega;
  c->ri1[0] = ri1[0];
  c->ri1[1] = ri1[1];
  if (q_host) MOM_TRY(copy_block_to_host(c, c->B, nsrc, q_host, ldq));
  return MOM_OK;
}

int mom_gpu_solve(mom_ctx *c, int32_t precision, double tol, int32_t maxit, double *x_host, int64_t ldx,
                  int32_t *iters_out) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  MOM_TRY(check_prec(c, precision));
  if (!c->assembled && c->factored != precision)
    return fail(c, MOM_ERR_STATE, "build the system matrix before solving");
  if (c->nsrc <= 0) return fail(c, MOM_ERR_STATE, "compute source vectors before solving");
  if (x_host && ldx < 2 * (int64_t)c->N) return fail(c, MOM_ERR_ARG, "ldx < 2N");
  if (precision == MOM_PREC_MIXED && (!c->A32 || maxit <= 0 || !(tol > 0)))
    return fail(c, MOM_ERR_ARG, "mixed solve needs a mixed sysmat and tol > 0, maxit > 0");
  MOM_CUDA(c, cudaSetDevice(c->device));
  // one factorisation and solve per representation (solve_systems, solver.f90:325-357)
  int it = 0;
  if (c->factored != precision) {
    for (int r = 0; r < c->nga; r++) {
      select_rep(c, r);
      const int rc = lu_factor(c, precision);
      if (rc != MOM_OK) {
        select_rep(c, 0);
        c->factored = -1;
        return rc;
      }
    }
  }
  for (int r = 0; r < c->nga; r++) {
    select_rep(c, r);
    int itr = 0;
    const size_t off = (size_t)r * c->nsrc * c->n;
    const int rc = lu_solve_ex(c, precision, 0, c->B + off, c->X + off, c->nsrc, tol, maxit, &itr);
    if (rc != MOM_OK) {
      select_rep(c, 0);
      return rc;
    }
    it = std::max(it, itr);
  }
  select_rep(c, 0);
  if (precision == MOM_PREC_FP64) c->assembled = 0;  // the matrices now hold their LU factors
  c->solved = true;
  if (iters_out) *iters_out = it;
  if (x_host) MOM_TRY(copy_block_to_host(c, c->X, c->nsrc, x_host, ldx));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  return MOM_OK;
}

int mom_gpu_solve_wavelength(mom_ctx *c, double omega, const double *ri, int32_t nsrc, const mom_src *src,
                             int32_t precision, double tol, int32_t maxit, double *x_host, int64_t ldx,
                             int32_t *iters_out) {
  int r = mom_gpu_sysmat(c, omega, ri, precision, nullptr, 0);
  if (r) return r;
  r = mom_gpu_srcvec(c, omega, ri, nsrc, src, nullptr, 0);
  if (r) return r;
  return mom_gpu_solve(c, precision, tol, maxit, x_host, ldx, iters_out);
}

int mom_gpu_shg_solve(mom_ctx *c, double omega, const double *ri, const double *shri, const mom_nls *nls,
                      int32_t precision, double tol, int32_t maxit, double *nlx_host, int64_t ldx,
                      int32_t *iters_out) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem before the second-harmonic solve");
  if (!ri || !shri || !nls || !(omega > 0)) return fail(c, MOM_ERR_ARG, "invalid omega, refractive indices or media");
  MOM_TRY(check_prec(c, precision));
  if (c->nsrc <= 0 || !c->solved) return fail(c, MOM_ERR_STATE, "solve at the fundamental frequency first");
  if (nlx_host && ldx < 2 * (int64_t)c->N) return fail(c, MOM_ERR_ARG, "ldx < 2N");
  if (precision == MOM_PREC_MIXED && (maxit <= 0 || !(tol > 0)))
    return fail(c, MOM_ERR_ARG, "mixed solve needs tol > 0, maxit > 0");
  MOM_CUDA(c, cudaSetDevice(c->device));
  if (precision == MOM_PREC_MIXED) MOM_TRY(ensure_a32(c));
  int it = 0;
  c->solved = false;  // the device solutions become the second harmonic's
  const int rc = shg_solve(c, omega, ri, shri, nls, precision, tol, maxit, &it);
  if (rc != MOM_OK) {
    c->factored = -1;
    return rc;
  }
  if (iters_out) *iters_out = it;
  if (nlx_host) MOM_TRY(copy_block_to_host(c, c->X, c->nsrc, nlx_host, ldx));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  return MOM_OK;
}

int mom_gpu_shg_source_coef(mom_ctx *c, int32_t dom, double *coef_host, int64_t ldc) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem || dom < 0 || dom >= c->ndom || !coef_host || ldc < 2 * (int64_t)c->N)
    return fail(c, MOM_ERR_ARG, "invalid domain or output for the second-harmonic source coefficients");
  if (dom >= (int)c->shg_slot.size() || c->shg_slot[dom] < 0 || !c->shg_c)
    return fail(c, MOM_ERR_STATE, "no second-harmonic source coefficients for this domain");
  MOM_CUDA(c, cudaSetDevice(c->device));
  const double2 *src = (const double2 *)c->shg_c + (size_t)c->shg_slot[dom] * c->n * c->nsrc * c->nga;
  return copy_block_to_host(c, src, c->nsrc, coef_host, ldc);
}

int mom_gpu_sweep(mom_ctx *c, int32_t nwl, const double *omega, const double *ri, int32_t nsrc, const mom_src *src,
                  int32_t precision, double tol, int32_t maxit, double *csca, double *cabs, int32_t *iters) {
  if (!c) return MOM_ERR_ARG;
  if (nwl <= 0 || !omega || !ri || nsrc <= 0 || !src || !csca || !cabs) return fail(c, MOM_ERR_ARG, "invalid sweep arguments");
  int ndom = 0;
  {
    std::lock_guard<std::mutex> g(c->mu);
    if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem first");
    ndom = c->ndom;
  }
  for (int w = 0; w < nwl; w++) {
    const double *r = ri + (size_t)w * 2 * ndom;
    int it = 0;
    MOM_TRY(mom_gpu_solve_wavelength(c, omega[w], r, nsrc, src, precision, tol, maxit, nullptr, 0, &it));
    MOM_TRY(mom_gpu_cross_sections(c, 0, omega[w], r, nsrc, src, nullptr, 0, csca + (size_t)w * nsrc,
                                   cabs + (size_t)w * nsrc));
    if (iters) iters[w] = it;
  }
  return MOM_OK;
}

int mom_gpu_sweep_many(int32_t nctx, mom_ctx **ctx, const int32_t *nwl, const double *const *omega,
                       const double *const *ri, int32_t nsrc, const mom_src *src, int32_t precision, double tol,
                       int32_t maxit, double *const *csca, double *const *cabs, int32_t *status) {
  if (nctx <= 0 || !ctx || !nwl || !omega || !ri || !csca || !cabs) return MOM_ERR_ARG;
  std::vector<int> st(nctx, MOM_OK);
  std::vector<std::thread> th;
  th.reserve(nctx);
  for (int i = 0; i < nctx; i++)
    th.emplace_back([&, i]() {
      st[i] = mom_gpu_sweep(ctx[i], nwl[i], omega[i], ri[i], nsrc, src, precision, tol, maxit, csca[i], cabs[i],
                            nullptr);
    });
  for (auto &t : th) t.join();
  int rc = MOM_OK;
  for (int i = 0; i < nctx; i++) {
    if (status) status[i] = st[i];
    if (rc == MOM_OK && st[i] != MOM_OK) rc = st[i];
  }
  return rc;
}

int mom_gpu_autotune_result(mom_ctx *c, int32_t precision, int32_t max_entries, int32_t *nent, int64_t *heights,
                            int32_t *ctas, double *us_per_column, double *tune_ms) {
  if (!c || !nent) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  for (const auto &t : c->tuned)
    if (t.n == c->n && t.precision == precision) {
      const int k = std::min<int>(max_entries, (int)t.m.size());
      for (int i = 0; i < k; i++) {
        if (heights) heights[i] = t.m[i];
        if (ctas) ctas[i] = t.P[i];
        if (us_per_column) us_per_column[i] = t.us[i];
      }
      *nent = (int32_t)t.m.size();
      if (tune_ms) *tune_ms = t.ms;
      return MOM_OK;
    }
  return fail(c, MOM_ERR_STATE, "no autotuning result for this matrix order and precision");
}

int mom_gpu_autotune_placement(mom_ctx *c, int32_t precision, int32_t max_entries, int32_t *nent, int32_t *chosen,
                               double *us_per_column) {
  if (!c || !nent || !chosen) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  for (const auto &t : c->tuned)
    if (t.n == c->n && t.precision == precision) {
      const int k = std::min<int>(max_entries, (int)t.xslot_us.size());
      for (int i = 0; us_per_column && i < k; i++) us_per_column[i] = t.xslot_us[i];
      *nent = (int32_t)t.xslot_us.size();
      *chosen = t.xslot;
      return MOM_OK;
    }
  return fail(c, MOM_ERR_STATE, "no autotuning result for this matrix order and precision");
}

int32_t mom_gpu_domain_nodes(mom_ctx *c, int32_t dom) {
  if (!c || !c->have_problem || dom < 0 || dom >= c->ndom) return -1;
  return c->dom[dom].nnodes;
}

// Shared set-up of the adjoint entry points: G = d sigma / dx of the solved
// sources and the adjoint currents A^T lambda = G (2 nsrc columns: ext, abs
// per source) in c->adj; returns the pointers.
static int adjoint_currents(mom_ctx *c, int32_t precision, double omega, const double *ri, int32_t nsrc,
                            const mom_src *src, double tol, int32_t maxit, double2 **G, double2 **lam,
                            double2 **xo, int32_t *iters) {
  MOM_TRY(check_prec(c, precision));
  if (c->factored != precision || !c->solved)
    return fail(c, MOM_ERR_STATE, "the adjoint needs the factors and solutions of a solve in this precision");
  if (nsrc != c->nsrc || nsrc <= 0 || !src || !ri || !(omega > 0))
    return fail(c, MOM_ERR_ARG, "the adjoint sources must be those of the last solve");
  if (precision == MOM_PREC_MIXED && (maxit <= 0 || !(tol > 0))) return fail(c, MOM_ERR_ARG, "mixed adjoint needs tol > 0, maxit > 0");
  const size_t col = sizeof(double2) * (size_t)c->n, R = 2 * (size_t)nsrc;
  MOM_TRY(ensure_buffer(c, &c->adj, &c->adj_bytes, 3 * R * col));
  *G = (double2 *)c->adj;
  *lam = (double2 *)((char *)c->adj + R * col);
  *xo = (double2 *)((char *)c->adj + 2 * R * col);
  MOM_TRY(cs_gradient(c, 0, omega, ri, nsrc, src, c->X, c->n, *G));
  int it = 0;
  MOM_TRY(lu_solve_ex(c, precision, 1, *G, *lam, (int)R, tol, maxit, &it));
  if (iters) *iters = it;
  for (int s = 0; s < nsrc; s++)
    for (int k = 0; k < 2; k++)
      MOM_CUDA(c, cudaMemcpyAsync((char *)*xo + (2 * s + k) * col, c->X + (size_t)s * c->n, col,
                                  cudaMemcpyDeviceToDevice, c->stream));
  return MOM_OK;
}

int mom_gpu_adjoint(mom_ctx *c, int32_t precision, double omega, const double *ri, int32_t nsrc, const mom_src *src,
                    int32_t eps_dom, double tol, int32_t maxit, double *deps, double *dnodes, int32_t *iters_out) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem first");
  if (nsrc < 1 || nsrc > 4) return fail(c, MOM_ERR_ARG, "per-source adjoint gradients take 1 to 4 sources");
  if (deps && (eps_dom < 1 || eps_dom >= c->ndom)) return fail(c, MOM_ERR_ARG, "eps_dom must be an interior domain");
  MOM_TRY(no_group(c, "adjoint gradients"));
  MOM_CUDA(c, cudaSetDevice(c->device));
  double2 *G = nullptr, *lam = nullptr, *xo = nullptr;
  MOM_TRY(adjoint_currents(c, precision, omega, ri, nsrc, src, tol, maxit, &G, &lam, &xo, iters_out));
  const int R = 2 * nsrc;
  if (deps) {
    std::vector<double> t(2 * R);
    MOM_TRY(adjoint_eps(c, omega, ri, eps_dom, R, lam, xo, nullptr, t.data()));
    // d sigma = -Re(lambda^T A' x d eps): d/dRe eps = -Re t', d/dIm eps = Im t'
    for (int o = 0; o < R; o++) {
      deps[2 * o] = -t[2 * o];
      deps[2 * o + 1] = t[2 * o + 1];
    }
  }
  if (dnodes) {
    std::vector<int> osrc(R), okind(R);
    for (int o = 0; o < R; o++) {
      osrc[o] = o / 2;
      okind[o] = o % 2;
    }
    MOM_TRY(adjoint_nodes(c, omega, ri, R, lam, xo, osrc.data(), okind.data(), nsrc, src, dnodes));
  }
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  return MOM_OK;
}

int mom_gpu_adjoint_mean_eps(mom_ctx *c, int32_t precision, double omega, const double *ri, int32_t nsrc,
                             const mom_src *src, int32_t eps_dom, double tol, int32_t maxit, double *dmean,
                             int32_t *iters_out) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem first");
  if (!dmean || eps_dom < 1 || eps_dom >= c->ndom) return fail(c, MOM_ERR_ARG, "eps_dom must be an interior domain");
  MOM_TRY(no_group(c, "adjoint gradients"));
  MOM_CUDA(c, cudaSetDevice(c->device));
  double2 *G = nullptr, *lam = nullptr, *xo = nullptr;
  MOM_TRY(adjoint_currents(c, precision, omega, ri, nsrc, src, tol, maxit, &G, &lam, &xo, iters_out));
  const int64_t n = c->n;
  MOM_TRY(ensure_buffer(c, &c->adjW, &c->adjW_bytes, sizeof(double2) * (size_t)n * n));
  double2 *W = (double2 *)c->adjW;
  for (int k = 0; k < 2; k++) {
    // W = (1/nsrc) sum_s lambda_{2s+k} x_s^T (a plain library GEMM, K = nsrc)
    const cuDoubleComplex al = make_cuDoubleComplex(1.0 / nsrc, 0.0), be = make_cuDoubleComplex(0.0, 0.0);
    MOM_BLAS(c, cublasSetMathMode(c->blas, CUBLAS_DEFAULT_MATH));
    MOM_BLAS(c, cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)n, (int)n, nsrc, &al,
                            (const cuDoubleComplex *)(lam + (size_t)k * n), (int)(2 * n),
                            (const cuDoubleComplex *)c->X, (int)n, &be, (cuDoubleComplex *)W, (int)n));
    c->blas_calls++;
    double t[2];
    MOM_TRY(adjoint_eps(c, omega, ri, eps_dom, 0, nullptr, nullptr, W, t));
    dmean[2 * k] = -t[0];
    dmean[2 * k + 1] = t[1];
  }
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  return MOM_OK;
}

int mom_gpu_cross_sections(mom_ctx *c, int32_t dom, double omega, const double *ri, int32_t nsrc,
                           const mom_src *src, const double *x_host, int64_t ldx, double *csca, double *cabs) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem first");
  if (dom < 0 || dom >= c->ndom || nsrc <= 0 || !src || !ri || !csca || !cabs || !(omega > 0))
    return fail(c, MOM_ERR_ARG, "invalid cross-section arguments");
  MOM_CUDA(c, cudaSetDevice(c->device));
  const double2 *xd = c->X;
  int64_t ld = c->n, xrep = (int64_t)c->nsrc * c->n;
  if (x_host) {
    if (ldx < 2 * (int64_t)c->N) return fail(c, MOM_ERR_ARG, "ldx < 2N");
    MOM_TRY(ensure_buffer(c, (void **)&c->Xh, &c->Xh_cap, sizeof(double2) * c->n * nsrc * c->nga));
    MOM_TRY(copy_block_to_device(c, x_host, ldx, nsrc, c->Xh));
    xd = c->Xh;
    xrep = (int64_t)nsrc * c->n;
  } else if (nsrc > c->nsrc) {
    return fail(c, MOM_ERR_STATE, "no device solution for that many sources");
  }
  return cross_sections(c, dom, omega, ri, nsrc, src, xd, ld, csca, cabs, xrep);
}

int mom_gpu_rcs(mom_ctx *c, int32_t dom, double omega, const double *ri, int32_t isrc, const double *x_host,
                int64_t ldx, int32_t ntheta, int32_t nphi, double *rcs) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem first");
  if (dom < 0 || dom >= c->ndom || ntheta < 2 || nphi < 2 || !rcs || !ri || isrc < 0 || !(omega > 0))
    return fail(c, MOM_ERR_ARG, "invalid far-field arguments");
  MOM_CUDA(c, cudaSetDevice(c->device));
  const double2 *xd;
  int64_t xrep;
  if (x_host) {
    if (ldx < 2 * (int64_t)c->N) return fail(c, MOM_ERR_ARG, "ldx < 2N");
    MOM_TRY(ensure_buffer(c, (void **)&c->Xh, &c->Xh_cap, sizeof(double2) * c->n * c->nga));
    MOM_TRY(copy_block_to_device(c, x_host + 2 * (size_t)isrc * c->nga * ldx, ldx, 1, c->Xh));
    xd = c->Xh;
    xrep = c->n;
  } else {
    if (isrc >= c->nsrc) return fail(c, MOM_ERR_STATE, "no device solution for that source");
    xd = c->X + (size_t)isrc * c->n;
    xrep = (int64_t)c->nsrc * c->n;
  }
  return far_field(c, dom, omega, ri, xd, ntheta, nphi, rcs, xrep);
}

int mom_gpu_scat_fields(mom_ctx *c, int32_t dom, double omega, const double *ri, int32_t nsrc, const mom_src *src,
                        const double *x_host, int64_t ldx, int32_t npts, const double *pts, double *e, double *h) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem first");
  if (dom < 0 || dom >= c->ndom || nsrc < 1 || npts < 1 || !pts || !e || !h || !ri || !(omega > 0))
    return fail(c, MOM_ERR_ARG, "invalid near-field arguments");
  MOM_TRY(no_group(c, "near fields"));
  MOM_CUDA(c, cudaSetDevice(c->device));
  const size_t pbytes = ((sizeof(double) * 3 * (size_t)npts + 255) / 256) * 256;
  const size_t fbytes = ((sizeof(double2) * 3 * (size_t)npts * nsrc + 255) / 256) * 256;
  const size_t xbytes = x_host ? sizeof(double2) * (size_t)c->n * nsrc : 0;
  const size_t sbytes = (size_t)128 * nsrc;
  MOM_TRY(ensure_buffer(c, &c->nf_buf, &c->nf_cap, pbytes + 2 * fbytes + sbytes + xbytes + 256));
  char *b = (char *)c->nf_buf;
  double *dp = (double *)b;
  double2 *dE = (double2 *)(b + pbytes), *dH = (double2 *)(b + pbytes + fbytes);
  void *dsrc = b + pbytes + 2 * fbytes;
  const double2 *xd;
  int64_t ldxd;
  if (x_host) {
    if (ldx < 2 * (int64_t)c->N) return fail(c, MOM_ERR_ARG, "ldx < 2N");
    double2 *xh = (double2 *)(b + pbytes + 2 * fbytes + ((sbytes + 255) / 256) * 256);
    MOM_CUDA(c, cudaMemcpy2DAsync(xh, sizeof(double2) * c->n, x_host, sizeof(double2) * ldx,
                                  sizeof(double2) * 2 * c->N, nsrc, cudaMemcpyHostToDevice, c->stream));
    xd = xh;
    ldxd = c->n;
  } else {
    if (nsrc > c->nsrc) return fail(c, MOM_ERR_STATE, "no device solutions for that many sources");
    xd = c->X;
    ldxd = c->n;
  }
  MOM_CUDA(c, cudaMemcpyAsync(dp, pts, sizeof(double) * 3 * npts, cudaMemcpyHostToDevice, c->stream));
  {
    ProfScope ps(c, kProfPost);
    MOM_TRY(scat_fields(c, dom, omega, ri, nsrc, xd, ldxd, npts, dp, dE, dH));
    if (src) MOM_TRY(add_incident_fields(c, omega, ri, nsrc, src, npts, dp, dE, dH, dsrc));
  }
  MOM_CUDA(c, cudaMemcpyAsync(e, dE, sizeof(double2) * 3 * (size_t)npts * nsrc, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaMemcpyAsync(h, dH, sizeof(double2) * 3 * (size_t)npts * nsrc, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  return MOM_OK;
}

int mom_gpu_set_wait_limits(mom_ctx *c, int64_t panel_polls, int64_t gemm_polls, int64_t solve_polls) {
  if (!c || panel_polls < 0 || gemm_polls < 0 || solve_polls < 0) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  c->wait_limit[0] = panel_polls;
  c->wait_limit[1] = gemm_polls;
  c->wait_limit[2] = solve_polls;
  return MOM_OK;
}

int mom_gpu_set_matrix(mom_ctx *c, int32_t precision, const double *A_host, int64_t lda) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem before the matrix");
  MOM_TRY(check_prec(c, precision));
  if (!A_host || lda < 2 * (int64_t)c->N) return fail(c, MOM_ERR_ARG, "invalid matrix or lda < 2N");
  MOM_TRY(no_group(c, "a caller's matrix"));
  MOM_CUDA(c, cudaSetDevice(c->device));
  if (precision == MOM_PREC_MIXED) MOM_TRY(ensure_a32(c));
  MOM_TRY(load_matrix(c, A_host, lda, precision));
  return MOM_OK;
}

int mom_gpu_surface_fields(mom_ctx *c, int32_t dom, double omega, const double *ri, int32_t isrc, const double *x_host,
                           int64_t ldx, double *e, double *h) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem first");
  if (dom < 0 || dom >= c->ndom || !ri || !e || !h || isrc < 0 || !(omega > 0))
    return fail(c, MOM_ERR_ARG, "invalid surface-field arguments");
  MOM_CUDA(c, cudaSetDevice(c->device));
  const size_t fbytes = ((sizeof(double2) * 3 * (size_t)c->dom[dom].F * c->nga + 255) / 256) * 256;
  const size_t xbytes = x_host ? sizeof(double2) * (size_t)c->n * c->nga : 0;
  MOM_TRY(ensure_buffer(c, &c->nf_buf, &c->nf_cap, 2 * fbytes + xbytes + 256));
  char *b = (char *)c->nf_buf;
  double2 *dE = (double2 *)b, *dH = (double2 *)(b + fbytes);
  const double2 *xd;
  int64_t xrep;
  if (x_host) {
    if (ldx < 2 * (int64_t)c->N) return fail(c, MOM_ERR_ARG, "ldx < 2N");
    double2 *xh = (double2 *)(b + 2 * fbytes);
    MOM_TRY(copy_block_to_device(c, x_host + 2 * (size_t)isrc * c->nga * ldx, ldx, 1, xh));
    xd = xh;
    xrep = c->n;
  } else {
    if (isrc >= c->nsrc) return fail(c, MOM_ERR_STATE, "no device solution for that source");
    xd = c->X + (size_t)isrc * c->n;
    xrep = (int64_t)c->nsrc * c->n;
  }
  MOM_TRY(surface_fields(c, dom, omega, ri, xd, xrep, dE, dH));
  const size_t out = sizeof(double2) * 3 * (size_t)c->dom[dom].F * c->nga;
  MOM_CUDA(c, cudaMemcpyAsync(e, dE, out, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaMemcpyAsync(h, dH, out, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  return MOM_OK;
}

int mom_gpu_group_action(mom_ctx *c, int32_t g, double *j, double *detj) {
  if (!c || !j || !detj) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem first");
  if (g < 0 || g >= c->nga) return fail(c, MOM_ERR_ARG, "group element out of range");
  for (int i = 0; i < 9; i++) j[i] = c->ga[g].j[i];
  *detj = c->ga[g].detj;
  return MOM_OK;
}

int mom_gpu_device_matrix(mom_ctx *c, void **A_dev, int64_t *lda) {
  if (!c || !A_dev || !lda) return MOM_ERR_ARG;
  *A_dev = c->A;
  *lda = c->lda;
  return MOM_OK;
}

int mom_gpu_device_solution(mom_ctx *c, void **x_dev, int64_t *ldx, int32_t *nsrc) {
  if (!c || !x_dev || !ldx || !nsrc) return MOM_ERR_ARG;
  *x_dev = c->X;
  *ldx = c->n;
  *nsrc = c->nsrc;
  return MOM_OK;
}

int mom_gpu_synchronize(mom_ctx *c) {
  if (!c) return MOM_ERR_ARG;
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  return MOM_OK;
}

int64_t mom_gpu_launch_count(mom_ctx *c) { return c ? c->launches : 0; }

void *mom_gpu_stream(mom_ctx *c) { return c ? (void *)c->stream : nullptr; }

int64_t mom_gpu_library_calls(mom_ctx *c) { return c ? c->blas_calls : 0; }

double mom_gpu_tensor_flops(mom_ctx *c) { return c ? c->tc_flops : 0.0; }

int mom_gpu_profile(mom_ctx *c, int32_t enable) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  cudaStreamSynchronize(c->stream);
  for (auto &v : c->prof_ev) {
    for (auto &e : v) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
    v.clear();
  }
  for (auto &n : c->prof_launch) n = 0;
  for (auto &t : c->prof_ms) t = 0;
  c->prof = enable != 0;
  return MOM_OK;
}

int mom_gpu_profile_read(mom_ctx *c, int32_t category, double *ms_total, int64_t *launches) {
  if (!c || category < 0 || category >= kProfCount || !ms_total || !launches) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  double t = 0;
  for (auto &e : c->prof_ev[category]) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, e.first, e.second) == cudaSuccess) t += ms;
  }
  *ms_total = t + c->prof_ms[category];
  *launches = c->prof_launch[category];
  return MOM_OK;
}

}  // extern "C"
