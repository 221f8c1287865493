// Symmetry groups of mirror planes (the nga > 1 path of the reference).
//
//   read_symm       (interface.f90:160-210): the group is the product of the
//                   named groups "id", "mxp", "myp", "mzp";
//   group_id / group_mp / product_group (symmetry.f90:45-103, 178-241):
//                   element k = n nb + m of a x b is a_n b_m, with J, det J,
//                   generator bits and field actions multiplied;
//   edge_bc         (bc.f90:28-117): per representation, the J (M)
//                   coefficient of a master edge on a mirror plane is removed
//                   when the field action (times det J) of that plane's
//                   mirror is not -1;
//   reduce_system / expand_solution (bc.f90:170-232): here the removed
//                   unknowns keep their place with an identity row and
//                   column and a zero right-hand side, so every
//                   representation keeps the order 2N and the solution is 0
//                   there, which is what expand_solution writes;
//   admissible_ga   (bc.f90:237-257): a mirror acts on an interior domain only
//                   if that domain has edges on the mirror's plane.
// Rotation groups (rN) are not supported.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "mom_internal.h"

namespace mom {
namespace {

constexpr int kGidIdentity = 1, kGidMxp = 2, kGidMyp = 3, kGidMzp = 4;

void ga_identity(GroupAction &g) {
  std::memset(&g, 0, sizeof g);
  g.j[0] = g.j[4] = g.j[8] = 1.0;
  g.detj = 1.0;
  g.id = kGidIdentity;
  g.genbits = 1u << kGidIdentity;
  g.ef[0] = 1.0;
}

// group_mp (symmetry.f90:60-103): {identity, mirror of axis np (1..3)}.
void ga_mirror(int np, GroupAction g[2]) {
  ga_identity(g[0]);
  g[0].ef[1] = 1.0;
  std::memset(&g[1], 0, sizeof g[1]);
  g[1].j[0] = g[1].j[4] = g[1].j[8] = 1.0;
  g[1].j[4 * (np - 1)] = -1.0;
  g[1].detj = -1.0;
  g[1].ef[0] = 1.0;
  g[1].ef[1] = -1.0;
  g[1].id = np == 1 ? kGidMxp : np == 2 ? kGidMyp : kGidMzp;
  g[1].genbits = 1u << g[1].id;
}

// product_group (symmetry.f90:178-241); returns the order or -1.
int ga_product(GroupAction *a, int na, const GroupAction *b, int nb) {
  if (na * nb > kMaxGroup) return -1;
  std::vector<GroupAction> t(na * nb);
  for (int n = 0; n < na; n++)
    for (int m = 0; m < nb; m++) {
      GroupAction &g = t[n * nb + m];
      std::memset(&g, 0, sizeof g);
      for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
          double v = 0;
          for (int l = 0; l < 3; l++) v += a[n].j[3 * i + l] * b[m].j[3 * l + k];
          g.j[3 * i + k] = v;
        }
      g.detj = a[n].detj * b[m].detj;
      g.genbits = a[n].genbits | b[m].genbits;
      g.id = 0;
      if (a[n].id == kGidIdentity && b[m].id == kGidIdentity) g.id = kGidIdentity;
      else if (a[n].id != 0 && a[n].id != kGidIdentity && b[m].id == kGidIdentity) g.id = a[n].id;
      else if (b[m].id != 0 && b[m].id != kGidIdentity && a[n].id == kGidIdentity) g.id = b[m].id;
      for (int n2 = 0; n2 < na; n2++)
        for (int m2 = 0; m2 < nb; m2++) g.ef[n2 * nb + m2] = a[n].ef[n2] * b[m].ef[m2];
    }
  std::copy(t.begin(), t.end(), a);
  return na * nb;
}

int plane_bnd(int id) { return id == kGidMxp ? MOM_BND_XPLANE : id == kGidMyp ? MOM_BND_YPLANE : MOM_BND_ZPLANE; }

// Identity rows and columns of the removed unknowns of one representation
// (after assembly, before the factorisation).
__global__ void bc_identity_kernel(double2 *A, int64_t lda, int64_t n, const int *rm, int nrm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (k >= nrm || i >= n) return;
  const int64_t r = rm[k];
  A[r + i * lda] = make_double2(i == r ? 1.0 : 0.0, 0.0);  // row r
  A[i + r * lda] = make_double2(i == r ? 1.0 : 0.0, 0.0);  // column r
}

__global__ void zero_rows_kernel(double2 *B, int64_t ldb, int ncol, const int *rm, int nrm) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (k >= nrm || s >= ncol) return;
  B[(size_t)s * ldb + rm[k]] = make_double2(0.0, 0.0);
}

}  // namespace

// Matrix of representation r after assembly: the boundary conditions.
int apply_bc_matrix(Ctx *c, int r) {
  const int nrm = c->removed_off[r + 1] - c->removed_off[r];
  if (nrm == 0) return MOM_OK;
  const dim3 grid((unsigned)((c->n + 255) / 256), (unsigned)nrm);
  bc_identity_kernel<<<grid, 256, 0, c->stream>>>(c->A_all + (size_t)r * c->lda * c->n, c->lda, c->n,
                                                   c->removed_dev + c->removed_off[r], nrm);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

// Right-hand sides of representation r (ncol columns, ld n): zero at the
// removed unknowns.
int apply_bc_rhs(Ctx *c, int r, double2 *B, int ncol) {
  const int nrm = c->removed_off[r + 1] - c->removed_off[r];
  if (nrm == 0 || ncol == 0) return MOM_OK;
  zero_rows_kernel<<<dim3((unsigned)((nrm + 127) / 128), (unsigned)ncol), 128, 0, c->stream>>>(
      B, c->n, ncol, c->removed_dev + c->removed_off[r], nrm);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

// Allocates the per-representation matrices and factors for nga
// representations (A32 / inv32 again on the next mixed sysmat).
int alloc_representations(Ctx *c, int nga) {
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  for (auto *g : c->lu_graphs) {
    g->reset();
    delete g;
  }
  c->lu_graphs.clear();
  cudaFree(c->A_all);
  cudaFree(c->A32_all);
  cudaFree(c->ipiv_all);
  cudaFree(c->perm_all);
  cudaFree(c->invd_all);
  cudaFree(c->inv32_all);
  c->A_all = nullptr;
  c->A32_all = nullptr;
  c->ipiv_all = c->perm_all = nullptr;
  c->invd_all = nullptr;
  c->inv32_all = nullptr;
  c->A32_bytes = 0;
  const size_t mat = (size_t)c->lda * c->n;
  c->A_bytes = sizeof(double2) * mat * nga;
  if (cudaMalloc(&c->A_all, c->A_bytes) != cudaSuccess ||
      cudaMalloc(&c->ipiv_all, sizeof(int) * c->n * nga) != cudaSuccess ||
      cudaMalloc(&c->perm_all, sizeof(int) * c->n * nga) != cudaSuccess ||
      cudaMalloc(&c->invd_all, sizeof(double2) * 2 * (size_t)c->nb * c->n * nga) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, MOM_ERR_ALLOC, "device allocation for the system matrices failed");
  }
  select_rep(c, 0);
  c->assembled = 0;
  c->factored = -1;
  return MOM_OK;
}

}  // namespace mom

using namespace mom;
struct mom_ctx : public Ctx {};

extern "C" {

int mom_gpu_set_symmetry(mom_ctx *c, int32_t nnames, const char *const *names, const int32_t *edge_bnd) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem before the symmetry group");
  if (nnames < 0 || (nnames > 0 && !names) || !edge_bnd) return fail(c, MOM_ERR_ARG, "invalid symmetry arguments");
  MOM_CUDA(c, cudaSetDevice(c->device));
  GroupAction ga[kMaxGroup];
  ga_identity(ga[0]);
  int n = 1;
  for (int i = 0; i < nnames; i++) {
    const std::string nm = names[i] ? names[i] : "";
    GroupAction two[2];
    if (nm == "id") {
      ga_identity(two[0]);
      n = ga_product(ga, n, two, 1);
    } else if (nm == "mxp" || nm == "myp" || nm == "mzp") {
      ga_mirror(nm[1] - 'w', two);
      n = ga_product(ga, n, two, 2);
    } else {
      return fail(c, MOM_ERR_ARG, "symmetry group '" + nm + "' is not supported (id, mxp, myp, mzp)");
    }
    if (n < 0) return fail(c, MOM_ERR_ARG, "symmetry group larger than " + std::to_string(kMaxGroup) + " elements");
  }
  for (int e = 0; e < c->N; e++)
    if (edge_bnd[e] < MOM_BND_NONE || edge_bnd[e] > MOM_BND_ZPLANE)
      return fail(c, MOM_ERR_ARG, "edge boundary type out of range");
  // edge_bc per representation
  std::vector<std::vector<int>> removed(n);
  for (int r = 0; r < n; r++) {
    std::vector<char> rm(2 * (size_t)c->N, 0);
    for (int k = 0; k < c->N; k++)
      for (int a = 0; a < n; a++) {
        const GroupAction &g = ga[a];
        if (g.id < kGidMxp || g.id > kGidMzp || edge_bnd[k] != plane_bnd(g.id)) continue;
        const double gae = g.ef[r], gah = g.ef[r] * g.detj;
        if (-gae < 0.99) rm[k] = 1;
        if (-gah < 0.99) rm[k + c->N] = 1;
      }
    for (int k = 0; k < 2 * c->N; k++)
      if (rm[k]) removed[r].push_back(k);
  }
  // actions on each domain: admissibility and the mapped test geometry
  std::vector<char> has(c->ndom * 5, 0);
  for (int d = 0; d < c->ndom; d++)
    for (int e : c->dom[d].h_epar) has[d * 5 + edge_bnd[e]] = 1;
  c->nga = n;
  std::copy(ga, ga + n, c->ga);
  c->edge_bnd.assign(edge_bnd, edge_bnd + c->N);
  c->removed = removed;
  c->removed_off.assign(n + 1, 0);
  std::vector<int> flat;
  for (int r = 0; r < n; r++) {
    flat.insert(flat.end(), removed[r].begin(), removed[r].end());
    c->removed_off[r + 1] = (int)flat.size();
  }
  cudaFree(c->removed_dev);
  c->removed_dev = nullptr;
  MOM_CUDA(c, cudaMalloc(&c->removed_dev, sizeof(int) * std::max<size_t>(1, flat.size())));
  if (!flat.empty())
    MOM_CUDA(c, cudaMemcpy(c->removed_dev, flat.data(), sizeof(int) * flat.size(), cudaMemcpyHostToDevice));
  for (int d = 0; d < c->ndom; d++) {
    DomDev &D = c->dom[d];
    free_actions(D);
    D.act.assign(n, ActDev());
    for (int a = 0; a < n; a++) {
      const GroupAction &g = ga[a];
      bool ok = true;
      if (d > 0) {
        if ((g.genbits >> kGidMxp & 1u) && !has[d * 5 + MOM_BND_XPLANE]) ok = false;
        if ((g.genbits >> kGidMyp & 1u) && !has[d * 5 + MOM_BND_YPLANE]) ok = false;
        if ((g.genbits >> kGidMzp & 1u) && !has[d * 5 + MOM_BND_ZPLANE]) ok = false;
      }
      D.act[a].admissible = ok;
      if (ok && a > 0) MOM_TRY(action_precompute(c, d, a));
    }
  }
  MOM_TRY(alloc_representations(c, n));
  return MOM_OK;
}

int32_t mom_gpu_group_order(mom_ctx *c) { return (c && c->have_problem) ? c->nga : -1; }

}  // extern "C"
