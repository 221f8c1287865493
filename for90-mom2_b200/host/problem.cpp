// Host-side problem set-up: the reference's mesh / ndom / sdom / fdom
// commands (interface.f90:32-123, 357-366) producing the flattened domain
// submeshes that mom_gpu_set_problem consumes.
//
// The topology must match the reference exactly, because the matrix and
// solution are indexed by it:
//   build_mesh (mesh.f90:1044-1137): unique edges in face order, local edge k
//     of a face = (node k, node k+1), the first face that meets an edge is
//     its "+" face with free vertex node k+2; a later face overwrites the
//     "-" slot.  The reference scans all edges found so far; a hash map keyed
//     by the unordered node pair gives the same numbering in O(F).
//   extract_submesh (mesh.f90:290-376), invert_faces (278-288),
//   submesh_edge_connectivity (378-452), orient_basis (454-558).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/mom_gpu.h"

namespace {

struct Mesh {
  int nnodes = 0, nfaces = 0, nedges = 0;
  std::vector<double> node;       // [nnodes][3]
  std::vector<int> node_parent;   // [nnodes]
  std::vector<int> face_node;     // [nfaces][3]
  std::vector<int> face_edge;     // [nfaces][3]
  std::vector<int> face_id;       // [nfaces]
  std::vector<int> face_parent;   // [nfaces]
  std::vector<int> edge_node;     // [nedges][2]
  std::vector<int> edge_face;     // [nedges][2]
  std::vector<int> edge_bnode;    // [nedges][2]
  std::vector<int> edge_parent;   // [nedges]
  std::vector<std::vector<std::pair<int, int>>> child;  // master only: (submesh, local edge)
};

inline uint64_t pair_key(int a, int b) {
  const uint32_t lo = (uint32_t)std::min(a, b), hi = (uint32_t)std::max(a, b);
  return ((uint64_t)hi << 32) | lo;
}

// build_mesh without the geometry part (the device library derives it).
void build_edges(Mesh &m, double scale) {
  for (auto &v : m.node) v = v * scale;
  m.face_edge.assign(3 * (size_t)m.nfaces, -1);
  m.edge_node.clear();
  m.edge_face.clear();
  m.edge_bnode.clear();
  std::unordered_map<uint64_t, int> seen;
  seen.reserve(3 * (size_t)m.nfaces);
  for (int n = 0; n < m.nfaces; n++) {
    for (int k = 0; k < 3; k++) {
      const int a = m.face_node[3 * n + k], b = m.face_node[3 * n + (k + 1) % 3];
      const int opp = m.face_node[3 * n + (k + 2) % 3];
      auto it = seen.find(pair_key(a, b));
      if (it != seen.end()) {
        const int l = it->second;
        m.edge_face[2 * l + 1] = n;
        m.edge_bnode[2 * l + 1] = opp;
        m.face_edge[3 * n + k] = l;
      } else {
        const int l = (int)(m.edge_node.size() / 2);
        seen.emplace(pair_key(a, b), l);
        m.edge_node.push_back(a);
        m.edge_node.push_back(b);
        m.edge_face.push_back(n);
        m.edge_face.push_back(-1);
        m.edge_bnode.push_back(opp);
        m.edge_bnode.push_back(-1);
        m.face_edge[3 * n + k] = l;
      }
    }
  }
  m.nedges = (int)(m.edge_node.size() / 2);
  m.edge_parent.assign(m.nedges, -1);
}

Mesh extract_submesh(const Mesh &ms, const std::vector<int> &ids) {
  Mesh s;
  std::vector<char> nmask(ms.nnodes, 0);
  auto hit = [&](int id) { return std::find(ids.begin(), ids.end(), id) != ids.end(); };
  for (int n = 0; n < ms.nfaces; n++)
    if (hit(ms.face_id[n]))
      for (int k = 0; k < 3; k++) nmask[ms.face_node[3 * n + k]] = 1;
  std::vector<int> loc(ms.nnodes, -1);
  for (int n = 0; n < ms.nnodes; n++)
    if (nmask[n]) {
      loc[n] = s.nnodes++;
      for (int i = 0; i < 3; i++) s.node.push_back(ms.node[3 * n + i]);
      s.node_parent.push_back(n);
    }
  for (int n = 0; n < ms.nfaces; n++)
    if (hit(ms.face_id[n])) {
      for (int k = 0; k < 3; k++) s.face_node.push_back(loc[ms.face_node[3 * n + k]]);
      s.face_parent.push_back(n);
      s.face_id.push_back(ms.face_id[n]);
      s.nfaces++;
    }
  return s;
}

void invert_faces(Mesh &m, int id) {
  for (int n = 0; n < m.nfaces; n++)
    if (m.face_id[n] == id) std::swap(m.face_node[3 * n], m.face_node[3 * n + 2]);
}

}  // namespace

struct mom_problem {
  Mesh master;
  bool have_mesh = false;
  std::vector<int> line_node;  // [nlines][2] line elements of the mesh file (master node indices)
  std::vector<int> line_id;    // [nlines] their physical ids
  std::vector<int> edge_bnd;   // [master nedges] boundary type (classify_edges), MOM_BND_NONE by default
  std::vector<Mesh> dom;
  std::vector<char> dom_set;
  bool finalized = false;
};

extern "C" {

int mom_problem_create(mom_problem **out) {
  if (!out) return MOM_ERR_ARG;
  *out = new (std::nothrow) mom_problem();
  return *out ? MOM_OK : MOM_ERR_ALLOC;
}

void mom_problem_destroy(mom_problem *p) { delete p; }

int mom_problem_set_mesh(mom_problem *p, int32_t nnodes, const double *nodes, int32_t nfaces, const int32_t *faces,
                         const int32_t *face_ids, double scale) {
  if (!p || nnodes <= 0 || nfaces <= 0 || !nodes || !faces || !face_ids) return MOM_ERR_ARG;
  for (int i = 0; i < 3 * nfaces; i++)
    if (faces[i] < 0 || faces[i] >= nnodes) return MOM_ERR_MESH;
  Mesh m;
  m.nnodes = nnodes;
  m.nfaces = nfaces;
  m.node.assign(nodes, nodes + 3 * (size_t)nnodes);
  m.face_node.assign(faces, faces + 3 * (size_t)nfaces);
  m.face_id.assign(face_ids, face_ids + nfaces);
  m.node_parent.resize(nnodes);
  m.face_parent.resize(nfaces);
  for (int i = 0; i < nnodes; i++) m.node_parent[i] = i;
  for (int i = 0; i < nfaces; i++) m.face_parent[i] = i;
  build_edges(m, scale);
  p->master = std::move(m);
  p->have_mesh = true;
  p->line_node.clear();
  p->line_id.clear();
  p->edge_bnd.assign(p->master.nedges, MOM_BND_NONE);
  p->dom.clear();
  p->dom_set.clear();
  p->finalized = false;
  return MOM_OK;
}

// load_mesh_gmsh (mesh.f90:610-736): Gmsh 2.1 / 2.2 ASCII, triangles (type 2)
// with the first tag as the physical id; other elements are skipped.
int mom_problem_load_gmsh(mom_problem *p, const char *path, double scale) {
  if (!p || !path) return MOM_ERR_ARG;
  std::ifstream in(path);
  if (!in) return MOM_ERR_IO;
  std::string tok;
  std::vector<double> nodes;
  std::vector<int> faces, ids, lines, line_ids;
  int nn = 0;
  bool have_nodes = false, have_elems = false;
  while (in >> tok) {
    if (tok == "$MeshFormat") {
      std::string ver;
      in >> ver;
      if (ver.compare(0, 3, "2.1") != 0 && ver.compare(0, 3, "2.2") != 0) return MOM_ERR_IO;  // unsupported version
      std::string line;
      std::getline(in, line);
      in >> tok;
      if (tok != "$EndMeshFormat") return MOM_ERR_IO;
    } else if (tok == "$Nodes") {
      in >> nn;
      if (!in || nn <= 0) return MOM_ERR_IO;
      nodes.assign(3 * (size_t)nn, 0.0);
      for (int i = 0; i < nn; i++) {
        long num;
        double x, y, z;
        in >> num >> x >> y >> z;
        if (!in || num < 1 || num > nn) return MOM_ERR_IO;
        nodes[3 * (num - 1)] = x;
        nodes[3 * (num - 1) + 1] = y;
        nodes[3 * (num - 1) + 2] = z;
      }
      in >> tok;
      if (tok != "$EndNodes") return MOM_ERR_IO;
      have_nodes = true;
    } else if (tok == "$Elements") {
      int ne = 0;
      in >> ne;
      if (!in || ne < 0) return MOM_ERR_IO;
      std::string line;
      std::getline(in, line);
      for (int i = 0; i < ne; i++) {
        if (!std::getline(in, line)) return MOM_ERR_IO;
        std::istringstream ls(line);
        long num;
        int type, ntags;
        ls >> num >> type >> ntags;
        if (!ls) return MOM_ERR_IO;
        std::vector<long> tags(ntags);
        for (int t = 0; t < ntags; t++) ls >> tags[t];
        if (type == 2) {
          long a, b, c;
          ls >> a >> b >> c;
          if (!ls || ntags < 1) return MOM_ERR_IO;
          faces.push_back((int)a - 1);
          faces.push_back((int)b - 1);
          faces.push_back((int)c - 1);
          ids.push_back((int)tags[0]);
        } else if (type == 1) {
          // line elements: boundary curves that sbnd classifies (mesh.f90:680-684)
          long a, b;
          ls >> a >> b;
          if (!ls || ntags < 1) return MOM_ERR_IO;
          lines.push_back((int)a - 1);
          lines.push_back((int)b - 1);
          line_ids.push_back((int)tags[0]);
        }
      }
      in >> tok;
      if (tok != "$EndElements") return MOM_ERR_IO;
      have_elems = true;
    }
  }
  if (!have_nodes || !have_elems || ids.empty()) return MOM_ERR_IO;
  for (int v : lines)
    if (v < 0 || v >= nn) return MOM_ERR_IO;
  const int rc = mom_problem_set_mesh(p, nn, nodes.data(), (int32_t)ids.size(), faces.data(), ids.data(), scale);
  if (rc != MOM_OK) return rc;
  p->line_node = lines;
  p->line_id = line_ids;
  return MOM_OK;
}

int mom_problem_set_lines(mom_problem *p, int32_t nlines, const int32_t *line_nodes, const int32_t *line_ids) {
  if (!p || !p->have_mesh) return MOM_ERR_STATE;
  if (nlines < 0 || (nlines > 0 && (!line_nodes || !line_ids))) return MOM_ERR_ARG;
  for (int i = 0; i < 2 * nlines; i++)
    if (line_nodes[i] < 0 || line_nodes[i] >= p->master.nnodes) return MOM_ERR_MESH;
  p->line_node.assign(line_nodes, line_nodes + 2 * (size_t)nlines);
  p->line_id.assign(line_ids, line_ids + nlines);
  return MOM_OK;
}

// classify_edges (mesh.f90:155-175): every master edge whose end nodes are
// those of a line element with physical id `id` gets boundary type bnd.
int mom_problem_classify_edges(mom_problem *p, int32_t id, int32_t bnd, int32_t *nclassified) {
  if (!p || !p->have_mesh) return MOM_ERR_STATE;
  if (bnd < MOM_BND_NONE || bnd > MOM_BND_ZPLANE) return MOM_ERR_ARG;
  const Mesh &ms = p->master;
  std::unordered_map<uint64_t, std::vector<int>> byedge;
  for (size_t l = 0; l < p->line_id.size(); l++)
    if (p->line_id[l] == id) byedge[pair_key(p->line_node[2 * l], p->line_node[2 * l + 1])].push_back((int)l);
  int cnt = 0;
  for (int e = 0; e < ms.nedges; e++) {
    auto it = byedge.find(pair_key(ms.edge_node[2 * e], ms.edge_node[2 * e + 1]));
    if (it == byedge.end()) continue;
    p->edge_bnd[e] = bnd;
    cnt += (int)it->second.size();  // the reference counts every matching line
  }
  if (nclassified) *nclassified = cnt;
  return MOM_OK;
}

int mom_problem_edge_bnd(const mom_problem *p, int32_t *bnd) {
  if (!p || !bnd) return MOM_ERR_ARG;
  if (!p->have_mesh) return MOM_ERR_STATE;
  std::copy(p->edge_bnd.begin(), p->edge_bnd.end(), bnd);
  return MOM_OK;
}

int mom_problem_set_ndom(mom_problem *p, int32_t ndom) {
  if (!p || ndom <= 0) return MOM_ERR_ARG;
  p->dom.assign(ndom, Mesh());
  p->dom_set.assign(ndom, 0);
  p->finalized = false;
  return MOM_OK;
}

int mom_problem_set_domain(mom_problem *p, int32_t dom, int32_t nsurf, const int32_t *surf_ids) {
  if (!p || !p->have_mesh) return MOM_ERR_STATE;
  if (dom < 0 || dom >= (int)p->dom.size() || nsurf <= 0 || !surf_ids) return MOM_ERR_ARG;
  std::vector<int> absid(nsurf);
  for (int i = 0; i < nsurf; i++) {
    if (surf_ids[i] == 0) return MOM_ERR_ARG;  // "Zero is not a valid surface id!" (interface.f90:80-83)
    absid[i] = std::abs(surf_ids[i]);
  }
  Mesh s = extract_submesh(p->master, absid);
  if (s.nfaces == 0) return MOM_ERR_MESH;
  for (int i = 0; i < nsurf; i++)
    if (surf_ids[i] < 0) invert_faces(s, -surf_ids[i]);
  build_edges(s, 1.0);
  p->dom[dom] = std::move(s);
  p->dom_set[dom] = 1;
  p->finalized = false;
  return MOM_OK;
}

int mom_problem_finalize(mom_problem *p) {
  if (!p || !p->have_mesh || p->dom.empty()) return MOM_ERR_STATE;
  for (char s : p->dom_set)
    if (!s) return MOM_ERR_STATE;
  Mesh &ms = p->master;
  const int nsub = (int)p->dom.size();
  // submesh_edge_connectivity: children ordered by submesh, then local edge.
  std::unordered_map<uint64_t, int> medge;
  medge.reserve(ms.nedges);
  for (int e = 0; e < ms.nedges; e++) medge.emplace(pair_key(ms.edge_node[2 * e], ms.edge_node[2 * e + 1]), e);
  ms.child.assign(ms.nedges, {});
  for (int s = 0; s < nsub; s++) {
    Mesh &sm = p->dom[s];
    for (int l = 0; l < sm.nedges; l++) {
      const int a = sm.node_parent[sm.edge_node[2 * l]], b = sm.node_parent[sm.edge_node[2 * l + 1]];
      auto it = medge.find(pair_key(a, b));
      if (it == medge.end()) return MOM_ERR_MESH;
      sm.edge_parent[l] = it->second;
      ms.child[it->second].push_back({s, l});
    }
  }
  for (int e = 0; e < ms.nedges; e++)
    if (ms.child[e].size() < 2) return MOM_ERR_MESH;  // "Submesh decomposition is inconsistent"
  // orient_basis (non-periodic part)
  for (int n = 0; n < ms.nedges; n++) {
    const auto &ch = ms.child[n];
    const int nchild = (int)ch.size();
    std::vector<char> oriented(nchild, 0);
    oriented[0] = 1;
    for (int it = 0; it < nchild; it++) {
      for (int l = 1; l < nchild; l++) {
        if (oriented[l]) continue;
        for (int k = 0; k < nchild; k++) {
          if (!oriented[k]) continue;
          Mesh &sl = p->dom[ch[l].first], &sk = p->dom[ch[k].first];
          const int el = ch[l].second, ek = ch[k].second;
          int pf1 = sl.edge_face[2 * el], nf1 = sl.edge_face[2 * el + 1];
          int pf2 = sk.edge_face[2 * ek], nf2 = sk.edge_face[2 * ek + 1];
          if (pf1 != -1) pf1 = sl.face_parent[pf1];
          if (nf1 != -1) nf1 = sl.face_parent[nf1];
          if (pf2 != -1) pf2 = sk.face_parent[pf2];
          if (nf2 != -1) nf2 = sk.face_parent[nf2];
          if (pf1 == pf2 || nf1 == nf2) {
            std::swap(sl.edge_face[2 * el], sl.edge_face[2 * el + 1]);
            std::swap(sl.edge_bnode[2 * el], sl.edge_bnode[2 * el + 1]);
          }
          if (pf1 == pf2 || nf1 == nf2 || pf1 == nf2 || nf1 == pf2) {
            oriented[l] = 1;
            break;
          }
        }
      }
      if (std::count(oriented.begin(), oriented.end(), 1) == nchild) break;
    }
  }
  p->finalized = true;
  return MOM_OK;
}

int32_t mom_problem_nedges(const mom_problem *p) { return (p && p->have_mesh) ? p->master.nedges : -1; }
int32_t mom_problem_ndom(const mom_problem *p) { return p ? (int32_t)p->dom.size() : -1; }

int mom_problem_domain(const mom_problem *p, int32_t dom, mom_mesh *out) {
  if (!p || !out) return MOM_ERR_ARG;
  if (dom == -1 ? !p->have_mesh : !p->finalized) return MOM_ERR_STATE;
  if (dom < -1 || dom >= (int)p->dom.size()) return MOM_ERR_ARG;
  const Mesh &m = dom < 0 ? p->master : p->dom[dom];
  out->nnodes = m.nnodes;
  out->nfaces = m.nfaces;
  out->nedges = m.nedges;
  out->nodes = m.node.data();
  out->face_nodes = m.face_node.data();
  out->face_edges = m.face_edge.data();
  out->edge_nodes = m.edge_node.data();
  out->edge_faces = m.edge_face.data();
  out->edge_bnodes = m.edge_bnode.data();
  out->edge_parent = m.edge_parent.data();
  return MOM_OK;
}

int mom_problem_node_parent(const mom_problem *p, int32_t dom, int32_t *parent) {
  if (!p || !parent) return MOM_ERR_ARG;
  if (!p->finalized) return MOM_ERR_STATE;
  if (dom < 0 || dom >= (int)p->dom.size()) return MOM_ERR_ARG;
  const Mesh &m = p->dom[dom];
  for (int i = 0; i < m.nnodes; i++) parent[i] = m.node_parent[i];
  return MOM_OK;
}

// Triangle rules of quad.f90 (tri_quad_data, quad.f90:277-315).  tri_gl13
// (quad.f90:115-171) and the tri_gl3 nodes (102-113) are default-real
// literals in the reference, i.e. rounded to single precision; the others
// carry the _dp suffix.
int32_t mom_tri_rule(const char *name, double *qw, double *qn) {
  if (!name || !qw || !qn) return -1;
  std::string s(name);
  std::vector<double> w;
  std::vector<double> f;  // [k][i] barycentric factor k of point i
  if (s == "tri_gl13") {
    static const float w13[13] = {-0.149570044467670f, 0.175615257433204f, 0.175615257433204f,
                                  0.175615257433204f,  0.053347235608839f, 0.053347235608839f,
                                  0.053347235608839f,  0.077113760890257f, 0.077113760890257f,
                                  0.077113760890257f,  0.077113760890257f, 0.077113760890257f,
                                  0.077113760890257f};
    static const float a = 0.333333333333333f, b = 0.479308067841923f, c = 0.260345966079038f,
                       d = 0.869739794195568f, e = 0.065130102902216f, g = 0.638444188569809f,
                       h = 0.312865496004875f, k = 0.048690315425316f;
    static const float f13[3][13] = {{a, b, c, c, d, e, e, g, g, h, h, k, k},
                                     {a, c, c, b, e, e, d, k, h, k, g, h, g},
                                     {a, c, b, c, e, d, e, h, k, g, k, g, h}};
    for (int i = 0; i < 13; i++) w.push_back((double)w13[i]);
    for (int kk = 0; kk < 3; kk++)
      for (int i = 0; i < 13; i++) f.push_back((double)f13[kk][i]);
  } else if (s == "tri_gl1") {
    w = {1.0};
    f = {0.333333333333333, 0.333333333333333, 0.333333333333333};
  } else if (s == "tri_gl3") {
    const double big = (double)0.666666666666667f, sml = (double)0.166666666666667f;
    w = {0.333333333333333, 0.333333333333333, 0.333333333333333};
    f = {big, sml, sml, sml, big, sml, sml, sml, big};
  } else if (s == "tri_gl4") {
    w = {-0.56250000, 0.52083333, 0.52083333, 0.52083333};
    f = {1.0 / 3.0, 0.6, 0.2, 0.2, 1.0 / 3.0, 0.2, 0.6, 0.2, 1.0 / 3.0, 0.2, 0.2, 0.6};
  } else if (s == "tri_gl7") {
    w = {0.22500000, 0.13239415, 0.13239415, 0.13239415, 0.12593918, 0.12593918, 0.12593918};
    f = {0.33333333, 0.05971587, 0.47014206, 0.47014206, 0.79742698, 0.10128650, 0.10128650,
         0.33333333, 0.47014206, 0.05971587, 0.47014206, 0.10128650, 0.79742698, 0.10128650,
         0.33333333, 0.47014206, 0.47014206, 0.05971587, 0.10128650, 0.10128650, 0.79742698};
  } else {
    return -1;  // "Unrecognized quadrature type" (quad.f90:312-313)
  }
  const int nq = (int)w.size();
  for (int i = 0; i < nq; i++) {
    qw[i] = w[i];
    for (int kk = 0; kk < 3; kk++) qn[3 * i + kk] = f[(size_t)kk * nq + i];
  }
  return nq;
}

int mom_problem_upload(const mom_problem *p, mom_ctx *ctx, const char *quad_name) {
  if (!p || !ctx) return MOM_ERR_ARG;
  if (!p->finalized) return MOM_ERR_STATE;
  double qw[13], qn[39];
  const int nq = mom_tri_rule(quad_name ? quad_name : "tri_gl13", qw, qn);
  if (nq < 0) return MOM_ERR_ARG;
  std::vector<mom_mesh> doms(p->dom.size());
  for (size_t d = 0; d < p->dom.size(); d++) mom_problem_domain(p, (int32_t)d, &doms[d]);
  return mom_gpu_set_problem(ctx, p->master.nedges, (int32_t)doms.size(), doms.data(), nq, qw, qn);
}

}  // extern "C"
