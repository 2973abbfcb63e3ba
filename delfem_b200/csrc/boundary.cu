// Boundary facets of a GiD volume mesh, derived as the reference's readers
// derive them after reading the elements (host only):
//
//  * tetrahedra (Msh::CMesh3D::ReadFromFile_GiDMsh, src/msh/mesh3d.cpp:
//    744-778): the faces no other tetrahedron shares with the opposite
//    orientation (Msh::MakeTetSurTet, src/msh/meshkernel3d.cpp:102-230, and
//    Msh::MakeOuterBoundTet, :514-539), in (tetrahedron, face) order with the
//    nodes counter-clockwise seen from outside; their edge neighbours
//    (Msh::MakeTriSurTri, :306-395); and colours, flat patches grown across
//    edges whose unit normals have a dot product above crt_dot
//    (Msh::MakeColorCoding_Tri3D, :905-947; the reader passes 0.2).
//  * triangles and quadrilaterals (Msh::CMesher2D::ReadFromFile_GiDMsh,
//    src/msh/mesher2d.cpp:2581-2760): the edges no other element shares
//    (Msh::MakeInnerRelationTri / Quad + MakeOuterBoundTri / Quad,
//    src/msh/meshkernel2d.cpp:1161-1323), split into chains of bars whose
//    successive unit directions have a dot product above crt_dot
//    (Msh::ColorCodeBarAry, :1941-2018; 0.8 there), and the chains' end
//    nodes as vertices, ascending.
//  * hexahedra: none (the reference's hexahedral boundary is commented out,
//    src/msh/mesh3d.cpp:724-727).
//
// The reference finds neighbours by scanning the elements around a node; here
// facets are grouped by their sorted node tuple and each group is resolved by
// the reference's rule (first partner in ascending element order, pairs
// linked both ways, later links overwriting earlier ones), which gives the
// same links on any mesh, manifold or not.  A colour is the set of facets
// reachable from its seed (the lowest uncoloured facet) over the neighbour
// links that pass the normal test, so it does not depend on the search
// order.  Elements with a repeated node are rejected.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <vector>

#include "dfm_internal.h"

namespace dfm {
namespace {

// Local node numbering conventions of the reference's element types
// (include/delfem/msh/meshkernel3d.h:52-57, include/delfem/msh/meshkernel2d.h:55-74):
// face f of a tetrahedron is opposite node f, counter-clockwise from outside.
constexpr int kTetFace[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
constexpr int kTriEdge[3][2] = {{1, 2}, {2, 0}, {0, 1}};
constexpr int kQuadEdge[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};

struct Key3 {
  unsigned a, b, c, id;  // sorted nodes, facet id = element * nface + local facet
};
struct Key2 {
  unsigned a, b, id;
};

// parity of a permutation of 0..3 (true = odd)
bool odd4(const int p[4]) {
  int inv = 0;
  for (int i = 0; i < 4; i++)
    for (int j = i + 1; j < 4; j++) inv += p[i] > p[j];
  return inv & 1;
}

// Which faces of the tetrahedra have a partner (MakeTetSurTet's g == -2).
// Two faces with the same nodes are partners when the tetrahedra meet with
// opposite orientation (the map of the second's local nodes onto the first's,
// apex onto apex, is odd); a same-orientation pair is the reference's
// "inverse element" and stays unlinked.
std::vector<char> tet_face_linked(unsigned ntet, const int* tet) {
  std::vector<Key3> k((size_t)ntet * 4);
  for (unsigned t = 0; t < ntet; t++)
    for (int f = 0; f < 4; f++) {
      unsigned n[3];
      for (int q = 0; q < 3; q++) n[q] = (unsigned)tet[4 * (size_t)t + kTetFace[f][q]];
      std::sort(n, n + 3);
      k[4 * (size_t)t + f] = {n[0], n[1], n[2], 4 * t + (unsigned)f};
    }
  std::sort(k.begin(), k.end(), [](const Key3& x, const Key3& y) {
    if (x.a != y.a) return x.a < y.a;
    if (x.b != y.b) return x.b < y.b;
    if (x.c != y.c) return x.c < y.c;
    return x.id < y.id;
  });
  std::vector<char> linked((size_t)ntet * 4, 0);
  // partners: the map of tet j's local nodes onto tet i's (face nodes onto
  // the same node, apex onto apex) must be odd
  auto partners = [&](unsigned fi, unsigned fj) {
    const unsigned ti = fi / 4, tj = fj / 4;
    const int ai = (int)(fi % 4);
    int p[4];
    for (int jl = 0; jl < 4; jl++) {
      const int g = tet[4 * (size_t)tj + jl];
      p[jl] = ai;
      for (int il = 0; il < 4; il++)
        if (il != ai && tet[4 * (size_t)ti + il] == g) p[jl] = il;
    }
    return odd4(p);
  };
  for (size_t s = 0; s < k.size();) {
    size_t e = s + 1;
    while (e < k.size() && k[e].a == k[s].a && k[e].b == k[s].b && k[e].c == k[s].c) e++;
    // members are in (tetrahedron, face) order; each looks for the first
    // partner in ascending tetrahedron order, skipping its own tetrahedron
    for (size_t m = s; m < e && e - s > 1; m++) {
      if (linked[k[m].id]) continue;
      for (size_t c = s; c < e; c++) {
        if (k[c].id / 4 == k[m].id / 4) continue;
        if (partners(k[m].id, k[c].id)) {
          linked[k[m].id] = linked[k[c].id] = 1;
          break;
        }
      }
    }
    s = e;
  }
  return linked;
}

// Edge neighbours of triangles (MakeTriSurTri's s2; -1 where none): members
// of an edge group, in (triangle, edge) order, each unlinked one taking the
// first other triangle of the group and linking both ways.
std::vector<long long> tri_edge_links(size_t ntri, const unsigned* tri) {
  std::vector<Key2> k(ntri * 3);
  for (size_t t = 0; t < ntri; t++)
    for (int d = 0; d < 3; d++) {
      unsigned a = tri[3 * t + kTriEdge[d][0]], b = tri[3 * t + kTriEdge[d][1]];
      if (a > b) std::swap(a, b);
      k[3 * t + d] = {a, b, (unsigned)(3 * t + d)};
    }
  std::sort(k.begin(), k.end(), [](const Key2& x, const Key2& y) {
    if (x.a != y.a) return x.a < y.a;
    if (x.b != y.b) return x.b < y.b;
    return x.id < y.id;
  });
  std::vector<long long> s2(ntri * 3, -1);
  std::vector<char> g2(ntri * 3, 0);
  for (size_t s = 0; s < k.size();) {
    size_t e = s + 1;
    while (e < k.size() && k[e].a == k[s].a && k[e].b == k[s].b) e++;
    for (size_t m = s; m < e && e - s > 1; m++) {
      const unsigned im = k[m].id;
      if (g2[im]) continue;
      for (size_t c = s; c < e; c++) {
        const unsigned ic = k[c].id;
        if (ic / 3 == im / 3) continue;
        s2[im] = ic / 3;
        s2[ic] = im / 3;
        g2[im] = g2[ic] = 1;
        break;
      }
    }
    s = e;
  }
  return s2;
}

// unit normal of triangle (p1, p2, p3) in the reference's operation order
// (Com::UnitNormal, include/delfem/vector3d.h:725-738)
void unit_normal(const double* p1, const double* p2, const double* p3, double n[3]) {
  n[0] = (p2[1] - p1[1]) * (p3[2] - p1[2]) - (p2[2] - p1[2]) * (p3[1] - p1[1]);
  n[1] = (p2[2] - p1[2]) * (p3[0] - p1[0]) - (p2[0] - p1[0]) * (p3[2] - p1[2]);
  n[2] = (p2[0] - p1[0]) * (p3[1] - p1[1]) - (p2[1] - p1[1]) * (p3[0] - p1[0]);
  const double r = 1.0 / std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  n[0] *= r;
  n[1] *= r;
  n[2] *= r;
}

struct Result {
  int nnofa = 0;
  std::vector<unsigned> facet;      // nfacet * nnofa
  std::vector<unsigned> group_ptr;  // ngroup + 1
  std::vector<unsigned> group_facet;
  std::vector<unsigned> vertex;
  std::vector<unsigned> group_ends;  // 2 per group (2-D)
};

void tet_boundary(const double* coord, unsigned ntet, const int* tet, double crt, Result& R) {
  R.nnofa = 3;
  const std::vector<char> linked = tet_face_linked(ntet, tet);
  for (unsigned t = 0; t < ntet; t++)
    for (int f = 0; f < 4; f++)
      if (!linked[4 * (size_t)t + f])
        for (int q = 0; q < 3; q++) R.facet.push_back((unsigned)tet[4 * (size_t)t + kTetFace[f][q]]);
  const size_t ntri = R.facet.size() / 3;
  const std::vector<long long> s2 = tri_edge_links(ntri, R.facet.data());
  std::vector<double> nrm(ntri * 3);
  for (size_t t = 0; t < ntri; t++)
    unit_normal(coord + 3 * (size_t)R.facet[3 * t], coord + 3 * (size_t)R.facet[3 * t + 1],
                coord + 3 * (size_t)R.facet[3 * t + 2], &nrm[3 * t]);
  std::vector<long long> color(ntri, -1);
  std::vector<size_t> stack;
  long long ncolor = 0;
  for (size_t seed = 0; seed < ntri; seed++) {
    if (color[seed] != -1) continue;
    color[seed] = ncolor;
    stack.assign(1, seed);
    while (!stack.empty()) {
      const size_t cur = stack.back();
      stack.pop_back();
      for (int d = 0; d < 3; d++) {
        const long long nb = s2[3 * cur + d];
        if (nb < 0 || color[nb] != -1) continue;
        const double* a = &nrm[3 * cur];
        const double* b = &nrm[3 * (size_t)nb];
        if (a[0] * b[0] + a[1] * b[1] + a[2] * b[2] > crt) {
          color[nb] = ncolor;
          stack.push_back((size_t)nb);
        }
      }
    }
    ncolor++;
  }
  // a colour's triangles in boundary order
  R.group_ptr.assign((size_t)ncolor + 1, 0);
  for (size_t t = 0; t < ntri; t++) R.group_ptr[color[t] + 1]++;
  for (long long c = 0; c < ncolor; c++) R.group_ptr[c + 1] += R.group_ptr[c];
  R.group_facet.resize(ntri);
  std::vector<unsigned> fill(R.group_ptr.begin(), R.group_ptr.end() - 1);
  for (size_t t = 0; t < ntri; t++) R.group_facet[fill[color[t]]++] = (unsigned)t;
}

void planar_boundary(unsigned nnode, const double* coord, int nnoel, unsigned nelem, const int* elem, double crt,
                     Result& R) {
  R.nnofa = 2;
  const int ned = nnoel;  // edges per element: 3 or 4
  std::vector<Key2> k((size_t)nelem * ned);
  for (unsigned t = 0; t < nelem; t++)
    for (int d = 0; d < ned; d++) {
      const int* ed = nnoel == 3 ? kTriEdge[d] : kQuadEdge[d];
      unsigned a = (unsigned)elem[(size_t)nnoel * t + ed[0]], b = (unsigned)elem[(size_t)nnoel * t + ed[1]];
      if (a > b) std::swap(a, b);
      k[(size_t)ned * t + d] = {a, b, (unsigned)((size_t)ned * t + d)};
    }
  std::sort(k.begin(), k.end(), [](const Key2& x, const Key2& y) {
    if (x.a != y.a) return x.a < y.a;
    if (x.b != y.b) return x.b < y.b;
    return x.id < y.id;
  });
  // an edge is outer when no other element has the same two nodes
  std::vector<char> inner((size_t)nelem * ned, 0);
  for (size_t s = 0; s < k.size();) {
    size_t e = s + 1;
    while (e < k.size() && k[e].a == k[s].a && k[e].b == k[s].b) e++;
    if (e - s > 1)
      for (size_t m = s; m < e; m++) inner[k[m].id] = 1;
    s = e;
  }
  for (unsigned t = 0; t < nelem; t++)
    for (int d = 0; d < ned; d++) {
      if (inner[(size_t)ned * t + d]) continue;
      const int* ed = nnoel == 3 ? kTriEdge[d] : kQuadEdge[d];
      R.facet.push_back((unsigned)elem[(size_t)nnoel * t + ed[0]]);
      R.facet.push_back((unsigned)elem[(size_t)nnoel * t + ed[1]]);
    }
  const std::vector<unsigned>& bar = R.facet;
  const size_t nbar = bar.size() / 2;
  // bars around each node, ascending; nodes with exactly two join them:
  // link[2*i + k] is the bar across node v[1-k] of bar i
  std::vector<unsigned> ptr((size_t)nnode + 1, 0), around(nbar * 2);
  for (size_t i = 0; i < nbar * 2; i++) ptr[bar[i] + 1]++;
  for (unsigned v = 0; v < nnode; v++) ptr[v + 1] += ptr[v];
  {
    std::vector<unsigned> f(ptr.begin(), ptr.end() - 1);
    for (size_t i = 0; i < nbar * 2; i++) around[f[bar[i]]++] = (unsigned)(i / 2);
  }
  std::vector<long long> link(nbar * 2, -1);
  for (unsigned v = 0; v < nnode; v++) {
    if (ptr[v + 1] - ptr[v] != 2) continue;
    const unsigned e0 = around[ptr[v]], e1 = around[ptr[v] + 1];
    const int k0 = bar[2 * (size_t)e0] == v ? 0 : 1, k1 = bar[2 * (size_t)e1] == v ? 0 : 1;
    link[2 * (size_t)e0 + (1 - k0)] = e1;
    link[2 * (size_t)e1 + (1 - k1)] = e0;
  }
  auto x = [&](unsigned n) { return coord[2 * (size_t)n]; };
  auto y = [&](unsigned n) { return coord[2 * (size_t)n + 1]; };
  std::vector<long long> color(nbar, -1);
  long long nchain = 0;
  R.group_ptr.assign(1, 0);
  for (size_t seed = 0; seed < nbar; seed++) {
    if (color[seed] != -1) continue;
    color[seed] = nchain;
    std::deque<unsigned> chain(1, (unsigned)seed);
    for (int dir = 0; dir < 2; dir++) {  // forward (across v[1]), then backward (across v[0])
      int k0 = dir;
      size_t b0 = seed;
      for (;;) {
        const long long nb = link[2 * b0 + k0];
        if (nb < 0 || color[nb] != -1) break;
        const unsigned b1 = (unsigned)nb;
        const unsigned iv0 = bar[2 * b0 + k0], iv1 = bar[2 * b0 + 1 - k0];
        const int k1 = bar[2 * (size_t)b1] == iv1 ? 1 : 0;  // b1's far end
        const unsigned iv2 = bar[2 * (size_t)b1 + k1];
        double ux = x(iv1) - x(iv0), uy = y(iv1) - y(iv0);
        double wx = x(iv2) - x(iv1), wy = y(iv2) - y(iv1);
        const double lu = std::sqrt(ux * ux + uy * uy), lw = std::sqrt(wx * wx + wy * wy);
        ux /= lu;
        uy /= lu;
        wx /= lw;
        wy /= lw;
        if (!(ux * wx + uy * wy > crt)) break;  // a corner ends the chain
        color[b1] = nchain;
        if (dir == 0) chain.push_back(b1);
        else chain.push_front(b1);
        b0 = b1;
        k0 = 1 - k1;
      }
    }
    R.group_facet.insert(R.group_facet.end(), chain.begin(), chain.end());
    R.group_ptr.push_back((unsigned)R.group_facet.size());
    nchain++;
  }
  // the chains' end nodes (first bar's v[0], last bar's v[1]), ascending
  std::map<unsigned, unsigned> ends;
  for (long long c = 0; c < nchain; c++) {
    ends[bar[2 * (size_t)R.group_facet[R.group_ptr[c]]]] = 0;
    ends[bar[2 * (size_t)R.group_facet[R.group_ptr[c + 1] - 1] + 1]] = 0;
  }
  unsigned iv = 0;
  for (auto& e : ends) {
    e.second = iv++;
    R.vertex.push_back(e.first);
  }
  for (long long c = 0; c < nchain; c++) {
    R.group_ends.push_back(ends[bar[2 * (size_t)R.group_facet[R.group_ptr[c]]]]);
    R.group_ends.push_back(ends[bar[2 * (size_t)R.group_facet[R.group_ptr[c + 1] - 1] + 1]]);
  }
}

int gid_boundary(int ndim, unsigned nnode, const double* coord, int nnoel, unsigned nelem, const int* elem,
                 double crt_dot, int* nnofa, unsigned* nfacet, unsigned* facet, unsigned* ngroup, unsigned* group_ptr,
                 unsigned* group_facet, unsigned* nvertex, unsigned* vertex, unsigned* group_ends) {
  if (!nnofa || !nfacet || !ngroup || !nvertex || (nelem && !elem) || (nnode && !coord)) return DFM_ERR_INVALID;
  const bool tet = ndim == 3 && nnoel == 4, hex = ndim == 3 && nnoel == 8,
             planar = ndim == 2 && (nnoel == 3 || nnoel == 4);
  if (!tet && !hex && !planar) return DFM_ERR_INVALID;
  if ((size_t)nelem * (size_t)nnoel >= (size_t)1 << 32) return DFM_ERR_INVALID;
  for (unsigned t = 0; t < nelem; t++)
    for (int q = 0; q < nnoel; q++) {
      const int v = elem[(size_t)nnoel * t + q];
      if (v < 0 || (unsigned)v >= nnode) return DFM_ERR_INVALID;
      for (int r = 0; r < q; r++)
        if (elem[(size_t)nnoel * t + r] == v) return DFM_ERR_INVALID;  // a repeated node
    }
  Result R;
  if (tet) tet_boundary(coord, nelem, elem, crt_dot, R);
  else if (planar) planar_boundary(nnode, coord, nnoel, nelem, elem, crt_dot, R);
  else R.group_ptr.assign(1, 0);
  *nnofa = hex ? 4 : R.nnofa;
  *nfacet = (unsigned)(R.facet.size() / (R.nnofa ? R.nnofa : 1));
  *ngroup = (unsigned)(R.group_ptr.size() - 1);
  *nvertex = (unsigned)R.vertex.size();
  if (!facet) return DFM_OK;
  std::copy(R.facet.begin(), R.facet.end(), facet);
  if (group_ptr) std::copy(R.group_ptr.begin(), R.group_ptr.end(), group_ptr);
  if (group_facet) std::copy(R.group_facet.begin(), R.group_facet.end(), group_facet);
  if (vertex) std::copy(R.vertex.begin(), R.vertex.end(), vertex);
  if (group_ends) std::copy(R.group_ends.begin(), R.group_ends.end(), group_ends);
  return DFM_OK;
}

}  // namespace
}  // namespace dfm

extern "C" {

int dfm_gid_boundary(int ndim, unsigned nnode, const double* coord, int nnoel, unsigned nelem, const int* elem,
                     double crt_dot, int* nnofa, unsigned* nfacet, unsigned* facet, unsigned* ngroup,
                     unsigned* group_ptr, unsigned* group_facet, unsigned* nvertex, unsigned* vertex,
                     unsigned* group_ends) {
  try {
    return dfm::gid_boundary(ndim, nnode, coord, nnoel, nelem, elem, crt_dot, nnofa, nfacet, facet, ngroup, group_ptr,
                             group_facet, nvertex, vertex, group_ends);
  } catch (const std::bad_alloc&) {
    return DFM_ERR_NOMEM;
  } catch (...) {
    return DFM_ERR_INVALID;
  }
}

}  // extern "C"
