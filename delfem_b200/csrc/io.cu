// On-disk formats that feed the solve path (host only).
//
// CZMatDia_BlkCrs(const std::string& file_path)
// (src/matvec/zmatdia_blkcrs.cpp:108-173) reads a complex matrix with scalar
// blocks as text: a line "nblk nnz", then nnz entries "icol irow re im"
// (0-based; icol is the row of the block-CRS, irow the column), grouped by
// non-decreasing icol; icol == irow gives the diagonal, and a row without one
// has a zero diagonal.  This reader produces the same pattern and values as
// the reference for every file the reference reads without hitting one of its
// asserts, with these definitions where the reference leaves memory
// uninitialised or keeps an order the block-CRS cannot hold:
//   * rows that have no entry at all get an empty row and a zero diagonal
//     (the reference leaves their row pointer - after the last listed row -
//     and their diagonal unset);
//   * off-diagonal entries of a row are sorted by column (the reference keeps
//     the file's order, and its ILU assumes ascending columns);
//   * a repeated diagonal keeps the last value, as in the reference; a
//     repeated off-diagonal column is an error (the reference would store it
//     twice).
// Malformed input (a bad count, an index out of range, a decreasing row, a
// missing or unparsable entry) is DFM_ERR_INVALID; an unreadable file is
// DFM_ERR_IO.  The reference prints and exit(1)s instead.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <new>
#include <numeric>
#include <vector>

#include "dfm_internal.h"

namespace dfm {
namespace {

struct Tokens {
  std::vector<char> buf;
  size_t pos = 0;
  void skip() {
    while (pos < buf.size() && (buf[pos] == ' ' || buf[pos] == '\t' || buf[pos] == '\n' || buf[pos] == '\r' ||
                                buf[pos] == '\v' || buf[pos] == '\f'))
      pos++;
  }
  bool integer(long long* v) {
    skip();
    if (pos >= buf.size()) return false;
    char* end = nullptr;
    errno = 0;
    *v = std::strtoll(buf.data() + pos, &end, 10);
    if (end == buf.data() + pos || errno == ERANGE) return false;
    pos = (size_t)(end - buf.data());
    return true;
  }
  bool real(double* v) {
    skip();
    if (pos >= buf.size()) return false;
    char* end = nullptr;
    *v = std::strtod(buf.data() + pos, &end);  // the conversion fscanf's %lf performs
    if (end == buf.data() + pos) return false;
    pos = (size_t)(end - buf.data());
    return true;
  }
};

int read_file(const char* path, std::vector<char>& buf) {
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return DFM_ERR_IO;
  char tmp[1 << 16];
  size_t n;
  while ((n = std::fread(tmp, 1, sizeof(tmp), fp)) > 0) buf.insert(buf.end(), tmp, tmp + n);
  const bool bad = std::ferror(fp) != 0;
  std::fclose(fp);
  if (bad) return DFM_ERR_IO;
  buf.push_back('\0');  // strtod / strtoll stop here
  return DFM_OK;
}

}  // namespace
}  // namespace dfm

using namespace dfm;

namespace dfm {
namespace {

int zmat_read_text(const char* path, unsigned* N, unsigned* ncrs, unsigned* rowptr, unsigned* colind, double* diag,
                   double* off) {
  if (!path || !N || !ncrs) return DFM_ERR_INVALID;
  Tokens t;
  int rc = read_file(path, t.buf);
  if (rc) return rc;
  long long nblk = 0, nnz = 0;
  if (!t.integer(&nblk) || !t.integer(&nnz) || nblk < 0 || nnz < 0 || nblk > 0x7fffffffLL) return DFM_ERR_INVALID;
  // every entry line holds four numbers, at least 8 bytes with separators: a
  // count the file cannot hold is malformed (and must not size an allocation)
  if ((unsigned long long)nnz > t.buf.size() / 8 + 1) return DFM_ERR_INVALID;
  const unsigned n = (unsigned)nblk;
  std::vector<unsigned> rp(n + 1, 0), cols;
  std::vector<double> dg(2 * (size_t)n, 0.0), vals;
  cols.reserve((size_t)nnz);
  vals.reserve(2 * (size_t)nnz);
  long long row_cur = 0;
  for (long long e = 0; e < nnz; e++) {
    long long icol, irow;
    double re, im;
    if (!t.integer(&icol) || !t.integer(&irow) || !t.real(&re) || !t.real(&im)) return DFM_ERR_INVALID;
    if (icol < 0 || icol >= nblk || irow < 0 || irow >= nblk || icol < row_cur) return DFM_ERR_INVALID;
    while (row_cur < icol) rp[++row_cur] = (unsigned)cols.size();  // rows up to icol start here
    if (icol == irow) {
      dg[2 * icol] = re;
      dg[2 * icol + 1] = im;
    } else {
      cols.push_back((unsigned)irow);
      vals.push_back(re);
      vals.push_back(im);
    }
  }
  while (row_cur < (long long)n) rp[++row_cur] = (unsigned)cols.size();
  // ascending columns inside every row, no repeats
  for (unsigned i = 0; i < n; i++) {
    const unsigned a = rp[i], b = rp[i + 1];
    bool sorted = true;
    for (unsigned s = a + 1; s < b; s++)
      if (cols[s] <= cols[s - 1]) sorted = false;
    if (sorted) continue;
    std::vector<unsigned> perm(b - a);
    std::iota(perm.begin(), perm.end(), a);
    std::stable_sort(perm.begin(), perm.end(), [&](unsigned x, unsigned y) { return cols[x] < cols[y]; });
    std::vector<unsigned> c2(b - a);
    std::vector<double> v2(2 * (size_t)(b - a));
    for (unsigned k = 0; k < b - a; k++) {
      c2[k] = cols[perm[k]];
      v2[2 * k] = vals[2 * (size_t)perm[k]];
      v2[2 * k + 1] = vals[2 * (size_t)perm[k] + 1];
      if (k > 0 && c2[k] == c2[k - 1]) return DFM_ERR_INVALID;
    }
    std::copy(c2.begin(), c2.end(), cols.begin() + a);
    std::copy(v2.begin(), v2.end(), vals.begin() + 2 * (size_t)a);
  }
  *N = n;
  *ncrs = (unsigned)cols.size();
  if (!rowptr) return DFM_OK;  // size query
  std::copy(rp.begin(), rp.end(), rowptr);
  if (colind) std::copy(cols.begin(), cols.end(), colind);
  if (diag) std::copy(dg.begin(), dg.end(), diag);
  if (off) std::copy(vals.begin(), vals.end(), off);
  return DFM_OK;
}

}  // namespace
}  // namespace dfm

// GiD ASCII mesh, as Msh::CMesh3D::ReadFromFile_GiDMsh (src/msh/mesh3d.cpp:
// 601-800) and Msh::CMesher2D::ReadFromFile_GiDMsh (src/msh/mesher2d.cpp:
// 2464-2640) read it: a header line
//   MESH dimension <ndim> ElemType <Tetrahedra|Hexahedra|Triangle|Quadrilateral> Nnode <n>
// then "Coordinates", lines "<id> x y z" (ids 1, 2, ... in order), "end
// coordinates", one line, "Elements", lines "<id> v1 .. vn [material]"
// (1-based nodes), "end elements".  Tetrahedra and hexahedra come out with 3-D
// coordinates.  Triangles and quadrilaterals come out as the 2-D mesher makes
// them: with ndim 3, the node cloud must be planar (the smallest of the three
// coordinate variances at most 1e-4 of their sum, the reference's test) and
// the axis of that smallest variance is dropped, the other two kept in cyclic
// order (y,z / z,x / x,y); with ndim 2 the lines carry x y.  The volume
// elements and coordinates are what the pattern and the assembly need; the
// boundary facets the reference derives from them are dfm_gid_boundary's
// (boundary.cu).
namespace dfm {
namespace {
struct Lines {
  std::vector<char> buf;
  size_t pos = 0;
  // next line (without the newline) or false at the end
  bool next(const char** b, const char** e) {
    if (pos >= buf.size() || buf[pos] == '\0') return false;
    const char* p = buf.data() + pos;
    size_t q = pos;
    while (q < buf.size() && buf[q] != '\n' && buf[q] != '\0') q++;
    *b = p;
    *e = buf.data() + q;
    pos = q < buf.size() && buf[q] == '\n' ? q + 1 : q;
    return true;
  }
};
bool starts(const char* b, const char* e, const char* w) {
  size_t n = std::strlen(w);
  return (size_t)(e - b) >= n && std::strncmp(b, w, n) == 0;
}
// whitespace-separated numbers of [b, e): integers or doubles
int parse_numbers(const char* b, const char* e, double* out, int max) {
  std::string line(b, e);
  const char* p = line.c_str();
  int n = 0;
  while (n < max) {
    char* q = nullptr;
    const double v = std::strtod(p, &q);
    if (q == p) break;
    out[n++] = v;
    p = q;
  }
  return n;
}
}  // namespace
}  // namespace dfm

namespace dfm {
namespace {

int gid_read_mesh(const char* path, int* ndim, unsigned* nnode, double* coord, int* nnoel, unsigned* nelem,
                  int* elem) {
  if (!path || !ndim || !nnode || !nnoel || !nelem) return DFM_ERR_INVALID;
  Lines L;
  int rc = read_file(path, L.buf);
  if (rc) return rc;
  const char *b, *e;
  if (!L.next(&b, &e)) return DFM_ERR_INVALID;
  char w1[64], w2[64], w3[64], type[64], w4[64];
  int nd = 0, nn = 0;
  {
    std::string h(b, e);
    if (std::sscanf(h.c_str(), "%63s %63s %d %63s %63s %63s %d", w1, w2, &nd, w3, type, w4, &nn) != 7)
      return DFM_ERR_INVALID;
  }
  const std::string t(type);
  int want = 0;
  bool surface = false;
  if (t == "Tetrahedra") want = 4;
  else if (t == "Hexahedra") want = 8;
  else if (t == "Triangle") { want = 3; surface = true; }
  else if (t == "Quadrilateral") { want = 4; surface = true; }
  if (!want || nn != want) return DFM_ERR_INVALID;
  if ((!surface && nd != 3) || (surface && nd != 2 && nd != 3)) return DFM_ERR_INVALID;
  if (!L.next(&b, &e)) return DFM_ERR_INVALID;  // "Coordinates"
  std::vector<double> xyz;
  unsigned count = 0;
  for (;;) {
    if (!L.next(&b, &e)) return DFM_ERR_INVALID;
    if (starts(b, e, "end coordinates")) break;
    double v[4];
    const int k = parse_numbers(b, e, v, 1 + nd);
    if (k != 1 + nd || v[0] != (double)(count + 1)) return DFM_ERR_INVALID;
    for (int d = 0; d < nd; d++) xyz.push_back(v[1 + d]);
    count++;
  }
  if (count == 0) return DFM_ERR_INVALID;
  int nd_out = nd, keep0 = 0, keep1 = 1;
  if (surface && nd == 3) {  // planar cloud -> the 2-D mesher's coordinates
    double ax = 0, ay = 0, az = 0, vx = 0, vy = 0, vz = 0;
    for (unsigned i = 0; i < count; i++) {
      const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
      ax += x; ay += y; az += z;
      vx += x * x; vy += y * y; vz += z * z;
    }
    vx /= count; vy /= count; vz /= count;
    ax /= count; ay /= count; az /= count;
    vx -= ax * ax; vy -= ay * ay; vz -= az * az;
    double vmin = vx;
    int dmin = 0;
    if (vy < vmin) { vmin = vy; dmin = 1; }
    if (vz < vmin) { vmin = vz; dmin = 2; }
    if (vmin > (vx + vy + vz) * 0.0001) return DFM_ERR_INVALID;  // not planar
    keep0 = dmin == 0 ? 1 : (dmin == 1 ? 2 : 0);
    keep1 = dmin == 0 ? 2 : (dmin == 1 ? 0 : 1);
    nd_out = 2;
  }
  if (!L.next(&b, &e)) return DFM_ERR_INVALID;  // the line after "end coordinates"
  if (!L.next(&b, &e)) return DFM_ERR_INVALID;  // "Elements"
  std::vector<int> conn;
  unsigned ne = 0;
  for (;;) {
    if (!L.next(&b, &e)) return DFM_ERR_INVALID;
    if (starts(b, e, "end elements")) break;
    double v[10];
    const int k = parse_numbers(b, e, v, 1 + want);
    if (k != 1 + want || v[0] != (double)(ne + 1)) return DFM_ERR_INVALID;
    for (int j = 0; j < want; j++) {
      if (!(v[1 + j] >= 1 && v[1 + j] <= (double)count) || v[1 + j] != std::floor(v[1 + j])) return DFM_ERR_INVALID;
      conn.push_back((int)v[1 + j] - 1);
    }
    ne++;
  }
  *ndim = nd_out;
  *nnode = count;
  *nnoel = want;
  *nelem = ne;
  if (coord) {
    for (unsigned i = 0; i < count; i++) {
      if (nd_out == 3) for (int d = 0; d < 3; d++) coord[3 * (size_t)i + d] = xyz[3 * (size_t)i + d];
      else if (nd == 3) { coord[2 * (size_t)i] = xyz[3 * (size_t)i + keep0]; coord[2 * (size_t)i + 1] = xyz[3 * (size_t)i + keep1]; }
      else { coord[2 * (size_t)i] = xyz[2 * (size_t)i]; coord[2 * (size_t)i + 1] = xyz[2 * (size_t)i + 1]; }
    }
  }
  if (elem) std::copy(conn.begin(), conn.end(), elem);
  return DFM_OK;
}

}  // namespace
}  // namespace dfm

// The readers build host containers sized by the file: a failed allocation
// (or any other exception) must not cross the C ABI.
extern "C" {

int dfm_zmat_read_text(const char* path, unsigned* N, unsigned* ncrs, unsigned* rowptr, unsigned* colind,
                       double* diag, double* off) {
  try {
    return dfm::zmat_read_text(path, N, ncrs, rowptr, colind, diag, off);
  } catch (const std::bad_alloc&) {
    return DFM_ERR_NOMEM;
  } catch (...) {
    return DFM_ERR_INVALID;
  }
}

int dfm_gid_read_mesh(const char* path, int* ndim, unsigned* nnode, double* coord, int* nnoel, unsigned* nelem,
                      int* elem) {
  try {
    return dfm::gid_read_mesh(path, ndim, nnode, coord, nnoel, nelem, elem);
  } catch (const std::bad_alloc&) {
    return DFM_ERR_NOMEM;
  } catch (...) {
    return DFM_ERR_INVALID;
  }
}

}  // extern "C"
