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
#include <cstdlib>
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

extern "C" {

int dfm_zmat_read_text(const char* path, unsigned* N, unsigned* ncrs, unsigned* rowptr, unsigned* colind,
                       double* diag, double* off) {
  if (!path || !N || !ncrs) return DFM_ERR_INVALID;
  Tokens t;
  int rc = read_file(path, t.buf);
  if (rc) return rc;
  long long nblk = 0, nnz = 0;
  if (!t.integer(&nblk) || !t.integer(&nnz) || nblk < 0 || nnz < 0 || nblk > 0x7fffffffLL) return DFM_ERR_INVALID;
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

}  // extern "C"
