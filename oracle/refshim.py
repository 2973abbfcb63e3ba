"""ctypes binding of oracle/_ref/libdfm_refshim.so - the reference's own CPU
implementation of the linear-solve path (DelFEM sources compiled by
oracle/Makefile).  TEST INFRASTRUCTURE ONLY: tests, fixture generation and the
bench's CPU-baseline leg use it as the checker / timed baseline."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libdfm_refshim.so")
REF_DIR = os.environ.get("DELFEM_REFERENCE", "/root/reference")  # the reference source tree

POISSON2D, SOLID2D, SOLID3D, HELMHOLTZ2D = 1, 2, 3, 4
PCG, PBICGSTAB, PCOCG, CG = 0, 1, 2, 3

_lib = None


def build(ref_dir: str = REF_DIR) -> bool:
    """Compile the reference + shim into oracle/_ref (needs the reference tree)."""
    if not os.path.isdir(ref_dir):
        return os.path.exists(LIB_PATH)
    r = subprocess.run(["make", "-s", "-C", HERE, f"REF={ref_dir}", "ref", "-j8"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference build failed:\n" + r.stdout + r.stderr)
    return True


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        dp, up, ip = C.POINTER(C.c_double), C.POINTER(C.c_uint), C.POINTER(C.c_int)
        L.dfm_ref_create.restype = P
        L.dfm_ref_create.argtypes = [C.c_int, C.c_int, C.c_int, dp, C.c_int, C.c_int, ip, C.c_int, C.c_int, ip]
        L.dfm_ref_destroy.argtypes = [P]
        L.dfm_ref_dims.argtypes = [P, up, up, up]
        L.dfm_ref_pattern.argtypes = [P, up, up]
        L.dfm_ref_assemble.argtypes = [P, dp, dp, dp, dp, dp]
        L.dfm_ref_get_system.argtypes = [P, dp, dp, dp]
        L.dfm_ref_get_bcflag.argtypes = [P, ip]
        L.dfm_ref_ilu.argtypes = [P, dp]
        L.dfm_ref_get_ilu.argtypes = [P, dp, dp]
        L.dfm_ref_solve.argtypes = [P, C.c_int, C.c_double, C.c_uint, up, dp, dp, dp]
        L.dfm_ref_mat_spmv.argtypes = [C.c_uint, C.c_uint, up, up, dp, dp, C.c_double, dp, C.c_double, dp]
        L.dfm_ref_mat_ilu0.argtypes = [C.c_uint, C.c_uint, up, up, dp, dp, dp, dp]
        L.dfm_ref_mat_precond.argtypes = [C.c_uint, C.c_uint, up, up, dp, dp, dp]
        L.dfm_ref_mat_solve.argtypes = [C.c_uint, C.c_uint, up, up, dp, dp, dp, C.c_int, C.c_double,
                                        C.c_uint, up, dp, dp, dp, dp]
        L.dfm_ref_mat_iluk.argtypes = [C.c_uint, C.c_uint, up, up, dp, dp, C.c_int, C.c_uint, up, up, dp, dp, up]
        L.dfm_ref_mat_iluk_rows.argtypes = [C.c_uint, C.c_uint, up, up, dp, dp, C.c_int, C.c_uint, up, C.c_uint, up,
                                            up, dp, dp, up]
        L.dfm_ref_mat_solve_lev.argtypes = [C.c_uint, C.c_uint, up, up, dp, dp, dp, C.c_int, C.c_double,
                                            C.c_uint, C.c_int, up, dp, dp, dp, dp]
        L.dfm_ref_boundary_residual.argtypes = [C.c_uint, C.c_uint, up, up, dp, dp, ip, dp, dp, C.c_uint, up, up,
                                                dp, up, dp]
        L.dfm_ref_gid_read.argtypes = [C.c_char_p, C.c_int, C.c_uint, C.c_uint, up, up, ip, dp, ip]
        L.dfm_ref_gid_boundary.argtypes = [C.c_char_p, C.c_int, C.c_uint, C.c_uint, C.c_uint, up, up, up, up, up, up,
                                            up, up, up]
        L.dfm_ref_zmat_read.argtypes = [C.c_char_p, C.c_uint, up, up, up, up, dp, dp]
        L.dfm_ref_zmat_spmv.argtypes = [C.c_uint, up, up, dp, dp, C.c_double, dp, C.c_double, dp]
        L.dfm_ref_zmat_ilu0.argtypes = [C.c_uint, up, up, dp, dp, dp, dp]
        L.dfm_ref_zmat_iluk.argtypes = [C.c_uint, up, up, dp, dp, C.c_int, C.c_uint, up, up, dp, dp, up]
        L.dfm_ref_set_fill.argtypes = [P, C.c_int]
        L.dfm_ref_rmat_spmv.argtypes = [C.c_uint, C.c_uint, C.c_uint, C.c_uint, up, up, dp, C.c_double, dp,
                                        C.c_double, dp]
        L.dfm_ref_newmark.argtypes = [C.c_int, C.c_int, dp, C.c_int, ip, C.c_int, ip, dp, C.c_double, C.c_double,
                                      C.c_double, dp, dp, dp, dp, dp, dp, dp, ip, dp, dp]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _u(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None


class RefSystem:
    """Field-level reference system built from a :class:`delfem_b200.meshes.Mesh`."""

    def __init__(self, kind: int, mesh):
        L = lib()
        self.kind = kind
        coord = np.ascontiguousarray(mesh.coord, dtype=np.float64)
        elem = np.ascontiguousarray(mesh.elem, dtype=np.int32)
        bnd = np.ascontiguousarray(mesh.bnd, dtype=np.int32)
        self._keep = (coord, elem, bnd)
        self.h = L.dfm_ref_create(kind, mesh.ndim, mesh.nnode, _d(coord), mesh.nnoel, elem.shape[0], _i(elem),
                                  bnd.shape[1] if bnd.size else 0, bnd.shape[0], _i(bnd) if bnd.size else None)
        if not self.h:
            raise RuntimeError("dfm_ref_create failed")
        N, b, n = C.c_uint(), C.c_uint(), C.c_uint()
        L.dfm_ref_dims(self.h, C.byref(N), C.byref(b), C.byref(n))
        self.N, self.b, self.ncrs = N.value, b.value, n.value
        self.cplx = kind == HELMHOLTZ2D
        self.vw = 2 if self.cplx else self.b * self.b     # doubles per block
        self.xw = 2 if self.cplx else self.b              # doubles per block row of a vector

    def __del__(self):
        if getattr(self, "h", None):
            lib().dfm_ref_destroy(self.h)
            self.h = None

    def pattern(self):
        rp = np.zeros(self.N + 1, np.uint32)
        ci = np.zeros(max(self.ncrs, 1), np.uint32)
        lib().dfm_ref_pattern(self.h, _u(rp), _u(ci))
        return rp, ci[: self.ncrs]

    def assemble(self, params, coef=None, load=None):
        p = np.ascontiguousarray(params, dtype=np.float64)
        c = None if coef is None else np.ascontiguousarray(coef, dtype=np.float64)
        l_ = None if load is None else np.ascontiguousarray(load, dtype=np.float64).ravel()
        res, sec = C.c_double(), C.c_double()
        rc = lib().dfm_ref_assemble(self.h, _d(p), _d(c), _d(l_), C.byref(res), C.byref(sec))
        if rc:
            raise RuntimeError("assemble failed")
        return res.value, sec.value

    def system(self):
        d = np.zeros(self.N * self.vw)
        o = np.zeros(max(self.ncrs, 1) * self.vw)
        r = np.zeros(self.N * self.xw)
        lib().dfm_ref_get_system(self.h, _d(d), _d(o), _d(r))
        return d, o[: self.ncrs * self.vw], r

    def bcflag(self):
        f = np.zeros(self.N * self.b, np.int32)
        lib().dfm_ref_get_bcflag(self.h, _i(f))
        return f

    def set_fill(self, lev):
        """SetFillInLevel(lev) + SetLinearSystem of the system's preconditioner."""
        lib().dfm_ref_set_fill(self.h, int(lev))

    def ilu(self):
        sec = C.c_double()
        rc = lib().dfm_ref_ilu(self.h, C.byref(sec))
        return rc, sec.value

    def ilu_factor(self):
        d = np.zeros(self.N * self.vw)
        o = np.zeros(max(self.ncrs, 1) * self.vw)
        rc = lib().dfm_ref_get_ilu(self.h, _d(d), _d(o))
        return rc, d, o[: self.ncrs * self.vw]

    def solve(self, method=PCG, tol=1e-10, maxit=10000):
        x = np.zeros(self.N * self.xw)
        it, conv, sec = C.c_uint(), C.c_double(), C.c_double()
        rc = lib().dfm_ref_solve(self.h, method, tol, maxit, C.byref(it), C.byref(conv), _d(x), C.byref(sec))
        return rc, x, it.value, conv.value, sec.value


def mat_spmv(N, b, rowptr, colind, diag, off, alpha, x, beta, y):
    y = np.array(y, dtype=np.float64, copy=True)
    lib().dfm_ref_mat_spmv(N, b, _u(rowptr), _u(colind), _d(diag), _d(off), alpha, _d(np.ascontiguousarray(x)), beta, _d(y))
    return y


def mat_ilu0(N, b, rowptr, colind, diag, off):
    fd = np.zeros_like(diag)
    fo = np.zeros(max(off.size, 1))
    rc = lib().dfm_ref_mat_ilu0(N, b, _u(rowptr), _u(colind), _d(diag), _d(off if off.size else fo), _d(fd), _d(fo))
    return rc, fd, fo[: off.size]


def mat_precond(N, b, rowptr, colind, fdiag, foff, vec):
    v = np.array(vec, dtype=np.float64, copy=True)
    fo = foff if foff.size else np.zeros(1)
    lib().dfm_ref_mat_precond(N, b, _u(rowptr), _u(colind), _d(fdiag), _d(fo), _d(v))
    return v


def mat_solve(N, b, rowptr, colind, diag, off, rhs, method=PCG, tol=1e-10, maxit=10000, lev=0):
    x = np.zeros(N * b)
    it, conv, ti, ts = C.c_uint(), C.c_double(), C.c_double(), C.c_double()
    rc = lib().dfm_ref_mat_solve_lev(N, b, _u(rowptr), _u(colind), _d(diag), _d(off),
                                     _d(np.ascontiguousarray(rhs)), method, tol, maxit, lev, C.byref(it),
                                     C.byref(conv), _d(x), C.byref(ti), C.byref(ts))
    return rc, x, it.value, conv.value, ti.value, ts.value


def mat_iluk(N, b, rowptr, colind, diag, off, lev, rows=None):
    """CMatDiaFrac_BlkCrs(lev, A) + SetValue_Initialize + DoILUDecomp:
    (rc, frowptr, fcolind, fdiag, foff).  rows: the SetFillBlk list
    (AddFracPtn(lev, aBlkFill) over CMatDiaFrac_BlkCrs(0, A))."""
    n = C.c_uint()
    o = off if off.size else np.zeros(1)
    rw = np.ascontiguousarray(rows if rows is not None else [], np.uint32)
    ra = (rw.size, _u(rw if rw.size else np.zeros(1, np.uint32)))
    lib().dfm_ref_mat_iluk_rows(N, b, _u(rowptr), _u(colind), _d(diag), _d(o), lev, *ra, 0, None, None, None, None,
                                C.byref(n))
    fr = np.zeros(N + 1, np.uint32)
    fc = np.zeros(max(n.value, 1), np.uint32)
    fd = np.zeros(N * b * b)
    fo = np.zeros(max(n.value, 1) * b * b)
    rc = lib().dfm_ref_mat_iluk_rows(N, b, _u(rowptr), _u(colind), _d(diag), _d(o), lev, *ra, n.value, _u(fr),
                                     _u(fc), _d(fd), _d(fo), C.byref(n))
    return rc, fr, fc[: n.value], fd, fo[: n.value * b * b]


def zmat_ilu0(N, rowptr, colind, diag, off):
    fd = np.zeros_like(diag)
    fo = np.zeros(max(off.size, 1))
    lib().dfm_ref_zmat_ilu0(N, _u(rowptr), _u(colind), _d(diag), _d(off if off.size else fo), _d(fd), _d(fo))
    return fd, fo[: off.size]


def zmat_spmv(N, rowptr, colind, diag, off, alpha, x, beta, y):
    y = np.array(y, dtype=np.float64, copy=True)
    lib().dfm_ref_zmat_spmv(N, _u(rowptr), _u(colind), _d(diag), _d(off), alpha, _d(np.ascontiguousarray(x)), beta, _d(y))
    return y


def zmat_read(path):
    """The reference's CZMatDia_BlkCrs(file_path): (N, rowptr, colind, diag, off)."""
    n, m = C.c_uint(), C.c_uint()
    p = os.fsencode(path)
    lib().dfm_ref_zmat_read(p, 0, C.byref(n), C.byref(m), None, None, None, None)
    rp = np.zeros(n.value + 1, np.uint32)
    ci = np.zeros(max(m.value, 1), np.uint32)
    d = np.zeros(max(2 * n.value, 1))
    o = np.zeros(max(2 * m.value, 1))
    lib().dfm_ref_zmat_read(p, m.value, C.byref(n), C.byref(m), _u(rp), _u(ci), _d(d), _d(o))
    return n.value, rp, ci[: m.value], d[: 2 * n.value], o[: 2 * m.value]


def gid_read(path, want2d):
    """The reference's GiD reader (2-D mesher or 3-D mesh): (rc, coord, elem)."""
    nn, ne, no = C.c_uint(), C.c_uint(), C.c_int()
    p = os.fsencode(path)
    rc = lib().dfm_ref_gid_read(p, int(want2d), 0, 0, C.byref(nn), C.byref(ne), C.byref(no), None, None)
    if rc == 1:
        return 1, None, None
    nd = 2 if want2d else 3
    coord = np.zeros((nn.value, nd))
    elem = np.zeros((ne.value, no.value), np.int32)
    rc = lib().dfm_ref_gid_read(p, int(want2d), nn.value, ne.value, C.byref(nn), C.byref(ne), C.byref(no),
                                _d(coord.reshape(-1)), _i(elem.reshape(-1)))
    return rc, coord, elem


def gid_boundary(path, want2d):
    """The boundary facets the reference's GiD readers derive and store: a
    dict with ``facets`` (grouped, [nfacet, 3] triangles or [nfacet, 2] bars),
    ``groups`` (index ranges of each colour / bar array into ``facets``),
    ``group_ids``, and for 2-D ``vertices`` (nodes), ``vertex_ids`` and
    ``ends`` (each chain's id_se as indices into ``vertices``); None when the
    reader refuses the file."""
    p = os.fsencode(path)
    nf, ng, nv = C.c_uint(), C.c_uint(), C.c_uint()
    z = None
    rc = lib().dfm_ref_gid_boundary(p, int(want2d), 0, 0, 0, C.byref(nf), C.byref(ng), C.byref(nv), z, z, z, z, z, z)
    if rc == 1:
        return None
    k = 2 if want2d else 3
    facet = np.zeros((max(nf.value, 1), k), np.uint32)
    gptr = np.zeros(ng.value + 1, np.uint32)
    gid = np.zeros(max(ng.value, 1), np.uint32)
    vert = np.zeros(max(nv.value, 1), np.uint32)
    vid = np.zeros(max(nv.value, 1), np.uint32)
    ends = np.zeros((max(ng.value, 1), 2), np.uint32)
    rc = lib().dfm_ref_gid_boundary(p, int(want2d), nf.value, ng.value, nv.value, C.byref(nf), C.byref(ng),
                                    C.byref(nv), _u(facet.reshape(-1)), _u(gptr), _u(gid), _u(vert), _u(vid),
                                    _u(ends.reshape(-1)))
    assert rc == 0
    return {"facets": facet[:nf.value], "groups": [np.arange(gptr[g], gptr[g + 1]) for g in range(ng.value)],
            "group_ids": gid[:ng.value], "vertices": vert[:nv.value], "vertex_ids": vid[:nv.value],
            "ends": ends[:ng.value] if want2d else np.zeros((0, 2), np.uint32)}


def boundary_residual(N, b, rowptr, colind, diag, off, flags, force, u):
    """The reference's CLinearSystem_Save boundary matrix (row by row, diagonal
    first) and MakeResidual's r = force - B u: (brow, bcol, bval, r)."""
    n = C.c_uint()
    r = np.zeros(N * b)
    fl = np.ascontiguousarray(flags, np.int32)
    o = off if off.size else np.zeros(1)
    ci = colind if colind.size else np.zeros(1, np.uint32)
    args = (N, b, _u(rowptr), _u(ci), _d(diag), _d(o), _i(fl), _d(np.ascontiguousarray(force)),
            _d(np.ascontiguousarray(u)))
    lib().dfm_ref_boundary_residual(*args, 0, None, None, None, C.byref(n), _d(r))
    brow = np.zeros(N + 1, np.uint32)
    bcol = np.zeros(max(n.value, 1), np.uint32)
    bval = np.zeros(max(n.value, 1) * b * b)
    lib().dfm_ref_boundary_residual(*args, n.value, _u(brow), _u(bcol), _d(bval), C.byref(n), _d(r))
    return brow, bcol[: n.value], bval[: n.value * b * b], r


def newmark(scheme, mesh, params, dt, gamma, beta, u, v, a, x, ncrs):
    """The reference's CLinearSystem_SaveDiaM_Newmark (scheme 1, diffusion) /
    _NewmarkBeta (scheme 2, 2-D solid) on a P1 triangle mesh whose boundary
    bars are fixed: its stored matrix (library layout over the mesh pattern,
    ncrs off-diagonal blocks), force, flags, MakeResidual's r and norm, and the
    state after UpdateValueOfField with the update x.  Returns a dict."""
    b = 1 if scheme == 1 else 2
    N = mesh.nnode
    u, v, x = (np.array(t, np.float64, copy=True).ravel() for t in (u, v, x))
    a = np.array(a if a is not None else np.zeros(N * b), np.float64, copy=True).ravel()
    bd, bo = np.zeros(N * b * b), np.zeros(max(ncrs, 1) * b * b)
    force, r, fl = np.zeros(N * b), np.zeros(N * b), np.zeros(N * b, np.int32)
    nrm = C.c_double()
    elem = np.ascontiguousarray(mesh.elem, np.int32)
    bnd = np.ascontiguousarray(mesh.bnd, np.int32)
    rc = lib().dfm_ref_newmark(scheme, N, _d(np.ascontiguousarray(mesh.coord, np.float64)), elem.shape[0], _i(elem),
                               bnd.shape[0], _i(bnd), _d(np.ascontiguousarray(params, np.float64)), dt, gamma, beta,
                               _d(u), _d(v), _d(a), _d(x), _d(bd), _d(bo), _d(force), _i(fl), _d(r), C.byref(nrm))
    if rc:
        raise RuntimeError(f"dfm_ref_newmark failed ({rc})")
    return dict(bdiag=bd, boff=bo[: ncrs * b * b], force=force, flags=fl, r=r, norm=nrm.value, u=u, v=v, a=a, x=x)


def zmat_iluk(N, rowptr, colind, diag, off, lev):
    """CZMatDiaFrac_BlkCrs(lev, A) + SetValue_Initialize + DoILUDecomp:
    (rc, frowptr, fcolind, fdiag, foff), complex values interleaved."""
    n = C.c_uint()
    o = off if off.size else np.zeros(2)
    ci = colind if colind.size else np.zeros(1, np.uint32)
    lib().dfm_ref_zmat_iluk(N, _u(rowptr), _u(ci), _d(diag), _d(o), lev, 0, None, None, None, None, C.byref(n))
    fr = np.zeros(N + 1, np.uint32)
    fc = np.zeros(max(n.value, 1), np.uint32)
    fd = np.zeros(2 * N)
    fo = np.zeros(max(n.value, 1) * 2)
    rc = lib().dfm_ref_zmat_iluk(N, _u(rowptr), _u(ci), _d(diag), _d(o), lev, n.value, _u(fr), _u(fc), _d(fd),
                                 _d(fo), C.byref(n))
    return rc, fr, fc[: n.value], fd, fo[: 2 * n.value]


def rmat_spmv(nrow, ncol, brow, bcol, rowptr, colind, val, alpha, x, beta, y):
    """The reference's CMat_BlkCrs::MatVec: returns the new y."""
    y = np.array(y, np.float64, copy=True)
    ci = np.ascontiguousarray(colind, np.uint32) if len(colind) else np.zeros(1, np.uint32)
    v = np.ascontiguousarray(val, np.float64) if len(val) else np.zeros(1)
    lib().dfm_ref_rmat_spmv(nrow, ncol, brow, bcol, _u(np.ascontiguousarray(rowptr, np.uint32)), _u(ci), _d(v), alpha,
                            _d(np.ascontiguousarray(x, np.float64)), beta, _d(y))
    return y
