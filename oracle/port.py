"""ctypes binding of oracle/_ref/libdfm_oracle.so, the plain-C restatement of
the reference's linear-solve path (oracle/dfm_oracle.c).  TEST INFRASTRUCTURE
ONLY: used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
as the checker, never as the product."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libdfm_oracle.so")
_lib = None

dp, up, ip = C.POINTER(C.c_double), C.POINTER(C.c_uint), C.POINTER(C.c_int)


def build():
    r = subprocess.run(["make", "-s", "-C", HERE, "port"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "dfm_oracle.c")
        if not os.path.exists(LIB_PATH) or (os.path.exists(src) and os.path.getmtime(src) > os.path.getmtime(LIB_PATH)):
            build()
        L = C.CDLL(LIB_PATH)
        U, D = C.c_uint, C.c_double
        L.dfo_pattern.argtypes = [C.c_int, C.c_int, C.c_int, ip, up, up, up]
        L.dfo_diaind.argtypes = [U, up, up, up]
        L.dfo_levels_fwd.argtypes = [U, up, up, up, up]
        L.dfo_levels_fwd.restype = U
        L.dfo_levels_bwd.argtypes = [U, up, up, up, up]
        L.dfo_levels_bwd.restype = U
        L.dfo_asm_poisson_tri.argtypes = [up, up, C.c_int, ip, dp, D, D, dp, dp, dp, dp, dp]
        L.dfo_asm_solid2d_tri.argtypes = [up, up, C.c_int, ip, dp, D, D, D, D, D, dp, dp, dp, dp, dp]
        L.dfo_asm_solid3d_tet.argtypes = [up, up, C.c_int, ip, dp, D, D, D, D, D, D, dp, dp, dp, dp]
        L.dfo_asm_helmholtz_tri.argtypes = [up, up, C.c_int, ip, dp, D, dp, dp, dp, dp]
        L.dfo_asm_sommerfeld_bar.argtypes = [up, up, C.c_int, ip, dp, D, dp, dp, dp, dp]
        L.dfo_apply_bc.argtypes = [U, U, up, up, ip, dp, dp, dp]
        L.dfo_spmv.argtypes = [U, U, up, up, dp, dp, D, dp, D, dp]
        L.dfo_ilu0.argtypes = [U, U, up, up, up, dp, dp]
        L.dfo_ilu0.restype = U
        L.dfo_fwd.argtypes = [U, U, up, up, up, dp, dp, dp]
        L.dfo_bwd.argtypes = [U, U, up, up, up, dp, dp]
        L.dfo_pcg.argtypes = [U, U, up, up, up, dp, dp, dp, dp, dp, dp, D, U, up, dp, dp]
        L.dfo_iluk_pattern.argtypes = [U, up, up, C.c_int, up, C.POINTER(up), C.POINTER(up)]
        L.dfo_iluk_pattern_rows.argtypes = [U, up, up, C.c_int, U, up, U, up, C.POINTER(up), C.POINTER(up)]
        L.dfo_free.argtypes = [C.c_void_p]
        L.dfo_iluk_init.argtypes = [U, U, up, up, dp, dp, up, up, dp, dp]
        L.dfo_pcg_fill.argtypes = [U, U, up, up, dp, dp, up, up, up, dp, dp, dp, dp, D, U, up, dp, dp]
        L.dfo_pbicgstab.argtypes = [U, U, up, up, up, dp, dp, dp, dp, dp, dp, D, U, up, dp]
        L.dfo_cg.argtypes = [U, U, up, up, dp, dp, dp, dp, D, U, up, dp]
        L.dfo_ziluk_init.argtypes = [U, up, up, dp, dp, up, up, dp, dp]
        L.dfo_pcocg_fill.argtypes = [U, up, up, dp, dp, up, up, up, dp, dp, dp, dp, D, U, up, dp]
        L.dfo_rmat_spmv.argtypes = [U, U, U, up, up, dp, D, dp, D, dp]
        L.dfo_mat_zero_rows.argtypes = [U, U, up, ip, dp, dp]
        L.dfo_newmark_residual.argtypes = [U, U, up, up, dp, dp, C.c_int, D, D, D, dp, dp, dp, dp, ip, dp, dp, dp]
        L.dfo_newmark_update.argtypes = [C.c_size_t, C.c_int, D, D, D, ip, dp, dp, dp, dp]
        L.dfo_zspmv.argtypes = [U, up, up, dp, dp, D, dp, D, dp]
        L.dfo_zilu0.argtypes = [U, up, up, up, dp, dp]
        L.dfo_zilu0.restype = U
        L.dfo_zfwdbwd.argtypes = [U, up, up, up, dp, dp, dp]
        L.dfo_pcocg.argtypes = [U, up, up, up, dp, dp, dp, dp, dp, dp, D, U, up, dp]
        _lib = L
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(dp)


def _u(a):
    return a.ctypes.data_as(up)


def _i(a):
    return None if a is None else a.ctypes.data_as(ip)


def _dz(a):
    """pointer to a (possibly empty) float64 array; empty arrays get a dummy."""
    if a is None:
        return None
    if a.size == 0:
        a = np.zeros(1)
    return a.ctypes.data_as(dp)


def pattern(nnode, elem):
    elem = np.ascontiguousarray(elem, dtype=np.int32)
    n = C.c_uint()
    L = lib()
    L.dfo_pattern(nnode, elem.shape[1], elem.shape[0], _i(elem), None, None, C.byref(n))
    rp = np.zeros(nnode + 1, np.uint32)
    ci = np.zeros(max(n.value, 1), np.uint32)
    L.dfo_pattern(nnode, elem.shape[1], elem.shape[0], _i(elem), _u(rp), _u(ci), C.byref(n))
    return rp, ci[: n.value]


def diaind(rowptr, colind):
    N = rowptr.size - 1
    d = np.zeros(max(N, 1), np.uint32)
    ci = colind if colind.size else np.zeros(1, np.uint32)
    lib().dfo_diaind(N, _u(rowptr), _u(ci), _u(d))
    return d[:N]


def iluk_pattern(rowptr, colind, lev_fill, rows=None, bound=None):
    """ILU(k) fill pattern (CMatDiaFrac_BlkCrs::AddFracPtn): (frowptr, fcolind, flev).
    rows: block rows with unlimited fill (AddFracPtn(lev, aBlkFill), the
    SetFillBlk list), acting on pairs of rows below bound (default: all)."""
    rowptr = np.ascontiguousarray(rowptr, np.uint32)
    colind = np.ascontiguousarray(colind, np.uint32)
    N = rowptr.size - 1
    fr = np.zeros(N + 1, np.uint32)
    pc, pl = C.POINTER(C.c_uint)(), C.POINTER(C.c_uint)()
    rw = np.ascontiguousarray(rows if rows is not None else [], np.uint32)
    rc = lib().dfo_iluk_pattern_rows(N, _u(rowptr), _u(colind if colind.size else np.zeros(1, np.uint32)),
                                     int(lev_fill), rw.size, _u(rw if rw.size else np.zeros(1, np.uint32)),
                                     N if bound is None else int(bound), _u(fr), C.byref(pc), C.byref(pl))
    if rc:
        raise ValueError("fill rows out of range")
    n = int(fr[-1])
    fc = np.ctypeslib.as_array(pc, shape=(max(n, 1),))[:n].copy()
    fl = np.ctypeslib.as_array(pl, shape=(max(n, 1),))[:n].copy()
    lib().dfo_free(C.cast(pc, C.c_void_p))
    lib().dfo_free(C.cast(pl, C.c_void_p))
    return fr, fc, fl


def levels(rowptr, colind, dia):
    N = rowptr.size - 1
    ci = colind if colind.size else np.zeros(1, np.uint32)
    lf = np.zeros(max(N, 1), np.uint32)
    lb = np.zeros(max(N, 1), np.uint32)
    nf = lib().dfo_levels_fwd(N, _u(rowptr), _u(ci), _u(dia), _u(lf))
    nb = lib().dfo_levels_bwd(N, _u(rowptr), _u(ci), _u(dia), _u(lb))
    return lf[:N], nf, lb[:N], nb


class System:
    """Block-CRS system (pattern, values) in the reference layout."""

    def __init__(self, rowptr, colind, b, cplx=False):
        self.rowptr = np.ascontiguousarray(rowptr, np.uint32)
        self.colind = np.ascontiguousarray(colind, np.uint32)
        self._ci = self.colind if self.colind.size else np.zeros(1, np.uint32)
        self.N = self.rowptr.size - 1
        self.ncrs = self.colind.size
        self.b = b
        self.cplx = cplx
        self.vw = 2 if cplx else b * b
        self.xw = 2 if cplx else b
        self.dia = diaind(self.rowptr, self.colind)
        self.diag = np.zeros(self.N * self.vw)
        self.off = np.zeros(self.ncrs * self.vw)
        self.rhs = np.zeros(self.N * self.xw)

    def zero(self):
        self.diag[:] = 0
        self.off[:] = 0
        self.rhs[:] = 0

    def asm_poisson(self, mesh, alpha, source, coef=None, u=None):
        e = np.ascontiguousarray(mesh.elem, np.int32)
        c = np.ascontiguousarray(mesh.coord, np.float64)
        cf = None if coef is None else np.ascontiguousarray(coef, np.float64)
        lib().dfo_asm_poisson_tri(_u(self.rowptr), _u(self._ci), e.shape[0], _i(e), _d(c), alpha, source,
                                  _d(cf), _d(u), _d(self.diag), _dz(self.off), _d(self.rhs))

    def asm_solid2d(self, mesh, lam, myu, rho, gx, gy, coef=None, u=None):
        e = np.ascontiguousarray(mesh.elem, np.int32)
        c = np.ascontiguousarray(mesh.coord, np.float64)
        cf = None if coef is None else np.ascontiguousarray(coef, np.float64)
        lib().dfo_asm_solid2d_tri(_u(self.rowptr), _u(self._ci), e.shape[0], _i(e), _d(c), lam, myu, rho, gx, gy,
                                  _d(cf), _d(u), _d(self.diag), _dz(self.off), _d(self.rhs))

    def asm_solid3d(self, mesh, lam, myu, rho, gx, gy, gz, u=None):
        e = np.ascontiguousarray(mesh.elem, np.int32)
        c = np.ascontiguousarray(mesh.coord, np.float64)
        lib().dfo_asm_solid3d_tet(_u(self.rowptr), _u(self._ci), e.shape[0], _i(e), _d(c), lam, myu, rho, gx, gy, gz,
                                  _d(u), _d(self.diag), _dz(self.off), _d(self.rhs))

    def asm_helmholtz(self, mesh, wave_length, u=None):
        e = np.ascontiguousarray(mesh.elem, np.int32)
        c = np.ascontiguousarray(mesh.coord, np.float64)
        lib().dfo_asm_helmholtz_tri(_u(self.rowptr), _u(self._ci), e.shape[0], _i(e), _d(c), wave_length,
                                    _d(u), _d(self.diag), _dz(self.off), _d(self.rhs))
        if mesh.bnd.size:
            bb = np.ascontiguousarray(mesh.bnd, np.int32)
            lib().dfo_asm_sommerfeld_bar(_u(self.rowptr), _u(self._ci), bb.shape[0], _i(bb), _d(c), wave_length,
                                         _d(u), _d(self.diag), _dz(self.off), _d(self.rhs))

    def apply_bc(self, flags):
        f = np.ascontiguousarray(flags, np.int32)
        lib().dfo_apply_bc(self.N, self.b, _u(self.rowptr), _u(self._ci), _i(f), _d(self.diag), _dz(self.off),
                           _d(self.rhs))

    def spmv(self, alpha, x, beta, y, diag=None, off=None):
        y = np.array(y, dtype=np.float64, copy=True)
        x = np.ascontiguousarray(x, np.float64)
        d = self.diag if diag is None else diag
        o = self.off if off is None else off
        if self.cplx:
            lib().dfo_zspmv(self.N, _u(self.rowptr), _u(self._ci), _d(d), _dz(o), alpha, _d(x), beta, _d(y))
        else:
            lib().dfo_spmv(self.N, self.b, _u(self.rowptr), _u(self._ci), _d(d), _dz(o), alpha, _d(x), beta, _d(y))
        return y

    def ilu0(self):
        fd = self.diag.copy()
        fo = self.off.copy()
        if self.cplx:
            ns = lib().dfo_zilu0(self.N, _u(self.rowptr), _u(self._ci), _u(self.dia), _d(fd), _dz(fo))
        else:
            ns = lib().dfo_ilu0(self.N, self.b, _u(self.rowptr), _u(self._ci), _u(self.dia), _d(fd), _dz(fo))
        return int(ns), fd, fo

    def iluk(self, lev_fill, rows=None):
        """ILU(lev_fill): fill pattern, SetValue_Initialize, DoILUDecomp on it.
        rows: the SetFillBlk list (unlimited fill through those block rows).
        Returns (ns, fpat, fd, fo) with fpat = (frowptr, fcolind, fdiaind)."""
        fr, fc, _ = iluk_pattern(self.rowptr, self.colind, lev_fill, rows)
        fdia = diaind(fr, fc)
        if self.cplx:  # CZMatDiaFrac_BlkCrs(lev, A): the same fill pattern, complex values
            fd = np.zeros_like(self.diag)
            fo = np.zeros(max(fc.size, 1) * 2)
            fcz = fc if fc.size else np.zeros(1, np.uint32)
            lib().dfo_ziluk_init(self.N, _u(self.rowptr), _u(self._ci), _d(self.diag), _dz(self.off), _u(fr),
                                 _u(fcz), _d(fd), _d(fo))
            ns = lib().dfo_zilu0(self.N, _u(fr), _u(fcz), _u(fdia), _d(fd), _d(fo))
            return int(ns), (fr, fc, fdia), fd, fo[: fc.size * 2]
        fd = np.zeros_like(self.diag)
        fo = np.zeros(max(fc.size, 1) * self.b * self.b)
        fcz = fc if fc.size else np.zeros(1, np.uint32)
        lib().dfo_iluk_init(self.N, self.b, _u(self.rowptr), _u(self._ci), _d(self.diag), _dz(self.off), _u(fr),
                            _u(fcz), _d(fd), _d(fo))
        ns = lib().dfo_ilu0(self.N, self.b, _u(fr), _u(fcz), _u(fdia), _d(fd), _d(fo))
        return int(ns), (fr, fc, fdia), fd, fo[: fc.size * self.b * self.b]

    def solve_fill(self, fpat, fd, fo, rhs=None, tol=1e-10, maxit=10000):
        """Solve_PCG (Solve_PCOCG for complex systems) with a factor in its own
        pattern fpat = (frowptr, fcolind, fdiaind)."""
        fr, fc, fdia = fpat
        r = np.array(self.rhs if rhs is None else rhs, dtype=np.float64, copy=True)
        x = np.zeros_like(r)
        it, conv = C.c_uint(), C.c_double()
        fcz = fc if fc.size else np.zeros(1, np.uint32)
        if self.cplx:
            ok = lib().dfo_pcocg_fill(self.N, _u(self.rowptr), _u(self._ci), _d(self.diag), _dz(self.off), _u(fr),
                                      _u(fcz), _u(fdia), _d(fd), _dz(fo), _d(r), _d(x), tol, maxit, C.byref(it),
                                      C.byref(conv))
            return dict(ok=bool(ok), x=x, iters=it.value, conv=conv.value, r=r)
        ok = lib().dfo_pcg_fill(self.N, self.b, _u(self.rowptr), _u(self._ci), _d(self.diag), _dz(self.off),
                                _u(fr), _u(fcz), _u(fdia), _d(fd), _dz(fo), _d(r), _d(x), tol, maxit,
                                C.byref(it), C.byref(conv), None)
        return dict(ok=bool(ok), x=x, iters=it.value, conv=conv.value, r=r)

    def solve_cg(self, rhs=None, tol=1e-10, maxit=10000):
        """Solve_CG (no preconditioner) from x = 0."""
        r = np.array(self.rhs if rhs is None else rhs, dtype=np.float64, copy=True)
        x = np.zeros_like(r)
        it, conv = C.c_uint(), C.c_double()
        ok = lib().dfo_cg(self.N, self.b, _u(self.rowptr), _u(self._ci), _d(self.diag), _dz(self.off), _d(r),
                          _d(x), tol, maxit, C.byref(it), C.byref(conv))
        return dict(ok=bool(ok), x=x, iters=it.value, conv=conv.value, r=r)

    def fwd(self, fd, fo, v):
        v = np.array(v, dtype=np.float64, copy=True)
        lib().dfo_fwd(self.N, self.b, _u(self.rowptr), _u(self._ci), _u(self.dia), _d(fd), _dz(fo), _d(v))
        return v

    def bwd(self, fo, v):
        v = np.array(v, dtype=np.float64, copy=True)
        lib().dfo_bwd(self.N, self.b, _u(self.rowptr), _u(self._ci), _u(self.dia), _dz(fo), _d(v))
        return v

    def precond_fill(self, fpat, fd, fo, v):
        """The ILU(k) preconditioner with a factor in its own pattern."""
        fr, fc, fdia = fpat
        fcz = fc if fc.size else np.zeros(1, np.uint32)
        v = np.array(v, dtype=np.float64, copy=True)
        if self.cplx:
            lib().dfo_zfwdbwd(self.N, _u(fr), _u(fcz), _u(fdia), _d(fd), _dz(fo), _d(v))
            return v
        lib().dfo_fwd(self.N, self.b, _u(fr), _u(fcz), _u(fdia), _d(fd), _dz(fo), _d(v))
        lib().dfo_bwd(self.N, self.b, _u(fr), _u(fcz), _u(fdia), _dz(fo), _d(v))
        return v

    def precond(self, fd, fo, v):
        if self.cplx:
            v = np.array(v, dtype=np.float64, copy=True)
            lib().dfo_zfwdbwd(self.N, _u(self.rowptr), _u(self._ci), _u(self.dia), _d(fd), _dz(fo), _d(v))
            return v
        return self.bwd(fo, self.fwd(fd, fo, v))

    def solve(self, fd, fo, rhs=None, method="pcg", tol=1e-10, maxit=10000, hist=False):
        r = np.array(self.rhs if rhs is None else rhs, dtype=np.float64, copy=True)
        x = np.zeros_like(r)
        it, conv = C.c_uint(), C.c_double()
        h = np.zeros(maxit) if hist else None
        args = (_u(self.rowptr), _u(self._ci), _u(self.dia))
        if method == "pcocg":
            ok = lib().dfo_pcocg(self.N, *args, _d(self.diag), _dz(self.off), _d(fd), _dz(fo), _d(r), _d(x), tol,
                                 maxit, C.byref(it), C.byref(conv))
        elif method == "pbicgstab":
            ok = lib().dfo_pbicgstab(self.N, self.b, *args, _d(self.diag), _dz(self.off), _d(fd), _dz(fo), _d(r),
                                     _d(x), tol, maxit, C.byref(it), C.byref(conv))
        else:
            ok = lib().dfo_pcg(self.N, self.b, *args, _d(self.diag), _dz(self.off), _d(fd), _dz(fo), _d(r), _d(x),
                               tol, maxit, C.byref(it), C.byref(conv), _d(h))
        out = dict(ok=bool(ok), x=x, iters=it.value, conv=conv.value, r=r)
        if hist:
            out["hist"] = h[: min(maxit, it.value + 1)]
        return out


def bc_flags_from_bnd(nnode, b, bnd):
    """Dirichlet flags of all DOFs of the nodes of the boundary elements."""
    f = np.zeros((nnode, b), np.int32)
    if bnd.size:
        f[np.unique(bnd.ravel())] = 1
    return f.ravel()


def mat_zero_rows(N, b, rowptr, flags, diag, off):
    """CMat_BlkCrs::SetBoundaryCondition_Row on copies of (diag, off)."""
    d, o = np.array(diag, np.float64, copy=True), np.array(off, np.float64, copy=True)
    fl = np.ascontiguousarray(flags, np.int32)
    lib().dfo_mat_zero_rows(N, b, _u(np.ascontiguousarray(rowptr, np.uint32)), fl.ctypes.data_as(ip), _d(d), _dz(o))
    return d, o


def newmark_residual(N, b, rowptr, colind, diag, off, scheme, dt, gamma, beta, force, u, v, a, flags):
    """MakeResidual of the Newmark stored systems: (r, |r|)."""
    n = N * b
    t, r, nrm = np.zeros(n), np.zeros(n), C.c_double()
    a = np.zeros(n) if a is None else np.ascontiguousarray(a, np.float64)
    ci = np.ascontiguousarray(colind, np.uint32)
    fl = np.ascontiguousarray(flags, np.int32)
    lib().dfo_newmark_residual(N, b, _u(np.ascontiguousarray(rowptr, np.uint32)), _u(ci if ci.size else
                               np.zeros(1, np.uint32)), _d(np.ascontiguousarray(diag, np.float64)),
                               _dz(np.ascontiguousarray(off, np.float64)), scheme, dt, gamma, beta,
                               _d(np.ascontiguousarray(force, np.float64)), _d(np.ascontiguousarray(u, np.float64)),
                               _d(np.ascontiguousarray(v, np.float64)), _d(a), fl.ctypes.data_as(ip), _d(t), _d(r),
                               C.byref(nrm))
    return r, nrm.value


def newmark_update(scheme, dt, gamma, beta, flags, x, u, v, a=None):
    """UpdateValueOfField of the Newmark stored systems on copies: (x, u, v, a)."""
    x, u, v = (np.array(t, np.float64, copy=True) for t in (x, u, v))
    a = np.zeros_like(u) if a is None else np.array(a, np.float64, copy=True)
    fl = np.ascontiguousarray(flags, np.int32)
    lib().dfo_newmark_update(u.size, scheme, dt, gamma, beta, fl.ctypes.data_as(ip), _d(x), _d(u), _d(v), _d(a))
    return x, u, v, a


def rmat_spmv(nrow, brow, bcol, rowptr, colind, val, alpha, x, beta, y):
    """CMat_BlkCrs::MatVec restated: returns the new y."""
    y = np.array(y, np.float64, copy=True)
    ci = np.ascontiguousarray(colind, np.uint32) if len(colind) else np.zeros(1, np.uint32)
    lib().dfo_rmat_spmv(nrow, brow, bcol, _u(np.ascontiguousarray(rowptr, np.uint32)), _u(ci),
                        _dz(np.ascontiguousarray(val, np.float64)), alpha, _d(np.ascontiguousarray(x, np.float64)),
                        beta, _d(y))
    return y
