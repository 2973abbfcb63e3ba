"""ctypes binding of the C ABI (include/dfm_b200.h) and thin Python handles.

The CUDA library is required: importing works without it, but every call that
needs it raises if delfem_b200/_lib/libdfm_b200.so is missing or no CUDA device
is visible.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libdfm_b200.so")

(OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, NOT_CONVERGED, BREAKDOWN, SINGULAR_PIVOT, WAIT_TIMEOUT, ERR_UNSUPPORTED,
 ERR_IO) = range(10)
REAL, COMPLEX = 0, 1
HOST, DEVICE = 0, 1
PCG, PBICGSTAB, PCOCG, PCG_MIXED, PCOCG_MIXED, CG = 0, 1, 2, 3, 4, 5

_lib = None

_vp, _u, _i, _d = C.c_void_p, C.c_uint, C.c_int, C.c_double
_up, _dp, _ip = C.POINTER(C.c_uint), C.POINTER(C.c_double), C.POINTER(C.c_int)

# name -> (restype, argtypes); every symbol declared in include/dfm_b200.h
PROTOS = {
    "dfm_status_string": (C.c_char_p, [_i]),
    "dfm_abi_version": (_i, []),
    "dfm_ctx_create": (_i, [_i, C.POINTER(_vp)]),
    "dfm_ctx_destroy": (_i, [_vp]),
    "dfm_ctx_set_stream": (_i, [_vp, _vp]),
    "dfm_ctx_sync": (_i, [_vp]),
    "dfm_ctx_set_wait_limit": (_i, [_vp, C.c_ulonglong]),
    "dfm_ctx_set_mixed_operator": (_i, [_vp, _i]),
    "dfm_ctx_get_mixed_operator": (_i, [_vp, _ip]),
    "dfm_ctx_take_error": (_i, [_vp, _ip, _ip]),
    "dfm_ctx_wait_selftest": (_i, [_vp, C.c_ulonglong]),
    "dfm_buf_alloc": (_i, [_vp, C.c_size_t, C.POINTER(_vp)]),
    "dfm_buf_free": (_i, [_vp, _vp]),
    "dfm_buf_copy": (_i, [_vp, _vp, _vp, C.c_size_t, _i]),
    "dfm_buf_zero": (_i, [_vp, _vp, C.c_size_t]),
    "dfm_vec_dot": (_i, [_vp, C.c_size_t, _vp, _vp, _dp]),
    "dfm_vec_copy": (_i, [_vp, C.c_size_t, _vp, _vp]),
    "dfm_vec_scal": (_i, [_vp, C.c_size_t, _d, _vp]),
    "dfm_vec_axpy": (_i, [_vp, C.c_size_t, _d, _vp, _vp]),
    "dfm_vec_gather": (_i, [_vp, C.c_size_t, _u, _vp, _vp, _vp]),
    "dfm_mat_create": (_i, [_vp, _u, _u, _i, _up, _up, C.POINTER(_vp)]),
    "dfm_mat_destroy": (_i, [_vp]),
    "dfm_mat_info": (_i, [_vp, _up, _up, _up, _ip]),
    "dfm_mat_set_zero": (_i, [_vp]),
    "dfm_mat_set_values": (_i, [_vp, _vp, _vp, _i]),
    "dfm_mat_get_values": (_i, [_vp, _vp, _vp, _i]),
    "dfm_mat_values_device": (_i, [_vp, C.POINTER(_vp), C.POINTER(_vp)]),
    "dfm_mat_set_spmv_lanes": (_i, [_vp, _i]),
    "dfm_mat_get_spmv_lanes": (_i, [_vp, _ip]),
    "dfm_mat_set_spmv_kernel": (_i, [_vp, _i]),
    "dfm_mat_get_spmv_kernel": (_i, [_vp, _ip]),
    "dfm_spmv": (_i, [_vp, _d, _vp, _d, _vp]),
    "dfm_time_spmv": (_i, [_vp, _vp, _vp, _i, C.POINTER(C.c_float)]),
    "dfm_zmat_read_text": (_i, [C.c_char_p, _up, _up, _up, _up, _dp, _dp]),
    "dfm_gid_read_mesh": (_i, [C.c_char_p, _ip, _up, _dp, _ip, _up, _ip]),
    "dfm_last_cuda_error": (_i, [C.c_char_p, C.c_size_t]),
    "dfm_gid_boundary": (_i, [_i, _u, _dp, _i, _u, _ip, _d, _ip, _up, _up, _up, _up, _up, _up, _up, _up]),
    "dfm_mat_zero_rows": (_i, [_vp, _vp]),
    "dfm_rmat_create": (_i, [_vp, _u, _u, _u, _u, _up, _up, C.POINTER(_vp)]),
    "dfm_rmat_destroy": (_i, [_vp]),
    "dfm_rmat_set_values": (_i, [_vp, _vp, _i]),
    "dfm_rmat_spmv": (_i, [_vp, _d, _vp, _d, _vp]),
    "dfm_newmark_residual": (_i, [_vp, _i, _d, _d, _d, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _dp]),
    "dfm_newmark_update": (_i, [_vp, C.c_size_t, _i, _d, _d, _d, _vp, _vp, _vp, _vp, _vp]),
    "dfm_boundary_matrix": (_i, [_u, _u, _up, _up, _dp, _dp, _ip, _up, _up, _dp, _dp, _up]),
    "dfm_mesh_create": (_i, [_vp, _i, _u, _dp, _u, _u, _ip, _u, _ip, C.POINTER(_vp)]),
    "dfm_mesh_destroy": (_i, [_vp]),
    "dfm_mesh_pattern": (_i, [_vp, _up, _up, C.POINTER(C.c_size_t)]),
    "dfm_assemble_poisson2d": (_i, [_vp, _vp, _d, _d, _vp, _vp, _vp, _vp]),
    "dfm_assemble_solid2d": (_i, [_vp, _vp, _d, _d, _d, _d, _d, _vp, _vp, _vp, _vp]),
    "dfm_assemble_solid3d": (_i, [_vp, _vp, _d, _d, _d, _d, _d, _d, _vp, _vp, _vp]),
    "dfm_assemble_helmholtz2d": (_i, [_vp, _vp, _d, _vp, _vp, _vp]),
    "dfm_apply_dirichlet": (_i, [_vp, _vp, _vp]),
    "dfm_coef_grad_poisson2d": (_i, [_vp, _d, _vp, _vp, _vp]),
    "dfm_coef_grad_solid2d": (_i, [_vp, _d, _d, _vp, _vp, _vp]),
    "dfm_ilu_create": (_i, [_vp, C.POINTER(_vp)]),
    "dfm_ilu_create_fill": (_i, [_vp, _i, C.POINTER(_vp)]),
    "dfm_ilu_create_fill_rows": (_i, [_vp, _i, _up, C.c_size_t, C.c_uint, C.POINTER(_vp)]),
    "dfm_ilu_pattern": (_i, [_vp, _up, _up, _up]),
    "dfm_ilu_destroy": (_i, [_vp]),
    "dfm_ilu_levels": (_i, [_vp, _up, _up, _up, _up]),
    "dfm_ilu_factor": (_i, [_vp, _vp, _up]),
    "dfm_ilu_get_values": (_i, [_vp, _vp, _vp, _i]),
    "dfm_ilu_set_values": (_i, [_vp, _vp, _vp, _i]),
    "dfm_ilu_apply": (_i, [_vp, _vp, _vp]),
    "dfm_time_ilu_apply": (_i, [_vp, _vp, _vp, _i, C.POINTER(C.c_float)]),
    "dfm_ilu_apply_static": (_i, [_vp, _vp, _vp]),
    "dfm_ilu_set_sweep": (_i, [_vp, _i]),
    "dfm_ilu_get_sweep": (_i, [_vp, _ip]),
    "dfm_ilu_set_sweep_warps": (_i, [_vp, _i, _i, _i]),
    "dfm_ilu_get_sweep_warps": (_i, [_vp, _ip, _ip, _ip]),
    "dfm_ilu_set_sweep_tuning": (_i, [_vp, _i, _u]),
    "dfm_ilu_set_sweep_partition": (_i, [_vp, _up, _u]),
    "dfm_sweep_partition_patches": (_i, [_u, _i, _dp, _u, _up, _up]),
    "dfm_solve_pcg": (_i, [_vp, _vp, _vp, _vp, _d, _u, _up, _dp]),
    "dfm_solve_cg": (_i, [_vp, _vp, _vp, _d, _u, _up, _dp]),
    "dfm_solve_pbicgstab": (_i, [_vp, _vp, _vp, _vp, _d, _u, _up, _dp]),
    "dfm_solve_pcocg": (_i, [_vp, _vp, _vp, _vp, _d, _u, _up, _dp]),
    "dfm_solve_pcg_mixed": (_i, [_vp, _vp, _vp, _vp, _d, _u, _up, _dp]),
    "dfm_solve_pcocg_mixed": (_i, [_vp, _vp, _vp, _vp, _d, _u, _up, _dp]),
    "dfm_batch_create": (_i, [_vp, _u, _up, C.POINTER(_vp)]),
    "dfm_batch_destroy": (_i, [_vp]),
    "dfm_batch_set_tuning": (_i, [_vp, _i, _i]),
    "dfm_batch_get_tuning": (_i, [_vp, _ip, _ip]),
    "dfm_batch_set_schedule": (_i, [_vp, _i, _i, _i]),
    "dfm_batch_get_schedule": (_i, [_vp, _ip, _ip, _ip]),
    "dfm_batch_solve_pcg": (_i, [_vp, _vp, _i, _vp, _i, _d, _u, _up, _dp, _ip]),
    "dfm_solve_host": (_i, [_vp, _vp, _i, _vp, _vp, _d, _u, _up, _dp]),
    "dfm_solve_pcg_host": (_i, [_vp, _vp, _vp, _vp, _d, _u, _up, _dp]),
}


class DfmError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        msg = lib().dfm_status_string(code).decode() if _lib is not None else str(code)
        if _lib is not None and code in (ERR_CUDA, ERR_NOMEM):  # the runtime call and its error
            buf = C.create_string_buffer(256)
            if _lib.dfm_last_cuda_error(buf, 256):
                msg += f" [{buf.value.decode(errors='replace')}]"
        super().__init__(f"{where}: {msg} ({code})")


def load(path: str = LIB_PATH):
    """Load the shared library (no GPU needed for loading)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing; build it with `python -m delfem_b200.build`")
        L = C.CDLL(path)
        for name, (res, args) in PROTOS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def lib():
    return load()


def check(rc: int, where: str = "", allow=(OK,)):
    if rc not in allow:
        raise DfmError(rc, where)
    return rc


def _ptr(t):
    """Device (or host) address of a torch tensor / numpy array."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return C.c_void_p(t.data_ptr())
    return t.ctypes.data_as(C.c_void_p)


def _sync_torch():
    """Order the caller's torch work (default stream) before a library call,
    which runs on the context's own stream."""
    import torch
    if torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.current_stream().synchronize()


def _require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("delfem_b200 needs a CUDA device (no CPU fallback)")
    return torch


class Context:
    def __init__(self, device: int = 0, use_torch_stream: bool = False):
        torch = _require_cuda()
        self.device = device
        h = C.c_void_p()
        check(lib().dfm_ctx_create(device, C.byref(h)), "dfm_ctx_create")
        self.h = h
        if use_torch_stream:
            s = torch.cuda.current_stream(device).cuda_stream
            check(lib().dfm_ctx_set_stream(self.h, C.c_void_p(s)), "dfm_ctx_set_stream")

    def close(self):
        if getattr(self, "h", None):
            lib().dfm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        check(lib().dfm_ctx_sync(self.h), "dfm_ctx_sync")

    def take_error(self):
        code, where = C.c_int(), C.c_int()
        check(lib().dfm_ctx_take_error(self.h, C.byref(code), C.byref(where)))
        return code.value, where.value

    def set_wait_limit(self, ns: int):
        check(lib().dfm_ctx_set_wait_limit(self.h, ns))

    def wait_selftest(self, ns: int) -> int:
        return lib().dfm_ctx_wait_selftest(self.h, ns)

    @property
    def mixed_operator(self) -> int:
        """Operator values of the mixed-precision solves: 0 FP64, 1 FP32."""
        v = C.c_int()
        check(lib().dfm_ctx_get_mixed_operator(self.h, C.byref(v)))
        return v.value

    @mixed_operator.setter
    def mixed_operator(self, fp32: int):
        check(lib().dfm_ctx_set_mixed_operator(self.h, int(fp32)), "dfm_ctx_set_mixed_operator")


class Matrix:
    """MatVec::CMatDia_BlkCrs on the device (reference block-CRS layout)."""

    def __init__(self, ctx: Context, rowptr, colind, b: int, vtype: int = REAL):
        self.ctx = ctx
        rp = np.ascontiguousarray(rowptr, np.uint32)
        ci = np.ascontiguousarray(colind, np.uint32)
        ci_ = ci if ci.size else np.zeros(1, np.uint32)
        h = C.c_void_p()
        check(lib().dfm_mat_create(ctx.h, rp.size - 1, b, vtype, rp.ctypes.data_as(_up), ci_.ctypes.data_as(_up),
                                   C.byref(h)), "dfm_mat_create")
        self.h = h
        self.N, self.b, self.ncrs, self.vtype = rp.size - 1, b, ci.size, vtype
        self.rowptr, self.colind = rp, ci
        self.vw = 2 if vtype == COMPLEX else b * b
        self.xw = 2 if vtype == COMPLEX else b

    def close(self):
        if getattr(self, "h", None):
            lib().dfm_mat_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_values(self, diag, off):
        where = DEVICE if hasattr(diag, "data_ptr") and diag.is_cuda else HOST
        if where == HOST:
            diag = np.ascontiguousarray(diag, np.float64)
            off = np.ascontiguousarray(off, np.float64)
        if where == DEVICE:
            _sync_torch()
        check(lib().dfm_mat_set_values(self.h, _ptr(diag), _ptr(off), where), "dfm_mat_set_values")

    def get_values(self):
        d = np.zeros(self.N * self.vw)
        o = np.zeros(max(self.ncrs, 1) * self.vw)
        check(lib().dfm_mat_get_values(self.h, _ptr(d), _ptr(o), HOST), "dfm_mat_get_values")
        return d, o[: self.ncrs * self.vw]

    def spmv(self, alpha, x, beta, y):
        _sync_torch()
        check(lib().dfm_spmv(self.h, alpha, _ptr(x), beta, _ptr(y)), "dfm_spmv")
        return y

    def time_spmv(self, x, y, reps=50):
        """Average seconds per launch of y = A x over `reps` back-to-back launches."""
        _sync_torch()
        ms = C.c_float()
        check(lib().dfm_time_spmv(self.h, _ptr(x), _ptr(y), int(reps), C.byref(ms)), "dfm_time_spmv")
        return ms.value / 1e3

    @property
    def lanes(self):
        v = C.c_int()
        check(lib().dfm_mat_get_spmv_lanes(self.h, C.byref(v)))
        return v.value

    @lanes.setter
    def lanes(self, v):
        check(lib().dfm_mat_set_spmv_lanes(self.h, int(v)))

    @property
    def spmv_kernel(self):
        v = C.c_int()
        check(lib().dfm_mat_get_spmv_kernel(self.h, C.byref(v)))
        return v.value

    @spmv_kernel.setter
    def spmv_kernel(self, v):
        check(lib().dfm_mat_set_spmv_kernel(self.h, int(v)), "dfm_mat_set_spmv_kernel")


class Mesh:
    """A P1 mesh on the device (triangles or tetrahedra, optional boundary bars)
    for the gather assembly kernels."""

    def __init__(self, ctx: Context, coord, elem, bars=None):
        self.ctx = ctx
        coord = np.ascontiguousarray(coord, np.float64)
        elem = np.ascontiguousarray(elem, np.int32)
        ndim = coord.shape[1]
        nnoel = elem.shape[1]
        bars = np.zeros((0, 2), np.int32) if bars is None else np.ascontiguousarray(bars, np.int32).reshape(-1, 2)
        b_ = bars if bars.size else np.zeros((1, 2), np.int32)
        e_ = elem if elem.size else np.zeros((1, nnoel), np.int32)
        h = C.c_void_p()
        check(lib().dfm_mesh_create(ctx.h, ndim, coord.shape[0], coord.ctypes.data_as(_dp), nnoel, elem.shape[0],
                                    e_.ctypes.data_as(_ip), bars.shape[0], b_.ctypes.data_as(_ip), C.byref(h)),
              "dfm_mesh_create")
        self.h = h
        self.ndim, self.nnode, self.nnoel, self.nelem, self.nbar = ndim, coord.shape[0], nnoel, elem.shape[0], \
            bars.shape[0]

    def close(self):
        if getattr(self, "h", None):
            lib().dfm_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pattern(self):
        """(rowptr, colind) of the mesh's block pattern (host numpy uint32)."""
        n = C.c_size_t()
        rp = np.zeros(self.nnode + 1, np.uint32)
        check(lib().dfm_mesh_pattern(self.h, rp.ctypes.data_as(_up), None, C.byref(n)), "dfm_mesh_pattern")
        ci = np.zeros(max(n.value, 1), np.uint32)
        check(lib().dfm_mesh_pattern(self.h, rp.ctypes.data_as(_up), ci.ctypes.data_as(_up), C.byref(n)),
              "dfm_mesh_pattern")
        return rp, ci[: n.value]

    def assemble_poisson(self, A: Matrix, alpha, source, rhs, coef=None, u=None, load=None):
        _sync_torch()
        check(lib().dfm_assemble_poisson2d(self.h, A.h, alpha, source, _ptr(coef), _ptr(u), _ptr(load), _ptr(rhs)),
              "dfm_assemble_poisson2d")
        return rhs

    def assemble_solid2d(self, A: Matrix, lam, myu, rho, gx, gy, rhs, coef=None, u=None, load=None):
        _sync_torch()
        check(lib().dfm_assemble_solid2d(self.h, A.h, lam, myu, rho, gx, gy, _ptr(coef), _ptr(u), _ptr(load),
                                         _ptr(rhs)), "dfm_assemble_solid2d")
        return rhs

    def assemble_solid3d(self, A: Matrix, lam, myu, rho, gx, gy, gz, rhs, u=None, load=None):
        _sync_torch()
        check(lib().dfm_assemble_solid3d(self.h, A.h, lam, myu, rho, gx, gy, gz, _ptr(u), _ptr(load), _ptr(rhs)),
              "dfm_assemble_solid3d")
        return rhs

    def assemble_helmholtz(self, A: Matrix, wave_length, rhs, u=None, load=None):
        _sync_torch()
        check(lib().dfm_assemble_helmholtz2d(self.h, A.h, wave_length, _ptr(u), _ptr(load), _ptr(rhs)),
              "dfm_assemble_helmholtz2d")
        return rhs


def coef_grad_solid2d(G: Mesh, lam_e, myu_e, lam, u, grad):
    _sync_torch()
    check(lib().dfm_coef_grad_solid2d(G.h, lam_e, myu_e, _ptr(lam), _ptr(u), _ptr(grad)), "dfm_coef_grad_solid2d")
    return grad


def coef_grad_poisson2d(G: Mesh, alpha, lam, u, grad):
    _sync_torch()
    check(lib().dfm_coef_grad_poisson2d(G.h, alpha, _ptr(lam), _ptr(u), _ptr(grad)), "dfm_coef_grad_poisson2d")
    return grad


def read_complex_matrix_text(path):
    """The reference's complex matrix text format (CZMatDia_BlkCrs(file_path)):
    (N, rowptr, colind, diag, off) on the host, values interleaved (re, im)."""
    L = lib()
    n, m = C.c_uint(), C.c_uint()
    p = os.fsencode(path)
    check(L.dfm_zmat_read_text(p, C.byref(n), C.byref(m), None, None, None, None), "dfm_zmat_read_text")
    rp = np.zeros(n.value + 1, np.uint32)
    ci = np.zeros(max(m.value, 1), np.uint32)
    d = np.zeros(max(2 * n.value, 1))
    o = np.zeros(max(2 * m.value, 1))
    check(L.dfm_zmat_read_text(p, C.byref(n), C.byref(m), rp.ctypes.data_as(_up), ci.ctypes.data_as(_up),
                               d.ctypes.data_as(_dp), o.ctypes.data_as(_dp)), "dfm_zmat_read_text")
    return n.value, rp, ci[: m.value], d[: 2 * n.value], o[: 2 * m.value]


def sweep_partition_patches(coord, max_parts):
    """(part, nparts): patches across the longest axis of the node coordinates
    (dfm_sweep_partition_patches), for ILU.set_sweep_partition."""
    coord = np.ascontiguousarray(coord, np.float64)
    n, ndim = coord.shape
    part = np.zeros(max(n, 1), np.uint32)
    k = C.c_uint()
    check(lib().dfm_sweep_partition_patches(n, ndim, coord.ctypes.data_as(_dp), int(max_parts),
                                            part.ctypes.data_as(_up), C.byref(k)), "dfm_sweep_partition_patches")
    return part[:n], k.value


def read_gid_mesh(path):
    """A GiD ASCII mesh as the reference reads it (dfm_gid_read_mesh):
    (coord[nnode, ndim], elem[nelem, nnoel]) on the host, elem 0-based."""
    L = lib()
    p = os.fsencode(path)
    nd, nn, ne, no = C.c_int(), C.c_uint(), C.c_uint(), C.c_int()
    check(L.dfm_gid_read_mesh(p, C.byref(nd), C.byref(nn), None, C.byref(no), C.byref(ne), None), "dfm_gid_read_mesh")
    coord = np.zeros((nn.value, nd.value))
    elem = np.zeros((ne.value, no.value), np.int32)
    check(L.dfm_gid_read_mesh(p, C.byref(nd), C.byref(nn), coord.ctypes.data_as(_dp), C.byref(no), C.byref(ne),
                              elem.ctypes.data_as(_ip)), "dfm_gid_read_mesh")
    return coord, elem


def gid_boundary(coord, elem, crt_dot=None):
    """The boundary facets the reference's GiD readers derive from a mesh
    (dfm_gid_boundary): a dict with ``facets`` [nfacet, nnofa] (boundary
    triangles of a tetrahedral mesh, outer bars of a planar one), ``groups``
    (per colour / bar chain, the facet indices in the reference's order),
    ``vertices`` (planar: the chains' end nodes, ascending) and ``ends``
    [ngroup, 2] (planar: each chain's first and last vertex index).
    ``crt_dot`` defaults to the reference's thresholds, 0.2 for the
    triangles' normals and 0.8 for the bars' directions."""
    coord = np.ascontiguousarray(coord, np.float64)
    elem = np.ascontiguousarray(elem, np.int32)
    ndim, nnoel = coord.shape[1], elem.shape[1]
    if crt_dot is None:
        crt_dot = 0.2 if ndim == 3 else 0.8
    L = lib()
    nf, nfa, ng, nv = C.c_int(), C.c_uint(), C.c_uint(), C.c_uint()
    args = (int(ndim), coord.shape[0], coord.ctypes.data_as(_dp), int(nnoel), elem.shape[0], elem.ctypes.data_as(_ip),
            float(crt_dot), C.byref(nf), C.byref(nfa))
    check(L.dfm_gid_boundary(*args, None, C.byref(ng), None, None, C.byref(nv), None, None), "dfm_gid_boundary")
    facet = np.zeros((nfa.value, nf.value), np.uint32)
    gptr = np.zeros(ng.value + 1, np.uint32)
    gfac = np.zeros(max(nfa.value, 1), np.uint32)
    vert = np.zeros(max(nv.value, 1), np.uint32)
    ends = np.zeros((max(ng.value, 1), 2), np.uint32)
    check(L.dfm_gid_boundary(*args, facet.ctypes.data_as(_up), C.byref(ng), gptr.ctypes.data_as(_up),
                             gfac.ctypes.data_as(_up), C.byref(nv), vert.ctypes.data_as(_up),
                             ends.ctypes.data_as(_up)), "dfm_gid_boundary")
    groups = [gfac[gptr[g]:gptr[g + 1]].copy() for g in range(ng.value)]
    return {"facets": facet, "groups": groups, "vertices": vert[:nv.value].copy(),
            "ends": ends[:ng.value].copy() if ndim == 2 else np.zeros((0, 2), np.uint32)}


def boundary_matrix(rowptr, colind, diag, off, flags, b):
    """CLinearSystem_Save's boundary matrix B from K's values before the
    Dirichlet elimination (dfm_boundary_matrix): (brow, bcol, bdiag, boff);
    MakeResidual is then r = Force - B u (Matrix.spmv(-1, u, 1, r))."""
    rowptr = np.ascontiguousarray(rowptr, np.uint32)
    colind = np.ascontiguousarray(colind if np.size(colind) else np.zeros(1), np.uint32)
    diag = np.ascontiguousarray(diag, np.float64)
    off = np.ascontiguousarray(off if np.size(off) else np.zeros(1), np.float64)
    flags = np.ascontiguousarray(flags, np.int32)
    N = rowptr.size - 1
    n = C.c_uint()
    args = (N, b, rowptr.ctypes.data_as(_up), colind.ctypes.data_as(_up), diag.ctypes.data_as(_dp),
            off.ctypes.data_as(_dp), flags.ctypes.data_as(_ip))
    L = lib()
    check(L.dfm_boundary_matrix(*args, None, None, None, None, C.byref(n)), "dfm_boundary_matrix")
    brow = np.zeros(N + 1, np.uint32)
    bcol = np.zeros(max(n.value, 1), np.uint32)
    bdiag = np.zeros(max(N * b * b, 1))
    boff = np.zeros(max(n.value * b * b, 1))
    check(L.dfm_boundary_matrix(*args, brow.ctypes.data_as(_up), bcol.ctypes.data_as(_up), bdiag.ctypes.data_as(_dp),
                                boff.ctypes.data_as(_dp), C.byref(n)), "dfm_boundary_matrix")
    return brow, bcol[: n.value], bdiag[: N * b * b], boff[: n.value * b * b]


def apply_dirichlet(A: Matrix, flags, rhs=None):
    """Dirichlet elimination with device int32 flags[N*b] (nonzero = fixed)."""
    _sync_torch()
    check(lib().dfm_apply_dirichlet(A.h, _ptr(flags), _ptr(rhs)), "dfm_apply_dirichlet")


class ILU:
    """LsSol::CPreconditioner_ILU on the device: ILU(0), or ILU(fill_level)
    (SetFillInLevel; -1 = no limit) with the factor in its own fill pattern.
    fill_rows: the SetFillBlk list (block rows whose fill has no level limit),
    acting on pairs of rows below fill_bound (default N)."""

    def __init__(self, A: Matrix, fill_level: int = 0, fill_rows=None, fill_bound=None):
        self.A = A
        self.fill_level = int(fill_level)
        h = C.c_void_p()
        if fill_rows is not None and len(fill_rows):
            rows = np.ascontiguousarray(fill_rows, np.uint32)
            bound = A.N if fill_bound is None else int(fill_bound)
            check(lib().dfm_ilu_create_fill_rows(A.h, self.fill_level, rows.ctypes.data_as(_up), rows.size, bound,
                                                 C.byref(h)), "dfm_ilu_create_fill_rows")
        elif self.fill_level == 0:
            check(lib().dfm_ilu_create(A.h, C.byref(h)), "dfm_ilu_create")
        else:
            check(lib().dfm_ilu_create_fill(A.h, self.fill_level, C.byref(h)), "dfm_ilu_create_fill")
        self.h = h
        n = C.c_uint()
        check(lib().dfm_ilu_pattern(h, None, None, C.byref(n)), "dfm_ilu_pattern")
        self.ncrs = n.value

    def pattern(self):
        """The factor's pattern (rowptr, colind)."""
        rp = np.zeros(self.A.N + 1, np.uint32)
        ci = np.zeros(max(self.ncrs, 1), np.uint32)
        check(lib().dfm_ilu_pattern(self.h, rp.ctypes.data_as(_up), ci.ctypes.data_as(_up), None),
              "dfm_ilu_pattern")
        return rp, ci[: self.ncrs]

    def close(self):
        if getattr(self, "h", None):
            lib().dfm_ilu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def levels(self):
        nf, nb = C.c_uint(), C.c_uint()
        lf = np.zeros(max(self.A.N, 1), np.uint32)
        lb = np.zeros(max(self.A.N, 1), np.uint32)
        check(lib().dfm_ilu_levels(self.h, C.byref(nf), C.byref(nb), lf.ctypes.data_as(_up),
                                   lb.ctypes.data_as(_up)))
        return lf[: self.A.N], nf.value, lb[: self.A.N], nb.value

    def factor(self, A: Matrix | None = None, allow=(OK,)):
        ns = C.c_uint()
        rc = lib().dfm_ilu_factor(self.h, (A or self.A).h, C.byref(ns))
        check(rc, "dfm_ilu_factor", allow)
        return rc, ns.value

    def get_values(self):
        d = np.zeros(self.A.N * self.A.vw)
        o = np.zeros(max(self.ncrs, 1) * self.A.vw)
        check(lib().dfm_ilu_get_values(self.h, _ptr(d), _ptr(o), HOST), "dfm_ilu_get_values")
        return d, o[: self.ncrs * self.A.vw]

    def set_values(self, diag, off):
        diag = np.ascontiguousarray(diag, np.float64)
        off = np.ascontiguousarray(off if np.size(off) else np.zeros(1), np.float64)
        check(lib().dfm_ilu_set_values(self.h, _ptr(diag), _ptr(off), HOST), "dfm_ilu_set_values")

    def apply(self, r, z):
        _sync_torch()
        check(lib().dfm_ilu_apply(self.h, _ptr(r), _ptr(z)), "dfm_ilu_apply")
        return z

    def set_sweep_partition(self, part=None, nparts=0):
        """Row partition of the range sweeps (part[i] = CTA of row i), or None."""
        if part is None:
            check(lib().dfm_ilu_set_sweep_partition(self.h, None, 0), "dfm_ilu_set_sweep_partition")
            return
        part = np.ascontiguousarray(part, np.uint32)
        check(lib().dfm_ilu_set_sweep_partition(self.h, part.ctypes.data_as(_up), int(nparts)),
              "dfm_ilu_set_sweep_partition")

    def time_apply(self, r, z, reps=20):
        """Average seconds per z = U^-1 L^-1 r over `reps` back-to-back applications."""
        _sync_torch()
        ms = C.c_float()
        check(lib().dfm_time_ilu_apply(self.h, _ptr(r), _ptr(z), int(reps), C.byref(ms)), "dfm_time_ilu_apply")
        return ms.value / 1e3

    @property
    def sweep(self):
        v = C.c_int()
        check(lib().dfm_ilu_get_sweep(self.h, C.byref(v)))
        return v.value

    @sweep.setter
    def sweep(self, v):
        check(lib().dfm_ilu_set_sweep(self.h, int(v)))

    @property
    def sweep_warps(self):
        """(compute warps, lanes per row, producer warps) of schedule 9."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().dfm_ilu_get_sweep_warps(self.h, C.byref(a), C.byref(b), C.byref(c)), "dfm_ilu_get_sweep_warps")
        return a.value, b.value, c.value

    @sweep_warps.setter
    def sweep_warps(self, v):
        check(lib().dfm_ilu_set_sweep_warps(self.h, *(int(t) for t in v)), "dfm_ilu_set_sweep_warps")


class Batch:
    """Many independent systems held as one block-diagonal matrix (see dfm_batch_create)."""

    def __init__(self, M: ILU, row_off):
        self.M = M
        ro = np.ascontiguousarray(row_off, np.uint32)
        self.ninst = ro.size - 1
        self.row_off = ro
        h = C.c_void_p()
        check(lib().dfm_batch_create(M.h, self.ninst, ro.ctypes.data_as(_up), C.byref(h)), "dfm_batch_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().dfm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def tuning(self):
        a, b = C.c_int(), C.c_int()
        check(lib().dfm_batch_get_tuning(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    @tuning.setter
    def tuning(self, v):
        check(lib().dfm_batch_set_tuning(self.h, int(v[0]), int(v[1])), "dfm_batch_set_tuning")

    @property
    def schedule(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().dfm_batch_get_schedule(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    @schedule.setter
    def schedule(self, v):
        v = tuple(v) + (0, 0)
        check(lib().dfm_batch_set_schedule(self.h, int(v[0]), int(v[1]), int(v[2])), "dfm_batch_set_schedule")

    def solve(self, b, x=None, tol=1e-8, maxit=10000, allow=(OK, NOT_CONVERGED)):
        """b, x: device tensors (x written) or host arrays (x returned).  Returns
        (status, x, iters[ninst], conv[ninst], status[ninst])."""
        it = np.zeros(self.ninst, np.uint32)
        cv = np.zeros(self.ninst)
        st = np.zeros(self.ninst, np.int32)
        dev = hasattr(b, "data_ptr")
        if not dev:
            b = np.ascontiguousarray(b, np.float64)
            x = np.zeros_like(b)
        else:
            _sync_torch()
        w = DEVICE if dev else HOST
        rc = lib().dfm_batch_solve_pcg(self.h, _ptr(b), w, _ptr(x), w, tol, maxit, it.ctypes.data_as(_up),
                                       cv.ctypes.data_as(_dp), st.ctypes.data_as(_ip))
        check(rc, "dfm_batch_solve_pcg", allow)
        return rc, x, it, cv, st


def solve_pcg(A: Matrix, M: ILU, r, x, tol=1e-10, maxit=10000, allow=(OK, NOT_CONVERGED)):
    """LsSol::Solve_PCG on device vectors; returns (status, iters, conv)."""
    it, conv = C.c_uint(), C.c_double()
    _sync_torch()
    rc = lib().dfm_solve_pcg(A.h, M.h, _ptr(r), _ptr(x), tol, maxit, C.byref(it), C.byref(conv))
    check(rc, "dfm_solve_pcg", allow)
    return rc, it.value, conv.value


class RMatrix:
    """A rectangular block-CRS matrix on the device (CMat_BlkCrs: a coupling
    of two segments), nrow x ncol blocks of brow x bcol."""

    def __init__(self, ctx: Context, nrow, ncol, brow, bcol, rowptr, colind):
        self.ctx = ctx
        rp = np.ascontiguousarray(rowptr, np.uint32)
        ci = np.ascontiguousarray(colind, np.uint32) if len(colind) else np.zeros(1, np.uint32)
        h = C.c_void_p()
        check(lib().dfm_rmat_create(ctx.h, int(nrow), int(ncol), int(brow), int(bcol), rp.ctypes.data_as(_up),
                                    ci.ctypes.data_as(_up), C.byref(h)), "dfm_rmat_create")
        self.h = h
        self.nrow, self.ncol, self.brow, self.bcol = int(nrow), int(ncol), int(brow), int(bcol)

    def set_values(self, val):
        v = np.ascontiguousarray(val, np.float64)
        check(lib().dfm_rmat_set_values(self.h, v.ctypes.data_as(C.c_void_p), HOST), "dfm_rmat_set_values")

    def spmv(self, alpha, x, beta, y):
        _sync_torch()
        check(lib().dfm_rmat_spmv(self.h, alpha, _ptr(x), beta, _ptr(y)), "dfm_rmat_spmv")

    def close(self):
        if getattr(self, "h", None):
            lib().dfm_rmat_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mat_zero_rows(B: Matrix, flags):
    """CMat_BlkCrs::SetBoundaryCondition_Row: zero the rows of fixed DOFs (device flags)."""
    _sync_torch()
    check(lib().dfm_mat_zero_rows(B.h, _ptr(flags)), "dfm_mat_zero_rows")


def newmark_residual(B: Matrix, scheme, dt, gamma, beta, force, u, v, a, flags, t, r) -> float:
    """MakeResidual of CLinearSystem_SaveDiaM_Newmark (scheme 1) / _NewmarkBeta (2); returns |r|."""
    nrm = C.c_double()
    _sync_torch()
    check(lib().dfm_newmark_residual(B.h, int(scheme), dt, gamma, beta, _ptr(force), _ptr(u), _ptr(v), _ptr(a),
                                     _ptr(flags), _ptr(t), _ptr(r), C.byref(nrm)), "dfm_newmark_residual")
    return nrm.value


def newmark_update(ctx: Context, scheme, dt, gamma, beta, flags, x, u, v, a=None):
    """UpdateValueOfField of the Newmark (1) / Newmark-beta (2) stored systems."""
    _sync_torch()
    check(lib().dfm_newmark_update(ctx.h, x.numel(), int(scheme), dt, gamma, beta, _ptr(flags), _ptr(x), _ptr(u),
                                   _ptr(v), _ptr(a)), "dfm_newmark_update")


def solve_cg(A: Matrix, r, x, tol=1e-10, maxit=10000, allow=(OK, NOT_CONVERGED)):
    """LsSol::Solve_CG (no preconditioner) on device vectors; returns (status, iters, conv)."""
    it, conv = C.c_uint(), C.c_double()
    _sync_torch()
    rc = lib().dfm_solve_cg(A.h, _ptr(r), _ptr(x), tol, maxit, C.byref(it), C.byref(conv))
    check(rc, "dfm_solve_cg", allow)
    return rc, it.value, conv.value


def vec_dot(ctx: Context, x, y) -> float:
    """CVector_Blk dot product of two device vectors (deterministic)."""
    out = C.c_double()
    _sync_torch()
    check(lib().dfm_vec_dot(ctx.h, x.numel(), _ptr(x), _ptr(y), C.byref(out)), "dfm_vec_dot")
    return out.value


def vec_gather(ctx, b, idx, x, y):
    """y[i b + c] := x[idx[i] b + c] (dfm_vec_gather): idx a device uint32
    tensor of block indices, x and y device float64 tensors."""
    _sync_torch()
    check(lib().dfm_vec_gather(ctx.h, idx.numel(), int(b), _ptr(idx), _ptr(x), _ptr(y)), "dfm_vec_gather")


def vec_axpy(ctx: Context, alpha: float, x, y):
    """y += alpha x on the context's stream."""
    _sync_torch()
    check(lib().dfm_vec_axpy(ctx.h, x.numel(), alpha, _ptr(x), _ptr(y)), "dfm_vec_axpy")


def vec_scal(ctx: Context, alpha: float, x):
    """x *= alpha on the context's stream."""
    _sync_torch()
    check(lib().dfm_vec_scal(ctx.h, x.numel(), alpha, _ptr(x)), "dfm_vec_scal")


def vec_copy(ctx: Context, x, y):
    """y := x on the context's stream."""
    _sync_torch()
    check(lib().dfm_vec_copy(ctx.h, x.numel(), _ptr(x), _ptr(y)), "dfm_vec_copy")


def solve_pbicgstab(A: Matrix, M: ILU, r, x, tol=1e-10, maxit=10000, allow=(OK, NOT_CONVERGED)):
    """LsSol::Solve_PBiCGSTAB on device vectors; returns (status, iters, conv)."""
    it, conv = C.c_uint(), C.c_double()
    _sync_torch()
    rc = lib().dfm_solve_pbicgstab(A.h, M.h, _ptr(r), _ptr(x), tol, maxit, C.byref(it), C.byref(conv))
    check(rc, "dfm_solve_pbicgstab", allow)
    return rc, it.value, conv.value


def solve_pcocg(A: Matrix, M: ILU, r, x, tol=1e-10, maxit=10000, allow=(OK, NOT_CONVERGED)):
    """Fem::Ls::Solve_PCOCG on device vectors (interleaved complex); returns (status, iters, conv)."""
    it, conv = C.c_uint(), C.c_double()
    _sync_torch()
    rc = lib().dfm_solve_pcocg(A.h, M.h, _ptr(r), _ptr(x), tol, maxit, C.byref(it), C.byref(conv))
    check(rc, "dfm_solve_pcocg", allow)
    return rc, it.value, conv.value


def solve_pcg_mixed(A: Matrix, M: ILU, r, x, tol=1e-10, maxit=10000, allow=(OK, NOT_CONVERGED)):
    """PCG with FP32 values inside FP64 residual replacement; returns (status, iters, conv)."""
    it, conv = C.c_uint(), C.c_double()
    _sync_torch()
    rc = lib().dfm_solve_pcg_mixed(A.h, M.h, _ptr(r), _ptr(x), tol, maxit, C.byref(it), C.byref(conv))
    check(rc, "dfm_solve_pcg_mixed", allow)
    return rc, it.value, conv.value


def solve_pcocg_mixed(A: Matrix, M: ILU, r, x, tol=1e-10, maxit=10000, allow=(OK, NOT_CONVERGED)):
    """PCOCG with complex64 values inside complex128 residual replacement."""
    it, conv = C.c_uint(), C.c_double()
    _sync_torch()
    rc = lib().dfm_solve_pcocg_mixed(A.h, M.h, _ptr(r), _ptr(x), tol, maxit, C.byref(it), C.byref(conv))
    check(rc, "dfm_solve_pcocg_mixed", allow)
    return rc, it.value, conv.value


def solve_host(A: Matrix, M: ILU, b, method=PCG, tol=1e-10, maxit=10000, allow=(OK, NOT_CONVERGED)):
    """End-to-end solve from host b to host x; returns (status, x, iters, conv)."""
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b)
    it, conv = C.c_uint(), C.c_double()
    rc = lib().dfm_solve_host(A.h, M.h if M is not None else None, method, _ptr(b), _ptr(x), tol, maxit,
                              C.byref(it), C.byref(conv))
    check(rc, "dfm_solve_host", allow)
    return rc, x, it.value, conv.value


def solve_pcg_host(A: Matrix, M: ILU, b, tol=1e-10, maxit=10000, allow=(OK, NOT_CONVERGED)):
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b)
    it, conv = C.c_uint(), C.c_double()
    rc = lib().dfm_solve_pcg_host(A.h, M.h, _ptr(b), _ptr(x), tol, maxit, C.byref(it), C.byref(conv))
    check(rc, "dfm_solve_pcg_host", allow)
    return rc, x, it.value, conv.value
