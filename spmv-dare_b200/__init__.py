"""spmv-dare_b200 -- B200-native SpMV engine behind the reference's format plugin API.

Host-side mirror of the reference's plugin interface (src/spmv_kernels/spmv_kernel.h:8-29):

    MF = csr_to_format(row_ptr, col_ind, values, m, n, nnz, symmetric, symmetry_expanded,
                       format="csr_naive", ...)
    MF.spmv(x, y)                 # Matrix_Format::spmv
    MF.mem_footprint, MF.csr_mem_footprint, MF.format_name, MF.m, MF.n, MF.nnz
    MF.statistics_start(); MF.statistics_print_data()
    statistics_print_labels()

Every call goes through the C ABI of libspmv_b200.so (include/spmv_b200.h).  The
conversion and the SpMV run on the GPU; there is no CPU fallback: without the built
library or without a CUDA device the calls raise.

``spmv(x, y)`` accepts host numpy arrays (the reference's contract: x and y are host
buffers, copied to and from the device inside the call) or CUDA torch tensors (the
device-resident path, enqueued on torch's current stream).
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_int, c_int64

import numpy as np

from . import _capi
from ._capi import FORMATS, VALUES_F32, VALUES_F64

__all__ = [
    "SpmvError", "Matrix_Format", "csr_to_format", "statistics_print_labels", "generate_artificial",
    "ArtificialMatrix", "FORMATS", "format_defaults", "library", "version", "Batch", "read_mtx", "MtxMatrix",
    "coo_to_csr", "expand_symmetric", "drop_upper", "rcm", "generate_artificial_device",
]


class SpmvError(RuntimeError):
    """Raised for every non-zero status of the C ABI (the reference prints and exits)."""

    def __init__(self, status, message):
        super().__init__(f"[status {status}] {message}")
        self.status = status


def library():
    return _capi.load()


def version():
    return library().spmv_version().decode()


def _raise(status):
    msg = library().spmv_last_error().decode(errors="replace")
    raise SpmvError(status, msg or "error")


def format_defaults(format="csr_naive"):
    """The reference's defaults for `format` as a dict of descriptor fields."""
    d = _capi.FormatDesc()
    library().spmv_format_desc_init(byref(d), FORMATS[format])
    return {name: getattr(d, name) for name, _ in _capi.FormatDesc._fields_ if name != "reserved"}


def _desc(format, params):
    if format not in FORMATS:
        raise ValueError(f"unknown format {format!r}; one of {sorted(FORMATS)}")
    d = _capi.FormatDesc()
    library().spmv_format_desc_init(byref(d), FORMATS[format])
    for k, v in params.items():
        if v is None:
            continue
        if k == "value_type":           # the descriptor's `values` field
            k = "values"
            v = {"f64": VALUES_F64, "f32": VALUES_F32}.get(v, v)
        if not hasattr(d, k) or k in ("format", "reserved"):
            raise TypeError(f"unknown format parameter {k!r}")
        setattr(d, k, v)
    return d


def _host(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _is_cuda_tensor(a):
    return getattr(a, "is_cuda", False) is True


CUDA_STREAM_LEGACY = 1   # cudaStreamLegacy: torch's default stream reports handle 0


def _torch_stream(device, stream=None):
    """Raw cudaStream_t of `stream` (a torch.cuda.Stream or raw handle) or of torch's current
    stream.  The legacy default stream (handle 0) is passed as cudaStreamLegacy, because a
    NULL stream means "the handle's own stream" in the C ABI."""
    import torch

    if stream is None:
        stream = torch.cuda.current_stream(device)
    h = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
    return h if h else CUDA_STREAM_LEGACY


class Matrix_Format:
    """A matrix converted to one GPU format (the reference's struct Matrix_Format)."""

    def __init__(self, handle, format):
        self._h = handle
        self._format = format
        info = _capi.Info()
        st = library().spmv_get_info(self._h, byref(info))
        if st:
            _raise(st)
        self.m = int(info.m)
        self.n = int(info.n)
        self.nnz = int(info.nnz)
        self.mem_footprint = float(info.mem_footprint)
        self.csr_mem_footprint = float(info.csr_mem_footprint)
        self.format_name = info.format_name.decode()
        self.stored_elems = int(info.stored_elems)
        self.device_bytes = int(info.device_bytes)
        self.convert_ms = float(info.convert_ms)
        self.alloc_ms = float(info.alloc_ms)
        self.copy_in_ms = float(info.copy_in_ms)
        self.x_span = (int(info.x_lo), int(info.x_hi))    # columns above 0 the matrix reads
        self.x_col0 = bool(info.x_col0)                    # x[0] read too (column 0 or padding)
        self.kernels_per_run = int(info.kernels_per_run)
        self.num_loops = 0

    @property
    def format(self):
        return self._format

    @property
    def handle(self):
        return self._h

    def spmv(self, x, y=None, stream=None):
        """y = A x.  Host numpy buffers: synchronous copy-in / copy-out (Matrix_Format::spmv).
        CUDA torch tensors: enqueued on `stream` (default: torch's current stream)."""
        if self._h is None:
            raise SpmvError(_capi.SPMV_ERR_ARG, "matrix already destroyed")
        self.num_loops += 1
        lib = library()
        if _is_cuda_tensor(x):
            import torch

            if y is None:
                y = torch.empty(self.m, dtype=x.dtype, device=x.device)
            if not (x.is_contiguous() and y.is_contiguous()):
                raise ValueError("x and y must be contiguous")
            if x.numel() < self.n or y.numel() < self.m:
                raise ValueError(f"x needs {self.n} and y {self.m} elements")
            s = _torch_stream(x.device, stream)
            if x.dtype == torch.float32:
                st = lib.spmv_run_device_f32(self._h, x.data_ptr(), y.data_ptr(), s)
            else:
                if x.dtype != torch.float64 or y.dtype != torch.float64:
                    raise TypeError("x and y must both be float64 (or both float32 for the FP32 variant)")
                st = lib.spmv_run_device(self._h, x.data_ptr(), y.data_ptr(), s)
            if st:
                _raise(st)
            return y
        if getattr(x, "dtype", None) == np.float32 and getattr(self, "_f32", False):
            xf = _host(x, np.float32)
            if y is None:
                y = np.empty(self.m, np.float32)
            if xf.size < self.n or not (isinstance(y, np.ndarray) and y.dtype == np.float32 and y.size >= self.m):
                raise ValueError("x / y must be float32 arrays of n / m elements")
            st = lib.spmv_run_f32(self._h, xf.ctypes.data, y.ctypes.data)
            if st:
                _raise(st)
            return y
        xh = _host(x, np.float64)
        if xh.size < self.n:
            raise ValueError(f"x needs {self.n} elements")
        if y is None:
            y = np.empty(self.m, np.float64)
        if not (isinstance(y, np.ndarray) and y.dtype == np.float64 and y.flags.c_contiguous and y.size >= self.m):
            raise ValueError("y must be a contiguous float64 numpy array with at least m elements")
        st = lib.spmv_run(self._h, xh.ctypes.data, y.ctypes.data)
        if st:
            _raise(st)
        return y

    def sync(self):
        st = library().spmv_sync(self._h)
        if st:
            _raise(st)

    def export(self, name):
        """One converted array as numpy (for array-for-array parity with the reference)."""
        aid, dt = _capi.ARRAYS[name]
        if name == "values" and self._format == "csr_naive" and getattr(self, "_f32", False):
            dt = "float32"
        cnt = c_int64(0)
        st = library().spmv_export(self._h, aid, None, byref(cnt))
        if st:
            _raise(st)
        out = np.empty(max(cnt.value, 1), dtype=dt)
        st = library().spmv_export(self._h, aid, out.ctypes.data, byref(cnt))
        if st:
            _raise(st)
        return out[: cnt.value]

    def statistics_start(self):
        self.num_loops = 0

    def statistics_print_data(self):
        buf = ctypes.create_string_buffer(1024)
        library().spmv_statistics_print_data(self._h, buf, len(buf))
        return buf.value.decode()

    def destroy(self):
        if self._h is not None:
            library().spmv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __repr__(self):
        return f"<Matrix_Format {self.format_name} m={self.m} n={self.n} nnz={self.nnz}>"


def csr_to_format(row_ptr, col_ind, values, m=None, n=None, nnz=None, symmetric=0, symmetry_expanded=1,
                  format="csr_naive", **params):
    """csr_to_format (spmv_kernel.h:28): convert a CSR matrix to `format` on the GPU.

    Inputs may be host arrays (copied, as every reference format deep-copies) or CUDA torch
    tensors (converted device-to-device).  `params` are spmv_format_desc fields
    (num_threads, vec_len, sellcs_c, sellcs_sigma, div_packet_vals, div_tolerance, exact,
    block_nnz, block_rows, stages, ctas_per_sm, threads, kernel) and value_type ("f64", or
    "f32" for the FP32 storage variant)."""
    desc = _desc(format, params)
    st = c_int(0)
    lib = library()
    if _is_cuda_tensor(row_ptr):
        import torch

        m = int(row_ptr.numel() - 1) if m is None else int(m)
        nnz = int(col_ind.numel()) if nnz is None else int(nnz)
        n = m if n is None else int(n)
        if symmetric and not symmetry_expanded:
            raise SpmvError(_capi.SPMV_ERR_UNSUPPORTED,
                            "symmetric matrices have to be expanded to be supported by this format")
        rp = row_ptr.contiguous()
        ci = col_ind.contiguous()
        vv = values.contiguous()
        if rp.dtype != torch.int32 or ci.dtype != torch.int32 or vv.dtype != torch.float64:
            raise TypeError("device CSR must be int32 row_ptr / col_ind and float64 values")
        h = lib.spmv_create_device(rp.data_ptr(), ci.data_ptr(), vv.data_ptr(), m, n, nnz, byref(desc),
                                   _torch_stream(rp.device), byref(st))
    else:
        rp = _host(row_ptr, np.int32)
        ci = _host(col_ind, np.int32)
        vv = _host(values, np.float64)
        m = rp.size - 1 if m is None else int(m)
        nnz = int(rp[m]) if nnz is None else int(nnz)
        n = m if n is None else int(n)
        h = lib.spmv_create(rp.ctypes.data, ci.ctypes.data if ci.size else None,
                            vv.ctypes.data if vv.size else None, m, n, nnz, int(symmetric), int(symmetry_expanded),
                            byref(desc), byref(st))
    if not h:
        _raise(st.value)
    mf = Matrix_Format(h, format)
    mf._f32 = desc.values == VALUES_F32
    return mf


class Batch:
    """Many matrices in one persistent launch (spmv_batch_* of the C ABI).

    matrices: list of (row_ptr, col_ind, values, m, n); formats: one format name (or
    dict of descriptor fields incl. "format") per matrix; geometry: block_nnz, stages,
    threads, exact for the whole batch.  x / y are the matrices' vectors concatenated
    (see x_offsets / y_offsets)."""

    def __init__(self, matrices, formats, **geometry):
        lib = library()
        cnt = len(matrices)
        if len(formats) != cnt:
            raise ValueError("one format per matrix")
        descs = (_capi.FormatDesc * max(cnt, 1))()
        self._keep = []
        rps = (ctypes.c_void_p * max(cnt, 1))()
        cis = (ctypes.c_void_p * max(cnt, 1))()
        vvs = (ctypes.c_void_p * max(cnt, 1))()
        ms = np.empty(max(cnt, 1), np.int64)
        ns = np.empty(max(cnt, 1), np.int64)
        for i, ((rp, ci, vv, m, n), f) in enumerate(zip(matrices, formats)):
            params = dict(f) if isinstance(f, dict) else {"format": f}
            fmt = params.pop("format")
            params.update(geometry)
            descs[i] = _desc(fmt, params)
            rp, ci, vv = _host(rp, np.int32), _host(ci, np.int32), _host(vv, np.float64)
            self._keep += [rp, ci, vv]
            rps[i], cis[i], vvs[i] = rp.ctypes.data, ci.ctypes.data if ci.size else None, vv.ctypes.data if vv.size else None
            ms[i], ns[i] = m, n
        st = c_int(0)
        self._b = lib.spmv_batch_create(cnt, ctypes.cast(rps, ctypes.c_void_p), ctypes.cast(cis, ctypes.c_void_p),
                                        ctypes.cast(vvs, ctypes.c_void_p), ms.ctypes.data, ns.ctypes.data,
                                        ctypes.cast(descs, ctypes.c_void_p), byref(st))
        self._keep = None
        if not self._b:
            _raise(st.value)
        tx, ty, tn, nb = c_int64(), c_int64(), c_int64(), c_int64()
        self.x_offsets = np.empty(max(cnt, 1), np.int64)
        self.y_offsets = np.empty(max(cnt, 1), np.int64)
        lib.spmv_batch_info(self._b, byref(tx), byref(ty), byref(tn), self.x_offsets.ctypes.data,
                            self.y_offsets.ctypes.data, byref(nb))
        self.x_offsets, self.y_offsets = self.x_offsets[:cnt], self.y_offsets[:cnt]
        self.total_x, self.total_y, self.total_nnz, self.num_blocks = tx.value, ty.value, tn.value, nb.value
        self.count = cnt

    def spmv(self, xd, yd, graph=False, stream=None):
        """xd, yd: CUDA float64 tensors of total_x / total_y elements."""
        s = _torch_stream(xd.device, stream)
        f = library().spmv_batch_run_graph if graph else library().spmv_batch_run_device
        st = f(self._b, xd.data_ptr(), yd.data_ptr(), s)
        if st:
            _raise(st)
        return yd

    def sync(self):
        st = library().spmv_batch_sync(self._b)
        if st:
            _raise(st)

    def destroy(self):
        if getattr(self, "_b", None):
            library().spmv_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def statistics_print_labels():
    buf = ctypes.create_string_buffer(1024)
    library().spmv_statistics_print_labels(buf, len(buf))
    return buf.value.decode()


STAT_NAMES = [
    "avg_nnz_per_row", "std_nnz_per_row", "min_nnz_per_row", "max_nnz_per_row", "skew",
    "avg_bw", "std_bw", "min_bw", "max_bw",
    "avg_sc", "std_sc", "min_sc", "max_sc",
    "avg_num_neighbours", "std_num_neighbours", "min_num_neighbours", "max_num_neighbours",
    "cross_row_similarity", "std_cross_row_similarity", "min_cross_row_similarity", "max_cross_row_similarity",
    "avg_clustering", "std_clustering", "min_clustering", "max_clustering",
    "avg_ngroups", "std_ngroups", "min_ngroups", "max_ngroups",
    "avg_dis", "std_dis", "min_dis", "max_dis",
    "avg_ngroups_size", "std_ngroups_size", "min_ngroups_size", "max_ngroups_size",
]


class ArtificialMatrix:
    """CSR arrays and structural statistics of one generated matrix."""

    def __init__(self, row_ptr, col_ind, values, stats, params):
        self.row_ptr = row_ptr
        self.col_ind = col_ind
        self.values = values
        self.stats = stats
        self.params = params

    @property
    def m(self):
        return self.row_ptr.size - 1

    @property
    def nnz(self):
        return int(self.row_ptr[-1])


def generate_artificial(rows, cols, avg_nnz_per_row, std_nnz_per_row, distribution, placement, avg_bw, skew,
                        avg_num_neighbours, cross_row_similarity, seed, threads=0):
    """The reference's artificial matrix generator (bench argv order, src/bench.cpp:564-578),
    restated natively; thread-count independent.  Values are U[0,1) as in the reference."""
    import os

    lib = library()
    st = c_int(0)
    threads = threads or (os.cpu_count() or 1)
    g = lib.spmv_artgen_create(int(rows), int(cols), float(avg_nnz_per_row), float(std_nnz_per_row),
                               distribution.encode(), placement.encode(), float(avg_bw), float(skew),
                               float(avg_num_neighbours), float(cross_row_similarity), int(seed) & 0xFFFFFFFF,
                               int(threads), byref(st))
    if not g:
        _raise(st.value)
    try:
        nnz = lib.spmv_artgen_nnz(g)
        rp = np.empty(rows + 1, np.int32)
        ci = np.empty(max(nnz, 1), np.int32)
        v = np.empty(max(nnz, 1), np.float64)
        stats = np.empty(37, np.float64)
        lib.spmv_artgen_get(g, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, stats.ctypes.data)
    finally:
        lib.spmv_artgen_destroy(g)
    params = dict(rows=rows, cols=cols, avg_nnz_per_row=avg_nnz_per_row, std_nnz_per_row=std_nnz_per_row,
                  distribution=distribution, placement=placement, avg_bw=avg_bw, skew=skew,
                  avg_num_neighbours=avg_num_neighbours, cross_row_similarity=cross_row_similarity, seed=seed)
    return ArtificialMatrix(rp, ci[:nnz], v[:nnz], dict(zip(STAT_NAMES, stats.tolist())), params)


class MtxMatrix:
    """CSR arrays of an imported Matrix-Market file, with the reference's CSR_reference_s
    flags (src/bench.cpp:196-207): symmetric, symmetry_expanded, nnz_diag, nnz_non_diag."""

    def __init__(self, row_ptr, col_ind, values, n, symmetric, symmetry_expanded, nnz_diag, nnz_non_diag):
        self.row_ptr, self.col_ind, self.values = row_ptr, col_ind, values
        self.n = n
        self.symmetric, self.symmetry_expanded = symmetric, symmetry_expanded
        self.nnz_diag, self.nnz_non_diag = nnz_diag, nnz_non_diag

    @property
    def m(self):
        return self.row_ptr.size - 1

    @property
    def nnz(self):
        return int(self.row_ptr[-1])


def read_mtx(path, expand_symmetry=True):
    """The reference's import_file (src/bench.cpp:127-238) for a Matrix-Market coordinate
    file: parsed on the host, COO -> CSR (columns sorted in every row) on the GPU.
    expand_symmetry=False keeps a symmetric file's stored triangle (KEEP_SYMMETRY)."""
    import os

    lib = library()
    st = c_int(0)
    x = lib.spmv_mtx_read(os.fsencode(path), 1 if expand_symmetry else 0, byref(st))
    if not x:
        _raise(st.value)
    try:
        m, n, nnz, nd, nn = c_int64(), c_int64(), c_int64(), c_int64(), c_int64()
        sym, exp = ctypes.c_int32(), ctypes.c_int32()
        lib.spmv_mtx_info(x, byref(m), byref(n), byref(nnz), byref(sym), byref(exp), byref(nd), byref(nn))
        rp = np.empty(m.value + 1, np.int32)
        ci = np.empty(max(nnz.value, 1), np.int32)
        v = np.empty(max(nnz.value, 1), np.float64)
        lib.spmv_mtx_get(x, rp.ctypes.data, ci.ctypes.data, v.ctypes.data)
    finally:
        lib.spmv_mtx_destroy(x)
    return MtxMatrix(rp, ci[:nnz.value], v[:nnz.value], n.value, sym.value, exp.value, nd.value, nn.value)


def coo_to_csr(rows, cols, values, m, n):
    """coo_to_csr (csr_gen.c:178-210, sorted columns) on the GPU for CUDA torch tensors
    (int32 rows / cols, float64 values or None): returns (row_ptr, col_ind, values) tensors."""
    import torch

    nnz = int(rows.numel())
    dev = rows.device
    rp = torch.empty(int(m) + 1, dtype=torch.int32, device=dev)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
    vv = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
    rows, cols = rows.contiguous(), cols.contiguous()
    values = values.contiguous() if values is not None else None
    st = library().spmv_coo_to_csr_device(rows.data_ptr(), cols.data_ptr(),
                                          values.data_ptr() if values is not None else None,
                                          int(m), int(n), nnz, rp.data_ptr(), ci.data_ptr(), vv.data_ptr(),
                                          _torch_stream(dev))
    if st:
        _raise(st)
    return rp, ci[:nnz], vv[:nnz]


def _csr_out(fn, row_ptr, col_ind, values, n, *extra):
    lib = library()
    rp, ci, vv = _host(row_ptr, np.int32), _host(col_ind, np.int32), _host(values, np.float64)
    m = rp.size - 1
    st = c_int(0)
    o = fn(rp.ctypes.data, ci.ctypes.data if ci.size else None, vv.ctypes.data if vv.size else None, m, int(n),
           int(rp[-1]), *extra, byref(st))
    if not o:
        _raise(st.value)
    try:
        mm, nn, nz, nd = c_int64(), c_int64(), c_int64(), c_int64()
        lib.spmv_csr_out_info(o, byref(mm), byref(nn), byref(nz), byref(nd))
        orp = np.empty(mm.value + 1, np.int32)
        oci = np.empty(max(nz.value, 1), np.int32)
        ov = np.empty(max(nz.value, 1), np.float64)
        perm = np.empty(max(mm.value, 1), np.int32)
        lib.spmv_csr_out_get(o, orp.ctypes.data, oci.ctypes.data, ov.ctypes.data, perm.ctypes.data)
    finally:
        lib.spmv_csr_out_destroy(o)
    return orp, oci[:nz.value], ov[:nz.value], perm[:mm.value], nd.value


def expand_symmetric(row_ptr, col_ind, values, n=None):
    """csr_expand_symmetric (csr_gen.c:256-336) on the GPU: (row_ptr, col_ind, values, nnz_diag)."""
    rp, ci, v, _, nd = _csr_out(library().spmv_expand_symmetric, row_ptr, col_ind, values,
                                len(row_ptr) - 1 if n is None else n)
    return rp, ci, v, nd


def drop_upper(row_ptr, col_ind, values, n=None):
    """csr_drop_upper (csr_gen.c:344-420) on the GPU: (row_ptr, col_ind, values, nnz_diag)."""
    rp, ci, v, _, nd = _csr_out(library().spmv_drop_upper, row_ptr, col_ind, values,
                                len(row_ptr) - 1 if n is None else n)
    return rp, ci, v, nd


def rcm(row_ptr, col_ind, values, symmetry_expanded=True):
    """The bench's rcm() (src/bench.cpp:280-358) on the GPU: (row_ptr, col_ind, values,
    permutation), permutation[old row] = new row."""
    rp, ci, v, perm, _ = _csr_out(library().spmv_rcm, row_ptr, col_ind, values, len(row_ptr) - 1,
                                  1 if symmetry_expanded else 0)
    return rp, ci, v, perm


def generate_artificial_device(rows, cols, avg_nnz_per_row, std_nnz_per_row, distribution, placement, avg_bw, skew,
                               avg_num_neighbours, cross_row_similarity, seed, device="cuda", stream=None):
    """The artificial generator run on the GPU (one thread per anchor segment): CUDA int32
    row_ptr / col_ind and float64 values (U[0,1)) tensors on `device`."""
    import torch

    lib = library()
    dev = torch.device(device)
    s = _torch_stream(dev, stream)
    st = c_int(0)
    g = lib.spmv_gen_create_device(int(rows), int(cols), float(avg_nnz_per_row), float(std_nnz_per_row),
                                   distribution.encode(), placement.encode(), float(avg_bw), float(skew),
                                   float(avg_num_neighbours), float(cross_row_similarity), int(seed) & 0xFFFFFFFF, s,
                                   byref(st))
    if not g:
        _raise(st.value)
    try:
        m, n, nnz = c_int64(), c_int64(), c_int64()
        lib.spmv_gen_info(g, byref(m), byref(n), byref(nnz))
        rp = torch.empty(m.value + 1, dtype=torch.int32, device=dev)
        ci = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev)
        v = torch.empty(max(nnz.value, 1), dtype=torch.float64, device=dev)
        st2 = lib.spmv_gen_copy_device(g, rp.data_ptr(), ci.data_ptr(), v.data_ptr(), s)
        if st2:
            _raise(st2)
    finally:
        lib.spmv_gen_destroy(g)     # its buffers are freed in stream order, after the copies
    return rp, ci[:nnz.value], v[:nnz.value]
