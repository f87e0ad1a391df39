"""ctypes front end of the oracle (TEST INFRASTRUCTURE ONLY).

Two CPU checkers live under oracle/:

* ``liboracle.so`` -- the plain-C restatement of the reference's SpMV hot path
  (oracle/spmv_oracle.c), always built by ``make -C oracle``;
* ``_ref/libref_*.so`` -- the reference itself, compiled from its own sources by
  ``make -C oracle ref`` where the reference checkout is present.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module.  The product package never does.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_double, c_int, c_long, c_void_p, c_char_p, c_uint

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def lib():
    """The restatement library (loaded on first use)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle restatement not built: {LIB_PATH} (run `make -C oracle`)")
        L = ctypes.CDLL(LIB_PATH)
        P = c_void_p
        sig = {
            "orc_nearest_index": (c_long, [P, c_long, c_long, c_long]),
            "orc_partition_prefix_sums": (None, [c_long, c_long, P, c_long, c_long, P, P]),
            "orc_partition_iterations": (None, [c_long, c_long, c_long, c_long, P, P]),
            "orc_csr_spmv": (None, [P, P, P, c_long, P, P]),
            "orc_csr_vec_spmv": (None, [P, P, P, c_long, c_long, P, P]),
            "orc_csr_gold": (None, [P, P, P, c_long, P, P, P]),
            "orc_csr_f32_dot2": (None, [P, P, P, c_long, P, P]),
            "orc_sell_size": (c_long, [P, c_long, c_long]),
            "orc_sell_convert": (None, [P, P, P, c_long, c_long, c_long, P, P, P, P]),
            "orc_sell_spmv": (None, [P, P, P, c_long, c_long, P, P]),
            "orc_sell_sorted_size": (c_long, [P, c_long, c_long, c_long]),
            "orc_sell_sorted_convert": (None, [P, P, P, c_long, c_long, c_long, P, P, P, P, P, P]),
            "orc_sell_sorted_spmv": (None, [P, P, P, P, c_long, c_long, P, P]),
            "orc_sellcs_size": (c_long, [P, c_long, c_long, c_long]),
            "orc_sellcs_convert": (c_int, [P, P, P, c_long, c_long, c_long, P, P, P, P, P]),
            "orc_sellcs_spmv": (None, [P, P, P, P, P, c_long, c_long, P, P]),
            "orc_div_build": (P, [P, P, P, c_long, c_long, c_long, c_long, c_long, c_double]),
            "orc_div_get": (c_long, [P, c_int, P]),
            "orc_div_free": (None, [P]),
            "orc_div_header_size": (c_long, [c_long]),
            "orc_div_spmv": (c_int, [P, c_long, P, c_long, c_long, P, P, c_int]),
            "orc_div_decode_coo": (c_long, [P, c_long, c_long, P, P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data if a is not None else None


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ------------------------------------------------------------------ partitioners
def partition_prefix_sums(T, t, sums, N, total):
    s, e = c_long(), c_long()
    sums = _c(sums, np.int32)
    lib().orc_partition_prefix_sums(T, t, _p(sums), N, total, ctypes.byref(s), ctypes.byref(e))
    return s.value, e.value


# ------------------------------------------------------------------ CSR
def csr_spmv(rp, ci, v, x):
    rp, ci, v, x = _c(rp, np.int32), _c(ci, np.int32), _c(v, np.float64), _c(x, np.float64)
    m = rp.size - 1
    y = np.empty(m, np.float64)
    lib().orc_csr_spmv(_p(rp), _p(ci), _p(v), m, _p(x), _p(y))
    return y


def csr_vec_spmv(rp, ci, v, x, L=4):
    rp, ci, v, x = _c(rp, np.int32), _c(ci, np.int32), _c(v, np.float64), _c(x, np.float64)
    m = rp.size - 1
    y = np.empty(m, np.float64)
    lib().orc_csr_vec_spmv(_p(rp), _p(ci), _p(v), m, L, _p(x), _p(y))
    return y


def csr_f32_dot2(rp, ci, v32, x32):
    """FP32 values / x, Dot2-compensated FP32 row sums."""
    rp, ci = _c(rp, np.int32), _c(ci, np.int32)
    v32, x32 = _c(v32, np.float32), _c(x32, np.float32)
    m = rp.size - 1
    y = np.empty(m, np.float32)
    lib().orc_csr_f32_dot2(_p(rp), _p(ci), _p(v32), m, _p(x32), _p(y))
    return y


def csr_gold(rp, ci, v, x):
    """(y_gold, sum |a x|) in binary128 arithmetic."""
    rp, ci, v, x = _c(rp, np.int32), _c(ci, np.int32), _c(v, np.float64), _c(x, np.float64)
    m = rp.size - 1
    y = np.empty(m, np.float64)
    a = np.empty(m, np.float64)
    lib().orc_csr_gold(_p(rp), _p(ci), _p(v), m, _p(x), _p(y), _p(a))
    return y, a


# ------------------------------------------------------------------ SELL family
def sell_convert(rp, ci, v, V=4, T=8):
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), _c(v, np.float64)
    m = rp.size - 1
    nc = (m + V - 1) // V
    size = lib().orc_sell_size(_p(rp), m, V)
    rcp = np.empty(nc + 1, np.int32)
    ja = np.empty(max(size, 1), np.int32)
    a = np.empty(max(size, 1), np.float64)
    ranges = np.empty(2 * T, np.int64)
    lib().orc_sell_convert(_p(rp), _p(ci), _p(v), m, V, T, _p(rcp), _p(ja), _p(a), _p(ranges))
    return dict(row_cluster_ptr=rcp, ja=ja[:size], a=a[:size], ranges=ranges)


def sell_spmv(arr, m, V, x):
    x = _c(x, np.float64)
    y = np.empty(m, np.float64)
    lib().orc_sell_spmv(_p(arr["row_cluster_ptr"]), _p(_c(arr["ja"], np.int32)), _p(_c(arr["a"], np.float64)),
                        m, V, _p(x), _p(y))
    return y


def sell_sorted_convert(rp, ci, v, V=4, T=8):
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), _c(v, np.float64)
    m = rp.size - 1
    nc = (m + V - 1) // V
    size = lib().orc_sell_sorted_size(_p(rp), m, V, T)
    rcp = np.empty(nc + 1, np.int32)
    ja = np.empty(max(size, 1), np.int32)
    a = np.empty(max(size, 1), np.float64)
    perm = np.empty(max(m, 1), np.int32)
    rev = np.empty(max(m, 1), np.int32)
    ranges = np.empty(2 * T, np.int64)
    lib().orc_sell_sorted_convert(_p(rp), _p(ci), _p(v), m, V, T, _p(rcp), _p(ja), _p(a), _p(perm), _p(rev),
                                  _p(ranges))
    return dict(row_cluster_ptr=rcp, ja=ja[:size], a=a[:size], permutation=perm[:m], rev_permutation=rev[:m],
                ranges=ranges)


def sell_sorted_spmv(arr, m, V, x):
    x = _c(x, np.float64)
    y = np.empty(m, np.float64)
    lib().orc_sell_sorted_spmv(_p(arr["row_cluster_ptr"]), _p(_c(arr["ja"], np.int32)),
                               _p(_c(arr["a"], np.float64)), _p(_c(arr["rev_permutation"], np.int32)),
                               m, V, _p(x), _p(y))
    return y


def sellcs_convert(rp, ci, v, C=32, sigma=512):
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), _c(v, np.float64)
    m = rp.size - 1
    ns = (m + C - 1) // C
    size = lib().orc_sellcs_size(_p(rp), m, C, sigma)
    ro = np.empty(max(m, 1), np.int32)
    w = np.empty(max(ns, 1), np.int32)
    ptr = np.empty(ns + 1, np.int64)
    cols = np.empty(max(size, 1), np.int32)
    vals = np.empty(max(size, 1), np.float64)
    rc = lib().orc_sellcs_convert(_p(rp), _p(ci), _p(v), m, C, sigma, _p(ro), _p(w), _p(ptr), _p(cols), _p(vals))
    if rc != 0:
        raise ValueError("SELL-C-sigma needs C a power of two and sigma a multiple of C")
    return dict(row_order=ro[:m], slice_widths=w[:ns], slice_pointers=ptr, column_indices=cols[:size],
                values=vals[:size])


def sellcs_spmv(arr, m, C, x):
    x = _c(x, np.float64)
    y = np.empty(m, np.float64)
    lib().orc_sellcs_spmv(_p(_c(arr["row_order"], np.int32)), _p(_c(arr["slice_widths"], np.int32)),
                          _p(_c(arr["slice_pointers"], np.int64)), _p(_c(arr["column_indices"], np.int32)),
                          _p(_c(arr["values"], np.float64)), m, C, _p(x), _p(y))
    return y


# ------------------------------------------------------------------ DIV-RF
def div_convert(rp, ci, v, n=None, T=8, L=4, packet_vals=16384, tolerance=0.0):
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), _c(v, np.float64)
    m = rp.size - 1
    n = m if n is None else n
    h = lib().orc_div_build(_p(rp), _p(ci), _p(v), m, n, T, L, packet_vals, float(tolerance))
    if not h:
        raise ValueError("invalid DIV-RF parameters")
    try:
        get = lib().orc_div_get
        nb = get(h, 0, None)
        data = np.empty(max(nb, 1), np.uint8)
        get(h, 0, _p(data))
        npk = get(h, 1, None)
        pkt = np.empty(npk, np.int64)
        get(h, 1, _p(pkt))
        tb = np.empty(T, np.int64)
        get(h, 2, _p(tb))
        tg = np.empty(T, np.int64)
        get(h, 3, _p(tg))
        ng = get(h, 4, None)
        gp = np.empty(ng, np.int64)
        get(h, 4, _p(gp))
        rg = np.empty(2 * T, np.int64)
        get(h, 5, _p(rg))
        err = get(h, 6, None)
    finally:
        lib().orc_div_free(h)
    if err:
        raise RuntimeError("DIV-RF oracle: inconsistent packet groups")
    return dict(data=data[:nb], packet_offsets=pkt, thread_bytes=tb, thread_groups=tg, group_pos=gp,
                ranges=rg, T=T, L=L)


def div_packet_offsets(data, L):
    """Byte offsets of the packets of a DIV-RF stream (walking the headers,
    div_kernels_rf.h:65-79 and :909-917); the last entry is the stream length."""
    data = np.ascontiguousarray(data, dtype=np.uint8)
    hsz = 28 + 4 * L
    offs = [0]
    pos = 0
    while pos < data.size:
        h = data[pos:pos + hsz]
        u32 = lambda o: int.from_bytes(h[o:o + 4].tobytes(), "little")
        nv, nu, nrf = u32(0), u32(4), u32(24)
        cb = (int(h[20]) + int(h[21]) + 7) >> 3
        lanes = sum(u32(28 + 4 * l) for l in range(L))
        pos += hsz + 8 * nrf + cb * nv + nu + lanes
        offs.append(pos)
    if pos != data.size:
        raise ValueError("DIV-RF stream does not end on a packet boundary")
    return np.array(offs, np.int64)


def div_zero_header_padding(data, L):
    """The two padding bytes after col_bits in struct packet_header are never written by the
    reference (their content is whatever the reused buffer held); zero them."""
    data = np.array(data, dtype=np.uint8, copy=True)
    for o in div_packet_offsets(data, L)[:-1]:
        data[o + 22:o + 24] = 0
    return data


def div_spmv(arr, m, x, fused=False):
    x = _c(x, np.float64)
    y = np.ones(m, np.float64)
    d = arr["data"]
    rc = lib().orc_div_spmv(_p(d), d.size, _p(arr["ranges"]), arr["T"], arr["L"], _p(x), _p(y), int(fused))
    if rc != 0:
        raise RuntimeError("DIV-RF oracle decode failed")
    return y


def div_decode_coo(data, L, nnz):
    data = _c(data, np.uint8)
    r = np.empty(max(nnz, 1), np.int32)
    c = np.empty(max(nnz, 1), np.int32)
    v = np.empty(max(nnz, 1), np.float64)
    k = lib().orc_div_decode_coo(_p(data), data.size, L, _p(r), _p(c), _p(v))
    if k < 0:
        raise RuntimeError("DIV-RF oracle decode failed")
    return r[:k], c[:k], v[:k]


# ------------------------------------------------------------------ reference (compiled from its sources)
def ref_available(name="gen"):
    return os.path.exists(os.path.join(REF_DIR, f"libref_{name}.so"))


_ref_cache = {}


def _ref(name):
    if name not in _ref_cache:
        path = os.path.join(REF_DIR, f"libref_{name}.so")
        if not os.path.exists(path):
            raise RuntimeError(f"reference build missing: {path} (run `make -C oracle ref`)")
        L = ctypes.CDLL(path)
        if name == "gen":
            L.ref_gen.restype = c_void_p
            L.ref_gen.argtypes = [c_long, c_long, c_double, c_double, c_char_p, c_uint, c_char_p,
                                  c_double, c_double, c_double, c_double, c_int]
            L.ref_gen_nnz.restype = c_long
            L.ref_gen_nnz.argtypes = [c_void_p]
            L.ref_gen_arrays.argtypes = [c_void_p] * 4
            L.ref_gen_stats.argtypes = [c_void_p, c_void_p]
            L.ref_gen_num_stats.restype = c_int
            L.ref_gen_free.argtypes = [c_void_p]
            L.ref_cross_row_similarity.restype = c_double
            L.ref_cross_row_similarity.argtypes = [c_void_p, c_void_p, c_long, c_long, c_long, c_int]
        elif name == "rcm":
            L.ref_sym_transform.restype = c_void_p
            L.ref_sym_transform.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_long, c_long, c_long, c_long, c_int]
            L.ref_sym_nnz.restype = c_long
            L.ref_sym_nnz.argtypes = [c_void_p]
            L.ref_sym_nnz_diag.restype = c_long
            L.ref_sym_nnz_diag.argtypes = [c_void_p]
            L.ref_sym_arrays.argtypes = [c_void_p] * 5
            L.ref_sym_free.argtypes = [c_void_p]
        elif name == "mtx":
            L.ref_mtx_import.restype = c_void_p
            L.ref_mtx_import.argtypes = [c_char_p, c_long, c_int]
            L.ref_mtx_info.argtypes = [c_void_p, c_void_p]
            L.ref_mtx_arrays.argtypes = [c_void_p] * 4
            L.ref_mtx_free.argtypes = [c_void_p]
        elif name == "sellcs":
            L.ref_sellcs_convert.restype = c_void_p
            L.ref_sellcs_convert.argtypes = [c_void_p] * 3 + [c_long] * 5
            L.ref_sellcs_nslices.restype = c_long
            L.ref_sellcs_nslices.argtypes = [c_void_p]
            L.ref_sellcs_size.restype = c_long
            L.ref_sellcs_size.argtypes = [c_void_p]
            L.ref_sellcs_export.argtypes = [c_void_p] * 6
            L.ref_sellcs_free.argtypes = [c_void_p]
        else:
            L.ref_convert.restype = c_void_p
            L.ref_convert.argtypes = [c_void_p] * 3 + [c_long] * 3 + [c_int]
            L.ref_spmv.argtypes = [c_void_p] * 3
            L.ref_free.argtypes = [c_void_p]
            L.ref_mem_footprint.restype = c_double
            L.ref_mem_footprint.argtypes = [c_void_p]
            L.ref_format_name.restype = c_char_p
            L.ref_format_name.argtypes = [c_void_p]
            L.ref_export.restype = c_long
            L.ref_export.argtypes = [c_void_p, c_int, c_void_p]
            L.ref_vec_len.restype = c_int
        _ref_cache[name] = L
    return _ref_cache[name]


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


def ref_generate(rows, cols, avg, std, distribution, placement, bw, skew, neigh, cross, seed, threads=8):
    """The reference generator (bench argv order, src/bench.cpp:564-578)."""
    L = _ref("gen")
    d = distribution.encode()
    p = placement.encode()
    h = L.ref_gen(rows, cols, avg, std, d, seed, p, bw, skew, neigh, cross, threads)
    try:
        nnz = L.ref_gen_nnz(h)
        rp = np.empty(rows + 1, np.int32)
        ci = np.empty(max(nnz, 1), np.int32)
        v = np.empty(max(nnz, 1), np.float64)
        L.ref_gen_arrays(h, _p(rp), _p(ci), _p(v))
        st = np.empty(L.ref_gen_num_stats(), np.float64)
        L.ref_gen_stats(h, _p(st))
    finally:
        L.ref_gen_free(h)
    return rp, ci[:nnz], v[:nnz], dict(zip(STAT_NAMES, st.tolist()))


def ref_cross_row_similarity(rp, ci, n, threads=8):
    """The reference's csr_cross_row_similarity (matrix_util.h:269-328), window 1."""
    rp, ci = _c(rp, np.int32), _c(ci, np.int32)
    return _ref("gen").ref_cross_row_similarity(_p(rp), _p(ci), rp.size - 1, n, int(rp[-1]), threads)


class RefFormat:
    """One reference format compiled from its sources (csr_naive, csr_vec, sell, sell_sorted, div_rf).

    The reference keeps per-thread state of a converted matrix in file-scope globals, so at
    most one RefFormat of a format may be alive: close() it before converting another."""

    def __init__(self, fmt, rp, ci, v, n=None, threads=8):
        self.L = _ref(fmt)
        self.fmt = fmt
        self.rp, self.ci, self.v = _c(rp, np.int32), _c(ci, np.int32), _c(v, np.float64)
        self.m = self.rp.size - 1
        self.n = self.m if n is None else n
        self.nnz = int(self.rp[-1])
        self.threads = threads
        self.h = self.L.ref_convert(_p(self.rp), _p(self.ci), _p(self.v), self.m, self.n, self.nnz, threads)

    def spmv(self, x, y=None):
        x = _c(x, np.float64)
        if y is None:
            y = np.ones(self.m + 64, np.float64)
        self.L.ref_spmv(self.h, _p(x), _p(y))
        return y

    def close(self):
        if self.h:
            self.L.ref_free(self.h)
            self.h = None

    @property
    def mem_footprint(self):
        return self.L.ref_mem_footprint(self.h)

    @property
    def format_name(self):
        return self.L.ref_format_name(self.h).decode()

    def export(self, what, dtype):
        cnt = self.L.ref_export(self.h, what, None)
        if cnt < 0:
            raise KeyError(what)
        out = np.empty(max(cnt, 1), dtype)
        self.L.ref_export(self.h, what, _p(out))
        return out[:cnt]

    def sell_arrays(self):
        d = dict(row_cluster_ptr=self.export(0, np.int32), ja=self.export(1, np.int32), a=self.export(2, np.float64),
                 ranges=self.export(5, np.int64))
        if self.fmt == "sell_sorted":
            d["permutation"] = self.export(3, np.int32)
            d["rev_permutation"] = self.export(4, np.int32)
        return d

    def div_arrays(self):
        T = self.L.ref_export(self.h, 10, None)
        streams = [self.export(100 + t, np.uint8) for t in range(T)]
        groups = [self.export(200 + t, np.int64) for t in range(T)]
        ranges = np.concatenate([self.export(300 + t, np.int64) for t in range(T)])
        return dict(data=np.concatenate(streams) if streams else np.empty(0, np.uint8),
                    thread_bytes=np.array([s.size for s in streams], np.int64),
                    group_pos=np.concatenate(groups), ranges=ranges, T=T)


def ref_read_mtx(path, expand_symmetry=True, threads=4):
    """The reference's import_file (src/bench.cpp:127-238) on a well-formed Matrix-Market
    file: dict of CSR arrays and the m, n, nnz, nnz_diag, nnz_non_diag, symmetric and
    expanded flags."""
    L = _ref("mtx")
    h = L.ref_mtx_import(os.fsencode(path), 1 if expand_symmetry else 0, threads)
    try:
        info = np.zeros(7, np.int64)
        L.ref_mtx_info(h, _p(info))
        m, n, nnz = int(info[0]), int(info[1]), int(info[2])
        rp = np.zeros(m + 1, np.int32)
        ci = np.zeros(max(nnz, 1), np.int32)
        v = np.zeros(max(nnz, 1), np.float64)
        L.ref_mtx_arrays(h, _p(rp), _p(ci), _p(v))
    finally:
        L.ref_mtx_free(h)
    return dict(row_ptr=rp, col_ind=ci[:nnz], values=v[:nnz], m=m, n=n, nnz=nnz, nnz_diag=int(info[3]),
                nnz_non_diag=int(info[4]), symmetric=int(info[5]), expanded=int(info[6]))


def ref_sym_transform(kind, rp, ci, v, n=None, expanded=1, threads=1):
    """The reference's csr_expand_symmetric (kind "expand"), csr_drop_upper ("drop") or the
    bench's rcm() ("rcm"): (row_ptr, col_ind, values, permutation or None, nnz_diag)."""
    L = _ref("rcm")
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), _c(v, np.float64)
    m = rp.size - 1
    k = {"expand": 0, "drop": 1, "rcm": 2}[kind]
    h = L.ref_sym_transform(k, _p(rp), _p(ci), _p(v), m, m if n is None else n, int(rp[-1]), expanded, threads)
    try:
        nnz = L.ref_sym_nnz(h)
        orp = np.zeros(m + 1, np.int32)
        oci = np.zeros(max(nnz, 1), np.int32)
        ov = np.zeros(max(nnz, 1), np.float64)
        perm = np.zeros(max(m, 1), np.int32)
        L.ref_sym_arrays(h, _p(orp), _p(oci), _p(ov), _p(perm) if k == 2 else None)
        nd = L.ref_sym_nnz_diag(h)
    finally:
        L.ref_sym_free(h)
    return orp, oci[:nnz], ov[:nnz], (perm[:m] if k == 2 else None), nd


def ref_sellcs_convert(rp, ci, v, C, sigma):
    L = _ref("sellcs")
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), _c(v, np.float64)
    m = rp.size - 1
    nnz = int(rp[-1])
    h = L.ref_sellcs_convert(_p(rp), _p(ci), _p(v), m, m, nnz, C, sigma)
    try:
        ns = L.ref_sellcs_nslices(h)
        size = L.ref_sellcs_size(h)
        ro = np.empty(max(m, 1), np.int64)
        w = np.empty(max(ns, 1), np.int64)
        ptr = np.empty(ns + 1, np.int64)
        cols = np.empty(max(size, 1), np.int64)
        vals = np.empty(max(size, 1), np.float64)
        L.ref_sellcs_export(h, _p(ro), _p(w), _p(ptr), _p(cols), _p(vals))
    finally:
        L.ref_sellcs_free(h)
    return dict(row_order=ro[:m], slice_widths=w[:ns], slice_pointers=ptr, column_indices=cols[:size],
                values=vals[:size])


# ------------------------------------------------------------------ learned selector
def features(rp, ci, m, n):
    """The 10 structural features in numpy FP64 (the statistics of
    artificial-matrix-generator/artificial_matrix_generation.c:529-570 and
    matrix_util.h:206-300 with window 1; cross-row similarity as csr_cross_row_similarity,
    the mean over non-empty rows)."""
    rp = np.asarray(rp, np.int64)
    ci = np.asarray(ci, np.int64)
    nnz = int(rp[-1]) if m > 0 else 0
    deg = np.diff(rp).astype(np.float64)
    md = float(m) if m > 0 else 1.0
    avg = deg.sum() / md
    var = (deg * deg).sum() / md - avg * avg
    ne = deg > 0
    first = np.where(ne, ci[np.minimum(rp[:-1], max(nnz - 1, 0))] if nnz else 0, 0)
    last = np.where(ne, ci[np.maximum(rp[1:] - 1, 0)] if nnz else 0, 0)
    bw = np.where(ne, last - first + 1, 0).astype(np.float64)
    rows = np.repeat(np.arange(m), np.diff(rp))
    same = rows[1:] == rows[:-1] if nnz > 1 else np.zeros(0, bool)
    d = np.diff(ci) if nnz > 1 else np.zeros(0, np.int64)
    consec = np.bincount(rows[1:][same & (d <= 1)], minlength=m) if nnz > 1 else np.zeros(m)
    newgrp = np.bincount(rows[1:][same & (d > 1)], minlength=m) if nnz > 1 else np.zeros(m)
    groups = np.where(ne, 1 + newgrp, 0)
    # cross-row similarity: each non-empty row against the next non-empty row
    nz_rows = np.nonzero(ne)[0]
    crs = 0.0
    if nz_rows.size > 1:
        nxt = np.full(m, -1, np.int64)
        nxt[nz_rows[:-1]] = nz_rows[1:]
        W = n + 3
        key = rows * W + ci
        tgt = nxt[rows]
        ok = tgt >= 0
        lo = tgt * W + ci - 1
        idx = np.searchsorted(key, lo, "left")
        hit = ok & (idx < nnz)
        hit[hit] = key[idx[hit]] <= (tgt * W + ci + 1)[hit]
        sim = np.bincount(rows[hit], minlength=m).astype(np.float64)
        crs = float(np.sum(np.where(ne, sim / np.maximum(deg, 1), 0.0)))
    out = np.zeros(10)
    out[0] = np.log2(m + 1.0)
    out[1] = np.log2(nnz + 1.0)
    out[2] = avg
    out[3] = np.sqrt(max(var, 0.0)) / avg if avg > 0 else 0.0
    out[4] = (deg.max() - avg) / avg if avg > 0 else 0.0
    out[5] = (bw / n).sum() / md if n > 0 else 0.0
    out[6] = np.where(ne, deg / np.maximum(bw, 1), 0.0).sum() / md
    out[7] = 2.0 * consec.sum() / nnz if nnz > 0 else 0.0
    out[8] = crs / nz_rows.size if nz_rows.size > 0 else 0.0
    out[9] = np.where(ne, groups / np.maximum(deg, 1), 0.0).sum() / md
    return out


def mlp_offsets(dims):
    """Offsets of W1, b1, W2, b2, W3, b3 in the flat parameter vector."""
    offs, o = [], 0
    for l in range(3):
        offs.append((o, o + dims[l + 1] * dims[l]))
        o += dims[l + 1] * dims[l] + dims[l + 1]
    return offs, o


def mlp_loss_grad(params, dims, X, labels):
    """FP64 forward + backward of the selector MLP (ReLU hidden layers, mean softmax
    cross-entropy): (loss, flat gradient, logits)."""
    p = np.asarray(params, np.float64)
    offs, total = mlp_offsets(dims)
    Ws = [p[w0:b0].reshape(dims[l + 1], dims[l]) for l, (w0, b0) in enumerate(offs)]
    bs = [p[b0:b0 + dims[l + 1]] for l, (w0, b0) in enumerate(offs)]
    X = np.asarray(X, np.float64)
    B = X.shape[0]
    z1 = X @ Ws[0].T + bs[0]
    a1 = np.maximum(z1, 0)
    z2 = a1 @ Ws[1].T + bs[1]
    a2 = np.maximum(z2, 0)
    z3 = a2 @ Ws[2].T + bs[2]
    mx = z3.max(1, keepdims=True)
    lse = mx[:, 0] + np.log(np.exp(z3 - mx).sum(1))
    y = np.asarray(labels, np.int64)
    loss = float(np.mean(lse - z3[np.arange(B), y]))
    d3 = np.exp(z3 - lse[:, None])
    d3[np.arange(B), y] -= 1.0
    d3 /= B
    g = np.zeros(total)
    acts = [X, a1, a2]
    zs = [z1, z2]
    d = d3
    for l in (2, 1, 0):
        w0, b0 = offs[l]
        g[w0:b0] = (d.T @ acts[l]).ravel()
        g[b0:b0 + dims[l + 1]] = d.sum(0)
        if l > 0:
            d = (d @ Ws[l]) * (zs[l - 1] > 0)
    return loss, g, z3
