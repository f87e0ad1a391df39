"""Matrix-Market import (the reference's real-matrix path, src/bench.cpp:127-238).

Fixtures: hand-written files in tests/golden/mtx/ (every field -- real, integer, complex,
pattern -- every symmetry -- general, symmetric, skew-symmetric, Hermitian -- a file
without banner, rectangular shapes, empty rows, entries out of order, extreme exponents),
with the CSR arrays the reference's own import produced for each (make_golden_mtx.py).

CPU: the oracle's harness (the reference compiled from its sources) is pinned on those
arrays, and malformed files are refused by the reader before any GPU work.
GPU: spmv_mtx_read (host parse, COO -> CSR on the GPU) gives the reference's arrays bit for
bit on every fixture and on generated files, and coo_to_csr on device arrays sorts like
the reference's coo_to_csr.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

MTX_DIR = os.path.join(GOLDEN, "mtx")
FIXTURES = sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(MTX_DIR, "*.mtx")))
INFO = ["m", "n", "nnz", "nnz_diag", "nnz_non_diag", "symmetric", "expanded"]


def _golden(name, e):
    with np.load(os.path.join(MTX_DIR, name + ".npz")) as z:
        return {k: z[f"e{e}_{k}"] for k in ("row_ptr", "col_ind", "values", "info")}


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("e", [1, 0])
def test_reference_harness_pinned_on_fixtures(orc, name, e):
    if not orc.ref_available("mtx"):
        pytest.skip("reference build (oracle/_ref) not present")
    g = _golden(name, e)
    r = orc.ref_read_mtx(os.path.join(MTX_DIR, name + ".mtx"), expand_symmetry=bool(e))
    assert np.array_equal(r["row_ptr"], g["row_ptr"]) and np.array_equal(r["col_ind"], g["col_ind"])
    assert np.array_equal(_bits(r["values"]), _bits(g["values"]))
    assert [r[k] for k in INFO] == g["info"].tolist()


BAD = {
    "array.mtx": "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",
    "field.mtx": "%%MatrixMarket matrix coordinate quaternion general\n1 1 1\n1 1 1\n",
    "symmetry.mtx": "%%MatrixMarket matrix coordinate real upper\n1 1 1\n1 1 1\n",
    "count.mtx": "%%MatrixMarket matrix coordinate real general\n3 3 3\n1 1 1\n2 2 2\n",
    "range.mtx": "%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1\n4 2 2\n",
    "value.mtx": "%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1\n2 2 abc\n",
    "subnormal.mtx": "%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1\n2 2 5e-324\n",
    "sizes.mtx": "%%MatrixMarket matrix coordinate real general\n3 x 2\n1 1 1\n2 2 2\n",
    "empty.mtx": "",
}


@pytest.mark.parametrize("name", sorted(BAD))
def test_malformed_files_are_refused(sb, tmp_path, name):
    """Each is an error in the reference's reader too (it prints and exits): the dense array
    format, unknown field or symmetry, a line count that differs from NNZ, a coordinate
    outside the matrix, a bad number, a strtod range error, bad sizes, an empty file."""
    p = tmp_path / name
    p.write_text(BAD[name])
    with pytest.raises(sb.SpmvError) as e:
        sb.read_mtx(str(p))
    assert e.value.status == 1


def test_missing_file_is_refused(sb, tmp_path):
    with pytest.raises(sb.SpmvError):
        sb.read_mtx(str(tmp_path / "nope.mtx"))


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("e", [1, 0])
def test_read_mtx_matches_reference_fixture(sb, name, e):
    g = _golden(name, e)
    r = sb.read_mtx(os.path.join(MTX_DIR, name + ".mtx"), expand_symmetry=bool(e))
    assert np.array_equal(r.row_ptr, g["row_ptr"]) and np.array_equal(r.col_ind, g["col_ind"])
    assert np.array_equal(_bits(r.values), _bits(g["values"]))
    assert [r.m, r.n, r.nnz, r.nnz_diag, r.nnz_non_diag, r.symmetric, r.symmetry_expanded] == g["info"].tolist()


def _write_random_mtx(path, m, n, nnz, symmetry, field, seed):
    rng = np.random.default_rng(seed)
    if symmetry == "general":
        flat = rng.choice(m * n, size=nnz, replace=False)
        r, c = flat // n, flat % n
    else:
        lo = [(i, j) for i in range(m) for j in range(i + (symmetry == "skew-symmetric"))]
        pick = rng.choice(len(lo), size=min(nnz, len(lo)), replace=False)
        r = np.array([lo[k][0] for k in pick])
        c = np.array([lo[k][1] for k in pick])
    lines = [f"%%MatrixMarket matrix coordinate {field} {symmetry}", "% generated", f"{m} {n} {r.size}"]
    for i, j in zip(r, c):
        if field == "real":
            lines.append(f"{i + 1} {j + 1} {rng.uniform(-1e3, 1e3):.17g}")
        elif field == "integer":
            lines.append(f"{i + 1} {j + 1} {int(rng.integers(-1000, 1000))}")
        else:
            lines.append(f"{i + 1} {j + 1}")
    path.write_text("\n".join(lines) + "\n")


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,nnz,symmetry,field", [(3000, 2000, 40000, "general", "real"),
                                                    (1500, 1500, 20000, "symmetric", "real"),
                                                    (800, 800, 9000, "skew-symmetric", "integer"),
                                                    (1200, 1200, 15000, "symmetric", "pattern")])
def test_read_mtx_matches_reference_generated(sb, orc, tmp_path, m, n, nnz, symmetry, field):
    """Generated files against the reference's import run on the same file, both
    expansions; then the imported matrix through csr_to_format + spmv against the
    reference's csr_naive on the reference's CSR (bit for bit)."""
    if not orc.ref_available("mtx"):
        pytest.fail("reference build (oracle/_ref) missing")
    p = tmp_path / "a.mtx"
    _write_random_mtx(p, m, n, nnz, symmetry, field, seed=m + nnz)
    for e in (True, False):
        ref = orc.ref_read_mtx(str(p), expand_symmetry=e)
        r = sb.read_mtx(str(p), expand_symmetry=e)
        assert np.array_equal(r.row_ptr, ref["row_ptr"]) and np.array_equal(r.col_ind, ref["col_ind"])
        assert np.array_equal(_bits(r.values), _bits(ref["values"]))
        assert (r.nnz_diag, r.nnz_non_diag, r.symmetric) == (ref["nnz_diag"], ref["nnz_non_diag"], ref["symmetric"])
    ref = orc.ref_read_mtx(str(p), expand_symmetry=True)
    r = sb.read_mtx(str(p), expand_symmetry=True)
    x = np.random.default_rng(1).uniform(-1, 1, r.n)
    mf = sb.csr_to_format(r.row_ptr, r.col_ind, r.values, r.m, r.n, r.nnz, r.symmetric, r.symmetry_expanded,
                          format="csr_naive")
    y = mf.spmv(x, np.full(r.m, 1.0))
    R = orc.RefFormat("csr_naive", ref["row_ptr"], ref["col_ind"], ref["values"], n=ref["n"], threads=8)
    try:
        assert np.array_equal(_bits(y), _bits(R.spmv(x)[:r.m]))
    finally:
        R.close()
    if r.symmetric:
        kept = sb.read_mtx(str(p), expand_symmetry=False)
        with pytest.raises(sb.SpmvError) as ex:      # every format rejects unexpanded symmetry (csr.cpp:131)
            sb.csr_to_format(kept.row_ptr, kept.col_ind, kept.values, kept.m, kept.n, kept.nnz, kept.symmetric,
                             kept.symmetry_expanded, format="sell")
        assert ex.value.status == 5


@pytest.mark.gpu
def test_coo_to_csr_device(sb):
    import torch

    rng = np.random.default_rng(3)
    m, n, nnz = 5000, 7000, 60000
    flat = rng.choice(m * n, size=nnz, replace=False)
    r, c = (flat // n).astype(np.int32), (flat % n).astype(np.int32)
    v = rng.uniform(-1, 1, nnz)
    rp, ci, vv = sb.coo_to_csr(torch.from_numpy(r).cuda(), torch.from_numpy(c).cuda(), torch.from_numpy(v).cuda(), m, n)
    order = np.lexsort((c, r))
    assert np.array_equal(rp.cpu().numpy(), np.concatenate([[0], np.cumsum(np.bincount(r, minlength=m))]))
    assert np.array_equal(ci.cpu().numpy(), c[order])
    assert np.array_equal(vv.cpu().numpy(), v[order])
    with pytest.raises(sb.SpmvError):
        bad = torch.from_numpy(np.array([0, m], np.int32)).cuda()
        sb.coo_to_csr(bad, bad, None, m, n)
