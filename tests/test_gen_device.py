"""The artificial generator on the GPU (spmv_gen_create_device, one thread per anchor
segment) against the native host generator, which is pinned bit for bit on the reference's
own generator (tests/test_artgen.py).

CPU: the GPU generator's per-segment code, run on the host with glibc's libm
(spmv_gen_host_check), is the host generator's output bit for bit -- the random stream
(glibc random_r TYPE_4, restated) and every step.
GPU: the same code with CUDA's libm.  Bars: the same nnz within 0.1%, at least 99% of rows
with the same columns, the structural features within 1% (distribution-equivalent), and
the matrices of the benchmark configurations identical where the two libms agree.
"""
import numpy as np
import pytest

CASES = [(100000, 100000, 10, 2, "normal", "random", 0.3, 0, 1.0, 0.5, 14),
         (400000, 400000, 20, 15, "gamma", "random", 0.05, 100, 2.0, 0.3, 7),
         (20000, 30000, 40, 30, "gamma", "diagonal", 0.2, 50, 1.5, 0.4, 3),
         (5000, 5000, 8, 0, "normal", "random", 0.5, 0, 0.0, 0.0, 99),
         (150, 300, 5, 2, "normal", "stripe", 0.1, 0, 1.0, 0.2, 1),
         (77, 77, 3, 1, "gamma", "random", 1.0, 2, 1.0, 0.5, 5)]


@pytest.mark.parametrize("case", CASES)
def test_generator_code_matches_host_generator_on_cpu(sb, case):
    g = sb.generate_artificial(*case)
    m, cap = case[0], g.nnz + 8
    rp, ci, v = np.zeros(m + 1, np.int32), np.zeros(cap, np.int32), np.zeros(cap)
    a = [case[0], case[1], case[2], case[3], case[4].encode(), case[5].encode()] + list(case[6:])
    nnz = sb.library().spmv_gen_host_check(*a, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, cap)
    assert nnz == g.nnz
    assert np.array_equal(rp, g.row_ptr) and np.array_equal(ci[:nnz], g.col_ind)
    assert np.array_equal(v[:nnz].view(np.uint64), g.values.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES + [(2000000, 2000000, 30, 30, "gamma", "random", 0.2, 150, 1.8, 0.4, 12345)])
def test_device_generator_is_distribution_equivalent(sb, case):
    from spmv_dare_b200 import selector

    rp_d, ci_d, v_d = sb.generate_artificial_device(*case)
    rp, ci, v = rp_d.cpu().numpy(), ci_d.cpu().numpy(), v_d.cpu().numpy()
    g = sb.generate_artificial(*case)
    m, n = case[0], case[1]
    assert abs(int(rp[-1]) - g.nnz) <= max(2, 1e-3 * g.nnz)
    assert np.all(np.diff(rp) >= 0) and np.all((ci >= 0) & (ci < n)) and np.all((v >= 0) & (v < 1))
    same = 0
    lens_h, lens_d = np.diff(g.row_ptr), np.diff(rp)
    for i in np.random.default_rng(0).choice(m, size=min(m, 3000), replace=False):
        if lens_h[i] == lens_d[i] and np.array_equal(ci[rp[i]:rp[i + 1]], g.col_ind[g.row_ptr[i]:g.row_ptr[i + 1]]):
            same += 1
    assert same >= 0.99 * min(m, 3000), same
    fh = selector.features(g.row_ptr, g.col_ind, m, n)
    fd = selector.features(rp, ci, m, n)
    assert np.allclose(fd, fh, rtol=1e-2, atol=1e-3), (fd, fh)
