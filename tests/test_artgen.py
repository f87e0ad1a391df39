"""The native artificial-matrix generator reproduces the reference generator bit for bit
(golden fixtures made by the reference; 100k-row and 4M-row regression numbers)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden


def _gen_args(g):
    a = [str(s) for s in g["gen_args"]]
    return (int(a[0]), int(a[1]), float(a[2]), float(a[3]), a[4], a[5], float(a[6]), float(a[7]), float(a[8]),
            float(a[9]), int(a[10]))


@pytest.mark.parametrize("name", [n for n in golden_names() if n.startswith("gen_")])
@pytest.mark.parametrize("threads", [1, 3, 8])
def test_generator_matches_reference_fixture(sb, name, threads):
    g = load_golden(name)
    m = sb.generate_artificial(*_gen_args(g), threads=threads)
    assert np.array_equal(m.row_ptr, g["row_ptr"])
    assert np.array_equal(m.col_ind, g["col_ind"])
    assert np.array_equal((2.0 * m.values - 1.0).view(np.uint64), g["values"].view(np.uint64))


def test_generator_normal100k_regression(sb):
    m = sb.generate_artificial(100000, 100000, 10, 2, "normal", "random", 0.3, 0, 1.0, 0.5, 14)
    assert m.nnz == 999475
    assert m.stats["max_nnz_per_row"] == 19
    assert abs(m.stats["avg_bw"] - 28758.15214) < 1e-4
    assert abs(m.stats["skew"] - 0.900998024) < 1e-8
    assert abs(m.stats["avg_num_neighbours"] - 0.8642897521) < 1e-9
    assert abs(m.stats["cross_row_similarity"] - 0.455818) < 1e-6


def test_generator_gamma4m_regression(sb):
    m = sb.generate_artificial(4000000, 4000000, 20, 15, "gamma", "random", 0.05, 100, 2.0, 0.3, 7)
    assert m.nnz == 80469735
    assert m.stats["max_nnz_per_row"] == 2040
    assert abs(m.stats["skew"] - 100.404584) < 1e-5
    assert abs(m.stats["avg_num_neighbours"] - 1.896619) < 1e-6
    assert abs(m.stats["cross_row_similarity"] - 0.299312) < 1e-6
    assert abs(m.stats["std_nnz_per_row"] - 15.0167) < 1e-4


def test_generator_rejects_bad_sizes(sb):
    with pytest.raises(sb.SpmvError):
        sb.generate_artificial(0, 10, 5, 1, "normal", "random", 0.3, 0, 1.0, 0.5, 1)
