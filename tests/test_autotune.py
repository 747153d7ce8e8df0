"""Launch-shape autotuner.

CPU: mode switches and argument checks, and the text table (load merges, save
writes back what was loaded). GPU: the shape it tunes (the cluster size of the
blocked RRQR) never changes results: factorizations explored with different
cluster sizes give bitwise identical preconditioner applications, in FP32 and
FP64, and a frozen table reproduces them too.
"""
import numpy as np
import pytest

from spaqr_public_b200 import FP32, FP64, Tree, _abi, autotune, matgen

TABLE = """# kind dev elem rows_log2 cols_log2 tasks_log2 candidate count best_cost
0 0 4 7 12 8 4 2 1.250000000e-09
0 0 4 7 12 8 8 2 2.500000000e-09
0 0 8 9 13 4 16 2 3.000000000e-09
"""


@pytest.fixture
def restore_tuner():
    mode = autotune()[0]
    yield
    autotune(mode=mode, reset=True)


def test_modes_and_argument_checks(restore_tuner):
    assert autotune(mode=0)[0] == 0
    assert autotune(mode=2)[0] == 2
    assert autotune(mode=1)[0] == 1
    L = _abi.lib()
    assert L.spq_autotune_set_mode(3) == 1
    assert b"autotune mode" in L.spq_last_error()
    assert L.spq_autotune_get(None, None, None) == 1
    assert L.spq_autotune_save(None) == 1


def test_table_load_save_roundtrip(tmp_path, restore_tuner):
    src = tmp_path / "in.txt"
    src.write_text(TABLE)
    autotune(reset=True)
    assert autotune(load=src)[1] == 3
    out = tmp_path / "out.txt"
    autotune(save=out)
    lines = [ln for ln in out.read_text().splitlines() if not ln.startswith("#")]
    want = [ln for ln in TABLE.splitlines() if not ln.startswith("#")]
    assert [ln.split()[:8] for ln in lines] == [ln.split()[:8] for ln in want]
    assert np.allclose([float(ln.split()[8]) for ln in lines], [float(ln.split()[8]) for ln in want])
    # loading merges, reset clears
    assert autotune(load=src)[1] == 3
    assert autotune(reset=True)[1] == 0
    bad = tmp_path / "bad.txt"
    bad.write_text("0 0 4 not a table\n")
    with pytest.raises(_abi.SpqError) as e:
        autotune(load=bad)
    assert e.value.code == 1
    with pytest.raises(_abi.SpqError):
        autotune(load=tmp_path / "missing.txt")


def _apply(name, prec, b):
    w = matgen.workload(name)
    A = matgen.column_normalize(w["A"])
    t = Tree(w["levels"], w["skip"], precision=prec)
    t.set_tol(w["tol"])
    t.set_scale(1)
    t.set_square(1)
    t.set_coords_grid(w["n"], w["d"])
    t.partition(A)
    t.assemble(A)
    t.factorize()
    y = t.solve(b)
    t.close()
    return y


@pytest.mark.gpu
@pytest.mark.parametrize("name,prec", [("advdiff3d_32", FP32), ("advdiff3d_32", FP64), ("advdiff2d_128", FP64)])
def test_tuned_shapes_do_not_change_results(gpu, name, prec, restore_tuner):
    w = matgen.workload(name)
    b = np.random.default_rng(5).standard_normal(w["A"][0])
    autotune(mode=1, reset=True)
    ys = []
    for _ in range(4):  # the default shape first, then the other fitting cluster sizes
        ys.append(_apply(name, prec, b))
    _, entries, _ = autotune()
    assert entries > 0
    assert all(np.array_equal(ys[0], y) for y in ys[1:])
    autotune(mode=2)  # frozen: the explored table only
    assert np.array_equal(ys[0], _apply(name, prec, b))
    autotune(mode=0)  # off: the built-in default
    assert np.array_equal(ys[0], _apply(name, prec, b))
