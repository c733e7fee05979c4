"""The stencil's launch-shape autotuner (ks_autotune_stencil) and its table: the choices are valid chunk counts, the
table round-trips through get / set / clear and a JSON file, and a tuned launch gives the same bits as the cost
model's -- H psi on host arrays and a whole H2 33^3 solve, with every count forced to the extreme chunkings."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def clean_table(ks):
    ks.clear_stencil_tuning()
    yield
    ks.clear_stencil_tuning()


def test_autotune_records_valid_choices(ks, clean_table, tmp_path):
    n = 47
    got = ks.autotune_stencil(n, [1, 8])
    assert set(got) == {1, 8}
    for k, modes in got.items():
        for c in modes.values():
            assert 1 <= c <= max(1, n // 8)
    table = sorted(ks.stencil_tuning())
    assert table == sorted([(n, k, 1, got[k]["hpsi"]) for k in got] + [(n, k, 2, got[k]["jacobi"]) for k in got])
    path = tmp_path / "tuning.json"
    ks.save_stencil_tuning(str(path))
    ks.clear_stencil_tuning()
    assert ks.stencil_tuning() == []
    ks.load_stencil_tuning(str(path))
    assert sorted(ks.stencil_tuning()) == table


def test_tuned_chunkings_give_the_same_bits(ks, oracle, clean_table):
    n, h = 33, 0.25
    x, y, z = oracle.grid_points(n, h)
    rng = np.random.default_rng(5)
    psi = rng.standard_normal((3, n ** 3))
    v = np.exp(-(x * x + y * y + z * z))
    ref = ks.apply_hamiltonian(n, h, psi, v)
    for c in (1, 2, 4):  # one chunk per tile column, two, the most for n = 33
        ks.set_stencil_tuning([(n, 3, 1, c)])
        assert np.array_equal(ks.apply_hamiltonian(n, h, psi, v), ref), c


def test_tuned_solve_is_bit_identical(ks, clean_table):
    """H2 on 33^3 with 1 + 3 bands per spin: every H psi and sweep shape the solve launches forced to one chunk, then to
    the most chunks, gives the untuned solve's energy and forces bit for bit."""
    nuc = [(0.7, 0.0, 0.0, 1), (-0.7, 0.0, 0.0, 1)]
    st = ks.ScfSettings(sigma=0.25, tol=1e-6)

    def solve():
        with ks.GpuSolver(33, 0.25, n_extra=3) as so:
            e = so.solve(ks.System(nuc, 1, 1), st)["energy"]["total"]
            return e, so.forces(nuc, 0.25)

    e0, f0 = solve()
    for c in (1, 4):
        ks.set_stencil_tuning([(33, k, mode, c) for k in range(1, 17) for mode in (1, 2)])
        e, f = solve()
        assert e == e0 and np.array_equal(f, f0), (c, e, e0)
