"""The guarded LOBPCG of the Fermi-Dirac channel solve (ks_lobpcg_guarded): the split stop test and the locked head,
after the reference's own test guarded_solve_locks_a_converged_head (crates/qm-gpu/src/eigen.rs:1118-1180) on the
harmonic oscillator 33^3 x 0.25 with k = 5: the head (1.5 and the 2.5 triplet, 4 columns) at tol = 3 x the f32 residual
floor, the fifth column (one of the 3.5 sextet) at the guard tolerance 1e-3."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, H, K, HEAD, GUARD = 33, 0.25, 5, 4, 1e-3
COEFF = [-205 / 72, 8 / 5, -1 / 5, 8 / 315, -1 / 560]


def floor_estimate(h):
    """The f32 residual floor model of crates/qm-gpu/src/eigen.rs:313-318."""
    s = 1.0 / (2.0 * h * h)
    mean = 3.0 * abs(COEFF[0]) * s
    var = 3.0 * 2.0 * sum(c * c for c in COEFF[1:]) * s * s
    return 2.4e-8 * np.sqrt(mean * mean + var)


@pytest.fixture(scope="module")
def rig(ks, oracle):
    x, y, z = oracle.grid_points(N, H)
    r2 = x * x + y * y + z * z
    v = (0.5 * r2).astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(11)
    guess = rng.uniform(-0.5, 0.5, (K + 1, N ** 3)) * np.exp(-r2 / 8.0)
    tol = 3.0 * floor_estimate(H)
    _, xs, _, _ = ks.lobpcg(N, H, v, guess[:K], tol=tol, max_iter=500)  # a converged 5-block: all at tol
    return v, xs, guess[K], tol


def guarded(ks, v, x, tol, **kw):
    return ks.lobpcg_guarded(N, H, v, x, tol, 1.5 * tol, HEAD, GUARD, K, max_iter=500, **kw)


def test_converged_block_is_accepted_at_the_guess(ks, rig):
    """(a) a block that meets both tiers is accepted at the guess, X bitwise; a fifth column whose residual sits between
    tol and the guard tolerance cannot push it into an iteration, which the block-wide test does on the same block."""
    v, xs, seed, tol = rig
    ev, x, res, st = guarded(ks, v, xs, tol)
    assert (st["iterations"], st["head_kept"]) == (0, True), st
    assert np.array_equal(x, xs)
    top = xs.copy()
    top[4] = xs[4] + 3e-6 * seed
    top = top.astype(np.float32).astype(np.float64)
    ev, x, res, st = guarded(ks, v, top, tol)
    assert 1.5 * tol < res[4] < GUARD, res
    assert (st["iterations"], st["head_kept"]) == (0, True), "a witness-tier residual never forces an iteration"
    assert np.array_equal(x, top)
    _, _, _, plain = ks.lobpcg_guarded(N, H, v, top, tol, 1.5 * tol, K, np.inf, K, max_iter=500, lock=False)
    assert plain["iterations"] > 0, ("the block-wide test iterates on the same block", plain)


@pytest.mark.parametrize("gram_mode", [0, 1])
def test_fresh_fifth_column_locks_the_head(ks, rig, gram_mode):
    """(b) the fifth column replaced by a fresh seed: the head is locked -- returned bitwise, head_kept -- and only the
    fifth column iterates, to the guard tolerance, landing on 3.5 Ha, orthogonal to the head; with the CUDA-core and
    the tensor-core Gram (the locked subspace [Y, X_a, W_a, P_a] has k + 2 (k - head) columns)."""
    v, xs, seed, tol = rig
    x0 = xs.copy()
    x0[4] = seed.astype(np.float32).astype(np.float64)
    ev, x, res, st = guarded(ks, v, x0, tol, gram_mode=gram_mode)
    assert st["iterations"] > 0 and st["head_kept"] and st["locked"] == HEAD, st
    assert np.array_equal(x[:HEAD], x0[:HEAD]), "the locked head is returned bitwise"
    assert res[4] < GUARD and abs(ev[4] - 3.5) < 2.0 * GUARD, (ev, res)
    gm = x @ x.T
    off = max(abs(gm[i, 4]) / np.sqrt(gm[i, i] * gm[4, 4]) for i in range(HEAD))
    assert off < 1e-5, f"the active column stays orthogonal to the head: max |cos| {off:.2e}"


def test_perturbed_head_iterates_the_whole_block(ks, rig):
    """(c) a head column perturbed: the whole block iterates (head_kept false), the head to tol and the fifth column to
    the guard tier (or a floor exit, which may leave it above its tier)."""
    v, xs, seed, tol = rig
    x0 = xs.copy()
    x0[0] = (xs[0] + 1e-2 * seed).astype(np.float32).astype(np.float64)
    ev, x, res, st = guarded(ks, v, x0, tol)
    assert st["iterations"] > 0 and not st["head_kept"] and st["locked"] == 0, st
    assert (res[:HEAD] < tol).all() and (res[4] < GUARD or st["stop"] == 1), (st, res)
    assert st["head_residual"] < tol, st


def test_untested_buffer_is_not_checked(ks, rig):
    """lobpcg_split with checked = 4: the fifth column is an untested buffer, so a fresh seed there leaves a converged
    head accepted at the guess (crates/qm-gpu/src/eigen.rs:613-618)."""
    v, xs, seed, tol = rig
    x0 = xs.copy()
    x0[4] = seed.astype(np.float32).astype(np.float64)
    ev, x, res, st = ks.lobpcg_guarded(N, H, v, x0, tol, 1.5 * tol, HEAD, GUARD, HEAD, max_iter=500, lock=False)
    assert st["iterations"] == 0 and st["head_kept"], st
    assert res[4] > GUARD  # measured, never tested
