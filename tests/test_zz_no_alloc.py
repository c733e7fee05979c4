"""ks_gram_device_noalloc, the Gram entry point that allocates no device memory, against the allocating
ks_gram (gram_mode 0): bit-for-bit the same matrix on two calls in a row (the static scratch is reused
without clearing), with and without a T block, and against the f64 products of the same f32 inputs to
the Gram tests' 2e-6 relative bound (an independent answer, not only the solver's own Gram); and a clear
KS_INVALID (ValueError) without any launch for a block beyond the 4 MiB scratch. This file is collected
last so that it also runs after every other GPU test in the same process."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_fields(torch, ks, n, dense):
    """(count, n^3) f64 host fields -> (count, n, n, P) f32 pitched device block, pads 0."""
    P = ks.field_pitch(n)
    count = dense.shape[0]
    out = torch.zeros(count, n, n, P, dtype=torch.float32, device="cuda:0")
    out[..., :n] = torch.from_numpy(dense.reshape(count, n, n, n)).to("cuda:0").float()
    return out


@pytest.mark.parametrize("m,mt", [(10, 14), (7, 0)])
def test_noalloc_gram_matches_ks_gram_on_two_calls(ks, m, mt):
    import torch

    n = 33
    rng = np.random.default_rng(11 + m + mt)
    s = rng.standard_normal((m, n ** 3))
    t = rng.standard_normal((mt, n ** 3))
    ref = ks.gram(n, s, t, gram_mode=0)
    S = _device_fields(torch, ks, n, s)
    T = _device_fields(torch, ks, n, t) if mt > 0 else None
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for _ in range(2):
        out = torch.full((m, m + mt), float("nan"), dtype=torch.float64, device="cuda:0")
        ks.gram_device_noalloc(stream, n, m, S.data_ptr(), mt, T.data_ptr() if T is not None else 0, out.data_ptr())
        outs.append(out)
    torch.cuda.synchronize()
    for out in outs:
        got = out.cpu().numpy()
        assert np.array_equal(got, ref), np.abs(got - ref).max()
    s32 = s.astype(np.float32).astype(np.float64)
    t32 = t.astype(np.float32).astype(np.float64)
    cols = np.concatenate([s32, t32]) if mt > 0 else s32
    want = s32 @ cols.T
    scale = np.sqrt(np.outer((s32 * s32).sum(1), (cols * cols).sum(1)))
    assert np.abs(outs[-1].cpu().numpy() - want).max() / scale.max() < 2e-6


def test_noalloc_gram_rejects_a_block_beyond_its_scratch(ks):
    import torch

    n, m, mt = 9, 40, 40  # 2 * 148 * 40 * 80 partials > 2^19
    S = torch.zeros(m + mt, n, n, ks.field_pitch(n), dtype=torch.float32, device="cuda:0")
    out = torch.zeros(m, m + mt, dtype=torch.float64, device="cuda:0")
    before = ks.launch_count()
    with pytest.raises(ValueError, match="static scratch"):
        ks.gram_device_noalloc(torch.cuda.current_stream().cuda_stream, n, m, S.data_ptr(), mt, S[m:].data_ptr(),
                               out.data_ptr())
    assert ks.launch_count() == before
