"""sj_mlp_loss_grad_noalloc against sj_mlp_loss_grad.

Some callers of this library cannot allocate device memory: work that is
being captured into a CUDA graph may not call cudaMalloc, and services that
reserve all of their GPU memory at start-up must not grow the device heap
afterwards.  sj_mlp_loss_grad_noalloc computes the estimator's loss and
gradient in caller-owned device buffers and keeps its per-sample scratch in a
fixed array inside the library.  These tests check it against the allocating
entry point on two calls in a row (the second with a different batch, so a
value left in the shared scratch or loss accumulator would show), and that a
batch larger than the fixed scratch is refused.
"""
import numpy as np
import pytest

import sjoin

pytestmark = pytest.mark.gpu


def _data(m, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((m, 16)).astype(np.float32)
    t = np.stack([x[:, :4].sum(1), np.abs(x[:, 4:8]).sum(1)], 1).astype(np.float32)
    return x, t


def test_noalloc_gradient_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    w = sjoin.mlp_init(7)
    wd = torch.from_numpy(w).to(dev)
    loss_d = torch.empty(1, dtype=torch.float32, device=dev)
    grad_d = torch.empty(w.size, dtype=torch.float32, device=dev)
    for m, seed in [(4096, 1), (777, 2)]:
        x, t = _data(m, seed)
        ref_loss, ref_grad = sjoin.mlp_loss_grad(x, t, w)
        xd = torch.from_numpy(x).to(dev)
        td = torch.from_numpy(t).to(dev)
        sjoin.mlp_loss_grad_noalloc(xd.data_ptr(), td.data_ptr(), m, wd.data_ptr(), loss_d.data_ptr(),
                                    grad_d.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize(dev)
        g = grad_d.cpu().numpy()
        loss = float(loss_d.item())
        # the tolerance of the estimator gradient tests (FP32 sums over samples)
        np.testing.assert_allclose(g, ref_grad, rtol=2e-3, atol=2e-5 * max(1.0, np.abs(ref_grad).max()))
        assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))


def test_noalloc_refuses_batches_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float32, device=dev)
    p = buf.data_ptr()
    with pytest.raises(sjoin.SJError) as e:
        sjoin.mlp_loss_grad_noalloc(p, p, sjoin.MLP_NOALLOC_MAX_SAMPLES + 1, p, p, p, 0)
    assert e.value.status == sjoin.SJ_ERR_BAD_INPUT
    assert "8192" in str(e.value)
