"""The tensor-core MLP (csrc/mlp.cu: tcgen05 GEMMs, BF16 operands, FP32
accumulate) against the FP64 reference (oracle/mlp.py), through the C ABI.

Tolerance: the GPU rounds every activation to BF16 (8-bit mantissa) between
layers, so outputs are compared as max |gpu - ref| / rms(ref) <= 3e-2 and
per-layer gradients as ||gpu - ref|| / ||ref|| <= 5e-2, with the reference
run on the same BF16-rounded weights and inputs."""
import numpy as np
import pytest

from oracle import mlp as M

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
S = pytest.importorskip("hackathon_b200.surrogate")


def _bf16(a):
    return torch.tensor(np.asarray(a, np.float32)).to(torch.bfloat16).to(torch.float64).numpy()


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = np.concatenate([rng.uniform(0, 1, (n, 64)), rng.uniform(-1, 0, (n, 1))], 1).astype(np.float32)
    y = rng.normal(size=(n, 5)).astype(np.float32)
    return x, y


def _rounded_params(net):
    p = net.get_params().astype(np.float64)
    layers = M.unflatten(p)
    return M.flatten([(_bf16(W), b) for W, b in layers])  # biases stay FP32 on the GPU


@pytest.mark.parametrize("n", [200, 1024])
def test_forward_matches_fp64_reference(n):
    net = S.Surrogate(batch_max=2048, seed=3)
    x, _ = _inputs(n, 1)
    out = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    net.sync()
    ref = M.forward(_rounded_params(net), _bf16(x))
    err = np.abs(out - ref).max() / np.sqrt((ref ** 2).mean())
    assert err <= 3e-2, err
    net.close()


@pytest.mark.parametrize("n", [256, 4096])
def test_gradients_match_fp64_reference(n):
    net = S.Surrogate(batch_max=4096, seed=4)
    x, y = _inputs(n, 2)
    loss, g = net.gradients(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda())
    ref_loss, ref = M.loss_and_grads(_rounded_params(net), _bf16(x), y.astype(np.float64))
    assert abs(loss - ref_loss) <= 1e-2 * ref_loss
    off = 0
    for i, o in M.DIMS:
        for k in (o * i, o):  # W then b
            a, b = g[off:off + k], ref[off:off + k]
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            assert rel <= 5e-2, (i, o, k, rel)
            off += k
    net.close()


def test_training_reduces_loss():
    net = S.Surrogate(batch_max=1024, seed=5)
    rng = np.random.default_rng(6)
    x = np.concatenate([rng.uniform(0, 1, (1024, 64)), rng.uniform(-1, 0, (1024, 1))], 1).astype(np.float32)
    # smooth targets of the inputs
    y = np.stack([x[:, :8].mean(1), x[:, 8:16].std(1) * 3, x[:, 64], np.sin(3 * x[:, 20]), x[:, 30] * x[:, 40]],
                 1).astype(np.float32)
    xt, yt = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    first = net.train_step(xt, yt, 1e-3, want_loss=True)
    for _ in range(300):
        net.train_step(xt, yt, 1e-3)
    last = net.train_step(xt, yt, 1e-3, want_loss=True)
    assert last < 0.1 * first, (first, last)
    net.close()


def test_rejects_bad_sizes():
    from hackathon_b200.engine import DdmArgError
    net = S.Surrogate(batch_max=64, seed=0)
    x = torch.zeros((65 * 72,), device="cuda").view(72, 65)
    with pytest.raises(DdmArgError):
        net.forward(x)  # 72 rows > batch_max
    with pytest.raises(DdmArgError):
        net.forward(x[:12])  # not a multiple of 8
    net.close()
