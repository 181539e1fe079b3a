"""The surrogate network's tensor-core kernels (include/sph_mlp.h) against a plain PyTorch
FP32 reference on the same bf16 operands."""
import ctypes

import numpy as np
import pytest
import torch

import sph_b200

pytestmark = pytest.mark.gpu

PF = ctypes.POINTER(ctypes.c_float)


def tc_gemm(A, B, heads, M, N, K):
    L = sph_b200.lib()
    L.sph_tc_gemm.argtypes = [ctypes.c_void_p, ctypes.c_void_p, PF, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    C = torch.full((heads, M, N), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    st = L.sph_tc_gemm(A.data_ptr(), B.data_ptr(), ctypes.cast(C.data_ptr(), PF), M, N, K,
                       heads, None)
    assert st == 0, sph_b200.STATUS.get(st, st)
    return C


@pytest.mark.parametrize("M,N,K,heads", [(128, 256, 64, 1), (256, 256, 256, 5),
                                         (128, 16, 128, 1), (256, 128, 1024, 2),
                                         (1024, 256, 256, 5)])
def test_tc_gemm_matches_fp32_reference(M, N, K, heads):
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K + heads)
    A = torch.randn(heads, M, K, generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn(heads, N, K, generator=g, device="cuda").to(torch.bfloat16)
    C = tc_gemm(A, B, heads, M, N, K)
    ref = torch.matmul(A.double(), B.double().transpose(1, 2))
    err = (C.double() - ref).abs().max().item()
    scale = ref.abs().max().item()
    # bf16 x bf16 products are exact in FP32; only the summation order differs
    assert err <= 1e-5 * scale, (err, scale)


# ---- the network (sph_surrogate.MLP) against the FP64 oracle (oracle/mlp_oracle.py) ----

def _batch(n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn(n, 6, generator=g, device="cuda")
    y = torch.randn(n, 4, generator=g, device="cuda")
    return x, y


@pytest.mark.parametrize("batch", [256, 1024])
def test_mlp_gradients_match_fp64_oracle(batch):
    """Batch 256: the weight gradients split K over 4 CTAs per tile; batch 1024: over 8, and
    the forward and input-gradient GEMMs take two column tiles per row tile."""
    import mlp_oracle
    import sph_surrogate

    net = sph_surrogate.MLP(heads=2, max_batch=batch, seed=3)
    x, y = _batch(batch, 1)
    loss, g = net.gradients(x, y)
    P = net.get_params()
    xs, ys = x.cpu().numpy(), y.cpu().numpy()
    for h in range(2):
        ref_loss, ref_g = mlp_oracle.loss_and_grads(P[h], xs, ys)
        assert abs(loss[h] - ref_loss) <= 1e-4 * ref_loss, (h, loss[h], ref_loss)
        for name, (a, b) in mlp_oracle.OFFS.items():
            num = np.linalg.norm(g[h, a:b] - ref_g[a:b])
            den = np.linalg.norm(ref_g[a:b])
            # FP32 (GPU) versus FP64 accumulation, plus rare one-ulp bf16 rounding flips of
            # an activation whose FP32 pre-image sits next to a rounding boundary
            assert num <= 2e-3 * den, (h, name, num / den)
    net.close()


def test_mlp_predict_matches_oracle_forward():
    import mlp_oracle
    import sph_surrogate

    net = sph_surrogate.MLP(heads=3, max_batch=256, seed=9)
    x, _ = _batch(640, 2)  # several chunks of max_batch
    out = net.predict(x).cpu().numpy()
    P = net.get_params()
    for h in range(3):
        ref, _ = mlp_oracle.forward(P[h], x.cpu().numpy())
        # an activation whose FP32 pre-image sits at a bf16 rounding boundary may round the
        # other way on the GPU (one bf16 ulp, 2^-8 relative): a few outputs move by up to a
        # few 1e-3 of the output scale, the typical output by far less
        diff = np.abs(out[h] - ref)
        scale = np.abs(ref).max()
        assert diff.max() <= 5e-3 * scale, (h, diff.max() / scale)
        assert np.sqrt(np.mean(diff ** 2)) <= 5e-4 * scale, (h, np.sqrt(np.mean(diff ** 2)) / scale)
    net.close()


def test_mlp_training_fits_and_is_reproducible():
    import sph_surrogate

    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.rand(4096, 6, generator=g, device="cuda") * 2 - 1
    Y = torch.stack([torch.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2], X[:, 3] ** 2 - X[:, 4],
                     torch.cos(X[:, 5] + X[:, 0]), X.sum(1) / 3], dim=1).contiguous()
    nets = [sph_surrogate.MLP(heads=5, max_batch=512, seed=1) for _ in range(2)]
    first = last = None
    for s in range(400):
        idx = torch.randint(0, 4096, (512,), device="cuda",
                            generator=torch.Generator(device="cuda").manual_seed(s))
        xb, yb = X[idx].contiguous(), Y[idx].contiguous()
        losses = [n.train_step(xb, yb, 1e-3, want_loss=(s in (0, 399))) for n in nets]
        if s == 0:
            first = losses[0]
        if s == 399:
            last = losses[0]
            assert np.array_equal(losses[0], losses[1])
    assert np.all(last < 0.2 * first), (first, last)
    # bit-reproducible: the same seed and batches give the same weights
    assert np.array_equal(nets[0].get_params(), nets[1].get_params())
    # the heads start from different weights and stay different
    p = nets[0].get_params()
    assert not np.array_equal(p[0], p[1])
    for n in nets:
        n.close()
