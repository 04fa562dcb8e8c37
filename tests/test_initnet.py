"""Learned initialiser: the tensor-core BF16 GEMM its layers run on, against an FP64
product of the same BF16 operands."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemm(A, B):
    import torch
    from sitk_b200 import _lib
    from sitk_b200.metric import default_context
    L = _lib.load()
    L.mi_gemm_bf16_tn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    L.mi_gemm_bf16_tn.restype = ctypes.c_int
    M, K = A.shape
    N = B.shape[0]
    C = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    ctx = default_context()
    _lib.check(L.mi_gemm_bf16_tn(ctx.handle, M, N, K, A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0),
                                 C.data_ptr(), C.stride(0)), ctx.handle)
    return C


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (300, 48, 200), (1000, 128, 1000), (64, 12, 256),
                                   (257, 256, 130), (130, 40, 54)])
def test_tensor_core_gemm_matches_fp64(M, N, K):
    import torch
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn((M, K), generator=g).to(torch.bfloat16).cuda()
    B = torch.randn((N, K), generator=g).to(torch.bfloat16).cuda()
    C = _gemm(A, B).cpu().double().numpy()
    ref = A.cpu().double().numpy() @ B.cpu().double().numpy().T
    # FP32 accumulation of K exact BF16 products
    tol = 1e-5 * np.sqrt(K) * (np.abs(A.cpu().double().numpy()) @ np.abs(B.cpu().double().numpy()).T) + 1e-6
    assert np.all(np.abs(C - ref) <= tol), np.max(np.abs(C - ref))


def test_tensor_core_gemm_strided_operands():
    import torch
    g = torch.Generator(device="cpu").manual_seed(5)
    A = torch.randn((200, 96), generator=g).to(torch.bfloat16).cuda()[:, :80]   # lda 96
    B = torch.randn((24, 88), generator=g).to(torch.bfloat16).cuda()[:, :80]    # ldb 88
    C = _gemm(A, B).cpu().double().numpy()
    ref = A.cpu().double().numpy() @ B.cpu().double().numpy().T
    assert np.max(np.abs(C - ref)) < 1e-3


# ---------------------------------------------------------------------------
# the network: forward and every layer's gradients against a torch-CPU FP64
# restatement that rounds to BF16 exactly where the device does (GEMM operands:
# the input, weights, activations and the output gradient fed to each GEMM)
# ---------------------------------------------------------------------------

def _bf(t):
    import torch
    return t.float().to(torch.bfloat16).double()


def _conv_w(w, cin):
    """Device weight (out × 27·cin, column ((kz·3+ky)·3+kx)·cin + c) → torch (out, cin, 3, 3, 3)."""
    import torch
    w = torch.as_tensor(np.asarray(w, dtype=np.float64))
    return w.reshape(w.shape[0], 3, 3, 3, cin).permute(0, 4, 1, 2, 3).contiguous()


def _conv_w_back(g):
    return g.permute(0, 2, 3, 4, 1).reshape(g.shape[0], -1).numpy()


def _reference(state, x, t):
    """Forward output and per-layer (dW, db) of the mean squared error, FP64."""
    import torch
    import torch.nn.functional as F
    from torch.nn.grad import conv3d_input, conv3d_weight
    chans = [2, 16, 32, 64, 128]
    W = [_bf(_conv_w(state[l][0], chans[l])) for l in range(4)] + \
        [_bf(torch.as_tensor(state[l][0].astype(np.float64))) for l in (4, 5)]
    b = [torch.as_tensor(state[l][1].astype(np.float64)) for l in range(6)]
    a = [_bf(torch.as_tensor(x.astype(np.float64)).permute(0, 4, 1, 2, 3))]  # GEMM inputs, NCDHW
    z = []
    for l in range(4):
        zl = F.conv3d(a[l], W[l], b[l], stride=2, padding=1)
        z.append(zl)
        a.append(_bf(torch.relu(zl)))
    B = x.shape[0]
    flat = a[4].permute(0, 2, 3, 4, 1).reshape(B, 1024)
    z4 = flat @ W[4].T + b[4]
    a5 = _bf(torch.relu(z4))
    out = a5 @ W[5].T + b[5]
    tt = torch.as_tensor(t.astype(np.float64))
    n = out.numel()
    grads = [None] * 6
    dz = 2.0 * (out - tt) / n
    grads[5] = ((_bf(dz).T @ a5).numpy(), dz.sum(0).numpy())
    dz4 = (_bf(dz) @ W[5]) * (z4 > 0)
    grads[4] = ((_bf(dz4).T @ flat).numpy(), dz4.sum(0).numpy())
    dx = (_bf(dz4) @ W[4]).reshape(B, 2, 2, 2, 128).permute(0, 4, 1, 2, 3)
    dzl = dx * (z[3] > 0)
    for l in (3, 2, 1, 0):
        gw = conv3d_weight(a[l], W[l].shape, _bf(dzl), stride=2, padding=1)
        grads[l] = (_conv_w_back(gw), dzl.sum((0, 2, 3, 4)).numpy())
        if l:
            dxl = conv3d_input(a[l].shape, W[l], _bf(dzl), stride=2, padding=1)
            dzl = dxl * (z[l - 1] > 0)
    return out.numpy(), grads, float(((out - tt) ** 2).mean())


def test_initnet_forward_and_gradients_match_fp64():
    import torch
    from sitk_b200.initnet import InitNet
    rng = np.random.default_rng(11)
    B = 3
    x = rng.standard_normal((B, 32, 32, 32, 2)).astype(np.float32)
    t = rng.standard_normal((B, 12)).astype(np.float32)
    net = InitNet(seed=5, max_batch=4)
    state = net.state()
    # biases 0 at creation: give them values so their path is exercised
    for l in range(6):
        w, b0 = state[l]
        b = (0.05 * rng.standard_normal(b0.shape)).astype(np.float32)
        net.set(l, w, b)
        state[l] = (w, b)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    out = net.forward(xd).cpu().double().numpy()
    ref_out, ref_grads, ref_loss = _reference(state, x, t)
    scale = np.max(np.abs(ref_out))
    assert np.max(np.abs(out - ref_out)) <= 1e-2 * scale, (np.max(np.abs(out - ref_out)), scale)
    loss = net.train_step(xd, td, lr=0.0)  # gradients only
    assert abs(loss - ref_loss) <= 1e-2 * ref_loss
    for l in range(6):
        gw, gb = net.get(l, grads=True)
        rw, rb = ref_grads[l]
        ew = np.max(np.abs(gw - rw)) / np.max(np.abs(rw))
        eb = np.max(np.abs(gb - rb)) / np.max(np.abs(rb))
        assert ew <= 1e-2 and eb <= 1e-2, (l, ew, eb)
    net.close()


def test_initnet_weights_round_trip_and_training_reduces_loss():
    import torch
    from sitk_b200.initnet import InitNet
    rng = np.random.default_rng(3)
    B = 8
    x = torch.from_numpy(rng.standard_normal((B, 32, 32, 32, 2)).astype(np.float32)).cuda()
    t = torch.from_numpy((0.5 * rng.standard_normal((B, 12))).astype(np.float32)).cuda()
    net = InitNet(seed=1, max_batch=B)
    w, b = net.get(2)
    net.set(2, w, b)
    w2, b2 = net.get(2)
    assert np.array_equal(w, w2) and np.array_equal(b, b2)
    first = net.train_step(x, t, lr=1e-3)
    for _ in range(60):
        last = net.train_step(x, t, lr=1e-3)
    assert last < 0.1 * first, (first, last)
    # the same seed gives the same weights, and the same steps the same result
    net2 = InitNet(seed=1, max_batch=B)
    assert np.array_equal(net2.get(0)[0], InitNet(seed=1, max_batch=1).get(0)[0])
    net.close()
    net2.close()


def test_initnet_prepare_matches_oracle_resample(oracle_lib):
    import torch
    from sitk_b200.initnet import prepare
    from sitk_b200.metric import DeviceImage
    from sitk_b200 import synth
    import oracle
    p = synth.make_pair(48, 8, 21, 10.0, 4.0)
    spacing, origin = (1.5, 1.0, 0.8), (3.0, -2.0, 1.0)
    f = DeviceImage.upload(p.fixed, spacing=spacing, origin=origin)
    m = DeviceImage.upload(p.moving, spacing=spacing, origin=origin)
    x = prepare(f, m).cpu().numpy()
    gi = oracle.make_geometry((48, 48, 48), spacing, origin)
    go = oracle.make_geometry((32, 32, 32), [s * 48 / 32 for s in spacing],
                              [o + s * (47 / 2 - 1.5 * 31 / 2) for o, s in zip(origin, spacing)])
    for ch, vol in enumerate((p.fixed, p.moving)):
        r = oracle.resample_linear(vol, gi, go).astype(np.float64)
        r = (r - r.mean()) / r.std()
        assert np.max(np.abs(x[..., ch] - r)) < 1e-4


def test_trained_initialiser_beats_centred_start():
    """A network trained on 1,024 labelled 64³ pairs (rotation ±20°, translation
    ±10 mm, scale 0.9–1.1): refined proposals reach the plain run's final metric value
    within 1e-3 on nearly every held-out pair, in fewer optimizer iterations, and land
    within 1 mm of the truth at least as often as the centred start does."""
    from sitk_b200 import initnet as I
    spec = I.PairSpec(n=64, nblobs=20, rot_deg=20.0, trans_mm=10.0)
    run = I.PlainRun(bins=32, percentage=0.2, iterations=200)
    data = I.labelled_set(range(100, 1124), spec, run)
    # the labels are the metric's optimum next to the generating affine
    c = [31.5] * 3
    assert np.median([I.target_error(l, t, c, 19.2) for l, t in zip(data["labels"], data["truth"])]) < 0.5
    net = I.InitNet(seed=2, max_batch=64)
    losses, _ = I.train(net, data["x"], data["labels"], epochs=10)
    assert losses[-1] < 0.5 * losses[0]
    ev = I.evaluate(net, range(500000, 500064), spec, run, single_pairs=2)
    assert ev["accepted"] >= 0.9, ev
    assert ev["iterations"]["learned"]["mean"] < ev["iterations"]["plain"]["mean"], ev
    assert ev["within_1mm"]["learned"] >= ev["within_1mm"]["plain"], ev
    net.close()
