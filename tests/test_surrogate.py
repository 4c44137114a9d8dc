"""Morphology surrogate: the FP64 oracle, the restated ga2d score, the BF16
tensor-core kernels against the oracle, training, and kMC labels."""
import os
import zlib

import numpy as np
import pytest

from oracle import cnn_oracle as C
from oracle import ga_score as G

HERE = os.path.dirname(os.path.abspath(__file__))


def rng_for(name):
    return np.random.default_rng(zlib.crc32(name.encode()))


# ---- CPU: the oracles ------------------------------------------------------------------------
def test_oracle_gradient_matches_finite_differences():
    """The FP64 oracle's analytic backward pass equals central differences."""
    rng = rng_for("fd")
    ph = (rng.random((2, 64, 128)) < 0.5).astype(np.uint8)
    P = C.init_params(1)
    y, cache = C.forward(ph, P, bf16=False)
    R = rng.standard_normal(y.shape)
    g = C.backward(R, cache, bf16=False)

    def loss(Q):
        return float((C.forward(ph, Q, bf16=False)[0] * R).sum())

    for ti in range(len(P)):
        scale = np.abs(g[ti]).max()
        for _ in range(2):
            idx = tuple(int(rng.integers(0, s)) for s in P[ti].shape)
            h = 1e-7  # small enough that no ReLU input crosses zero
            Pp = [p.copy() for p in P]
            Pm = [p.copy() for p in P]
            Pp[ti][idx] += h
            Pm[ti][idx] -= h
            fd = (loss(Pp) - loss(Pm)) / (2 * h)
            assert abs(fd - g[ti][idx]) <= 1e-5 * max(abs(g[ti][idx]), 1e-3 * scale), (ti, idx)


def test_round_bf16_nearest_even():
    v = np.array([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, 1 + 2 ** -7 + 2 ** -9, -3.14159, 0.0])
    assert C.round_bf16(v).tolist() == [1.0, 1.0, 1.015625, 1.0078125, -3.140625, 0.0]


def test_ga_score_matches_score_cache():
    """Restated ga.py:score on images of ga2d/score.cache (fixture of every sixth
    binary image): most equal the cached value to its 3 printed decimals, all
    agree within 0.05 (the score is a sum of terms of order 2e8)."""
    d = np.load(os.path.join(HERE, "golden", "ga_score.npz"))
    H, W = d["shape"]
    exact = 0
    for bits, cached in zip(d["images"], d["cached"]):
        im = (np.unpackbits(bits)[:H * W].reshape(H, W) * 255).astype(np.uint8)
        s = G.score(im)
        assert abs(s - cached) <= 0.05
        exact += abs(s - cached) <= 5e-4
    assert exact >= 0.8 * len(d["cached"])


def test_grf_morphology_fraction_and_correlation():
    torch = pytest.importorskip("torch")
    from langmuir_b200 import surrogate as S
    ph, ell, f = S.grf_morphologies(6, size=128, seed=3, device="cpu")
    assert ph.shape == (6, 128, 128) and ph.dtype == torch.uint8
    donor = (ph == 0).float().mean(dim=(1, 2))
    assert torch.allclose(donor, f, atol=1.0 / 128 ** 2 + 1e-6)
    assert bool(((ell >= 2) & (ell <= 16)).all()) and bool(((f >= 0.4) & (f <= 0.6)).all())
    # longer correlation -> fewer donor/acceptor bonds
    bonds = ((ph[:, 1:] != ph[:, :-1]).sum(dim=(1, 2)) + (ph[:, :, 1:] != ph[:, :, :-1]).sum(dim=(1, 2)))
    order = torch.argsort(ell)
    assert bonds[order[0]] > bonds[order[-1]]
    # same seed, same morphologies
    ph2, _, _ = S.grf_morphologies(6, size=128, seed=3, device="cpu")
    assert torch.equal(ph, ph2)


def test_label_arithmetic():
    from langmuir_b200 import surrogate as S
    c0 = [0] * 20
    c1 = [0] * 20
    c1[S._E_DRAIN_R], c1[S._E_DRAIN_L] = 70, 4
    c1[S._H_DRAIN_L], c1[S._H_DRAIN_R] = 66, 2
    c1[S._XSRC] = 200
    cur, eff, gen, rec = S._label_from_counters(c0, c1, 1000)
    assert cur == pytest.approx(130 / 1000) and eff == pytest.approx(130 / 400) and gen == 200


# ---- GPU: kernels against the oracle ---------------------------------------------------------
def _bf16(torch, a):
    return torch.as_tensor(np.asarray(a, np.float32)).to(torch.bfloat16).cuda()


def _f64(t):
    return t.float().cpu().numpy().astype(np.float64)


@pytest.mark.gpu
@pytest.mark.parametrize("cin,H,W,B", [(1, 64, 128, 2), (32, 32, 64, 3), (32, 16, 16, 5)])
def test_conv_forward_matches_oracle(cin, H, W, B):
    import torch
    from langmuir_b200 import surrogate as S
    rng = rng_for(f"conv{cin}{H}{W}")
    x = C.round_bf16(rng.standard_normal((B, H, W, cin)))
    w = C.round_bf16(rng.standard_normal((32, 9 * cin)) * np.sqrt(2.0 / (9 * cin)))
    b = rng.standard_normal(32) * 0.1
    pre = C.conv3x3(x, w, b)
    relu = np.maximum(pre, 0)
    w16 = S.conv_weights_bf16(torch.as_tensor(w, dtype=torch.float32).cuda(), cin)
    act, pooled = S.conv3x3_mma(_bf16(torch, x), w16,
                                torch.as_tensor(b, dtype=torch.float32).cuda(), H, W)
    torch.cuda.synchronize()
    # one BF16 rounding of an FP32 sum: within 2^-8 relative, plus FP32 order
    scale = np.abs(relu).max()
    assert np.all(np.abs(_f64(act) - relu) <= 2 ** -8 * np.abs(relu) + 1e-5 * scale)
    ref_pool = C.avgpool2(relu)
    assert np.all(np.abs(_f64(pooled) - ref_pool) <= 2 ** -8 * np.abs(ref_pool) + 1e-5 * scale)
    # no ReLU, no bias
    act2, _ = S.conv3x3_mma(_bf16(torch, x), w16, None, H, W, relu=False, pool=False)
    torch.cuda.synchronize()
    pre0 = C.conv3x3(x, w)
    assert np.all(np.abs(_f64(act2) - pre0) <= 2 ** -8 * np.abs(pre0) + 1e-5 * np.abs(pre0).max())


@pytest.mark.gpu
@pytest.mark.parametrize("H,W,B", [(8, 16, 1), (16, 16, 5), (32, 64, 3), (64, 64, 9)])
def test_tcgen05_conv_matches_oracle_and_mma_sync(H, W, B):
    """The tcgen05 kernel against the FP64 oracle (one BF16 rounding) and
    against the mma.sync kernel, in every output mode, with no device error."""
    import torch
    from langmuir_b200 import surrogate as S
    rng = rng_for(f"tc{H}{W}{B}")
    x = C.round_bf16(rng.standard_normal((B, H, W, 32)))
    w = C.round_bf16(rng.standard_normal((32, 288)) * np.sqrt(2.0 / 288))
    b = rng.standard_normal(32) * 0.1
    relu = np.maximum(C.conv3x3(x, w, b), 0)
    scale = np.abs(relu).max()
    x16, w16 = _bf16(torch, x), _bf16(torch, w)
    bt = torch.as_tensor(b, dtype=torch.float32).cuda()
    act, pooled = S.conv3x3_tc(x16, w16, bt, H, W)
    act_m, pooled_m = S.conv3x3_mma(x16, w16, bt, H, W)
    torch.cuda.synchronize()
    assert S.device_errors() == 0
    assert np.all(np.abs(_f64(act) - relu) <= 2 ** -8 * np.abs(relu) + 1e-5 * scale)
    ref_pool = C.avgpool2(relu)
    assert np.all(np.abs(_f64(pooled) - ref_pool) <= 2 ** -8 * np.abs(ref_pool) + 1e-5 * scale)
    # the two tensor-core paths differ at most by one BF16 rounding
    assert np.all(np.abs(_f64(act) - _f64(act_m)) <= 2 ** -7 * np.abs(_f64(act_m)) + 1e-5 * scale)
    # pooled only; then no bias, no ReLU, activation only (the input-gradient use)
    _, pooled2 = S.conv3x3_tc(x16, w16, bt, H, W, keep_act=False)
    act3, _ = S.conv3x3_tc(x16, w16, None, H, W, relu=False, pool=False)
    torch.cuda.synchronize()
    assert torch.equal(pooled2, pooled)
    pre0 = C.conv3x3(x, w)
    assert np.all(np.abs(_f64(act3) - pre0) <= 2 ** -8 * np.abs(pre0) + 1e-5 * np.abs(pre0).max())
    assert S.device_errors() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("cin,H,W,B", [(1, 64, 128, 3), (32, 32, 64, 4), (32, 16, 16, 7)])
def test_conv_wgrad_matches_oracle(cin, H, W, B):
    import torch
    from langmuir_b200 import surrogate as S
    rng = rng_for(f"wgrad{cin}{H}{W}")
    x = C.round_bf16(rng.standard_normal((B, H, W, cin)))
    dA = C.round_bf16(rng.standard_normal((B, H, W, 32)))
    dw_ref, db_ref = C.conv_wgrad(x, dA)
    kp = 16 if cin == 1 else 9 * cin
    dW = torch.zeros(32, kp, device="cuda")
    db = torch.zeros(32, device="cuda")
    S.conv3x3_wgrad(_bf16(torch, x), _bf16(torch, dA), dW, db, H, W)
    torch.cuda.synchronize()
    dw = dW.cpu().numpy().astype(np.float64)
    assert np.all(dw[:, 9 * cin:] == 0)
    err = np.linalg.norm(dw[:, :9 * cin] - dw_ref) / np.linalg.norm(dw_ref)
    assert err <= 1e-5, err
    assert np.linalg.norm(db.cpu().numpy() - db_ref) / np.linalg.norm(db_ref) <= 1e-5


@pytest.mark.gpu
def test_conv_dgrad_matches_oracle():
    import torch
    from langmuir_b200 import surrogate as S
    rng = rng_for("dgrad")
    B, H, W = 3, 32, 32
    dA = C.round_bf16(rng.standard_normal((B, H, W, 32)))
    w = C.round_bf16(rng.standard_normal((32, 288)) * 0.08)
    ref = C.conv_dgrad(dA, w, 32)
    dx = S.conv3x3_dgrad(_bf16(torch, dA), _bf16(torch, w), H, W)
    torch.cuda.synchronize()
    got = _f64(dx)
    assert np.all(np.abs(got - ref) <= 2 ** -8 * np.abs(ref) + 1e-5 * np.abs(ref).max())


@pytest.mark.gpu
def test_gemm_strides_bias_relu_accumulate():
    import torch
    from langmuir_b200 import surrogate as S
    rng = rng_for("gemm")
    M, N_, K = 37, 19, 45
    A = C.round_bf16(rng.standard_normal((K, M)))        # A(m, k) = A[k][m]
    Bm = C.round_bf16(rng.standard_normal((N_, K)))      # B(k, n) = Bm[n][k]
    bias = rng.standard_normal(N_)
    ref = np.maximum(A.T @ Bm.T + bias, 0)
    out = S.gemm(_bf16(torch, A), 1, M, _bf16(torch, Bm), 1, K, M, N_, K,
                 bias=torch.as_tensor(bias, dtype=torch.float32).cuda(), relu=True)
    torch.cuda.synchronize()
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()
    acc = torch.ones(M, N_, device="cuda")
    S.gemm(_bf16(torch, A), 1, M, _bf16(torch, Bm), 1, K, M, N_, K, out=acc)
    torch.cuda.synchronize()
    assert np.abs(acc.cpu().numpy() - (1 + A.T @ Bm.T)).max() <= 1e-4 * np.abs(A.T @ Bm.T).max()


def _network_case(seed, B=3, H=64, W=128):
    rng = rng_for(f"net{seed}")
    # a smooth-ish two-phase image so that activations are not degenerate
    ph = (rng.random((B, H, W)) < 0.5).astype(np.uint8)
    P = C.init_params(seed)
    return ph, P, rng


@pytest.mark.gpu
def test_network_forward_backward_match_oracle():
    """Whole network through SurrogateFn (autograd) vs the FP64 oracle with
    the kernels' BF16 rounding points (tolerance 1e-2 of each tensor's norm)
    and vs the exact FP64 network (5e-2)."""
    import torch
    from langmuir_b200 import surrogate as S
    ph, P, rng = _network_case(5)
    params = [torch.as_tensor(p, dtype=torch.float32).cuda().requires_grad_(True) for p in P]
    x16 = S.phases_to_input(ph)
    y = S.SurrogateFn.apply(x16, *params)
    R = rng.standard_normal(y.shape)
    (y * torch.as_tensor(R, dtype=torch.float32).cuda()).sum().backward()
    torch.cuda.synchronize()
    P32 = [p.astype(np.float32).astype(np.float64) for p in P]
    for bf16, tol in ((True, 1e-2), (False, 5e-2)):
        y_ref, cache = C.forward(ph, P32, bf16=bf16)
        g_ref = C.backward(R, cache, bf16=bf16)
        yg = y.detach().cpu().numpy()
        assert np.linalg.norm(yg - y_ref) <= tol * np.linalg.norm(y_ref), bf16
        for i, (p, gr) in enumerate(zip(params, g_ref)):
            gg = p.grad.cpu().numpy().astype(np.float64)
            assert gg.shape == gr.shape
            err = np.linalg.norm(gg - gr) / max(np.linalg.norm(gr), 1e-30)
            assert err <= tol, (S.PARAM_SHAPES[i][0], bf16, err)


@pytest.mark.gpu
def test_inference_path_equals_training_forward():
    import torch
    from langmuir_b200 import surrogate as S
    ph, P, _ = _network_case(9, B=4, H=128, W=128)
    params = [torch.as_tensor(p, dtype=torch.float32).cuda() for p in P]
    x16 = S.phases_to_input(ph)
    y_keep, _ = S.network_forward(x16, params, keep=True)
    y_inf, _ = S.network_forward(x16, params, keep=False)
    torch.cuda.synchronize()
    assert torch.equal(y_keep, y_inf)


@pytest.mark.gpu
def test_training_fits_a_morphology_property():
    """Trained by the native kernels, the network learns the donor fraction
    and the interface density of GRF morphologies (held-out R^2 > 0.9)."""
    import torch
    from langmuir_b200 import surrogate as S
    ph, ell, f = S.grf_morphologies(640, size=128, seed=11, device="cuda")
    bonds = ((ph[:, 1:] != ph[:, :-1]).sum(dim=(1, 2)) +
             (ph[:, :, 1:] != ph[:, :, :-1]).sum(dim=(1, 2))).float() / (2 * 128 * 127)
    y = torch.stack([1 - ph.float().mean(dim=(1, 2)), bonds], 1).cpu().numpy()
    # the donor fraction is not invariant under the phase exchange, so no
    # symmetry augmentation and linear targets here
    model = S.Surrogate(members=1, seed=2, log_targets=False, augment=False)
    hist = model.fit(ph[:512], y[:512], epochs=20, batch=64, lr=3e-3)
    assert hist[-1][2] < 0.5 * hist[0][2]
    mean, _ = model.predict(ph[512:])
    pred = mean.cpu().numpy()
    for k in range(2):
        yt = y[512:, k]
        r2 = 1 - ((pred[:, k] - yt) ** 2).sum() / ((yt - yt.mean()) ** 2).sum()
        assert r2 > 0.9, (k, r2)


@pytest.mark.gpu
def test_batched_labels_equal_single_replica():
    """A label from the batch equals the same morphology stepped alone."""
    import torch
    from langmuir_b200 import KMC
    from langmuir_b200 import surrogate as S
    ph, _, _ = S.grf_morphologies(3, size=128, seed=21, device="cuda")
    ph = ph.cpu().numpy()
    lab = S.kmc_labels(ph, steps=600, burn_in=200, seed=5, replica0=40)
    for i in range(3):
        p = S.solar_label_params(size=128, seed=5)
        with KMC(p, device=0, replica=40 + i) as k:
            k.set_morphology(ph[i].reshape(-1))
            k.run(200)
            c0 = k.stats()["counters"]
            k.run(400)
            c1 = k.stats()["counters"]
        cur, eff, gen, _ = S._label_from_counters(c0, c1, 400)
        assert lab["current"][i] == cur and lab["efficiency"][i] == eff
        assert lab["generated"][i] == gen
    assert lab["generated"].sum() > 0


@pytest.mark.gpu
def test_labels_through_a_process_group_equal_plain():
    """The sharded path of kmc_labels (labels of the rank's slice, then an
    all_gather) on a one-rank gloo group gives the plain labels."""
    import os
    import socket
    import torch.distributed as dist
    from langmuir_b200 import surrogate as S
    ph, _, _ = S.grf_morphologies(5, size=64, seed=8, device="cuda")
    ph = ph.cpu().numpy()
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        got = S.kmc_labels(ph, steps=500, burn_in=100, seed=3, replica0=60, chunk=2,
                           group=dist.group.WORLD)
    finally:
        dist.destroy_process_group()
    want = S.kmc_labels(ph, steps=500, burn_in=100, seed=3, replica0=60)
    for k in S.LABEL_KEYS:
        np.testing.assert_array_equal(got[k], want[k])


@pytest.mark.gpu
def test_surrogate_gain_over_descriptor_regression():
    """What the trained network gains over the method without it: on held-out
    morphologies labelled by kMC, the CNN trained on batched-kMC labels ranks
    efficiency far better than the reference's descriptor regression
    (ga.py:83-141, restated in oracle/ga_score.py), and the candidates it
    puts first are better under kMC than the regression's first picks."""
    import torch
    from langmuir_b200 import surrogate as S
    ph_tr, _, _ = S.grf_morphologies(1024, seed=101)
    ph_ho, _, _ = S.grf_morphologies(256, seed=102)
    lab_tr = S.kmc_labels(ph_tr, steps=12000, burn_in=3000, seed=3)
    lab_ho = S.kmc_labels(ph_ho, steps=12000, burn_in=3000, seed=3, replica0=1 << 20)
    model = S.Surrogate(members=2, seed=1)
    model.fit(ph_tr, np.stack([lab_tr["current"], lab_tr["efficiency"]], 1), epochs=30)
    pred = model.predict(ph_ho)[0][:, 1].cpu().numpy()
    eff = lab_ho["efficiency"]
    ga = np.array([G.score(G.phases_to_image(p)) for p in ph_ho.cpu().numpy()])
    rho_cnn, rho_ga = S._spearman(pred, eff), S._spearman(ga, eff)
    top_cnn = eff[np.argsort(-pred)[:16]].mean()
    top_ga = eff[np.argsort(-ga)[:16]].mean()
    print(f"spearman cnn {rho_cnn:.3f} ga {rho_ga:.3f}; top-16 kMC efficiency cnn {top_cnn:.4f} "
          f"ga {top_ga:.4f} all {eff.mean():.4f}")
    assert rho_cnn > 0.7 and rho_cnn > rho_ga + 0.15
    assert top_cnn > top_ga
