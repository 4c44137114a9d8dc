"""Morphology surrogate: a CNN that maps a 2-D donor/acceptor morphology to
solar-cell current and efficiency, trained on labels from the batched GPU kMC.

The reference screens ga2d morphologies with a regression over image
descriptors (LangmuirPython/ga2d/ga.py:83-141) and generates candidates from
Gaussian-blurred noise thresholded at the mean (ga2d/generators/iso.py:49-72).
Here:

* ``grf_morphologies``   seeded Gaussian random fields with a correlation
  length and a donor fraction per image, thresholded at that fraction's
  quantile (phase 0 donor / holes, 1 acceptor / electrons);
* ``kmc_labels``         batched solar-cell kMC on each morphology (carriers
  confined to their phase, excitons split across donor-acceptor bonds,
  recombination at interface pairs); current = net drain rate per step as
  LangmuirPython/langmuir/analyze.py:120-127 defines it, efficiency =
  collected pairs / generated excitons over a steady-state window;
* ``SurrogateFn``        the network's forward and backward on the BF16
  tensor-core kernels of include/langmuir_b200_cnn.h, as a
  torch.autograd.Function;
* ``Surrogate``          an ensemble of CNNs (spread = uncertainty), trained
  with Adam on FP32 master weights;
* ``screen``             rank candidates by predicted efficiency and send the
  top ones plus every high-uncertainty prediction back to kMC.

The CUDA library is required: every network pass runs in it.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np
import torch

from . import _native as N
from .kmc import KMCBatch, Params

CH = 32          # conv channels (LGM_CNN_CHANNELS)
HIDDEN = 64      # fully connected hidden width
OUTPUTS = 2      # current, efficiency

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
N.SIGNATURES.update({
    "lgm_cnn_conv3x3_fwd": (_i32, [_i32, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _i32, _i32, _vp]),
    "lgm_cnn_conv3x3_wgrad": (_i32, [_i32, _vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp]),
    "lgm_cnn_flip_weights": (_i32, [_i32, _vp, _vp, _vp]),
    "lgm_cnn_gemm": (_i32, [_vp, _i32, _i32, _vp, _i32, _i32, _vp, _vp, _i32, _i32, _i32, _i32,
                            _i32, _vp]),
    "lgm_cnn_relu_pool_bwd": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32, _i32, _vp]),
    "lgm_cnn_gap_fwd": (_i32, [_vp, _vp, _vp, _i32, _i32, _vp]),
    "lgm_cnn_gap_relu_bwd": (_i32, [_vp, _vp, _vp, _i32, _i32, _vp]),
    "lgm_cnn_to_bf16": (_i32, [_vp, _vp, _i32, _vp, _vp]),
    "lgm_cnn_conv3x3_fwd_tc": (_i32, [_vp, _vp, _vp, _vp, _vp, _i32, _i32, _i32, _i32, _vp]),
    "lgm_cnn_error": (_i32, [ctypes.POINTER(ctypes.c_uint32)]),
})
_CNN_SYMBOLS = [k for k in N.SIGNATURES if k.startswith("lgm_cnn_")]
if N._lib is not None:
    for _name in _CNN_SYMBOLS:
        _fn = getattr(N._lib, _name)
        _fn.restype, _fn.argtypes = N.SIGNATURES[_name]


def _p(t):
    return None if t is None else t.data_ptr()


def _ok(st):
    if st != N.OK:
        raise N.LgmError(st, N.lib().lgm_status_string(st).decode())


def _stream():
    return torch.cuda.current_stream().cuda_stream


# ---- kernel wrappers -----------------------------------------------------------------------
def conv3x3(x, w16, bias, H, W, relu=True, keep_act=True, pool=True):
    """x: [B,H,W,cin] bf16, w16: [CH, 16 or 9*CH] bf16 -> (act or None, pooled or None).
    32 input channels run on the tcgen05 kernel, 1 input channel on mma.sync."""
    B, cin = x.shape[0], x.shape[-1]
    if cin == CH:
        return conv3x3_tc(x, w16, bias, H, W, relu, keep_act, pool)
    return conv3x3_mma(x, w16, bias, H, W, relu, keep_act, pool)


def conv3x3_mma(x, w16, bias, H, W, relu=True, keep_act=True, pool=True):
    """The mma.sync kernel (lgm_cnn_conv3x3_fwd), for 1 or 32 input channels."""
    B, cin = x.shape[0], x.shape[-1]
    act = torch.empty(B, H, W, CH, dtype=torch.bfloat16, device=x.device) if keep_act else None
    pooled = (torch.empty(B, H // 2, W // 2, CH, dtype=torch.bfloat16, device=x.device)
              if pool else None)
    _ok(N.lib().lgm_cnn_conv3x3_fwd(cin, _p(x), _p(w16), _p(bias), _p(act), _p(pooled), B, H, W,
                                    int(relu), _stream()))
    return act, pooled


def conv3x3_tc(x, w16, bias, H, W, relu=True, keep_act=True, pool=True):
    """conv3x3 for 32 input channels on the tcgen05 tensor cores."""
    B = x.shape[0]
    act = torch.empty(B, H, W, CH, dtype=torch.bfloat16, device=x.device) if keep_act else None
    pooled = (torch.empty(B, H // 2, W // 2, CH, dtype=torch.bfloat16, device=x.device)
              if pool else None)
    _ok(N.lib().lgm_cnn_conv3x3_fwd_tc(_p(x), _p(w16), _p(bias), _p(act), _p(pooled), B, H, W,
                                       int(relu), _stream()))
    return act, pooled


def device_errors() -> int:
    """Error bits the tensor-core kernels raised since the last call (0 = none)."""
    v = ctypes.c_uint32()
    N.lib().lgm_cnn_error(ctypes.byref(v))
    return v.value


def conv3x3_wgrad(x, dA, dW, db, H, W):
    B, cin = x.shape[0], x.shape[-1]
    _ok(N.lib().lgm_cnn_conv3x3_wgrad(cin, _p(x), _p(dA), _p(dW), _p(db), B, H, W, _stream()))


def conv3x3_dgrad(dA, w16, H, W):
    """Input gradient of a CH -> CH layer: conv with flipped, transposed weights."""
    wd = torch.empty(CH, 9 * CH, dtype=torch.bfloat16, device=dA.device)
    _ok(N.lib().lgm_cnn_flip_weights(CH, _p(w16), _p(wd), _stream()))
    dx, _ = conv3x3(dA, wd, None, H, W, relu=False, keep_act=True, pool=False)
    return dx


def gemm(A, sam, sak, Bm, sbk, sbn, M, N_, K, bias=None, relu=False, out=None):
    C = out if out is not None else torch.empty(M, N_, dtype=torch.float32, device=A.device)
    _ok(N.lib().lgm_cnn_gemm(_p(A), sam, sak, _p(Bm), sbk, sbn, _p(C), _p(bias), M, N_, K,
                             int(relu), int(out is not None), _stream()))
    return C


def to_bf16(x, relu_mask=None):
    out = torch.empty(x.shape, dtype=torch.bfloat16, device=x.device)
    _ok(N.lib().lgm_cnn_to_bf16(_p(x), _p(out), x.numel(), _p(relu_mask), _stream()))
    return out


def relu_pool_bwd(act, dP, pooled):
    B, H, W, _ = act.shape
    dA = torch.empty_like(act)
    _ok(N.lib().lgm_cnn_relu_pool_bwd(_p(act), _p(dP), _p(dA), B, H, W, int(pooled), _stream()))
    return dA


def gap_fwd(act):
    B, H, W, _ = act.shape
    g32 = torch.empty(B, CH, dtype=torch.float32, device=act.device)
    g16 = torch.empty(B, CH, dtype=torch.bfloat16, device=act.device)
    _ok(N.lib().lgm_cnn_gap_fwd(_p(act), _p(g32), _p(g16), B, H * W, _stream()))
    return g32, g16


def gap_relu_bwd(act, dg):
    B, H, W, _ = act.shape
    dA = torch.empty_like(act)
    _ok(N.lib().lgm_cnn_gap_relu_bwd(_p(act), _p(dg), _p(dA), B, H * W, _stream()))
    return dA


def conv_weights_bf16(w, cin):
    """FP32 master [CH, 9*cin] -> kernel layout (cin == 1 padded to 16 columns)."""
    if cin == 1:
        w16 = torch.zeros(CH, 16, dtype=torch.bfloat16, device=w.device)
        w16[:, :9] = w.to(torch.bfloat16)
        return w16
    return w.to(torch.bfloat16).contiguous()


# ---- the network ---------------------------------------------------------------------------
PARAM_SHAPES = [("c1w", (CH, 9)), ("c1b", (CH,)), ("c2w", (CH, 9 * CH)), ("c2b", (CH,)),
                ("c3w", (CH, 9 * CH)), ("c3b", (CH,)), ("c4w", (CH, 9 * CH)), ("c4b", (CH,)),
                ("f1w", (HIDDEN, CH)), ("f1b", (HIDDEN,)), ("f2w", (OUTPUTS, HIDDEN)),
                ("f2b", (OUTPUTS,))]


def check_image_shape(H, W):
    if H % 64 or W % 128:
        raise ValueError(f"image {H}x{W}: the kernels need H % 64 == 0 and W % 128 == 0")


def network_forward(x16, params, keep=True):
    """x16: [B,H,W,1] bf16; params: FP32 masters in PARAM_SHAPES order.
    Returns y [B,2] fp32 and (keep) the tensors the backward pass reads."""
    c1w, c1b, c2w, c2b, c3w, c3b, c4w, c4b, f1w, f1b, f2w, f2b = params
    B, H, W, _ = x16.shape
    check_image_shape(H, W)
    w1 = conv_weights_bf16(c1w, 1)
    w2, w3, w4 = (conv_weights_bf16(w, CH) for w in (c2w, c3w, c4w))
    a1, p1 = conv3x3(x16, w1, c1b, H, W, keep_act=keep)
    a2, p2 = conv3x3(p1, w2, c2b, H // 2, W // 2, keep_act=keep)
    a3, p3 = conv3x3(p2, w3, c3b, H // 4, W // 4, keep_act=keep)
    a4, _ = conv3x3(p3, w4, c4b, H // 8, W // 8, keep_act=True, pool=False)
    g32, g16 = gap_fwd(a4)
    f1w16, f2w16 = f1w.to(torch.bfloat16), f2w.to(torch.bfloat16)
    # h = relu(g W1^T + b1): A(b, c) = g16[b][c], B(c, j) = W1[j][c]
    h32 = gemm(g16, CH, 1, f1w16, 1, CH, B, HIDDEN, CH, bias=f1b, relu=True)
    h16 = to_bf16(h32)
    y = gemm(h16, HIDDEN, 1, f2w16, 1, HIDDEN, B, OUTPUTS, HIDDEN, bias=f2b)
    saved = (x16, w2, w3, w4, f1w16, f2w16, a1, p1, a2, p2, a3, p3, a4, g16, h32, h16) if keep else None
    return y, saved


def network_backward(dy, saved):
    """Gradients of the FP32 masters (PARAM_SHAPES order) from dL/dy."""
    x16, w2, w3, w4, f1w16, f2w16, a1, p1, a2, p2, a3, p3, a4, g16, h32, h16 = saved
    B, H, W, _ = x16.shape
    dev = dy.device
    dy16 = to_bf16(dy.contiguous())
    ones = torch.ones(B, dtype=torch.bfloat16, device=dev)
    z = lambda *s: torch.zeros(*s, dtype=torch.float32, device=dev)
    # head: dW2 = dy^T h, db2 = 1^T dy, dh = dy W2 (masked by h > 0)
    df2w = gemm(dy16, 1, OUTPUTS, h16, HIDDEN, 1, OUTPUTS, HIDDEN, B, out=z(OUTPUTS, HIDDEN))
    df2b = gemm(ones, 0, 1, dy16, OUTPUTS, 1, 1, OUTPUTS, B, out=z(1, OUTPUTS)).view(OUTPUTS)
    dh = gemm(dy16, OUTPUTS, 1, f2w16, HIDDEN, 1, B, HIDDEN, OUTPUTS)
    dh16 = to_bf16(dh, relu_mask=h32)
    df1w = gemm(dh16, 1, HIDDEN, g16, CH, 1, HIDDEN, CH, B, out=z(HIDDEN, CH))
    df1b = gemm(ones, 0, 1, dh16, HIDDEN, 1, 1, HIDDEN, B, out=z(1, HIDDEN)).view(HIDDEN)
    dg = gemm(dh16, HIDDEN, 1, f1w16, CH, 1, B, CH, HIDDEN)
    # conv stack
    dA4 = gap_relu_bwd(a4, dg)
    dc4w, dc4b = z(CH, 9 * CH), z(CH)
    conv3x3_wgrad(p3, dA4, dc4w, dc4b, H // 8, W // 8)
    dp3 = conv3x3_dgrad(dA4, w4, H // 8, W // 8)
    dA3 = relu_pool_bwd(a3, dp3, True)
    dc3w, dc3b = z(CH, 9 * CH), z(CH)
    conv3x3_wgrad(p2, dA3, dc3w, dc3b, H // 4, W // 4)
    dp2 = conv3x3_dgrad(dA3, w3, H // 4, W // 4)
    dA2 = relu_pool_bwd(a2, dp2, True)
    dc2w, dc2b = z(CH, 9 * CH), z(CH)
    conv3x3_wgrad(p1, dA2, dc2w, dc2b, H // 2, W // 2)
    dp1 = conv3x3_dgrad(dA2, w2, H // 2, W // 2)
    dA1 = relu_pool_bwd(a1, dp1, True)
    dc1w16, dc1b = z(CH, 16), z(CH)
    conv3x3_wgrad(x16, dA1, dc1w16, dc1b, H, W)
    dc1w = dc1w16[:, :9].contiguous()
    return (dc1w, dc1b, dc2w, dc2b, dc3w, dc3b, dc4w, dc4b, df1w, df1b, df2w, df2b)


class SurrogateFn(torch.autograd.Function):
    """y = CNN(x); forward and backward on the native BF16 tensor-core kernels."""

    @staticmethod
    def forward(ctx, x16, *params):
        y, saved = network_forward(x16, params, keep=True)
        ctx.saved = saved
        return y

    @staticmethod
    def backward(ctx, dy):
        grads = network_backward(dy, ctx.saved)
        ctx.saved = None
        return (None, *grads)


def init_params(seed, device="cuda"):
    """He-normal conv/linear weights, zero biases, FP32 masters."""
    g = torch.Generator(device="cpu").manual_seed(int(seed))
    out = []
    for name, shape in PARAM_SHAPES:
        if name.endswith("b"):
            t = torch.zeros(shape)
        else:
            fan_in = shape[1]
            t = torch.randn(shape, generator=g) * math.sqrt(2.0 / fan_in)
        out.append(t.to(device).requires_grad_(True))
    return out


def phases_to_input(phases, device="cuda", ramp=0.0):
    """uint8 phases [B,H,W] (0 donor, 1 acceptor) -> bf16 [B,H,W,1]: -1 donor,
    +1 acceptor, plus ``ramp`` * (2x/(W-1) - 1) along x (the axis between the
    electrodes).  The global pool of the network makes it blind to where a
    feature sits; the ramp tells it how far a site is from either electrode.
    Mirroring x and exchanging the phases maps the input to minus its mirror
    image, ramp included, so the device symmetries stay a sign flip."""
    t = torch.as_tensor(phases, device=device)
    x = t.to(torch.float32) * 2.0 - 1.0
    if ramp:
        W = x.shape[-1]
        x = x + ramp * torch.linspace(-1.0, 1.0, W, device=x.device)
    return x.to(torch.bfloat16).unsqueeze(-1).contiguous()


# ---- morphologies --------------------------------------------------------------------------
def grf_morphologies(n, size=128, seed=0, corr=(2.0, 16.0), frac=(0.4, 0.6), device="cuda"):
    """``n`` binary morphologies [n,size,size] uint8 (0 donor, 1 acceptor).

    Per image: correlation length l ~ U(corr), donor fraction f ~ U(frac);
    white noise on a padded square is blurred by a Gaussian of standard
    deviation l (in Fourier space, so the padding removes the wrap-around)
    and the lowest f of the cropped field become donor.  The reference's
    makeIsotropic (ga2d/generators/iso.py:49-72) blurs uniform noise with a
    Gaussian filter and thresholds at the mean (f = 1/2 on average).
    Returns (phases, l, f)."""
    g = torch.Generator(device=device).manual_seed(int(seed))
    ell = corr[0] + (corr[1] - corr[0]) * torch.rand(n, generator=g, device=device)
    f = frac[0] + (frac[1] - frac[0]) * torch.rand(n, generator=g, device=device)
    pad = int(3 * corr[1])
    P = size + 2 * pad
    k = torch.fft.fftfreq(P, device=device)
    k2 = (k[:, None] ** 2 + k[None, :] ** 2)
    out = torch.empty(n, size, size, dtype=torch.uint8, device=device)
    S = size * size
    chunk = 1024
    for i0 in range(0, n, chunk):
        i1 = min(n, i0 + chunk)
        noise = torch.randn(i1 - i0, P, P, generator=g, device=device)
        filt = torch.exp(-2.0 * math.pi ** 2 * k2[None] * ell[i0:i1, None, None] ** 2)
        field = torch.fft.ifft2(torch.fft.fft2(noise) * filt).real[:, pad:pad + size, pad:pad + size]
        flat = field.reshape(i1 - i0, S)
        srt = flat.sort(dim=1).values
        kk = (f[i0:i1] * S).round().long().clamp(1, S - 1)
        thr = srt.gather(1, kk[:, None])
        out[i0:i1] = (flat >= thr).to(torch.uint8).view(i1 - i0, size, size)
    return out, ell, f


# ---- kMC labels ----------------------------------------------------------------------------
# the field of the reference's solar-cell example (examples/solar.inp: 7.5 V
# across grid.x = 96), in volts per lattice site
EXAMPLE_FIELD = 7.5 / 96


def solar_label_params(size=128, seed=1, generation=0.05, recombination=1e-3, field=EXAMPLE_FIELD,
                       cutoff=30, capacity=0.04):
    """Solar-cell kMC set-up of the labels: 2-D size x size lattice, point
    charges (coulomb.gaussian.sigma cannot be used in 2-D, parameters.h:631-634),
    holes confined to donor and electrons to acceptor sites, excitons split
    across a random donor-acceptor bond with probability ``generation`` per
    step (no area scaling), recombination of interface pairs with probability
    ``recombination``, ``field`` volts per site across x (voltage.right =
    field * size), drains at both x faces."""
    p = Params.default()
    keys = dict(simulation_type="solarcell", grid_x=size, grid_y=size, grid_z=1,
                electron_percentage=capacity, hole_percentage=capacity, seed_charges=0.0,
                defect_percentage=0.0, trap_percentage=0.0, voltage_left=0.0,
                voltage_right=field * size, coulomb_carriers=1, electrostatic_cutoff=cutoff,
                generation_rate=generation, source_scale_area=0.0,
                recombination_rate=recombination, recombination_range=1,
                morphology_confine=1, generation_interface=1, random_seed=int(seed),
                iterations_real=1000, iterations_print=10)
    for k, v in keys.items():
        p.set(k, v)
    return p.check()


# counters: (attempts, successes) of eSourceL, eSourceR, hSourceL, hSourceR,
# eDrainL, eDrainR, hDrainL, hDrainR, exciton source, recombination
_E_DRAIN_L, _E_DRAIN_R, _H_DRAIN_L, _H_DRAIN_R, _XSRC, _RECOMB = 9, 11, 13, 15, 17, 19


def _label_from_counters(c0, c1, steps):
    d = np.asarray(c1, np.int64) - np.asarray(c0, np.int64)
    e_net = d[_E_DRAIN_R] - d[_E_DRAIN_L]
    h_net = d[_H_DRAIN_L] - d[_H_DRAIN_R]
    gen = d[_XSRC]
    current = (e_net + h_net) / float(steps)
    eff = (e_net + h_net) / (2.0 * gen) if gen > 0 else 0.0
    return current, eff, int(gen), int(d[_RECOMB])


LABEL_KEYS = ("current", "efficiency", "generated", "recombined")


def shard_range(n, world, rank):
    """Rank ``rank``'s contiguous share [lo, hi) of n morphologies (the shares
    of a world differ in size by at most one)."""
    return rank * n // world, (rank + 1) * n // world


def _label_slice(ph, replica_start, steps, burn_in, seed, device, chunk, setup):
    """Labels of the morphologies ph [m,H,W]; morphology i is replica
    replica_start + i, so its label does not depend on how the set is split."""
    m, H, _ = ph.shape
    out = {k: np.zeros(m) for k in LABEL_KEYS}
    for i0 in range(0, m, chunk):
        i1 = min(m, i0 + chunk)
        params = [solar_label_params(size=H, seed=seed, **setup) for _ in range(i0, i1)]
        with KMCBatch(params, device=device, replica0=replica_start + i0) as b:
            reps = [b.replica(i) for i in range(i1 - i0)]
            for i, r in enumerate(reps):
                # the site order is x fastest: site = x + X*y, image[y][x]
                r.set_morphology(ph[i0 + i].reshape(-1))
            b.run(burn_in)
            c0 = [r.stats()["counters"] for r in reps]
            b.run(steps - burn_in)
            c1 = [r.stats()["counters"] for r in reps]
        for i in range(i1 - i0):
            lab = _label_from_counters(c0[i], c1[i], steps - burn_in)
            for k, v in zip(LABEL_KEYS, lab):
                out[k][i0 + i] = v
    return out


def gather_labels(local, n, group=None):
    """Every rank's share of the labels (``local``, the arrays of its
    shard_range) assembled into n-long arrays on every rank: one all_gather of
    a padded [keys, ceil(n/world)] FP64 tensor (on the GPU for NCCL, on the
    host for gloo).  The wall time is the longest rank's."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    dev = (torch.device("cuda", torch.cuda.current_device())
           if dist.get_backend(group) == "nccl" else torch.device("cpu"))
    cap = -(-n // world)
    lo, hi = shard_range(n, world, rank)
    buf = torch.zeros(len(LABEL_KEYS), cap, dtype=torch.float64, device=dev)
    for j, k in enumerate(LABEL_KEYS):
        buf[j, : hi - lo] = torch.as_tensor(np.asarray(local[k], np.float64))
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    t = torch.tensor([float(local.get("seconds", 0.0))], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    out = {k: np.zeros(n) for k in LABEL_KEYS}
    for r, part in enumerate(parts):
        a, b = shard_range(n, world, r)
        arr = part.cpu().numpy()
        for j, k in enumerate(LABEL_KEYS):
            out[k][a:b] = arr[j, : b - a]
    out["seconds"] = float(t.item())
    return out


def kmc_labels(phases, steps=50000, burn_in=10000, seed=1, replica0=0, device=0, chunk=4096,
               group=None, **setup):
    """Current and efficiency of every morphology from the batched GPU kMC.

    phases: uint8 [n,H,W] (numpy or torch).  The window [burn_in, steps)
    defines the labels (the first burn_in steps fill the device).  Returns a
    dict of numpy arrays plus the wall time.  With a process group ``group``
    (torch.distributed, one GPU per rank) each rank labels its shard_range of
    the morphologies on its own GPU and the labels are gathered to every
    rank; morphology i is replica replica0 + i either way, so the labels equal
    the single-GPU ones."""
    ph = phases.cpu().numpy() if torch.is_tensor(phases) else np.asarray(phases)
    ph = np.ascontiguousarray(ph, dtype=np.uint8)
    n, H, W = ph.shape
    if H != W:
        raise ValueError("square morphologies only")
    t0 = time.perf_counter()
    if group is None:
        out = _label_slice(ph, replica0, steps, burn_in, seed, device, chunk, setup)
        out["seconds"] = time.perf_counter() - t0
        return out
    import torch.distributed as dist
    lo, hi = shard_range(n, dist.get_world_size(group), dist.get_rank(group))
    local = _label_slice(ph[lo:hi], replica0 + lo, steps, burn_in, seed, device, chunk, setup)
    local["seconds"] = time.perf_counter() - t0
    return gather_labels(local, n, group)


# ---- ensemble ------------------------------------------------------------------------------
def symmetry(x16, k):
    """The device's symmetries on a bf16 input [B,H,W,1] (x = +-1 per phase):
    k = 0 identity, 1 mirror in y, 2 mirror in x with the phases exchanged
    (electrons and holes, collected at opposite electrodes, trade places),
    3 both.  kMC labels are invariant under all four."""
    if k & 1:
        x16 = x16.flip(1)
    if k & 2:
        x16 = (-x16).flip(2)
    return x16.contiguous()


class Surrogate:
    """Ensemble of CNNs on standardised log(current), log(efficiency).

    Training draws one of the four device symmetries per mini-batch, which is
    right for kMC labels (invariant under them) and wrong for targets that are
    not, such as the donor fraction (augment=False there); ``tta`` > 1
    averages predictions over that many symmetries."""

    def __init__(self, members=4, seed=0, device="cuda", log_targets=True, augment=True, tta=1,
                 ramp=0.0):
        self.device = device
        self.members = [init_params(seed * 1000 + m, device) for m in range(members)]
        self.mean = torch.zeros(OUTPUTS, device=device)
        self.std = torch.ones(OUTPUTS, device=device)
        self.log_targets, self.augment, self.tta = log_targets, augment, tta
        self.ramp = float(ramp)

    def _encode(self, y):
        return torch.log(y.clamp_min(1e-6)) if self.log_targets else y

    def fit(self, phases, targets, epochs=30, batch=64, lr=2e-3, seed=0, log=None):
        """phases uint8 [n,H,W], targets float [n,2] (current, efficiency)."""
        x = phases_to_input(phases, self.device, self.ramp)
        y = self._encode(torch.as_tensor(np.asarray(targets, np.float32), device=self.device))
        self.mean = y.mean(0)
        self.std = y.std(0).clamp_min(1e-6)
        yn = (y - self.mean) / self.std
        n = x.shape[0]
        history = []
        for m, params in enumerate(self.members):
            opt = torch.optim.Adam(params, lr=lr)
            sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=epochs)
            g = torch.Generator(device="cpu").manual_seed(int(seed) * 7919 + m)
            for ep in range(epochs):
                perm = torch.randperm(n, generator=g).to(self.device)
                tot = 0.0
                for i0 in range(0, n - batch + 1, batch):
                    idx = perm[i0:i0 + batch]
                    xb = x[idx]
                    if self.augment:
                        xb = symmetry(xb, int(torch.randint(0, 4, (1,), generator=g)))
                    pred = SurrogateFn.apply(xb, *params)
                    loss = ((pred - yn[idx]) ** 2).mean()
                    opt.zero_grad(set_to_none=True)
                    loss.backward()
                    opt.step()
                    tot += float(loss.detach()) * batch
                sched.step()
                history.append((m, ep, tot / max(1, (n // batch) * batch)))
                if log:
                    log(f"member {m} epoch {ep} loss {history[-1][2]:.4f}")
        return history

    @torch.no_grad()
    def predict(self, phases=None, x16=None, batch=1024):
        """Ensemble mean and spread in target units: two [n,2] tensors.  With
        log targets the mean is the geometric mean over members and the spread
        is mean * (std of the log predictions)."""
        if x16 is None:
            x16 = phases_to_input(phases, self.device, self.ramp)
        n = x16.shape[0]
        views = max(1, self.tta)
        preds = torch.zeros(len(self.members), n, OUTPUTS, device=self.device)
        for m, params in enumerate(self.members):
            for i0 in range(0, n, batch):
                xb = x16[i0:i0 + batch]
                for k in range(views):
                    y, _ = network_forward(symmetry(xb, k) if k else xb, params, keep=False)
                    preds[m, i0:i0 + batch] += y / views
        preds = preds * self.std + self.mean
        mu = preds.mean(0)
        sd = preds.std(0) if len(self.members) > 1 else torch.zeros_like(mu)
        if self.log_targets:
            mu = torch.exp(mu)
            sd = mu * sd
        return mu, sd

    def state_dict(self):
        return {"members": [[p.detach().cpu() for p in ps] for ps in self.members],
                "mean": self.mean.cpu(), "std": self.std.cpu(), "log_targets": self.log_targets,
                "tta": self.tta, "ramp": self.ramp}

    def load_state_dict(self, sd):
        self.members = [[p.to(self.device).requires_grad_(True) for p in ps] for ps in sd["members"]]
        self.mean, self.std = sd["mean"].to(self.device), sd["std"].to(self.device)
        self.log_targets, self.tta = sd.get("log_targets", False), sd.get("tta", 1)
        self.ramp = float(sd.get("ramp", 0.0))


def screen(model, candidates, top=256, uncertainty_quantile=0.9975, batch=1024):
    """Rank candidates by predicted efficiency.  Returns (order of the top
    ``top``, indices whose efficiency spread is above the quantile, mean, std)."""
    mean, std = model.predict(candidates, batch=batch)
    eff, sig = mean[:, 1], std[:, 1]
    top_idx = torch.argsort(eff, descending=True)[:top]
    thr = torch.quantile(sig.float(), uncertainty_quantile) if sig.numel() > 1 else sig.max()
    unc_idx = torch.nonzero(sig > thr).flatten()
    return top_idx, unc_idx, mean, std


# ---- the screening pipeline ----------------------------------------------------------------
def _spearman(a, b):
    ra = np.argsort(np.argsort(a)).astype(np.float64)
    rb = np.argsort(np.argsort(b)).astype(np.float64)
    return float(np.corrcoef(ra, rb)[0, 1])


def error_report(pred, truth):
    """Surrogate error against kMC labels: absolute and relative efficiency
    errors, the share within 5 % (relative) of kMC, R^2 and rank correlation."""
    pred, truth = np.asarray(pred, np.float64), np.asarray(truth, np.float64)
    err = pred - truth
    mae = float(np.mean(np.abs(err)))
    rel = np.abs(err) / np.maximum(np.abs(truth), 1e-12)
    ss = float(np.sum((truth - truth.mean()) ** 2))
    return {"n": int(truth.size), "mae": mae, "rmse": float(np.sqrt(np.mean(err ** 2))),
            "relative_mae": mae / float(np.mean(np.abs(truth))),
            "median_relative_error": float(np.median(rel)),
            "share_within_5pct": float(np.mean(rel <= 0.05)),
            "r2": 1.0 - float(np.sum(err ** 2)) / ss if ss > 0 else float("nan"),
            "spearman": _spearman(pred, truth) if truth.size > 2 else float("nan")}


def save_labels(path, phases, labels):
    """Morphologies (bit-packed) and their kMC labels in one .npz."""
    ph = phases.cpu().numpy() if torch.is_tensor(phases) else np.asarray(phases)
    np.savez_compressed(path, bits=np.packbits(ph.astype(bool), axis=None), shape=np.array(ph.shape),
                        **{k: np.asarray(v) for k, v in labels.items()})


def load_labels(path, device="cuda"):
    d = np.load(path)
    shape = tuple(int(v) for v in d["shape"])
    ph = np.unpackbits(d["bits"])[:int(np.prod(shape))].reshape(shape).astype(np.uint8)
    labels = {k: (d[k] if d[k].ndim else float(d[k])) for k in d.files if k not in ("bits", "shape")}
    return torch.as_tensor(ph, device=device), labels


def run_pipeline(n_train=4096, n_holdout=512, n_candidates=100000, steps=50000, burn_in=10000,
                 members=4, epochs=300, top=256, seed=0, labels_cache="", lr=4e-3, log=print,
                 holdout_steps=None, train_steps=None, **model_kw):
    """Generate, label, train, evaluate on kMC-labelled holdouts, screen
    candidates and re-simulate the picks.  Returns a report dict.  With
    ``labels_cache`` the training and holdout labels are read from (or, the
    first time, written to) that prefix.  ``train_steps`` / ``holdout_steps``
    (default ``steps``) set the length of the training and holdout label runs:
    a label's noise falls as the square root of its window, and the holdout
    labels are the yardstick of the surrogate's error."""
    import os
    train_steps = train_steps or steps
    holdout_steps = holdout_steps or steps
    rep = {"config": dict(n_train=n_train, n_holdout=n_holdout, n_candidates=n_candidates,
                          steps=steps, train_steps=train_steps, holdout_steps=holdout_steps,
                          burn_in=burn_in, members=members, epochs=epochs, top=top,
                          seed=seed, size=128, lr=lr, **model_kw)}
    sync = torch.cuda.synchronize
    cached = labels_cache and os.path.exists(labels_cache + "_train.npz")
    if cached:
        ph_tr, lab_tr = load_labels(labels_cache + "_train.npz")
        ph_ho, lab_ho = load_labels(labels_cache + "_holdout.npz")
    else:
        ph_tr, _, _ = grf_morphologies(n_train, seed=seed * 10 + 1)
        ph_ho, _, _ = grf_morphologies(n_holdout, seed=seed * 10 + 2)
        lab_tr = kmc_labels(ph_tr, steps=train_steps, burn_in=burn_in, seed=seed + 1, replica0=0)
        log(f"labels: {n_train} morphologies x {train_steps} steps in {lab_tr['seconds']:.1f} s")
        lab_ho = kmc_labels(ph_ho, steps=holdout_steps, burn_in=burn_in, seed=seed + 1,
                            replica0=1 << 24)
        if labels_cache:
            save_labels(labels_cache + "_train.npz", ph_tr, lab_tr)
            save_labels(labels_cache + "_holdout.npz", ph_ho, lab_ho)
    rep["labels_from_cache"] = bool(cached)
    rep["kmc"] = {"train_seconds": lab_tr["seconds"], "holdout_seconds": lab_ho["seconds"],
                  "morphs_per_s": n_train / lab_tr["seconds"] * train_steps / steps,
                  "efficiency_percentiles": np.percentile(lab_tr["efficiency"], [5, 50, 95]).tolist(),
                  "generated_median": float(np.median(lab_tr["generated"]))}
    y_tr = np.stack([lab_tr["current"], lab_tr["efficiency"]], 1)
    model = Surrogate(members=members, seed=seed, **model_kw)
    t0 = time.perf_counter()
    hist = model.fit(ph_tr, y_tr, epochs=epochs, batch=64, lr=lr, seed=seed)
    sync()
    rep["train"] = {"seconds": time.perf_counter() - t0, "final_loss": [h[2] for h in hist
                                                                        if h[1] == epochs - 1]}
    mean, std = model.predict(ph_ho)
    mean, std = mean.cpu().numpy(), std.cpu().numpy()
    rep["holdout"] = {"efficiency": error_report(mean[:, 1], lab_ho["efficiency"]),
                      "current": error_report(mean[:, 0], lab_ho["current"]),
                      "mean_predicted_spread": float(std[:, 1].mean())}
    log(f"holdout efficiency error: {rep['holdout']['efficiency']}")
    # screening
    cand, _, _ = grf_morphologies(n_candidates, seed=seed * 10 + 3)
    model.predict(cand[:1024])
    sync()
    t0 = time.perf_counter()
    top_idx, unc_idx, cmean, cstd = screen(model, cand, top=top)
    sync()
    screen_s = time.perf_counter() - t0
    picks = torch.unique(torch.cat([top_idx, unc_idx])).cpu()
    # the picks are labelled as the holdouts are, so that both judge the
    # surrogate on labels of one protocol
    lab_pk = kmc_labels(cand[picks.to(cand.device)], steps=holdout_steps, burn_in=burn_in,
                        seed=seed + 1, replica0=1 << 25)
    pk_mean = cmean[picks.to(cmean.device)].cpu().numpy()
    is_top = torch.isin(picks, top_idx.cpu()).numpy()
    is_unc = torch.isin(picks, unc_idx.cpu()).numpy()
    rep["screen"] = {
        "seconds": screen_s, "morphs_per_s": n_candidates / screen_s,
        "speedup_vs_kmc": (n_candidates / screen_s) / rep["kmc"]["morphs_per_s"],
        "resimulated": int(picks.numel()), "top": int(is_top.sum()), "high_uncertainty": int(is_unc.sum()),
        "top_error": error_report(pk_mean[is_top, 1], lab_pk["efficiency"][is_top]),
        "uncertain_error": (error_report(pk_mean[is_unc, 1], lab_pk["efficiency"][is_unc])
                            if is_unc.sum() > 2 else None),
        "best_kmc_efficiency_picked": float(lab_pk["efficiency"][is_top].max()),
        "mean_kmc_efficiency_top": float(lab_pk["efficiency"][is_top].mean()),
        "mean_kmc_efficiency_train": float(lab_tr["efficiency"].mean()),
        "best_kmc_efficiency_train": float(lab_tr["efficiency"].max())}
    log(f"screen: {rep['screen']}")
    rep["_arrays"] = {"holdout_phases": ph_ho.cpu().numpy(), "holdout_eff": lab_ho["efficiency"],
                      "holdout_pred": mean[:, 1]}
    rep["_model"] = model
    return rep


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the morphology surrogate on GPU kMC labels "
                                             "and screen candidates")
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--holdout", type=int, default=512)
    ap.add_argument("--candidates", type=int, default=100000)
    ap.add_argument("--steps", type=int, default=50000,
                    help="kMC steps per label (the screened picks; the cost screening is set "
                         "against)")
    ap.add_argument("--train-steps", type=int, default=0, help="training labels (0: --steps)")
    ap.add_argument("--holdout-steps", type=int, default=0, help="holdout labels (0: --steps)")
    ap.add_argument("--burn-in", type=int, default=10000)
    ap.add_argument("--members", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--lr", type=float, default=4e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--tta", type=int, default=1, help="symmetry views averaged per prediction")
    ap.add_argument("--ramp", type=float, default=0.5, help="x-position ramp added to the input")
    ap.add_argument("--labels-cache", default="", help="prefix of cached training/holdout labels")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    rep = run_pipeline(a.train, a.holdout, a.candidates, a.steps, a.burn_in, a.members, a.epochs,
                       seed=a.seed, labels_cache=a.labels_cache, lr=a.lr, tta=a.tta,
                       ramp=a.ramp, holdout_steps=a.holdout_steps or None,
                       train_steps=a.train_steps or None)
    arrays = rep.pop("_arrays")
    model = rep.pop("_model")
    text = json.dumps(rep, indent=1)
    print(text)
    if a.out:
        stem = a.out.rsplit(".", 1)[0]
        with open(a.out, "w") as fh:
            fh.write(text)
        np.savez_compressed(stem + "_holdout.npz", **arrays)
        torch.save(model.state_dict(), stem + "_model.pt")


if __name__ == "__main__":
    main()
