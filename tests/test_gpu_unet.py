"""The learned denoiser (RtxUnet*, RtxSetDenoiser, RtxReadAovs) against a
plain PyTorch FP32 restatement of the same network, run on the CPU.

The CUDA network keeps activations and the 3x3 weights in BF16 and
accumulates in FP32; the PyTorch restatement rounds the same tensors to BF16
in its forward pass (straight-through in the backward pass) and computes
everything else in FP32. Tolerances: loss within 0.5% relative; each
layer's gradient within 5% relative L2 error with cosine similarity above
0.99 (the CUDA backward also rounds the pre-activation gradient to BF16);
inference within 0.05 absolute in log(1 + radiance)."""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

import scenes
from native_api import Unet

pytestmark = pytest.mark.gpu

WIDTHS = (32, 48, 64, 96, 128)


def layer_table():
    """(input channels, output channels) of the 18 3x3 layers; input padded to 16."""
    layers, prev = [], 16
    for w in WIDTHS:
        layers += [(prev, w), (w, w)]
        prev = w
    for w in WIDTHS[3::-1]:
        layers += [(prev + w, w), (w, w)]
        prev = w
    return layers


def unpack(flat):
    """Flat parameters -> [(weight OIHW, bias)] * 18 + [(w[32][3], b[3])]."""
    out, off = [], 0
    for ci, co in layer_table():
        w = flat[off:off + 9 * ci * co].reshape(3, 3, ci, co)
        off += 9 * ci * co
        out.append([torch.tensor(w).permute(3, 2, 0, 1).contiguous().requires_grad_(),
                    torch.tensor(flat[off:off + co]).requires_grad_()])
        off += co
    out.append([torch.tensor(flat[off:off + 96].reshape(32, 3)).requires_grad_(),
                torch.tensor(flat[off + 96:off + 99]).requires_grad_()])
    assert off + 99 == flat.size
    return out


def pack_grads(params):
    parts = []
    for w, b in params[:-1]:
        parts += [w.grad.permute(2, 3, 1, 0).reshape(-1), b.grad]
    parts += [params[-1][0].grad.reshape(-1), params[-1][1].grad]
    return torch.cat(parts).numpy()


def bf(x):
    return x + (x.to(torch.bfloat16).float() - x).detach()


def features(aovs):
    """The network input (N, 16, H, W) from AOVs (N, H, W, 10)."""
    a = np.asarray(aovs, np.float32)
    x = np.zeros(a.shape[:3] + (16,), np.float32)
    x[..., 0:3] = np.log1p(np.maximum(a[..., 0:3], 0))
    x[..., 3:9] = a[..., 3:9]
    x[..., 9] = np.log1p(np.maximum(a[..., 9], 0))
    return torch.tensor(x).permute(0, 3, 1, 2)


def forward(x, params):
    x = bf(x)
    skips, k = [], 0
    for level in range(5):
        if level:
            x = bf(F.avg_pool2d(x, 2))
        for _ in range(2):
            w, b = params[k]
            k += 1
            x = bf(F.relu(F.conv2d(x, bf(w), b, padding=1)))
        skips.append(x)
    for level in (3, 2, 1, 0):
        x = torch.cat([F.interpolate(x, scale_factor=2, mode='nearest'), skips[level]], 1)
        for _ in range(2):
            w, b = params[k]
            k += 1
            x = bf(F.relu(F.conv2d(x, bf(w), b, padding=1)))
    wo, bo = params[-1]
    return torch.einsum('nchw,ck->nkhw', x, wo) + bo[None, :, None, None]


def synthetic(rng, n, h, w):
    """Noisy radiance around a smooth target, with albedo, normals, depth."""
    yy, xx = np.mgrid[0:h, 0:w] / max(h, w)
    target = np.empty((n, h, w, 3), np.float32)
    aovs = np.empty((n, h, w, 10), np.float32)
    for i in range(n):
        base = rng.uniform(0.1, 2.0, 3)
        target[i] = (base * (0.5 + 0.5 * np.sin(3 * xx + 2 * yy + i))[..., None]).astype(np.float32)
        aovs[i, ..., 0:3] = target[i] * rng.exponential(1.0, (h, w, 3))
        aovs[i, ..., 3:6] = rng.uniform(0, 1, 3)
        nrm = rng.normal(size=(h, w, 3))
        aovs[i, ..., 6:9] = nrm / np.linalg.norm(nrm, axis=-1, keepdims=True)
        aovs[i, ..., 9] = 1.0 + 4.0 * yy
    return aovs, target


@pytest.fixture(scope='module')
def net(lib):
    n = Unet(lib, seed=5)
    yield n
    n.close()


def test_parameter_layout(net):
    table = layer_table()
    assert net.param_count == sum(9 * ci * co + co for ci, co in table) + 32 * 3 + 3 == 1_017_379
    p = net.params()
    w0 = p[:9 * 16 * 32].reshape(9, 16, 32)
    assert (w0[:, 10:, :] == 0).all() and np.abs(w0[:, :10, :]).max() > 0  # padding channels stay zero
    q = np.random.default_rng(1).normal(0, 0.05, p.size).astype(np.float32)
    net.set_params(q)
    assert np.array_equal(net.params(), q)
    net.set_params(p)


def test_loss_and_gradient_match_pytorch(net):
    rng = np.random.default_rng(3)
    aovs, target = synthetic(rng, 2, 32, 48)
    flat = net.params()
    loss, grads = net.loss_grad(aovs, target)
    params = unpack(flat)
    pred = forward(features(aovs), params)
    t = torch.tensor(np.log1p(target)).permute(0, 3, 1, 2)
    ref = (pred - t).abs().mean()
    ref.backward()
    assert abs(loss - ref.item()) <= 5e-3 * ref.item(), (loss, ref.item())
    expect = pack_grads(params)
    off = 0
    sizes = [9 * ci * co for ci, co in layer_table()]
    chunks = []
    for (ci, co), size in zip(layer_table(), sizes):
        chunks += [('w', size), ('b', co)]
    chunks += [('w', 96), ('b', 3)]
    for i, (kind, size) in enumerate(chunks):
        g, e = grads[off:off + size].astype(np.float64), expect[off:off + size].astype(np.float64)
        off += size
        norm = np.linalg.norm(e)
        assert norm > 0, i
        rel = np.linalg.norm(g - e) / norm
        cos = g @ e / (np.linalg.norm(g) * norm)
        assert rel < 5e-2 and cos > 0.99, (i // 2, kind, rel, cos)
    assert off == grads.size


def test_inference_any_size_matches_pytorch(net):
    rng = np.random.default_rng(4)
    aovs, _ = synthetic(rng, 1, 37, 23)
    out = net.infer(aovs[0])
    assert out.shape == (37, 23, 3) and np.isfinite(out).all() and (out >= 0).all()
    padded = np.pad(aovs, ((0, 0), (0, 48 - 37), (0, 32 - 23), (0, 0)), mode='edge')
    with torch.no_grad():
        pred = forward(features(padded), unpack(net.params()))[0].permute(1, 2, 0).numpy()[:37, :23]
    expect = np.maximum(np.expm1(pred), 0)
    diff = np.abs(np.log1p(out) - np.log1p(expect))
    assert diff.max() < 5e-2 and diff.mean() < 5e-3, (diff.max(), diff.mean())


def test_training_reduces_loss_and_checkpoints(lib, tmp_path):
    rng = np.random.default_rng(6)
    aovs, target = synthetic(rng, 8, 32, 32)
    net = Unet(lib, seed=9)
    try:
        before, _ = net.loss_grad(aovs, target)
        losses = net.train(aovs, target, steps=80, batch=4, lr=2e-3, seed=1)
        assert losses.shape == (80,) and np.isfinite(losses).all()
        after, _ = net.loss_grad(aovs, target)
        assert after < 0.7 * before, (before, after)
        path = tmp_path / 'net.bin'
        net.save(path)
        assert path.stat().st_size == 32 + 4 * net.param_count
        net.save(tmp_path / 'state.bin', optimizer_state=True)
        assert (tmp_path / 'state.bin').stat().st_size == 32 + 12 * net.param_count
        other = Unet(lib, seed=10)
        try:
            assert not np.array_equal(other.params(), net.params())
            other.load(path)
            assert np.array_equal(other.params(), net.params())
            other.load(tmp_path / 'state.bin')
            assert np.array_equal(other.params(), net.params())
            (tmp_path / 'bad.bin').write_bytes(path.read_bytes()[:-4])
            with pytest.raises(Exception, match='checkpoint'):
                other.load(tmp_path / 'bad.bin')
            with pytest.raises(Exception, match='cannot read'):
                other.load(tmp_path / 'missing.bin')
        finally:
            other.close()
        with pytest.raises(Exception, match='multiples of 16'):
            net.loss_grad(aovs[:, :30], target[:, :30])
    finally:
        net.close()


def test_session_aovs_and_learned_denoise(lib, session, net):
    """RtxReadAovs is the accumulation divided by the sample count (normal
    normalised, first-hit distance added); RtDenoise with a network equals
    tonemapping RtxUnetInfer of those AOVs; uncovered pixels stay black."""
    tris, camera, settings, _, _ = scenes.cornell_sphere()
    w, h = 45, 33
    camera.aspect = w / h
    settings.raysPerPixel = 4
    session.initialize(tris, w, h)
    session.render(camera, settings)
    spp = session.sample_count()
    acc = session.accumulation()
    aovs = session.aovs()
    inv = np.float32(1) / np.float32(spp)

    def vec(field):
        return np.stack([acc[field][k] for k in 'xyz'], -1)
    assert np.array_equal(aovs[..., 0:3].reshape(-1, 3), vec('radiance') * inv)
    assert np.array_equal(aovs[..., 3:6].reshape(-1, 3), vec('albedo') * inv)
    covered = acc['covered'].reshape(h, w) != 0
    assert covered.mean() > 0.9
    lengths = np.linalg.norm(aovs[..., 6:9], axis=-1)
    assert np.abs(lengths[covered] - 1).max() < 1e-5
    depth = aovs[..., 9]
    assert (depth[covered] > 0).all() and (depth[covered] < 100).all() and (depth[~covered] == 0).all()
    plain, _ = session.denoise()
    session.set_denoiser(net)
    learned, ms = session.denoise()
    assert ms > 0 and 0 < session.render_stats()['denoiseMs'] <= ms  # device time of the kernels, within the call
    radiance = net.infer(aovs)
    c = 1 - np.exp(-np.maximum(radiance, 0) * np.float32(settings.exposure))
    c = np.where(c <= 0.0031308, 12.92 * c, 1.055 * np.power(c, 1 / 2.4) - 0.055)
    expect = np.floor(255 * np.minimum(c, 1) + 0.5) * covered[..., None]
    got = learned.reshape(h, w, 4)
    assert (got[..., 3] == 255).all()
    assert np.abs(got[..., :3].astype(int) - expect).max() <= 1
    session.set_denoiser(None)
    again, _ = session.denoise()
    assert np.array_equal(again, plain)
    camera.origin.x = 10000
    lib.RtReset(session.handle)
    session.render(camera, settings)
    session.set_denoiser(net)
    dark, _ = session.denoise()
    assert (dark.reshape(-1, 4)[:, :3] == 0).all()
    session.set_denoiser(None)


def test_trained_network_gains_over_the_filter(lib):
    """The committed network against the guided filter and the raw 4-spp
    image (the input it was trained on), on held-out rooms (seeds outside
    the training range) scored against their 1024-path renders: PSNR on
    8-bit display values."""
    from native_api import DENOISER_WEIGHTS
    import train_denoiser as td
    net = Unet(lib)
    try:
        net.load(DENOISER_WEIGHTS)
        gains = []
        for seed in (950_001, 950_002, 950_003):
            inputs, target, exposure, filtered = td.render_room(lib, seed, 128, 1024, (4,))
            ref = td.display(target, exposure)
            raw = td.psnr(td.display(inputs[0][..., 0:3], exposure), ref)
            guided = td.psnr(filtered[0], ref)
            learned = td.psnr(td.display(net.infer(inputs[0]), exposure), ref)
            gains.append((raw, guided, learned))
        raw, guided, learned = np.mean(gains, axis=0)
        assert learned > guided + 1.5 and learned > raw + 6.0, gains
    finally:
        net.close()


def test_conv_kernels_agree(lib, net):
    """The warp-specialised, TMA-fed convolution (the default wherever its
    shared memory allows) and the single-role kernel for every layer
    (RtxSetConvPath(1)) give the same inference and training gradients to
    BF16 rounding: at image sizes with partial 128-pixel column tiles, the
    concatenated decoder inputs (two passes in the default path, read in
    place by the single-role kernel), and tiny deep levels."""
    import ctypes as c
    rng = np.random.default_rng(12)

    def counts():
        pipe, single = c.c_longlong(), c.c_longlong()
        lib.RtxConvLaunchCounts(c.byref(pipe), c.byref(single))
        return pipe.value, single.value
    try:
        before = counts()
        aovs, _ = synthetic(rng, 1, 64, 256)
        net.infer(aovs[0])
        after = counts()
        # 18 layers; the concatenated decoder layers whose two halves fit the
        # pipelined kernel (80 -> 32, 112 -> 48, 160 -> 64) run as two
        # convolutions each (the upsampled half at half resolution, then the
        # skip half adding it): 21 convolutions, all but 224 -> 96 pipelined.
        pipe, single = after[0] - before[0], after[1] - before[1]
        assert pipe == 20 and single == 1, (before, after)
        for h, w in ((64, 256), (72, 136), (37, 23)):
            aovs, _ = synthetic(rng, 1, h, w)
            assert lib.RtxSetConvPath(1)
            old = net.infer(aovs[0])
            assert lib.RtxSetConvPath(0)
            new = net.infer(aovs[0])
            diff = np.abs(np.log1p(new) - np.log1p(old))
            assert diff.max() < 5e-2 and diff.mean() < 2e-3, (h, w, diff.max(), diff.mean())
        aovs, target = synthetic(rng, 2, 32, 160)
        lib.RtxSetConvPath(1)
        loss_old, grad_old = net.loss_grad(aovs, target)
        lib.RtxSetConvPath(0)
        loss_new, grad_new = net.loss_grad(aovs, target)
        assert abs(loss_new - loss_old) <= 2e-3 * loss_old
        g, e = grad_new.astype(np.float64), grad_old.astype(np.float64)
        assert np.linalg.norm(g - e) <= 2e-2 * np.linalg.norm(e)
    finally:
        lib.RtxSetConvPath(0)


def test_stacked_row_issue_identical(lib, net):
    """The pipelined kernel's default form stages input rows as swizzled
    slabs of 16-64 channels (one TMA box each) and, for unsplit 32-channel
    layers, issues one MMA per input row and column tap over the three kernel
    rows' weights side by side (accumulator blocks per output row in a ring);
    RtxSetConvPath(2) stages rows as planes of 8 channels and issues every tap
    per output tile. The MMAs see the same operands and each output row
    receives the taps in the same order either way, so inference is
    bit-identical: at sizes whose strips end mid-image, with a partial column
    tile, and with one-row strips. Training agrees to FP32 summation order
    (the loss and the bias and head gradients sum with atomics, whose order
    varies from run to run)."""
    rng = np.random.default_rng(21)
    try:
        for h, w in ((200, 300), (37, 130), (16, 16)):
            aovs, _ = synthetic(rng, 1, h, w)
            assert lib.RtxSetConvPath(2)
            tap = net.infer(aovs[0])
            assert lib.RtxSetConvPath(0)
            stacked = net.infer(aovs[0])
            assert np.array_equal(tap, stacked), (h, w)
        aovs, target = synthetic(rng, 3, 48, 144)
        lib.RtxSetConvPath(2)
        loss_tap, grad_tap = net.loss_grad(aovs, target)
        lib.RtxSetConvPath(0)
        loss_stacked, grad_stacked = net.loss_grad(aovs, target)
        assert abs(loss_tap - loss_stacked) <= 1e-6 * loss_tap
        g, e = grad_stacked.astype(np.float64), grad_tap.astype(np.float64)
        assert np.linalg.norm(g - e) <= 1e-5 * np.linalg.norm(e)
        assert not lib.RtxSetConvPath(3)
    finally:
        lib.RtxSetConvPath(0)


def test_conv_wait_limit_reports_and_recovers(lib):
    """A pipelined convolution whose tensor-core issuer waits on a barrier
    that nothing completes gives up after its (2 ms) limit, reports through
    the error flag, frees its tensor memory and loads, and the next launch
    on the same device computes the right output."""
    assert lib.RtxDebugConvWaitProbe() == 1
