"""The orientation-proposal network: its CPU oracle pinned by finite
differences, and the GPU kernels' loss and gradients against the oracle."""
import numpy as np
import pytest

from oracle.pnet_oracle import bf16, layers, loss_and_grads


def _params(rng, nc):
    out = []
    for kind, cin, cout, *_ in layers(nc):
        fan = 9 * cin if kind == 0 else cin
        out += [rng.normal(0., np.sqrt(2. / fan), cout * fan), rng.normal(0., 0.05, cout)]
    return np.concatenate(out)


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    nc = 12
    p = _params(rng, nc)
    x = np.log1p(rng.poisson(0.7, (3, 1024)).astype(np.float64))
    y = np.array([1, 5, 11])
    loss, g = loss_and_grads(p, x, y, nc, round_weights=False)
    idx = rng.choice(p.size, 40, replace=False)
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp, _ = loss_and_grads(q, x, y, nc, round_weights=False)
        q[i] -= 2 * h
        lm, _ = loss_and_grads(q, x, y, nc, round_weights=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_oracle_soft_target_gradients_match_finite_differences():
    """The oracle's soft cross-entropy (the checker of the soft-target
    training) against finite differences; one-hot targets give the
    hard-label loss."""
    rng = np.random.default_rng(1)
    nc = 12
    p = _params(rng, nc)
    x = np.log1p(rng.poisson(0.7, (3, 1024)).astype(np.float64))
    T = rng.random((3, nc)) * (rng.random((3, nc)) < 0.3)
    T[:, 0] += 0.1
    T /= T.sum(1, keepdims=True)
    loss, g = loss_and_grads(p, x, None, nc, round_weights=False, targets=T)
    idx = rng.choice(p.size, 40, replace=False)
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp, _ = loss_and_grads(q, x, None, nc, round_weights=False, targets=T)
        q[i] -= 2 * h
        lm, _ = loss_and_grads(q, x, None, nc, round_weights=False, targets=T)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])
    y = np.array([1, 5, 11])
    onehot = np.eye(nc)[y]
    l1, g1 = loss_and_grads(p, x, y, nc)
    l2, g2 = loss_and_grads(p, x, None, nc, targets=onehot)
    assert abs(l1 - l2) <= 1e-12 * abs(l1) and np.allclose(g1, g2, rtol=1e-12, atol=1e-15)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-30], np.float32)
    r = bf16(x)
    # BF16 keeps 8 mantissa bits: 1 + 2^-8 rounds to even (1.0), 1 + 3 * 2^-9 up
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] - x[3]) <= 2 ** -8 * abs(x[3])


@pytest.mark.gpu
def test_gpu_gradients_match_oracle():
    from dragonfly_b200._lib import ProposalNet
    rng = np.random.default_rng(1)
    nc = 40
    net = ProposalNet(nc, batch=8, seed=3)
    net.set_option("tensor_core_training", 0)   # the FP32 path
    p = net.params().astype(np.float64)
    x = np.log1p(rng.poisson(0.5, (8, 1024)).astype(np.float64))
    y = rng.integers(0, nc, 8)
    net.set_images(x)
    g, loss = net.gradients(y)
    loss_ref, g_ref = loss_and_grads(p, x.astype(np.float32).astype(np.float64), y, nc)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref), (loss, loss_ref)
    # per layer: relative L2 of the gradient (FP32 accumulation on the GPU)
    o = 0
    for kind, cin, cout, *_ in layers(nc):
        fan = 9 * cin if kind == 0 else cin
        for n in (cout * fan, cout):
            a, b = g[o:o + n].astype(np.float64), g_ref[o:o + n]
            o += n
            assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b) + 1e-9, (kind, cin, cout, n)
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("nc,batch", [(40, 8), (420, 64)])
def test_gpu_tensor_core_gradients_match_oracle(nc, batch):
    """Mixed-precision training: the forward products of layers 1-5 and their
    weight and input gradients on the tcgen05 tensor cores (BF16 activations,
    output gradients and weights; FP32 accumulation, the weight gradients
    split over the batch rows), layer 0, the biases and the loss in FP32.
    Against the oracle with the same roundings (loss_and_grads(mixed=True)):
    the loss and every layer's gradients. Activations summed in FP32 on the
    GPU and in FP64 by the oracle (relative differences of order 1e-6) round
    to different BF16 neighbours now and then, and those flips move the
    gradients: the bound per layer is twice the oracle's own change under a
    1e-6 relative perturbation of the weights (measured here; 1e-4 to 3e-2 on
    these inputs), at least 5e-3. Against the unrounded oracle the BF16
    roundings themselves account for 0.01 % to 10 % per layer (largest
    towards the input, where five products' roundings have added up), with
    the direction kept."""
    from dragonfly_b200._lib import ProposalNet
    rng = np.random.default_rng(11)
    net = ProposalNet(nc, batch=batch, seed=3)
    p = net.params().astype(np.float64)
    x = np.log1p(rng.poisson(0.5, (batch, 1024)).astype(np.float64))
    y = rng.integers(0, nc, batch)
    net.set_images(x)
    g, loss = net.gradients(y)
    x64 = x.astype(np.float32).astype(np.float64)
    loss_mix, g_mix = loss_and_grads(p, x64, y, nc, mixed=True)
    loss_ref, g_ref = loss_and_grads(p, x64, y, nc)
    # the mixed-precision gradients' own sensitivity to rounding flips
    sens = np.zeros_like(g_mix)
    for seed in (1, 2):
        pr = p * (1. + 1e-6 * np.random.default_rng(seed).standard_normal(p.size))
        sens = np.maximum(sens, np.abs(loss_and_grads(pr, x64, y, nc, mixed=True)[1] - g_mix))
    print("loss: tensor cores %.6f, mixed-precision oracle %.6f, oracle %.6f" % (loss, loss_mix, loss_ref))
    assert abs(loss - loss_mix) <= 5e-4 * abs(loss_mix), (loss, loss_mix)
    o, errs = 0, []
    for kind, cin, cout, *_ in layers(nc):
        fan = 9 * cin if kind == 0 else cin
        for n in (cout * fan, cout):
            a, m, b = g[o:o + n].astype(np.float64), g_mix[o:o + n], g_ref[o:o + n]
            sv = np.linalg.norm(sens[o:o + n]) / np.linalg.norm(m)
            o += n
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
            errs.append((kind, cout, n, np.linalg.norm(a - m) / np.linalg.norm(m), sv,
                         np.linalg.norm(a - b) / np.linalg.norm(b), cos))
    for r in errs:
        print("layer kind %d cout %4d size %7d: vs mixed-precision oracle %.2e (its flip sensitivity %.2e), "
              "vs oracle %.2e, cosine %.6f" % r)
    for kind, cout, n, e_mix, sv, e_ref, cos in errs:
        assert e_mix <= max(2. * sv, 5e-3), (kind, cout, n, e_mix, sv)
        assert e_ref <= 0.15 and cos >= 0.99, (kind, cout, n, e_ref, cos)
    # the FP32 path on the same network: FP32 activations against FP64 (2.8e-4
    # of the whole gradient at 420 classes and 64 images, where ReLU masks of
    # near-zero activations flip now and then)
    net.set_option("tensor_core_training", 0)
    g32, _ = net.gradients(y)
    assert np.linalg.norm(g32 - g_ref) <= 1e-3 * np.linalg.norm(g_ref)
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("nc", [40, 420])
def test_gpu_tensor_core_inference_matches_oracle(nc):
    """Inference on the tcgen05 tensor cores (layers 1-5: BF16 activations and
    weights, FP32 accumulation in TMEM) against the oracle's forward pass with
    the same roundings, and against the FP32 path training uses; 3000 images
    (two inference batches, the second partial; 420 classes: two N tiles of
    256, the second partial)."""
    from dragonfly_b200._lib import ProposalNet
    from oracle.pnet_oracle import logits
    rng = np.random.default_rng(4)
    net = ProposalNet(nc, batch=64, seed=5)
    p = net.params().astype(np.float64)
    x = np.log1p(rng.poisson(0.8, (3000, 1024)).astype(np.float64)).astype(np.float32)
    net.set_images(x)
    z_tc = net.logits().astype(np.float64)
    net.set_tensor_cores(False)
    z_fp = net.logits().astype(np.float64)
    sel = rng.choice(3000, 64, replace=False)
    ref_tc = logits(p, x[sel].astype(np.float64), nc, round_activations=True)
    ref_fp = logits(p, x[sel].astype(np.float64), nc, round_activations=False)
    e_tc = np.linalg.norm(z_tc[sel] - ref_tc) / np.linalg.norm(ref_tc)
    e_fp = np.linalg.norm(z_fp[sel] - ref_fp) / np.linalg.norm(ref_fp)
    e_mix = np.linalg.norm(z_tc - z_fp) / np.linalg.norm(z_fp)
    print("logits: tensor cores vs oracle %.2e, FP32 path vs oracle %.2e, tensor cores vs FP32 path %.2e"
          % (e_tc, e_fp, e_mix))
    # activations computed in FP32 on the GPU and in FP64 by the oracle round
    # to different BF16 neighbours now and then (one BF16 step is 2^-8), so the
    # rounded paths agree to a few 1e-4, several times closer than the two
    # forms of the product are to each other
    assert e_fp <= 1e-4, e_fp
    assert e_tc <= 2e-3 and e_tc * 3 < e_mix, (e_tc, e_mix)
    assert e_mix <= 3e-2, e_mix
    net.close()


@pytest.mark.gpu
def test_gpu_mass_covering_topk_matches_the_logits():
    """dfg_pnet_topk_mass: per image the classes by decreasing logit, K_min
    of them and then more until their softmax probabilities reach the mass,
    at most K_max, -1 in the unused slots; the plain top-K is its prefix."""
    from dragonfly_b200._lib import ProposalNet
    rng = np.random.default_rng(8)
    net = ProposalNet(420, batch=64, seed=5)
    x = np.log1p(rng.poisson(0.8, (500, 1024)).astype(np.float64)).astype(np.float32)
    net.set_images(x)
    z = net.logits().astype(np.float64)
    p = np.exp(z - z.max(1, keepdims=True))
    p /= p.sum(1, keepdims=True)
    K_min, K_max, mass = 4, 40, 0.5
    sel = net.topk_mass(K_min, K_max, mass)
    top = net.topk(K_max)
    np.testing.assert_array_equal(net.topk(K_min), top[:, :K_min])
    # up to 256 picks come from the radix-select kernel, more from the
    # per-pick arg-max kernel: the two agree, and with a stable sort of the
    # logits (value descending, index ascending)
    wide = net.topk(300)
    np.testing.assert_array_equal(wide[:, :K_max], top)
    np.testing.assert_array_equal(net.topk(256), wide[:, :256])
    ref = np.argsort(-z, axis=1, kind="stable")[:, :256]
    np.testing.assert_array_equal(net.topk(256), ref)
    for i in range(len(x)):
        n = int((sel[i] >= 0).sum())
        assert K_min <= n <= K_max and np.all(sel[i, n:] == -1)
        np.testing.assert_array_equal(sel[i, :n], top[i, :n])
        cum = np.cumsum(p[i, top[i]])
        # the first count at or after K_min whose cumulative probability
        # reaches the mass (FP32 sums on the device: a 1e-5 margin)
        if n < K_max:
            assert cum[n - 1] >= mass - 1e-5
        if n > K_min:
            assert cum[n - 2] < mass + 1e-5
    net.close()


@pytest.mark.gpu
def test_gpu_tensor_core_wait_gives_up_and_the_network_recovers():
    """Failure detection of the network's tensor-core products without a GPU
    fault: with one stage's copies withheld (test hook) the waits on it run
    out after a short limit and dfg_pnet_logits reports DFG_ERR_CUDA; with the
    hook off the next call on the same network gives the logits of before.
    Training on the tensor cores reports the same at the end of its epoch
    (its products are invalid, so the weights are put back before the
    network is used again)."""
    from dragonfly_b200._lib import DFG_ERR_CUDA, DFGError, ProposalNet
    rng = np.random.default_rng(6)
    net = ProposalNet(40, batch=64, seed=5)
    x = np.log1p(rng.poisson(0.8, (600, 1024)).astype(np.float64)).astype(np.float32)
    net.set_images(x)
    z = net.logits()
    net.set_option("wait_cycles", 2e7)          # about 10 ms per wait
    net.set_option("withhold_stage", 1)
    with pytest.raises(DFGError) as e:
        net.logits()
    assert e.value.code == DFG_ERR_CUDA and "gave up" in str(e.value)
    p0 = net.params()
    with pytest.raises(DFGError) as e:
        net.train(np.arange(600) % 40, epochs=1, lr=1e-3)
    assert e.value.code == DFG_ERR_CUDA and "gave up" in str(e.value)
    net.set_option("withhold_stage", -1)
    net.set_option("wait_cycles", 2e9)
    net.set_params(p0)
    np.testing.assert_array_equal(net.logits(), z)
    net.train(np.arange(600) % 40, epochs=1, lr=1e-3)   # the products run to the end again
    net.close()


@pytest.mark.gpu
def test_gpu_soft_target_gradients_match_oracle():
    """Soft targets (a distribution over a few classes per image, as the
    full search's probabilities aggregated per coarse cell give them): loss
    and gradients against the oracle's soft cross-entropy."""
    from dragonfly_b200._lib import ProposalNet
    rng = np.random.default_rng(2)
    nc = 40
    net = ProposalNet(nc, batch=8, seed=4)
    net.set_option("tensor_core_training", 0)   # the FP32 path
    p = net.params().astype(np.float64)
    x = np.log1p(rng.poisson(0.5, (8, 1024)).astype(np.float64))
    net.set_images(x)
    T = np.zeros((8, nc))
    off, cls, w = [0], [], []
    for i in range(8):
        c = rng.choice(nc, rng.integers(1, 5), replace=False)
        q = rng.random(c.size).astype(np.float32)
        q /= q.sum()
        T[i, c] = q
        cls.extend(c.tolist())
        w.extend(q.tolist())
        off.append(len(cls))
    net.set_targets(np.array(off), np.array(cls), np.array(w, np.float32))
    g, loss = net.gradients()
    loss_ref, g_ref = loss_and_grads(p, x.astype(np.float32).astype(np.float64), None, nc, targets=T)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref), (loss, loss_ref)
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref), np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    # training against the targets (on the tensor cores) lowers their
    # cross-entropy
    net.set_option("tensor_core_training", 1)
    l1 = net.train(epochs=20, lr=1e-3)
    assert l1 < loss, (l1, loss)
    with pytest.raises(RuntimeError):
        net.set_targets(np.array([0, 2] + [2] * 7), np.array([3, 3]), np.array([0.5, 0.5], np.float32))
    net.close()


def test_oracle_logits_agree_with_the_loss_forward():
    """The oracle's inference forward (BF16 weights, FP64 activations) gives
    the loss that loss_and_grads computes from its own forward pass; with
    rounded activations it stays within a BF16 step's effect."""
    from oracle.pnet_oracle import logits
    rng = np.random.default_rng(5)
    nc = 12
    p = _params(rng, nc)
    x = np.log1p(rng.poisson(0.7, (4, 1024)).astype(np.float64))
    y = np.array([0, 3, 7, 11])
    z = logits(p, x, nc)
    m = z.max(1, keepdims=True)
    loss = float(np.mean(np.log(np.exp(z - m).sum(1)) + m[:, 0] - z[np.arange(4), y]))
    ref, _ = loss_and_grads(p, x, y, nc)
    assert abs(loss - ref) <= 1e-12 * abs(ref)
    zr = logits(p, x, nc, round_activations=True)
    assert np.linalg.norm(zr - z) <= 2e-2 * np.linalg.norm(z)
