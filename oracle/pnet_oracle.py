"""CPU oracle of the orientation-proposal network (TEST INFRASTRUCTURE ONLY:
used by tests/ to check the GPU kernels of dragonfly_b200/csrc/proposal.cu).

float64 numpy forward and backward passes of the same network: NHWC
activations, 3x3 convolutions as im2col products with weights [cout][9 cin]
(rows ordered ky, kx, c), ReLU, fully connected layers, softmax
cross-entropy against class labels, mean over the batch. The products use
the weights rounded to BF16 (round to nearest even), as the GPU does; the
gradients are those of that network. Parameters are flat as
dfg_pnet_get_params lays them out: per layer the weights, then the biases.
"""
import numpy as np

IMG = 32


def layers(num_classes):
    """(kind, cin, cout, hin, stride, hout) per layer; kind 0 = conv 3x3."""
    return [(0, 1, 32, 32, 1, 32), (0, 32, 32, 32, 2, 16), (0, 32, 64, 16, 1, 16), (0, 64, 64, 16, 2, 8),
            (1, 4096, 256, 0, 0, 0), (1, 256, num_classes, 0, 0, 0)]


def bf16(x):
    """Round float values to BF16 (nearest even) and back to float64."""
    a = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (a + 0x7FFF + ((a >> 16) & 1)) >> 16 << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unflatten(params, num_classes):
    out, o = [], 0
    for kind, cin, cout, *_ in layers(num_classes):
        fan = 9 * cin if kind == 0 else cin
        w = np.asarray(params[o:o + cout * fan], np.float64).reshape(cout, fan)
        o += cout * fan
        b = np.asarray(params[o:o + cout], np.float64)
        o += cout
        out.append((w, b))
    return out


def im2col(x, s, ho):
    """x [B][H][H][C] -> cols [B*ho*ho][9*C] (ky, kx, c), zero padding 1."""
    B, H, _, C = x.shape
    xp = np.zeros((B, H + 2, H + 2, C))
    xp[:, 1:H + 1, 1:H + 1] = x
    cols = np.empty((B, ho, ho, 3, 3, C))
    for ky in range(3):
        for kx in range(3):
            cols[:, :, :, ky, kx] = xp[:, ky:ky + s * ho:s, kx:kx + s * ho:s]
    return cols.reshape(B * ho * ho, 9 * C)


def col2im(dcols, B, H, C, s, ho):
    d = dcols.reshape(B, ho, ho, 3, 3, C)
    dxp = np.zeros((B, H + 2, H + 2, C))
    for ky in range(3):
        for kx in range(3):
            dxp[:, ky:ky + s * ho:s, kx:kx + s * ho:s] += d[:, :, :, ky, kx]
    return dxp[:, 1:H + 1, 1:H + 1]


def logits(params, images, num_classes, round_activations=False):
    """Forward pass of the images [B][1024] to logits [B][classes] with BF16
    weights; with round_activations the inputs of layers 1-5 are rounded to
    BF16 too (the tensor-core inference path: BF16 operands, FP32 sums)."""
    L = layers(num_classes)
    P = unflatten(params, num_classes)
    B = images.shape[0]
    a = np.asarray(images, np.float64).reshape(B, IMG, IMG, 1)
    for l, ((kind, cin, cout, hin, s, ho), (w, b)) in enumerate(zip(L, P)):
        x = bf16(a) if (round_activations and l > 0) else a
        cols = im2col(x, s, ho) if kind == 0 else x.reshape(B, -1)
        y = cols @ bf16(w).T + b
        y = y.reshape(B, ho, ho, cout) if kind == 0 else y
        a = np.maximum(y, 0.) if l < len(L) - 1 else y
    return a


def loss_and_grads(params, images, labels, num_classes, round_weights=True, targets=None, mixed=False):
    """Mean softmax cross-entropy of the images [B][1024] and its gradient
    with respect to the flat parameters; against the labels, or (targets
    [B][classes], rows summing to 1) against soft targets. mixed: the
    roundings of mixed-precision training on the tensor cores -- the inputs
    of layers 1-5 rounded to BF16 in the forward products and in their
    weight gradients, the output gradients of layers 1-5 rounded to BF16 in
    their weight and input gradients (bias gradients and layer 0 from the
    unrounded values)."""
    L = layers(num_classes)
    P = unflatten(params, num_classes)
    B = images.shape[0]
    x = np.asarray(images, np.float64).reshape(B, IMG, IMG, 1)
    acts, colss = [x], []
    for l, ((kind, cin, cout, hin, s, ho), (w, b)) in enumerate(zip(L, P)):
        wr = bf16(w) if round_weights else w
        a_in = bf16(acts[-1]) if (mixed and l > 0) else acts[-1]
        if kind == 0:
            cols = im2col(a_in, s, ho)
            y = (cols @ wr.T + b).reshape(B, ho, ho, cout)
        else:
            cols = a_in.reshape(B, -1)
            y = cols @ wr.T + b
        colss.append(cols)
        acts.append(np.maximum(y, 0.) if l < len(L) - 1 else y)
    z = acts[-1]
    m = z.max(1, keepdims=True)
    e = np.exp(z - m)
    sm = e / e.sum(1, keepdims=True)
    if targets is None:
        targets = np.zeros_like(z)
        targets[np.arange(B), labels] = 1.
    loss = float(np.mean(np.log(e.sum(1)) + m[:, 0] - (targets * z).sum(1)))
    dy = (sm - targets) / B
    grads = [None] * len(L)
    for l in range(len(L) - 1, -1, -1):
        kind, cin, cout, hin, s, ho = L[l]
        w = P[l][0]
        wr = bf16(w) if round_weights else w
        if l < len(L) - 1:
            dy = dy * (acts[l + 1] > 0)
        d2 = dy.reshape(-1, cout)
        gb = d2.sum(0)
        if mixed and l > 0:
            d2 = bf16(d2)
        gw = d2.T @ colss[l]
        grads[l] = (gw, gb)
        if l > 0:
            dc = d2 @ wr
            dy = col2im(dc, B, hin, cin, s, ho) if kind == 0 else dc.reshape(acts[l].shape)
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat
