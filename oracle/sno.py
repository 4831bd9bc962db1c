"""FP64 CPU restatement of the surrogate far-field network (forward, loss and
backward) - test infrastructure only: the checker for the library's tcgen05
forward / adjoint / weight-gradient kernels.

There is no reference counterpart: the reference has no learned component.
The network is the one the library defines (a U-Net over the 4 x 4-cell patch
grid: 4 levels, 32 channels, 3x3x3 convolutions, 1x2x2 stride-2 down/up
transfers with additive skips, a 1x1x1 head; no biases, no activations).
Weights are a flat array, per layer [cout][tap][cin] in layer order, the
layout of mms_sno_set_weights.  Arrays here are [batch, z, y, x, channel].
"""
from __future__ import annotations

import numpy as np

PATCH = 4
CH = 32
LEVELS = 4
CIN0 = PATCH * PATCH
CONV3, DOWN, UP, POINT = 0, 1, 2, 3
TAPS = {CONV3: 27, DOWN: 4, UP: 4, POINT: 1}


def architecture():
    """(layers, node_levels, node_channels); a layer is a dict with pat, inp,
    out, skip, cin, cout, w_off"""
    lev, ch, layers = [], [], []
    off = [0]

    def node(level, c):
        lev.append(level)
        ch.append(c)
        return len(lev) - 1

    def add(pat, inp, out, skip=-1):
        d = dict(pat=pat, inp=inp, out=out, skip=skip, cin=ch[inp], cout=ch[out], w_off=off[0])
        off[0] += d["cout"] * TAPS[pat] * d["cin"]
        layers.append(d)

    x = node(0, CIN0)
    a = [node(0, CH)]
    add(CONV3, x, a[0])
    for level in range(1, LEVELS):
        d = node(level, CH)
        add(DOWN, a[level - 1], d)
        a.append(node(level, CH))
        add(CONV3, d, a[level])
    cur = node(LEVELS - 1, CH)
    add(CONV3, a[LEVELS - 1], cur)
    for level in range(LEVELS - 2, -1, -1):
        u = node(level, CH)
        add(UP, cur, u, a[level])
        c = node(level, CH)
        add(CONV3, u, c)
        cur = c
    y = node(0, CIN0)
    add(POINT, cur, y)
    return layers, lev, ch


def num_params():
    layers, _, _ = architecture()
    last = layers[-1]
    return last["w_off"] + last["cout"] * last["cin"]


def level_dims(Y, X):
    H, W = [-(-Y // PATCH)], [-(-X // PATCH)]
    for _ in range(1, LEVELS):
        H.append((H[-1] + 1) // 2)
        W.append((W[-1] + 1) // 2)
    return H, W


def layer_weights(w, layer):
    T = TAPS[layer["pat"]]
    n = layer["cout"] * T * layer["cin"]
    return np.asarray(w[layer["w_off"]:layer["w_off"] + n], np.float64).reshape(layer["cout"], T, layer["cin"])


def patchify(u, H, W):
    """[B, Z, Y, X] cells -> [B, Z, H, W, 16] (channel = 4 * row-in-patch + column)"""
    B, Z, Y, X = u.shape
    pad = np.zeros((B, Z, H * PATCH, W * PATCH))
    pad[:, :, :Y, :X] = u
    return pad.reshape(B, Z, H, PATCH, W, PATCH).transpose(0, 1, 2, 4, 3, 5).reshape(B, Z, H, W, CIN0)


def unpatchify(p, Y, X):
    B, Z, H, W, _ = p.shape
    return p.reshape(B, Z, H, W, PATCH, PATCH).transpose(0, 1, 2, 4, 3, 5).reshape(B, Z, H * PATCH, W * PATCH)[
        :, :, :Y, :X]


def _conv3_taps():
    for t in range(27):
        yield t, t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1


def _shift(a, dz, dy, dx):
    """s[.., z, y, x, :] = a[.., z + dz, y + dy, x + dx, :], zero outside"""
    B, Z, H, W, C = a.shape
    s = np.zeros_like(a)
    zs, ys, xs = slice(max(0, -dz), min(Z, Z - dz)), slice(max(0, -dy), min(H, H - dy)), slice(max(0, -dx),
                                                                                              min(W, W - dx))
    zt, yt, xt = slice(max(0, dz), min(Z, Z + dz)), slice(max(0, dy), min(H, H + dy)), slice(max(0, dx),
                                                                                            min(W, W + dx))
    s[:, zs, ys, xs] = a[:, zt, yt, xt]
    return s


def _apply(layer, Wl, a, out_hw):
    """forward of one layer (without the skip)"""
    pat = layer["pat"]
    if pat == CONV3:
        out = np.zeros(a.shape[:4] + (Wl.shape[0],))
        for t, dz, dy, dx in _conv3_taps():
            out += _shift(a, dz, dy, dx) @ Wl[:, t, :].T
        return out
    if pat == POINT:
        return a @ Wl[:, 0, :].T
    Ho, Wo = out_hw
    B, Z = a.shape[:2]
    out = np.zeros((B, Z, Ho, Wo, Wl.shape[0]))
    if pat == DOWN:
        Hi, Wi = a.shape[2:4]
        pad = np.zeros((B, Z, 2 * Ho, 2 * Wo, a.shape[4]))
        pad[:, :, :Hi, :Wi] = a
        for t in range(4):
            out += pad[:, :, (t >> 1)::2, (t & 1)::2][:, :, :Ho, :Wo] @ Wl[:, t, :].T
        return out
    # UP
    for t in range(4):
        dy, dx = t >> 1, t & 1
        src = a[:, :, :(Ho - dy + 1) // 2, :(Wo - dx + 1) // 2]
        out[:, :, dy::2, dx::2] = src @ Wl[:, t, :].T
    return out


def forward(w, u):
    """network output in patch layout and every node activation; u: [B, Z, Y, X]"""
    layers, lev, ch = architecture()
    B, Z, Y, X = u.shape
    H, W = level_dims(Y, X)
    acts = [None] * len(lev)
    acts[0] = patchify(np.asarray(u, np.float64), H[0], W[0])
    for layer in layers:
        lo = lev[layer["out"]]
        out = _apply(layer, layer_weights(w, layer), acts[layer["inp"]], (H[lo], W[lo]))
        if layer["skip"] >= 0:
            out = out + acts[layer["skip"]]
        acts[layer["out"]] = out
    return acts[-1], acts


def far_field(w, u):
    """network output as cells [B, Z, Y, X]"""
    y, _ = forward(w, u)
    return unpatchify(y, u.shape[2], u.shape[3])


def loss_and_grad(w, u, far):
    """loss = mean_b |y_b - t_b|^2 / |t_b|^2 and d loss / d w (flat, FP64)"""
    layers, lev, ch = architecture()
    B, Z, Y, X = u.shape
    H, W = level_dims(Y, X)
    y, acts = forward(w, u)
    t = patchify(np.asarray(far, np.float64), H[0], W[0])
    t2 = (t ** 2).reshape(B, -1).sum(1)
    t2 = np.where(t2 > 0, t2, 1.0)
    e = (y - t)
    loss = float(((e ** 2).reshape(B, -1).sum(1) / t2).mean())
    grads = [np.zeros_like(a) if a is not None else None for a in acts]
    grads[-1] = 2 * e / (B * t2)[:, None, None, None, None]
    gw = np.zeros(num_params())
    for layer in reversed(layers):
        Wl = layer_weights(w, layer)
        d = grads[layer["out"]]
        a = acts[layer["inp"]]
        if layer["skip"] >= 0:
            grads[layer["skip"]] += d
        pat = layer["pat"]
        T = TAPS[pat]
        gl = np.zeros_like(Wl)
        din = np.zeros_like(a)
        C = d.shape[-1]
        if pat == CONV3:
            for tt, dz, dy, dx in _conv3_taps():
                sa = _shift(a, dz, dy, dx)
                gl[:, tt, :] = d.reshape(-1, C).T @ sa.reshape(-1, a.shape[-1])
                din += _shift(d @ Wl[:, tt, :], -dz, -dy, -dx)
        elif pat == POINT:
            gl[:, 0, :] = d.reshape(-1, C).T @ a.reshape(-1, a.shape[-1])
            din = d @ Wl[:, 0, :]
        elif pat == DOWN:
            Ho, Wo = d.shape[2:4]
            Hi, Wi = a.shape[2:4]
            pad = np.zeros(a.shape[:2] + (2 * Ho, 2 * Wo, a.shape[4]))
            pad[:, :, :Hi, :Wi] = a
            dpad = np.zeros_like(pad)
            for tt in range(4):
                sl = (slice(None), slice(None), slice(tt >> 1, None, 2), slice(tt & 1, None, 2))
                src = pad[sl][:, :, :Ho, :Wo]
                gl[:, tt, :] = d.reshape(-1, C).T @ src.reshape(-1, a.shape[-1])
                dpad[sl][:, :, :Ho, :Wo] += d @ Wl[:, tt, :]
            din = dpad[:, :, :Hi, :Wi]
        else:  # UP
            Ho, Wo = d.shape[2:4]
            for tt in range(4):
                dy, dx = tt >> 1, tt & 1
                hs, ws = (Ho - dy + 1) // 2, (Wo - dx + 1) // 2
                dd = d[:, :, dy::2, dx::2]
                src = a[:, :, :hs, :ws]
                gl[:, tt, :] = dd.reshape(-1, C).T @ src.reshape(-1, a.shape[-1])
                din[:, :, :hs, :ws] += dd @ Wl[:, tt, :]
        n = gl.size
        gw[layer["w_off"]:layer["w_off"] + n] = gl.ravel()
        if layer["inp"] != 0:
            grads[layer["inp"]] += din
    return loss, gw


def init_weights(seed):
    """scaled uniform initialisation (per layer +-sqrt(3 / fan_in) x gain),
    seeded Philox"""
    layers, _, _ = architecture()
    g = np.random.Generator(np.random.Philox(seed))
    w = np.zeros(num_params(), np.float32)
    for layer in layers:
        T = TAPS[layer["pat"]]
        fan_in = T * layer["cin"] if layer["pat"] != UP else layer["cin"]
        n = layer["cout"] * T * layer["cin"]
        lim = np.sqrt(3.0 / fan_in)
        w[layer["w_off"]:layer["w_off"] + n] = g.uniform(-lim, lim, n)
    return w


def round_bf16(w):
    """round-to-nearest-even FP32 -> BF16, returned as FP32 values"""
    b = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)
