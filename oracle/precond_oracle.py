"""CPU restatement of the learned multilevel convolutional preconditioner.

THIS IS TEST INFRASTRUCTURE: the checker of the GPU network's forward pass,
loss and parameter gradients.  Nothing in the product path imports it.

The reference (SimiLie) has no learned preconditioner; this file restates
the network the GPU library defines (similie_b200/csrc/precond_net.cuh):

  M(r): e1 = w D^-1 r; r1 = r - K e1; s = rms(D^-1/2 r1);
        x = pool2x2([D^-1/2 r1/s, log(nu)/log(1000)]);  v = s D^-1/2 up2x2(net(x)) (0 on the boundary);
        e2 = e1 + v;  M(r) = e2 + w D^-1 (r - K e2),  w = 0.8
  net:  h0 = relu(inc(x));  per level l >= 1: p_l = relu(down(pool(h_{l-1}))), h_l = relu(enc(p_l));
        g_{D-1} = h_{D-1};  g_l = relu(dec(h_l + up(g_{l+1})));  out = outc(g_0)
  loss: 1 - (u.b)^2 / ((u.K u)(x.b)), u = M(b), mean over the batch.

Images are stored padded with a zero border ((h+2) x (w+2) pixels, channels
last).  With `emulate=True` every value the GPU stores in BF16 (activations,
pooled inputs, masked gradients fed to the tensor cores, the 32->32 weights)
is rounded to BF16 here at the same point (the decoder input skip +
up(coarse) is a sum of two BF16 tensors that the tensor core accumulates in
FP32 in the GPU's training pass, so it is not rounded; the GPU's inference
pass rounds that sum to BF16 once before its decoder convolution, which
this restatement does not), so the GPU's training-pass results differ only
by FP32 summation order; with
`emulate=False` the whole computation is float64, which the finite-difference
test uses to pin the backward pass.
"""
import math

import numpy as np

C = 32
TAPS = 9
BIG_W = C * TAPS * C
BIG_P = BIG_W + C
IN_W = C * TAPS * 2
OUT_W = TAPS * C
OFF_IN = 0
OFF_BIG = IN_W + C
OFF_OUT = OFF_BIG + 9 * BIG_P
NUM_PARAMS = OFF_OUT + OUT_W + 1
OMEGA = 0.8
DOWN, ENC, DEC = 0, 1, 2


def bf16(a):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


class Rounder:
    def __init__(self, emulate):
        self.emulate = emulate

    def __call__(self, a):
        if not self.emulate:
            return np.asarray(a, dtype=np.float64)
        return bf16(np.asarray(a, dtype=np.float32)).astype(np.float64)


# ----------------------------------------------------------------- parameters

def big_slice(kind, wl):
    j = wl * 3 + kind
    o = OFF_BIG + j * BIG_P
    return o, o + BIG_W, o + BIG_P


def unpack(params, rnd):
    """Weights as arrays: big[kind][wl] = (W[co, tap, ci] (BF16-rounded when emulating), bias)."""
    p = np.asarray(params, dtype=np.float64)
    win = p[OFF_IN:OFF_IN + IN_W].reshape(C, TAPS, 2)
    bin_ = p[OFF_IN + IN_W:OFF_IN + IN_W + C]
    big = [[None] * 3 for _ in range(3)]
    for kind in range(3):
        for wl in range(3):
            a, b, e = big_slice(kind, wl)
            big[kind][wl] = (rnd(p[a:b].reshape(C, TAPS, C)), p[b:e])
    wout = p[OFF_OUT:OFF_OUT + OUT_W].reshape(TAPS, C)
    bout = p[OFF_OUT + OUT_W]
    return win, bin_, big, wout, bout


# ----------------------------------------------------------------- image ops

def shifted(xp, tap):
    """Interior-sized view of the padded image xp shifted by tap (dy, dx) in {-1,0,1}^2."""
    dy, dx = tap // 3, tap % 3
    H, W = xp.shape[0] - 2, xp.shape[1] - 2
    return xp[dy:dy + H, dx:dx + W]


def conv(xp, w, b=None):
    """3x3 convolution of the padded image xp [H+2, W+2, ci] with w [co, tap, ci]: interior [H, W, co]."""
    out = 0.0
    for tap in range(TAPS):
        out = out + shifted(xp, tap) @ w[:, tap, :].T
    if b is not None:
        out = out + b
    return out


def pad(x):
    return np.pad(x, ((1, 1), (1, 1)) + ((0, 0),) * (x.ndim - 2))


def pool(xp):
    """2x2 average of the interior of a padded fine image (the zero border fills odd edges)."""
    H, W = xp.shape[0] - 2, xp.shape[1] - 2
    h, w = (H + 1) // 2, (W + 1) // 2
    q = np.zeros((2 * h + 2, 2 * w + 2) + xp.shape[2:])
    q[:H + 2, :W + 2] = xp
    blk = q[1:2 * h + 1, 1:2 * w + 1]
    return (blk[0::2, 0::2] + blk[0::2, 1::2] + blk[1::2, 0::2] + blk[1::2, 1::2]) * 0.25


def up(cp, H, W):
    """Nearest upsampling of a padded coarse image's interior to H x W."""
    c = cp[1:-1, 1:-1]
    return np.repeat(np.repeat(c, 2, axis=0), 2, axis=1)[:H, :W]


def up_adjoint(d, h, w):
    """Sum of the fine interior gradient d [H, W, ...] over each coarse pixel's children: [h, w, ...]."""
    H, W = d.shape[:2]
    q = np.zeros((2 * h, 2 * w) + d.shape[2:])
    q[:H, :W] = d
    return q[0::2, 0::2] + q[0::2, 1::2] + q[1::2, 0::2] + q[1::2, 1::2]


def depth_of(h, w):
    d = 1
    while min(h, w) >= 16:
        h, w = (h + 1) // 2, (w + 1) // 2
        d += 1
    return d


# ----------------------------------------------------------------- network

def net_forward(params, featp, emulate=True):
    """featp: padded [h+2, w+2, 2] features.  Returns (out [h, w], cache)."""
    rnd = Rounder(emulate)
    win, bin_, big, wout, bout = unpack(params, rnd)
    h0 = rnd(np.maximum(conv(featp, win, bin_), 0.0))
    H, W = featp.shape[0] - 2, featp.shape[1] - 2
    D = depth_of(H, W)
    hs, ps, pins = [pad(h0)], [None], [None]
    for l in range(1, D):
        wl = min(l - 1, 2)
        pin = pad(rnd(pool(hs[l - 1])))
        w, b = big[DOWN][wl]
        p = pad(rnd(np.maximum(conv(pin, w, b), 0.0)))
        w, b = big[ENC][wl]
        hh = pad(rnd(np.maximum(conv(p, w, b), 0.0)))
        hs.append(hh)
        ps.append(p)
        pins.append(pin)
    gs = [None] * D
    uins = [None] * D
    gs[D - 1] = hs[D - 1]
    for l in range(D - 2, -1, -1):
        wl = min(l, 2)
        Hl, Wl = hs[l].shape[0] - 2, hs[l].shape[1] - 2
        # the tensor core sums conv(skip) + conv(up(coarse)): no rounding of the sum
        uin = pad(hs[l][1:-1, 1:-1] + up(gs[l + 1], Hl, Wl))
        w, b = big[DEC][wl]
        gs[l] = pad(rnd(np.maximum(conv(uin, w, b), 0.0)))
        uins[l] = uin
    out = conv(gs[0], wout.reshape(1, TAPS, C))[..., 0] + bout
    cache = dict(featp=featp, hs=hs, ps=ps, pins=pins, gs=gs, uins=uins, D=D)
    return out, cache


def conv_wgrad(dz, xp):
    """dW[co, tap, ci] = sum_p dz[p, co] x[p + tap, ci]; db = sum_p dz."""
    dw = np.stack([np.einsum("hwo,hwi->oi", dz, shifted(xp, tap)) for tap in range(TAPS)], axis=1)
    return dw, dz.sum(axis=(0, 1))


def conv_data(dz, w):
    """Adjoint of conv: dx[p, ci] = sum_tap sum_co dz[p - tap, co] w[co, tap, ci] (interior)."""
    wt = w[:, ::-1, :].transpose(2, 1, 0)  # [ci, 8 - tap, co]
    return conv(pad(dz), wt)


def net_backward(params, cache, dout, emulate=True):
    """Gradient of sum(out * dout) with respect to the parameters (flat float64)."""
    rnd = Rounder(emulate)
    win, bin_, big, wout, bout = unpack(params, rnd)
    grad = np.zeros(NUM_PARAMS)
    hs, ps, pins, gs, uins, D = (cache[k] for k in ("hs", "ps", "pins", "gs", "uins", "D"))
    featp = cache["featp"]
    # output convolution
    dwo, dbo = conv_wgrad(dout[..., None], gs[0])
    grad[OFF_OUT:OFF_OUT + OUT_W] = dwo[0].ravel()
    grad[OFF_OUT + OUT_W] = dbo[0]
    dg = [None] * D
    dh = [np.zeros_like(h[1:-1, 1:-1]) for h in hs]
    dg[0] = conv_data(dout[..., None], wout.reshape(1, TAPS, C))
    for l in range(D - 1):
        dg[l + 1] = np.zeros_like(gs[l + 1][1:-1, 1:-1]) if dg[l + 1] is None else dg[l + 1]
    for l in range(0, D - 1):
        wl = min(l, 2)
        w, b = big[DEC][wl]
        dz = rnd(dg[l] * (gs[l][1:-1, 1:-1] > 0))
        dw, db = conv_wgrad(dz, uins[l])
        a, bb, e = big_slice(DEC, wl)
        grad[a:bb] += dw.ravel()
        grad[bb:e] += db
        dx = conv_data(dz, w)
        dh[l] += dx
        hc, wc = gs[l + 1].shape[0] - 2, gs[l + 1].shape[1] - 2
        dg[l + 1] = dg[l + 1] + up_adjoint(dx, hc, wc)
    dh[D - 1] = dh[D - 1] + (dg[D - 1] if D > 1 else 0.0)
    if D == 1:
        dh[0] = dh[0] + dg[0]
    for l in range(D - 1, 0, -1):
        wl = min(l - 1, 2)
        w, b = big[ENC][wl]
        dz = rnd(dh[l] * (hs[l][1:-1, 1:-1] > 0))
        dw, db = conv_wgrad(dz, ps[l])
        a, bb, e = big_slice(ENC, wl)
        grad[a:bb] += dw.ravel()
        grad[bb:e] += db
        dp = conv_data(dz, w)
        w, b = big[DOWN][wl]
        dz2 = rnd(dp * (ps[l][1:-1, 1:-1] > 0))
        dw, db = conv_wgrad(dz2, pins[l])
        a, bb, e = big_slice(DOWN, wl)
        grad[a:bb] += dw.ravel()
        grad[bb:e] += db
        dpin = conv_data(dz2, w)
        Hf, Wf = hs[l - 1].shape[0] - 2, hs[l - 1].shape[1] - 2
        dh[l - 1] = dh[l - 1] + 0.25 * up(pad(dpin), Hf, Wf)
    dz0 = dh[0] * (hs[0][1:-1, 1:-1] > 0)
    dw, db = conv_wgrad(dz0, featp)
    grad[OFF_IN:OFF_IN + IN_W] = dw.ravel()
    grad[OFF_IN + IN_W:OFF_IN + IN_W + C] = db
    return grad


# ----------------------------------------------------------------- operator and wrapper

def k_apply(a, nu):
    """2D magnetostatics residual operator on [ny, nx] arrays (identity boundary rows)."""
    a = np.asarray(a, dtype=np.float64)
    y = a.copy()
    ny, nx = a.shape
    c = a[1:-1, 1:-1]
    r = np.zeros_like(c)
    # sampled node below (j-1 >= 1), the node itself, left neighbour (i-1 >= 1)
    r[1:, :] += (c[1:, :] - a[1:-2, 1:-1][:, :]) * nu[1:-2, 1:-1]
    r += (c - a[2:, 1:-1]) * nu[1:-1, 1:-1]
    r[:, 1:] += (c[:, 1:] - a[1:-1, 1:-2]) * nu[1:-1, 1:-2]
    r += (c - a[1:-1, 2:]) * nu[1:-1, 1:-1]
    y[1:-1, 1:-1] = r
    return y


def dinv_of(nu):
    ny, nx = nu.shape
    d = np.ones_like(nu)
    dd = 2.0 * nu[1:-1, 1:-1]
    dd[1:, :] += nu[1:-2, 1:-1]
    dd[:, 1:] += nu[1:-1, 1:-2]
    d[1:-1, 1:-1] = dd
    return 1.0 / d


def interior_mask(ny, nx):
    m = np.zeros((ny, nx))
    m[1:-1, 1:-1] = 1.0
    return m


def precond(params, nu, r, emulate=True, keep=False):
    """M(r) for one [ny, nx] sample."""
    nu = np.asarray(nu, dtype=np.float64)
    r = np.asarray(r, dtype=np.float64)
    ny, nx = r.shape
    dinv = dinv_of(nu)
    e1 = OMEGA * dinv * r
    r1 = r - k_apply(e1, nu)
    sq = np.sqrt(dinv)
    s = math.sqrt(np.mean(dinv * r1 * r1))
    inv_s = 1.0 / s if s > 0 else 0.0
    f = np.stack([sq * r1 * inv_s, np.log(nu) / math.log(1000.0)], axis=-1)
    featp = pad(pool(pad(f)))
    out, cache = net_forward(params, featp, emulate)
    v = s * sq * up(pad(out), ny, nx) * interior_mask(ny, nx)
    e2 = e1 + v
    u = e2 + OMEGA * dinv * (r - k_apply(e2, nu))
    if keep:
        return u, dict(cache=cache, s=s, dinv=dinv, featp=featp, out=out)
    return u


def loss_and_grad(params, samples, emulate=True):
    """samples: list of (nu, b, x) [ny, nx] arrays.  Mean loss, per-sample losses, gradient."""
    n = len(samples)
    grad = np.zeros(NUM_PARAMS)
    losses = []
    for nu, b, x in samples:
        nu = np.asarray(nu, dtype=np.float64)
        b = np.asarray(b, dtype=np.float64)
        x = np.asarray(x, dtype=np.float64)
        u, aux = precond(params, nu, b, emulate, keep=True)
        ku = k_apply(u, nu)
        ub, uku, xb = float(np.sum(u * b)), float(np.sum(u * ku)), float(np.sum(x * b))
        losses.append(1.0 - ub * ub / (uku * xb))
        den = uku * uku * xb * n
        gu = (-2.0 * ub * uku / den) * b + (2.0 * ub * ub / den) * ku
        ge2 = gu - OMEGA * k_apply(aux["dinv"] * gu, nu)
        ny, nx = b.shape
        hc, wc = aux["out"].shape
        gnet = aux["s"] * up_adjoint(np.sqrt(aux["dinv"]) * ge2 * interior_mask(ny, nx), hc, wc)
        grad += net_backward(params, aux["cache"], gnet, emulate)
    return float(np.mean(losses)), losses, grad


def init_params(seed):
    """He-normal weights like the GPU initialiser's distribution (not its exact draws)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NUM_PARAMS)
    p[OFF_IN:OFF_IN + IN_W] = rng.normal(0, math.sqrt(2.0 / (TAPS * 2)), IN_W)
    for j in range(9):
        o = OFF_BIG + j * BIG_P
        p[o:o + BIG_W] = rng.normal(0, math.sqrt(2.0 / (TAPS * C)), BIG_W)
        p[o + BIG_W:o + BIG_P] = rng.normal(0, 0.05, C)
    p[OFF_OUT:OFF_OUT + OUT_W] = 0.5 * rng.normal(0, math.sqrt(2.0 / (TAPS * C)), OUT_W)
    p[OFF_IN + IN_W:OFF_IN + IN_W + C] = rng.normal(0, 0.05, C)
    p[OFF_OUT + OUT_W] = 0.01
    return p.astype(np.float32)
