"""ORACLE — test infrastructure only.  Imported by tests/ alone.

CPU restatement of the learned surrogate (no reference counterpart: ph_brush
has no surrogate, so these functions restate the engine's own definitions):

* `descriptor(...)`: the rows of one move -- per changed particle, 16 radial
  shells of width 0.5 sigma to 8 sigma x 4 classes (+1, -1, neutral
  titratable, permanent +1) of the environment (changed particles excluded):
  exact particle distances in the 27 cells around the descriptor centre,
  class counts binned by cell-centre distance for the other cells of the
  8-sigma cell range; then z / height, the one-hot state, pKa - pH and
  log10(salt).  Every float operation is float32 and rounded once, so the
  rows must match the engine's bit for bit.
* `forward / loss_grad`: the MLP n_in -> H -> H -> H -> 1 with GELU.  With
  `bf16=True` the weights, the standardised inputs, the hidden activations and
  the back-propagated pre-activation gradients are rounded to BF16 where the
  GPU kernels round them; sums are FP64 (the GPU's are FP32).  With
  `bf16=False` everything is FP64: the exact gradient that finite differences
  pin.
* `adam_step`: Adam (Kingma & Ba 2015), beta 0.9 / 0.999, eps 1e-8.
"""
import math

import numpy as np
from scipy.special import erf

from ph_brush_b200 import _abi

SHELLS, CLASSES, RMAX = 16, 4, 8.0
K_IN, ROWS = _abi.SUR_INPUTS, _abi.SUR_ROWS
f32 = np.float32


# ---------------------------------------------------------------------------
# descriptor
# ---------------------------------------------------------------------------
def desc_class(flags, q):
    """Class of present particles: 0 (+1: charged site, cation), 1 (-1), 2 (neutral
    titratable site), 3 (permanent +1); -1 none."""
    flags = np.asarray(flags)
    q = np.asarray(q, np.float32)
    c = np.full(flags.shape, -1, np.int32)
    titr = (flags & _abi.F_TITRATABLE) != 0
    c[titr & (q != 0)] = 0
    c[titr & (q == 0)] = 2
    nt = ~titr
    c[nt & (q < 0)] = 1
    c[nt & (q > 0) & ((flags & _abi.F_CATION) != 0)] = 0
    c[nt & (q > 0) & ((flags & _abi.F_CATION) == 0)] = 3
    c[(flags & _abi.F_GHOST) != 0] = -1
    return c


def row_state(titr, q):
    if titr:
        return 0 if q != 0 else 1
    return 2 if q < 0 else (3 if q > 0 else -1)


class Geometry:
    """Cell grid of one replica as the engine builds it (cells >= the largest cutoff)."""

    def __init__(self, box, dims, params):
        self.L = np.asarray(box, np.float32)
        self.n = np.asarray(dims, np.int64)
        self.scale = np.float32(self.n.astype(np.float32) / self.L)  # float(ncell) / L
        self.w = (self.L / self.n.astype(np.float32)).astype(np.float32)
        r = np.maximum(1, np.ceil(RMAX * self.n / np.asarray(box, np.float64)).astype(np.int64))
        self.dnk = np.minimum(2 * r + 1, self.n)
        # a window over the whole axis is centred: it holds -1, 0, +1 and every other cell once
        self.dnr = np.where(self.dnk < 2 * r + 1, (self.dnk - 1) // 2, r)
        walls = params.wall_hi > params.wall_lo
        self.z0 = f32(params.wall_lo) if walls else f32(0.0)
        self.h = f32(f32(params.wall_hi) - f32(params.wall_lo)) if walls else self.L[2]
        self.pk = f32(params.pKa - params.pH)
        self.salt = f32(math.log10(params.salt_conc)) if params.salt_conc > 0 else f32(-10.0)

    def cell3(self, x, y, z):
        c = []
        for k, v in enumerate((x, y, z)):
            i = (np.asarray(v, np.float32) * self.scale[k]).astype(np.int64)  # truncation, v >= 0
            c.append(np.clip(i, 0, self.n[k] - 1))
        return c

    def flat(self, cx, cy, cz):
        return (cz * self.n[1] + cy) * self.n[0] + cx


def min_image(d, L):
    d = np.asarray(d, np.float32)
    return (d - f32(L) * np.rint(d / f32(L)).astype(np.float32)).astype(np.float32)


def shell(dx, dy, dz):
    r2 = (dx * dx + dy * dy) + dz * dz  # float32, one rounding per operation
    return (np.sqrt(r2.astype(np.float32)) * f32(2.0)).astype(np.int64)


def descriptor(state, geo, changes):
    """Rows (ROWS x K_IN float32), signs and row count of one move.

    state: dict x, y, z, q (float32), flags (int) of every slot.
    changes: list of (slot, present_new, (x, y, z, q)) in the move's order.
    """
    x, y, z, q, fl = (state[k] for k in ("x", "y", "z", "q", "flags"))
    present = (fl & _abi.F_GHOST) == 0
    cls = desc_class(fl, q)
    cx, cy, cz = geo.cell3(x, y, z)
    cell = np.where(present, geo.flat(cx, cy, cz), -1)
    ncell = int(np.prod(geo.n))
    counts = np.zeros((ncell, CLASSES), np.int64)
    ok = present & (cls >= 0)
    np.add.at(counts, (cell[ok], cls[ok]), 1)
    changed = np.zeros(len(x), bool)
    for (i, _, _) in changes:
        changed[i] = True
    rows = np.zeros((ROWS, K_IN), np.float32)
    signs = np.zeros(ROWS, np.float32)
    nr = 0
    for (i, pres_new, pn) in changes:
        pres_old = bool(present[i])
        p = np.asarray(pn if pres_new else (x[i], y[i], z[i], q[i]), np.float32)
        hist = np.zeros((SHELLS, CLASSES), np.int64)
        c0 = [int(c[0]) for c in geo.cell3(p[0:1], p[1:2], p[2:3])]
        # cell range of the sphere
        offs = [np.arange(geo.dnk[k]) - geo.dnr[k] for k in range(3)]
        ox, oy, oz = np.meshgrid(offs[0], offs[1], offs[2], indexing="ij")
        ox, oy, oz = ox.ravel(), oy.ravel(), oz.ravel()
        ccx, ccy, ccz = (c0[0] + ox) % geo.n[0], (c0[1] + oy) % geo.n[1], (c0[2] + oz) % geo.n[2]
        cid = geo.flat(ccx, ccy, ccz)
        inner = (np.abs(ox) <= 1) & (np.abs(oy) <= 1) & (np.abs(oz) <= 1)
        # outer cells: class counts minus the changed particles' current classes
        oc = counts[cid[~inner]].copy()
        for (j, _, _) in changes:
            if present[j] and cls[j] >= 0:
                oc[cid[~inner] == cell[j], cls[j]] -= 1
        xc = ((ccx[~inner].astype(np.float32) + f32(0.5)) * geo.w[0]).astype(np.float32)
        yc = ((ccy[~inner].astype(np.float32) + f32(0.5)) * geo.w[1]).astype(np.float32)
        zc = ((ccz[~inner].astype(np.float32) + f32(0.5)) * geo.w[2]).astype(np.float32)
        sh = shell(min_image(xc - p[0], geo.L[0]), min_image(yc - p[1], geo.L[1]), min_image(zc - p[2], geo.L[2]))
        m = sh < SHELLS
        for c in range(CLASSES):
            np.add.at(hist[:, c], sh[m], oc[m, c])
        # inner cells: particles, exact shells
        inner_cells = set(int(v) for v in cid[inner])
        sel = ok & ~changed & np.isin(cell, list(inner_cells))
        idx = np.nonzero(sel)[0]
        sh = shell(min_image(x[idx] - p[0], geo.L[0]), min_image(y[idx] - p[1], geo.L[1]),
                   min_image(z[idx] - p[2], geo.L[2]))
        m = sh < SHELLS
        np.add.at(hist, (sh[m], cls[idx][m]), 1)
        titr = pres_old and bool(fl[i] & _abi.F_TITRATABLE)
        zf = np.float32((p[2] - geo.z0) / geo.h)
        states = []
        if pres_old:
            states.append((row_state(titr, float(q[i])), -1.0))
        if pres_new:
            states.append((row_state(titr, float(pn[3])), 1.0))
        for st, sg in states:
            r = rows[nr]
            r[:64] = hist.reshape(-1)
            r[64] = zf
            if st >= 0:
                r[65 + st] = 1.0
            r[69] = geo.pk
            r[70] = geo.salt
            signs[nr] = sg
            nr += 1
    return rows, signs, nr


# ---------------------------------------------------------------------------
# network
# ---------------------------------------------------------------------------
def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def unpack(p, nin, H):
    p = np.asarray(p)
    if p.dtype != np.float64:
        p = p.astype(np.float32)
    o = 0
    out = []
    for shape in ((nin, H), (H,), (H, H), (H,), (H, H), (H,), (H,), (1,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def forward(p, nin, H, mu, sd, x, bf=True):
    """Per-row outputs y (standardised units) and the activations."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p, nin, H)
    rnd = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    X = ((np.asarray(x, np.float32) - np.asarray(mu, np.float32)) / np.asarray(sd, np.float32)).astype(np.float32)
    X = rnd(X).astype(np.float64)
    acts = [X]
    Zs = []
    h = X
    for W, b in ((W1, b1), (W2, b2), (W3, b3)):
        Z = h @ rnd(W).astype(np.float64) + b.astype(np.float64)
        Zs.append(Z)
        h = rnd(gelu(Z).astype(np.float32) if bf else gelu(Z)).astype(np.float64)
        acts.append(h)
    y = h @ rnd(w4).astype(np.float64) + float(b4[0])
    return y, acts, Zs


def loss_grad(p, nin, H, mu, sd, scale, x, sign, t, clip, bf=True):
    """Loss 1/2 mean((sum_r sign_r y_r - clip(t)/scale)^2) and its flat gradient."""
    n = len(t)
    xr = np.asarray(x, np.float32).reshape(n * ROWS, nin)
    sg = np.asarray(sign, np.float64).reshape(n, ROWS)
    y, acts, Zs = forward(p, nin, H, mu, sd, xr, bf)
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p, nin, H)
    rnd = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    pred = (sg * y.reshape(n, ROWS)).sum(1)
    tt = np.clip(np.asarray(t, np.float64), -clip, clip) / scale
    d = pred - tt
    loss = 0.5 * np.mean(d * d)
    dy = (sg * (d / n)[:, None]).reshape(-1)
    H3 = acts[3]
    g_w4 = H3.T @ dy
    g_b4 = np.array([dy.sum()])
    w4r = rnd(w4).astype(np.float64)
    dZ = dy[:, None] * w4r[None, :] * gelu_grad(Zs[2])
    dZ = rnd(dZ.astype(np.float32) if bf else dZ).astype(np.float64)
    grads = {}
    Ws = [W1, W2, W3]
    for layer in (2, 1, 0):
        grads[layer] = (acts[layer].T @ dZ, dZ.sum(0))
        if layer > 0:
            back = dZ @ rnd(Ws[layer]).astype(np.float64).T
            dZ = back * gelu_grad(Zs[layer - 1])
            dZ = rnd(dZ.astype(np.float32) if bf else dZ).astype(np.float64)
    flat = np.concatenate([grads[0][0].ravel(), grads[0][1], grads[1][0].ravel(), grads[1][1],
                           grads[2][0].ravel(), grads[2][1], g_w4, g_b4])
    return loss, flat


def adam_step(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
