"""CPU oracle of the refinement indicator (test infrastructure only).

Nothing in the product imports this file; tests and the benchmark's CPU
baseline use it to test the GPU kernels against.

* ``tag_plain``: the plain geometric criterion, the two loops of the case
  hook ``AMR::TagtheBox`` (Userfunction_cy_naca15.cpp:560-635, rftag in
  Box.H:11-61) over the rule description of ``ibgpu_tag_rule``; pinned
  bit-exactly against the tags the reference itself produced
  (``tests/golden/*tags*``, written by ``oracle/ref_driver.cpp``).
* ``naca_rule``: the rule of the oracle's NACA0012 case
  (``oracle/cases/case_naca.cpp``), as an ``ibgpu_tag_rule``-shaped dict.
* ``features``: the learned indicator's inputs from a primitive-state field.
* ``mlp_forward`` / ``mlp_grad``: the MLP's forward pass and the gradient of
  the class-weighted cross entropy in FP64, rounding to BF16 exactly where
  the tensor-core kernels do (inputs, weights, hidden activations and each
  layer's output gradient); ``rounding=False`` gives the plain FP64 network
  for finite-difference checks.
"""
from __future__ import annotations

import numpy as np

MAXL = 16
N_IN, N_STENCIL, N_HID, N_OUT = 112, 100, 64, 3
P_W1 = 0
P_B1 = P_W1 + N_HID * N_IN
P_W2 = P_B1 + N_HID
P_B2 = P_W2 + N_HID * N_HID
P_W3 = P_B2 + N_HID
P_B3 = P_W3 + N_OUT * N_HID
P_COUNT = P_B3 + N_OUT
TAG_REFINE, TAG_COARSEN = 1, 2
GELU_A = np.float64(np.float32(0.7978845608028654))
GELU_B = np.float64(np.float32(0.044715))


# ---------------------------------------------------------------- plain rule
def empty_rule() -> dict:
    z = lambda: np.zeros(MAXL)  # noqa: E731
    return dict(body_left_x=0.0, body_right_x=0.0, body_center_y=0.0, body_half_height=0.0,
                n_rect=0, n_rect_coarsen=0,
                torefine=np.zeros(MAXL, np.int32), toderefine=np.zeros(MAXL, np.int32),
                rect_up=z(), rect_down=z(), rect_half=z(), band_lo=z(), band_hi=z(),
                near_margin=z(), derect_up=z(), derect_down=z(), derect_half=z(),
                deband_lo=z(), deband_hi=z(), denear_margin=z())


def naca_rule(nlevels: int, dh: np.ndarray, le_x: float = 9.5, le_y: float = 10.0,
              chord: float = 1.0) -> dict:
    """The oracle NACA case's TagtheBox regions (case_naca.cpp, naca_region):
    rectangles up=4s, down=8s, half=4s (s = 0.5^k) for k < nlevels-2, then
    the band -3 dh_k < signdis < max(0.25, 16 dh_finest) inside the body box
    grown by the band's upper limit.  Coarsening of level l uses region(l-1)."""
    r = empty_rule()
    r.update(body_left_x=le_x, body_right_x=le_x + chord, body_center_y=le_y,
             body_half_height=0.5 * chord, n_rect=nlevels - 2, n_rect_coarsen=nlevels - 2)
    re = max(0.25, 16.0 * dh[nlevels - 1])
    for k in range(nlevels):
        s = 0.5 ** k
        for pre in ("", "de"):
            r[pre + "rect_up"][k] = 4.0 * s
            r[pre + "rect_down"][k] = 8.0 * s
            r[pre + "rect_half"][k] = 4.0 * s
            r[pre + "band_lo"][k] = -3.0 * dh[k]
            r[pre + "band_hi"][k] = re
            r[pre + "near_margin"][k] = re
    r["torefine"][:nlevels] = 1
    r["toderefine"][1:nlevels] = 1
    return r


def _region(r: dict, pre: str, nrect: int, k, x, y, sd):
    k = np.asarray(k)
    rect = ((x - r["body_left_x"] > -r[pre + "rect_up"][k]) &
            (x - r["body_right_x"] < r[pre + "rect_down"][k]) &
            (np.abs(y - r["body_center_y"]) < r[pre + "rect_half"][k]))
    m = r[pre + "near_margin"][k]
    near = ((x > r["body_left_x"] - m) & (x < r["body_right_x"] + m) &
            (np.abs(y - r["body_center_y"]) < r["body_half_height"] + m))
    near = np.where(m > 0.0, near, True)
    band = near & (sd > r[pre + "band_lo"][k]) & (sd < r[pre + "band_hi"][k])
    return np.where(k < nrect, rect, band)


def tag_plain(r: dict, level, xc, yc, sd) -> np.ndarray:
    """IBGPU_TAG_REFINE | IBGPU_TAG_COARSEN bits per box."""
    level = np.asarray(level, np.int64)
    out = np.zeros(len(level), np.uint8)
    ref = (r["torefine"][level] != 0) & _region(r, "", r["n_rect"], level, xc, yc, sd)
    lm1 = np.maximum(level - 1, 0)
    co = ((level >= 1) & (r["toderefine"][level] != 0) &
          ~_region(r, "de", r["n_rect_coarsen"], lm1, xc, yc, sd))
    out[ref] |= TAG_REFINE
    out[co] |= TAG_COARSEN
    return out


def tags_from_rftag(tag, detag) -> np.ndarray:
    """rftag (tag, detag) fields (0 = set, -1 = clear) as IBGPU_TAG_* bits."""
    return ((np.asarray(tag) == 0) * TAG_REFINE + (np.asarray(detag) == 0) * TAG_COARSEN).astype(np.uint8)


def classes_from_tags(bits) -> np.ndarray:
    """Learned classes: 0 refine (tag set), 1 coarsen (detag only), 2 keep."""
    bits = np.asarray(bits)
    return np.where(bits & TAG_REFINE, 0, np.where(bits & TAG_COARSEN, 1, 2)).astype(np.uint8)


# ------------------------------------------------------------------- numerics
def bf16_round(x) -> np.ndarray:
    """Round to the nearest BF16 (ties to even) via float32, returned as f64."""
    f = np.asarray(x, np.float64).astype(np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(x) -> np.ndarray:
    return (bf16_round(x).astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)


def bits_to_f64(b) -> np.ndarray:
    return (np.asarray(b, np.uint32) << 16).view(np.float32).astype(np.float64)


def features(state: dict, cells: dict, rule: dict, initvar, gama: float, dh) -> np.ndarray:
    """Feature rows (BF16 bits) of the boxes.  state: dict (level, ix, iy) ->
    (rho, u, v, p) of every box of the mesh; cells: level, ix, iy, xc, yc,
    signdis arrays.  Absent stencil cells take the centre's value."""
    rho_inf, p_inf = float(initvar[0]), float(initvar[4])
    inv_rho, inv_p = 1.0 / rho_inf, 1.0 / p_inf
    inv_c = 1.0 / np.sqrt(gama * p_inf / rho_inf)
    inv_chord = 1.0 / (rule["body_right_x"] - rule["body_left_x"])
    n = len(cells["level"])
    out = np.zeros((n, N_IN), np.float64)
    for i in range(n):
        l, x, y = int(cells["level"][i]), int(cells["ix"][i]), int(cells["iy"][i])
        c = state[(l, x, y)]
        for dy in range(-2, 3):
            for dx in range(-2, 3):
                q = state.get((l, x + dx, y + dy), c)
                k = (dy + 2) * 5 + (dx + 2)
                out[i, k] = np.float32(q[0] * inv_rho - 1.0)
                out[i, 25 + k] = np.float32(q[1] * inv_c)
                out[i, 50 + k] = np.float32(q[2] * inv_c)
                out[i, 75 + k] = np.float32(q[3] * inv_p - 1.0)
        sd = cells["signdis"][i]
        out[i, 100] = min(max(sd / dh[l], -8.0), 8.0) * 0.125
        out[i, 101] = min(max(sd * inv_chord, -4.0), 4.0) * 0.25
        rx = (cells["xc"][i] - rule["body_left_x"]) * inv_chord * 0.125
        ry = (cells["yc"][i] - rule["body_center_y"]) * inv_chord * 0.125
        out[i, 102], out[i, 103], out[i, 104] = rx, ry, abs(ry)
        out[i, 105 + min(l, 6)] = 1.0
    return bf16_bits(out.astype(np.float32).astype(np.float64))


def unpack(P):
    P = np.asarray(P, np.float64)
    W1 = P[P_W1:P_B1].reshape(N_HID, N_IN)
    b1 = P[P_B1:P_W2]
    W2 = P[P_W2:P_B2].reshape(N_HID, N_HID)
    b2 = P[P_B2:P_W3]
    W3 = P[P_W3:P_B3].reshape(N_OUT, N_HID)
    b3 = P[P_B3:P_COUNT]
    return W1, b1, W2, b2, W3, b3


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initial weights, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    P = np.zeros(P_COUNT, np.float32)
    P[P_W1:P_B1] = rng.normal(0, np.sqrt(2.0 / N_IN), N_HID * N_IN)
    P[P_W2:P_B2] = rng.normal(0, np.sqrt(2.0 / N_HID), N_HID * N_HID)
    P[P_W3:P_B3] = rng.normal(0, np.sqrt(1.0 / N_HID), N_OUT * N_HID)
    return P


def _gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GELU_A * (z + GELU_B * z ** 3)))


def _gelu_grad(z):
    th = np.tanh(GELU_A * (z + GELU_B * z ** 3))
    return 0.5 * (1.0 + th) + 0.5 * z * (1.0 - th * th) * GELU_A * (1.0 + 3.0 * GELU_B * z * z)


def mlp_forward(P, X_bits=None, X=None, rounding: bool = True):
    """Logits (n x 3) and the intermediates of the forward pass."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    r = bf16_round if rounding else (lambda a: np.asarray(a, np.float64))
    if X is None:
        X = bits_to_f64(X_bits)
    X = np.asarray(X, np.float64)
    W1r, W2r, W3r = r(W1), r(W2), r(W3)
    f32 = (lambda a: a.astype(np.float32).astype(np.float64)) if rounding else (lambda a: a)
    z1 = X @ W1r.T + f32(b1)
    h1 = r(_gelu(z1))
    z2 = h1 @ W2r.T + f32(b2)
    h2 = r(_gelu(z2))
    z3 = h2 @ W3r.T + f32(b3)
    return z3, dict(X=X, z1=z1, h1=h1, z2=z2, h2=h2, W1=W1r, W2=W2r, W3=W3r)


def mlp_loss_grad(P, labels, class_weight, X_bits=None, X=None, rounding: bool = True):
    """(loss, gradient as a flat P_COUNT array, number correct)."""
    z3, c = mlp_forward(P, X_bits=X_bits, X=X, rounding=rounding)
    r = bf16_round if rounding else (lambda a: np.asarray(a, np.float64))
    n = len(z3)
    y = np.asarray(labels, np.int64)
    valid = (y >= 0) & (y < N_OUT)
    yv = np.where(valid, y, 0)
    w = np.where(valid, np.asarray(class_weight, np.float64)[yv], 0.0) / n
    m = z3.max(axis=1, keepdims=True)
    e = np.exp(z3 - m)
    se = e.sum(axis=1, keepdims=True)
    p = e / se
    lse = (np.log(se) + m)[:, 0]
    loss = float(np.sum(w * (lse - z3[np.arange(n), yv])))
    onehot = np.zeros_like(p)
    onehot[np.arange(n), yv] = 1.0
    dz3 = r(w[:, None] * (p - onehot))
    dh2 = dz3 @ c["W3"]
    dz2 = r(dh2 * _gelu_grad(c["z2"]))
    dh1 = dz2 @ c["W2"]
    dz1 = r(dh1 * _gelu_grad(c["z1"]))
    g = np.zeros(P_COUNT)
    g[P_W1:P_B1] = (dz1.T @ c["X"]).ravel()
    g[P_B1:P_W2] = dz1.sum(axis=0)
    g[P_W2:P_B2] = (dz2.T @ c["h1"]).ravel()
    g[P_B2:P_W3] = dz2.sum(axis=0)
    g[P_W3:P_B3] = (dz3.T @ c["h2"]).ravel()
    g[P_B3:P_COUNT] = dz3.sum(axis=0)
    correct = int(np.sum(valid & (np.argmax(z3, axis=1) == y)))
    return loss, g, correct


def adam(P, g, m, v, step: int, lr: float):
    """One bias-corrected Adam step (beta1 0.9, beta2 0.999, eps 1e-8)."""
    b1, b2, eps = 0.9, 0.999, 1e-8
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return P - lr * mh / (np.sqrt(vh) + eps), m, v
