"""Learned AMR refinement indicator (replaces the per-box decision of the case
hook AMR::TagtheBox, Userfunction_cy_naca15.cpp:533-650).

The plain criterion stays the label source and the fallback: ``tag_plain``
runs it on the GPU; ``LearnedIndicator`` trains the MLP of
``ibgpu_mlp_*`` (BF16 tensor-core forward/backward, FP32 accumulation, Adam)
on its tags and deploys it through ``ibgpu_tag_learned``.  ``Regridder``
applies the deployment policy: the learned decision on ordinary regrids, the
plain criterion on every ``judge_every``-th regrid, which also measures the
mismatch.  Device memory comes from torch (allocation only); every kernel is
the CUDA library's.
"""
from __future__ import annotations

import numpy as np

from . import ibgpu

CLASS_REFINE, CLASS_COARSEN, CLASS_KEEP = 0, 1, 2


def classes_from_tags(bits: np.ndarray) -> np.ndarray:
    """Plain-criterion tag bits -> classes (refine wins over coarsen)."""
    bits = np.asarray(bits)
    return np.where(bits & ibgpu.TAG_REFINE, CLASS_REFINE,
                    np.where(bits & ibgpu.TAG_COARSEN, CLASS_COARSEN, CLASS_KEEP)).astype(np.uint8)


def tags_from_classes(cls: np.ndarray) -> np.ndarray:
    cls = np.asarray(cls)
    return np.where(cls == CLASS_REFINE, ibgpu.TAG_REFINE,
                    np.where(cls == CLASS_COARSEN, ibgpu.TAG_COARSEN, 0)).astype(np.uint8)


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases (float32, ibgpu_mlp parameter layout)."""
    H, I, O = ibgpu.MLP_HIDDEN, ibgpu.MLP_IN, ibgpu.MLP_CLASSES
    rng = np.random.default_rng(seed)
    P = np.zeros(ibgpu.MLP_PARAMS, np.float32)
    o = 0
    P[o:o + H * I] = rng.normal(0.0, np.sqrt(2.0 / I), H * I)
    o += H * I + H
    P[o:o + H * H] = rng.normal(0.0, np.sqrt(2.0 / H), H * H)
    o += H * H + H
    P[o:o + O * H] = rng.normal(0.0, np.sqrt(1.0 / H), O * H)
    return P


def balanced_weights(labels: np.ndarray, power: float = 0.5) -> np.ndarray:
    """Class weights (n / (3 n_c))^power, 0 for absent classes."""
    counts = np.bincount(np.asarray(labels, np.int64), minlength=3)[:3].astype(np.float64)
    n = counts.sum()
    w = np.where(counts > 0, (n / (3.0 * np.maximum(counts, 1))) ** power, 0.0)
    return w.astype(np.float32)


class LearnedIndicator:
    """MLP parameters and Adam state on the solver's device."""

    def __init__(self, solver: "ibgpu.FlowSolver", seed: int = 0, params: np.ndarray | None = None):
        import torch
        self.torch = torch
        self.solver = solver
        dev = torch.device("cuda")
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        self.params = torch.from_numpy(p.copy()).to(dev)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.stats = torch.zeros(2, dtype=torch.float32, device=dev)
        self.step = 0

    # ---------------------------------------------------------------- data
    def features(self, rule: dict, boxes: dict):
        """Device feature rows (int16 tensor holding BF16 bits, n x 112) of
        boxes = dict(level, ix, iy, xc, yc, signdis) from the solver's state."""
        n = len(boxes["level"])
        feat = self.torch.empty((max(n, 1), ibgpu.MLP_IN), dtype=self.torch.int16, device="cuda")
        self.solver.indicator_features(rule, boxes["level"], boxes["ix"], boxes["iy"], boxes["xc"],
                                       boxes["yc"], boxes["signdis"], feat.data_ptr())
        return feat[:n]

    # ------------------------------------------------------------- training
    def train(self, feat, labels: np.ndarray, steps: int, batch: int = 8192, lr: float = 3e-3,
              class_weight=None, seed: int = 0) -> list:
        """Adam on minibatches of a once-shuffled copy of the rows; returns the
        per-step (loss, accuracy) history."""
        torch = self.torch
        n = feat.shape[0]
        labels = np.asarray(labels, np.uint8)
        cw = balanced_weights(labels) if class_weight is None else np.asarray(class_weight, np.float32)
        perm = np.random.default_rng(seed).permutation(n)
        X = feat[torch.from_numpy(perm).to(feat.device)].contiguous()
        Y = torch.from_numpy(labels[perm].copy()).to(feat.device)
        hist = []
        b = min(batch, n)
        off = 0
        for _ in range(steps):
            if off + b > n:
                off = 0
            self.stats.zero_()
            self.step += 1
            self.solver.mlp_train_step(self.params.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                                       self.grad.data_ptr(), self.step, lr, b,
                                       X[off:].data_ptr(), Y[off:].data_ptr(), cw,
                                       self.stats.data_ptr())
            s = self.stats.cpu().numpy()
            hist.append((float(s[0]), float(s[1]) / b))
            off += b
        return hist

    def gradient(self, feat, labels: np.ndarray, class_weight) -> tuple:
        """(loss, gradient, correct) of the rows at the current parameters."""
        torch = self.torch
        Y = torch.from_numpy(np.asarray(labels, np.uint8).copy()).to(feat.device)
        g = torch.zeros_like(self.params)
        st = torch.zeros(2, dtype=torch.float32, device=feat.device)
        self.solver.mlp_grad(self.params.data_ptr(), feat.shape[0], feat.data_ptr(), Y.data_ptr(),
                             class_weight, g.data_ptr(), st.data_ptr())
        s = st.cpu().numpy()
        return float(s[0]), g.cpu().numpy(), int(round(float(s[1])))

    # ------------------------------------------------------------ inference
    def predict(self, feat, logits: bool = False):
        torch = self.torch
        n = feat.shape[0]
        cls = torch.empty(max(n, 1), dtype=torch.uint8, device=feat.device)
        lg = torch.empty((max(n, 1), 3), dtype=torch.float32, device=feat.device) if logits else None
        self.solver.mlp_forward(self.params.data_ptr(), n, feat.data_ptr(), cls.data_ptr(),
                                lg.data_ptr() if logits else 0)
        out = cls[:n].cpu().numpy()
        return (out, lg[:n].cpu().numpy()) if logits else out

    def tags(self, rule: dict, boxes: dict) -> np.ndarray:
        """IBGPU_TAG_* bits of the boxes from the learned decision."""
        return self.solver.tag_learned(rule, boxes["level"], boxes["ix"], boxes["iy"], boxes["xc"],
                                       boxes["yc"], boxes["signdis"], self.params.data_ptr())


class Regridder:
    """Deployment policy: the learned indicator decides the ordinary regrids
    and the plain criterion re-judges every ``judge_every``-th one (its tags
    are then the ones used), recording the mismatch of the learned decision."""

    def __init__(self, indicator: LearnedIndicator, rule: dict, judge_every: int = 10):
        self.ind = indicator
        self.rule = rule
        self.judge_every = judge_every
        self.count = 0
        self.mismatch = []  # (regrid index, fraction of boxes whose decision differs)

    def tags(self, boxes: dict) -> np.ndarray:
        k = self.count
        self.count += 1
        if self.judge_every > 0 and k % self.judge_every == 0:
            plain = self.ind.solver.tag_plain(self.rule, boxes["level"], boxes["xc"], boxes["yc"],
                                              boxes["signdis"], boxes["ix"], boxes["iy"])
            learned = self.ind.tags(self.rule, boxes)
            diff = classes_from_tags(plain) != classes_from_tags(learned)
            self.mismatch.append((k, float(diff.mean()) if len(diff) else 0.0))
            return plain
        return self.ind.tags(self.rule, boxes)
