"""The learned cut: training data, training and loading of the cut-refinement MLP.

    python -m antiradiancecuts_b200.learned train [--scenes 64] [--samples 20000000] [--out PATH]

Training data come from the exact gather itself: for each training scene (room variants with
seeds 100..163: 0-16 random boxes, random light position and wall albedo) rendered at the
evaluation scale (1920x1080 G-buffer, 1,048,576 AVPLs), the GPU walks the trees of the 8x8 tiles in
a few seeded 64x64-pixel windows with the exact refine/accept decision and records the features,
label and error of every node the selection would score (arc_cut_training_samples).  The network
is then trained on the GPU by the library's own tensor-core forward/backward kernels
(arc_mlp_train_step, Adam) as a classifier of the 0/1 labels (weighted binary cross-entropy); the
selection refines a node when the predicted probability reaches the threshold.  A regression of
log2 of each node's exact relative error (squared loss; refine when the predicted error reaches
the threshold) is the alternative objective.
"""
from __future__ import annotations

import argparse
import ctypes as C
import math
import os
import sys
import time

import numpy as np

from . import _lib as L
from . import api, scene

PKG = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(PKG, "models", "cutnet.npz")
NUM_PARAMS = 9473

# training set-up (the learned-cut configuration)
TRAIN_SEEDS = range(100, 164)
TRAIN_W, TRAIN_H, TRAIN_AVPLS = 1920, 1080, 1 << 20
TRAIN_CROPS, TRAIN_CROP = 16, 32  # windows per scene and their size in pixels
LABEL_DELTA = 1e-4  # label: refine when the node's true error exceeds this fraction of the tile value
LOG2_FLOOR = -30.0  # regression targets: log2 of the relative error, at least this
# analytic pre-acceptance shared by labelling and selection: nodes whose error bound is within
# PREACCEPT_EPS of the tile estimate (antiradiance-uncertain nodes weighted by PREACCEPT_K) are
# accepted, nodes whose bound exceeds PREACCEPT_BAND times that are refined, both without the
# network; the network decides the nodes in between (it prunes refinements of the analytic cut)
PREACCEPT_EPS = 2e-3
PREACCEPT_K = 16.0
PREACCEPT_BAND = 64.0


class Model:
    """An arc_mlp handle with its parameters, its loss (L.ARC_MLP_LOSS_*) and the selection
    threshold recommended for it (probability for a classifier, relative error for a regressor)."""

    def __init__(self, ctx: api.Context, params: np.ndarray | None = None, seed: int = 1,
                 loss: int = L.ARC_MLP_LOSS_BCE, threshold: float | None = None, band: float = PREACCEPT_BAND):
        self.ctx = ctx
        h = C.c_void_p()
        L.check(ctx.lib.arc_mlp_create(ctx.handle, seed, C.byref(h)), "arc_mlp_create")
        self.handle = h
        ctx._children.add(self)
        L.check(ctx.lib.arc_mlp_set_loss(h, int(loss)), "arc_mlp_set_loss")
        self.loss = int(loss)
        self.threshold = threshold if threshold is not None else (0.5 if loss == L.ARC_MLP_LOSS_BCE else 1e-4)
        self.band = float(band)  # the analytic refine band the network was trained within
        if params is not None:
            self.set_params(params)

    def save(self, path: str) -> None:
        np.savez(path, params=self.params(), loss=np.int32(self.loss), threshold=np.float32(self.threshold),
                 band=np.float32(self.band))

    @classmethod
    def load(cls, ctx: api.Context, path: str) -> "Model":
        z = np.load(path)
        return cls(ctx, z["params"], loss=int(z["loss"]), threshold=float(z["threshold"]),
                   band=float(z["band"]) if "band" in z else PREACCEPT_BAND)

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        L.check(self.ctx.lib.arc_mlp_set_params(self.handle, p.ctypes.data_as(C.POINTER(C.c_float)), len(p)), "set")

    def params(self) -> np.ndarray:
        p = np.zeros(NUM_PARAMS, np.float32)
        L.check(self.ctx.lib.arc_mlp_get_params(self.handle, p.ctypes.data_as(C.POINTER(C.c_float)), NUM_PARAMS), "get")
        return p

    def forward(self, feats, logits) -> None:
        L.check(self.ctx.lib.arc_mlp_forward(self.handle, C.c_void_p(feats.data_ptr()), feats.shape[0],
                                             C.c_void_p(logits.data_ptr())), "arc_mlp_forward")

    def close(self):
        if self.handle and self.ctx.handle:
            self.ctx.lib.arc_mlp_destroy(self.handle)
        self.handle = None


def cut_params(model: Model, threshold: float | None = None, **kw):
    """ArcCutParams of the learned cut with the pre-acceptance the model was trained with."""
    kw.setdefault("mlp_band", model.band)
    return api.cut_params(L.ARC_CUT_LEARNED, error_bound=PREACCEPT_EPS, ar_uncertain_factor=PREACCEPT_K,
                          model=model.handle.value,
                          mlp_threshold=model.threshold if threshold is None else threshold, **kw)


def load_default_model(ctx: api.Context, path: str = DEFAULT_MODEL) -> Model:
    if not os.path.exists(path):
        raise FileNotFoundError(f"no trained cut model at {path}")
    return Model.load(ctx, path)


def scene_samples(ctx: api.Context, seed: int, capacity: int, width=TRAIN_W, height=TRAIN_H, num_avpls=TRAIN_AVPLS,
                  delta=LABEL_DELTA, error_bound=PREACCEPT_EPS, ar_uncertain=PREACCEPT_K, band=PREACCEPT_BAND,
                  crops=TRAIN_CROPS, crop=TRAIN_CROP):
    """(features bf16 [k,16], labels [k], errors [k]) torch CUDA tensors for one training scene: the
    tiles of `crops` seeded crop x crop windows of the width x height G-buffer (crops=0: all of it)."""
    import torch

    desc = scene.scene_desc(L.ARC_SCENE_TRAIN_VARIANT, seed)
    avpls, _ = scene.trace_avpls(desc, seed, num_avpls, 3)
    pos, nrm = scene.gbuffer(desc, width, height)
    mats, _, _, _ = scene.materials(desc)
    ctx.upload_materials(mats)
    dv = ctx.upload_avpls(avpls)
    bvh = api.AvplBvh(ctx)
    bvh.build(dv)
    gb = api.GBuffer(pos, nrm)
    prm = api.gather_params(L.ARC_AR_CONE, 30.0, 0.01)
    cut = api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=error_bound, ar_uncertain_factor=ar_uncertain,
                         mlp_band=band)
    feats = torch.empty((capacity, 16), dtype=torch.bfloat16, device="cuda")
    labels = torch.empty(capacity, dtype=torch.float32, device="cuda")
    errs = torch.empty(capacity, dtype=torch.float32, device="cuda")
    cam = (desc.camera_position.x, desc.camera_position.y, desc.camera_position.z)
    full = gb.view()
    if crops:
        rng = np.random.default_rng(seed)
        # windows on the 8-pixel tile grid, inside the image
        xs = rng.integers(0, (width - crop) // 8 + 1, crops) * 8
        ys = rng.integers(0, (height - crop) // 8 + 1, crops) * 8
        views = [L.ArcGBufferView(full.position + 16 * (int(y) * width + int(x)), full.normal + 16 * (int(y) * width + int(x)),
                                  crop, crop, width) for x, y in zip(xs, ys)]
    else:
        views = [full]
    k = 0
    for gv in views:
        count = C.c_int32()
        o = k
        L.check(ctx.lib.arc_cut_training_samples(ctx.handle, bvh.handle, C.byref(gv), L.f3(cam), C.byref(prm),
                                                 C.byref(cut), delta, C.c_void_p(feats[o:].data_ptr()),
                                                 C.c_void_p(labels[o:].data_ptr()), C.c_void_p(errs[o:].data_ptr()),
                                                 None, capacity - o, C.byref(count)), "arc_cut_training_samples")
        word = ctx.synchronize()
        if word:
            raise RuntimeError(f"device error word 0x{word:x} while labelling scene {seed}")
        k = min(capacity, o + count.value)
        if k >= capacity:
            break
    bvh.close()
    return feats[:k].clone(), labels[:k].clone(), errs[:k].clone()


def train(ctx: api.Context, feats, labels, epochs: float = 3.0, batch: int = 8192, lr: float = 2e-3,
          pos_weight: float = 2.0, seed: int = 1, log=print, loss: int = L.ARC_MLP_LOSS_BCE) -> Model:
    """Adam with a cosine learning rate on the weighted BCE of 0/1 labels (refine samples weighted
    pos_weight), or on the squared error of real-valued labels."""
    import torch

    model = Model(ctx, seed=seed, loss=loss)
    n = feats.shape[0]
    steps = max(1, int(epochs * n / batch))
    g = torch.Generator(device="cuda").manual_seed(seed)
    if loss == L.ARC_MLP_LOSS_BCE:
        weights = torch.where(labels > 0.5, torch.full_like(labels, pos_weight), torch.ones_like(labels))
    else:
        weights = torch.ones_like(labels)
    loss_acc = torch.zeros(1, device="cuda")
    t0 = time.time()
    perm = torch.randperm(n, device="cuda", generator=g)
    pi = 0
    for step in range(steps):
        if pi + batch > n:
            perm = torch.randperm(n, device="cuda", generator=g)
            pi = 0
        idx = perm[pi:pi + batch]
        pi += batch
        xb = feats[idx].contiguous()
        yb = labels[idx].contiguous()
        wb = weights[idx].contiguous()
        cur_lr = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))
        L.check(ctx.lib.arc_mlp_train_step(model.handle, C.c_void_p(xb.data_ptr()), C.c_void_p(yb.data_ptr()),
                                           C.c_void_p(wb.data_ptr()), batch, float(wb.sum().item()), cur_lr,
                                           C.c_void_p(loss_acc.data_ptr())), "arc_mlp_train_step")
        if (step + 1) % max(1, steps // 10) == 0:
            l = loss_acc.item() / max(1, steps // 10)
            loss_acc.zero_()
            log(f"  step {step + 1}/{steps} loss {l:.4f} ({time.time() - t0:.1f} s)")
    return model


def evaluate(ctx: api.Context, model: Model, feats, labels, delta: float = LABEL_DELTA):
    """Decision quality on held-out rows: for a regressor, `labels` are log2 relative errors and
    the decision is "error >= delta"; also the regression's RMS error in log2 units."""
    import torch

    logits = torch.empty(feats.shape[0], device="cuda")
    model.forward(feats, logits)
    ctx.synchronize()
    extra = {}
    if model.loss == L.ARC_MLP_LOSS_SQUARED:
        t = math.log2(delta)
        pred, lab = logits >= t, labels >= t
        extra["rms_log2"] = float(torch.sqrt(torch.mean((logits - labels) ** 2)).item())
    else:
        pred, lab = logits > 0, labels > 0.5
    acc = (pred == lab).float().mean().item()
    fn = (~pred & lab).float().sum().item() / max(1.0, lab.float().sum().item())
    fp = (pred & ~lab).float().sum().item() / max(1.0, (~lab).float().sum().item())
    return {"accuracy": acc, "missed_refine_rate": fn, "extra_refine_rate": fp, "rows": int(feats.shape[0]),
            "refine_fraction": lab.float().mean().item(), **extra}


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    tr = sub.add_parser("train")
    tr.add_argument("--scenes", type=int, default=64)
    tr.add_argument("--samples", type=int, default=20_000_000)
    tr.add_argument("--epochs", type=float, default=4.0)
    tr.add_argument("--delta", type=float, default=LABEL_DELTA)
    tr.add_argument("--objective", choices=["regression", "classification"], default="classification")
    tr.add_argument("--band", type=float, default=PREACCEPT_BAND)
    tr.add_argument("--threshold", type=float, default=None, help="selection threshold stored with the model")
    tr.add_argument("--out", default=DEFAULT_MODEL)
    a = ap.parse_args(argv)
    import torch

    ctx = api.Context(0)
    regress = a.objective == "regression"
    per_scene = max(1, a.samples // a.scenes)
    fs, ls = [], []
    t0 = time.time()
    seeds = list(TRAIN_SEEDS)[: a.scenes]
    for s in seeds:
        f, l, e = scene_samples(ctx, s, capacity=24 * per_scene, delta=a.delta, band=a.band)
        if regress:
            l = torch.log2(torch.clamp(e, min=2.0 ** LOG2_FLOOR))
        if f.shape[0] > per_scene:  # uniform subsample to the per-scene budget
            keep = torch.randperm(f.shape[0], device="cuda")[:per_scene]
            f, l = f[keep], l[keep]
        fs.append(f)
        ls.append(l)
        stat = f"mean log2 error {l.mean().item():.2f}" if regress else f"refine fraction {l.mean().item():.3f}"
        print(f"scene {s}: {f.shape[0]} samples, {stat} ({time.time() - t0:.1f} s)", flush=True)
    feats = torch.cat(fs)
    labels = torch.cat(ls)
    # hold out 2% for a validation report
    n = feats.shape[0]
    perm = torch.randperm(n, device="cuda")
    nv = max(1, n // 50)
    val, trn = perm[:nv], perm[nv:]
    loss = L.ARC_MLP_LOSS_SQUARED if regress else L.ARC_MLP_LOSS_BCE
    model = train(ctx, feats[trn].contiguous(), labels[trn].contiguous(), epochs=a.epochs, loss=loss)
    model.band = a.band
    # the shipped classifier refines at P(refine) >= 0.05: within 1% RMSE on the held-out scene
    model.threshold = a.threshold if a.threshold is not None else (0.05 if not regress else 1e-4)
    print("validation:", evaluate(ctx, model, feats[val].contiguous(), labels[val].contiguous(), a.delta), flush=True)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    model.save(a.out)
    print("saved", a.out, f"({time.time() - t0:.1f} s total)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
