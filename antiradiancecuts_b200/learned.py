"""The learned cut: training data, training and loading of the cut-refinement MLP.

    python -m antiradiancecuts_b200.learned train [--scenes 64] [--samples 20000000] [--out PATH]

Training data come from the exact gather itself: for each training scene (room variants with
seeds 100..163: 0-16 random boxes, random light position and wall albedo) the GPU walks every
8x8 tile's tree with the exact refine/accept decision and records the features, label and error
of every node the analytic bound cannot decide (arc_cut_training_samples).  The network is then
trained on the GPU by the library's own tensor-core forward/backward kernels (arc_mlp_train_step,
Adam, weighted binary cross-entropy).
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
DEFAULT_MODEL = os.path.join(PKG, "models", "cutnet.npy")
NUM_PARAMS = 9473

# training set-up (the learned-cut configuration)
TRAIN_SEEDS = range(100, 164)
TRAIN_W, TRAIN_H, TRAIN_AVPLS = 256, 192, 65536
LABEL_DELTA = 1.5e-4  # refine when the node's true error exceeds this fraction of the tile value
# analytic pre-acceptance shared by labelling and selection: nodes whose error bound is within
# PREACCEPT_EPS of the tile estimate (antiradiance-uncertain nodes weighted by PREACCEPT_K) are
# accepted without the network; the network decides every other node
PREACCEPT_EPS = 1e-3
PREACCEPT_K = 64.0


class Model:
    """An arc_mlp handle with its parameters."""

    def __init__(self, ctx: api.Context, params: np.ndarray | None = None, seed: int = 1):
        self.ctx = ctx
        h = C.c_void_p()
        L.check(ctx.lib.arc_mlp_create(ctx.handle, seed, C.byref(h)), "arc_mlp_create")
        self.handle = h
        ctx._children.add(self)
        if params is not None:
            self.set_params(params)

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


def cut_params(model: Model, threshold: float = 0.5, **kw):
    """ArcCutParams of the learned cut with the pre-acceptance the model was trained with."""
    return api.cut_params(L.ARC_CUT_LEARNED, error_bound=PREACCEPT_EPS, ar_uncertain_factor=PREACCEPT_K,
                          model=model.handle.value, mlp_threshold=threshold, **kw)


def load_default_model(ctx: api.Context, path: str = DEFAULT_MODEL) -> Model:
    if not os.path.exists(path):
        raise FileNotFoundError(f"no trained cut model at {path}")
    return Model(ctx, np.load(path))


def scene_samples(ctx: api.Context, seed: int, capacity: int, width=TRAIN_W, height=TRAIN_H, num_avpls=TRAIN_AVPLS,
                  delta=LABEL_DELTA, error_bound=PREACCEPT_EPS, ar_uncertain=PREACCEPT_K):
    """(features bf16 [k,16], labels [k], errors [k]) torch CUDA tensors for one training scene."""
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
    cut = api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=error_bound, ar_uncertain_factor=ar_uncertain)
    feats = torch.empty((capacity, 16), dtype=torch.bfloat16, device="cuda")
    labels = torch.empty(capacity, dtype=torch.float32, device="cuda")
    errs = torch.empty(capacity, dtype=torch.float32, device="cuda")
    count = C.c_int32()
    cam = (desc.camera_position.x, desc.camera_position.y, desc.camera_position.z)
    gv = gb.view()
    L.check(ctx.lib.arc_cut_training_samples(ctx.handle, bvh.handle, C.byref(gv), L.f3(cam), C.byref(prm), C.byref(cut),
                                             delta, C.c_void_p(feats.data_ptr()), C.c_void_p(labels.data_ptr()),
                                             C.c_void_p(errs.data_ptr()), capacity, C.byref(count)),
            "arc_cut_training_samples")
    word = ctx.synchronize()
    if word:
        raise RuntimeError(f"device error word 0x{word:x} while labelling scene {seed}")
    k = count.value
    bvh.close()
    return feats[:k].clone(), labels[:k].clone(), errs[:k].clone()


def train(ctx: api.Context, feats, labels, epochs: float = 3.0, batch: int = 8192, lr: float = 2e-3,
          pos_weight: float = 2.0, seed: int = 1, log=print) -> Model:
    """Adam on the weighted BCE (refine samples weighted pos_weight) with a cosine learning rate."""
    import torch

    model = Model(ctx, seed=seed)
    n = feats.shape[0]
    steps = max(1, int(epochs * n / batch))
    g = torch.Generator(device="cuda").manual_seed(seed)
    weights = torch.where(labels > 0.5, torch.full_like(labels, pos_weight), torch.ones_like(labels))
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


def evaluate(ctx: api.Context, model: Model, feats, labels):
    import torch

    logits = torch.empty(feats.shape[0], device="cuda")
    model.forward(feats, logits)
    ctx.synchronize()
    pred = logits > 0
    lab = labels > 0.5
    acc = (pred == lab).float().mean().item()
    fn = (~pred & lab).float().sum().item() / max(1.0, lab.float().sum().item())
    fp = (pred & ~lab).float().sum().item() / max(1.0, (~lab).float().sum().item())
    return {"accuracy": acc, "missed_refine_rate": fn, "extra_refine_rate": fp, "rows": int(feats.shape[0]),
            "refine_fraction": lab.float().mean().item()}


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    tr = sub.add_parser("train")
    tr.add_argument("--scenes", type=int, default=64)
    tr.add_argument("--samples", type=int, default=20_000_000)
    tr.add_argument("--epochs", type=float, default=3.0)
    tr.add_argument("--delta", type=float, default=LABEL_DELTA)
    tr.add_argument("--out", default=DEFAULT_MODEL)
    a = ap.parse_args(argv)
    import torch

    ctx = api.Context(0)
    per_scene = max(1, a.samples // a.scenes)
    fs, ls = [], []
    t0 = time.time()
    seeds = list(TRAIN_SEEDS)[: a.scenes]
    for s in seeds:
        f, l, e = scene_samples(ctx, s, capacity=4 * per_scene, delta=a.delta)
        if f.shape[0] > per_scene:  # uniform subsample to the per-scene budget
            keep = torch.randperm(f.shape[0], device="cuda")[:per_scene]
            f, l = f[keep], l[keep]
        fs.append(f)
        ls.append(l)
        print(f"scene {s}: {f.shape[0]} samples, refine fraction {l.mean().item():.3f} ({time.time() - t0:.1f} s)",
              flush=True)
    feats = torch.cat(fs)
    labels = torch.cat(ls)
    # hold out 2% for a validation report
    n = feats.shape[0]
    perm = torch.randperm(n, device="cuda")
    nv = max(1, n // 50)
    val, trn = perm[:nv], perm[nv:]
    model = train(ctx, feats[trn].contiguous(), labels[trn].contiguous(), epochs=a.epochs)
    print("validation:", evaluate(ctx, model, feats[val].contiguous(), labels[val].contiguous()), flush=True)
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    np.save(a.out, model.params())
    print("saved", a.out, f"({time.time() - t0:.1f} s total)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
