"""Training of the radiance-predictor network on data from the project's own
delta tracker (the learned part; replaces dataGen.cu and the offline
training that produced NNWeight.cuh).

Per scene configuration (seeded fBm cloud, extinction scale, albedo, g,
light direction) the GPU
  1. samples training points with mr_train_points (MeanFreePathSample),
  2. computes FP64-accumulated multiple-scattering labels with
     mr_train_labels (GetSample over `spp` paths),
  3. draws the inference frames (mr_train_frames) and gathers the 576-value
     descriptors with mr_gather_descriptors,
and the network is trained with mr_trainer_step (hand-written forward /
backward kernels, fp32 master weights, Adam). Device memory comes from torch.

    python -m internship_b200.train --configs 32 --samples 5000000 --spp 4096 --out weights.npy
"""
import argparse
import ctypes as C
import json
import math
import time

import numpy as np

from . import _lib, scenes
from ._lib import check
from .volume import Network, builtin_stencil, xavier_weights


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def scene_configs(n, seed=0, resolutions=(128, 256, 512), alpha_range=(16.0, 256.0), albedo_range=(0.9, 1.0),
                  g_range=(0.7, 0.9)):
    """n seeded scene configurations: cloud resolution cycles through
    `resolutions`; extinction scale, albedo and g uniform in their ranges;
    light direction uniform on the sphere."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(n):
        L = rng.normal(size=3)
        L /= np.linalg.norm(L)
        out.append(dict(res=int(resolutions[c % len(resolutions)]), cloud_seed=int(1000 + c),
                        alpha=float(rng.uniform(*alpha_range)), albedo=float(rng.uniform(*albedo_range)),
                        g=float(rng.uniform(*g_range)), light=[float(x) for x in L]))
    return out


def generate(configs, samples_per_config, spp, max_bounces=512, seed=0, lut_seed=0, stencil=None):
    """Training rows for every configuration: (desc n x 576, aux n x 5,
    label n) as float32 CUDA tensors."""
    import torch
    L_ = _lib.load()
    st = builtin_stencil() if stencil is None else stencil
    net = Network(xavier_weights(1), st)  # the gather needs the stencil only
    descs, auxs, labels = [], [], []
    for ci, cfg in enumerate(configs):
        res = cfg["res"]
        from .volume import VolumeRender
        v = VolumeRender(res)
        dens = torch.empty(res ** 3, device="cuda", dtype=torch.float32)
        scenes.generate_cloud_device(res, cfg["cloud_seed"], dens.data_ptr())
        check(L_.mr_volume_set_data_device(v.handle, _ptr(dens), dens.numel(), None))
        check(L_.mr_volume_update(v.handle, None))
        light = _lib.f3(cfg["light"])
        check(L_.mr_volume_update_tr(v.handle, light, cfg["alpha"], None))
        check(L_.mr_volume_update_hglut(v.handle, cfg["g"], lut_seed, None))
        cap = samples_per_config
        pos = torch.empty(cap, 3, device="cuda")
        dirs = torch.empty(cap, 3, device="cuda")
        n_rays = 2 * cap
        cnt = C.c_int32()
        for _ in range(6):
            check(L_.mr_train_points(v.handle, cfg["alpha"], cfg["g"], seed * 7919 + ci, n_rays, cap, _ptr(pos),
                                     _ptr(dirs), C.byref(cnt), None))
            if cnt.value >= cap:
                break
            n_rays *= 2
        n = cnt.value
        if n == 0:
            v.close()
            continue
        pos, dirs = pos[:n].contiguous(), dirs[:n].contiguous()
        sums = torch.zeros(n, device="cuda", dtype=torch.float64)
        check(L_.mr_train_labels(v.handle, _ptr(pos), _ptr(dirs), n, light, cfg["alpha"], cfg["g"], cfg["albedo"],
                                 max_bounces, spp, seed * 7919 + ci, _ptr(sums), None))
        frames = torch.empty(n, 12, device="cuda")
        check(L_.mr_train_frames(_ptr(dirs), n, light, seed * 7919 + ci, _ptr(frames), None))
        desc = torch.empty(n, 576, device="cuda")
        aux = torch.empty(n, 5, device="cuda")
        a = cfg["albedo"]
        check(L_.mr_gather_descriptors(v.handle, net.handle, _ptr(pos), _ptr(frames), n, cfg["alpha"], cfg["g"],
                                       _lib.f3((a, a, a)), _ptr(desc), _ptr(aux), None))
        torch.cuda.synchronize()
        descs.append(desc)
        auxs.append(aux)
        labels.append((sums / spp).float())
        v.close()
    net.close()
    return torch.cat(descs), torch.cat(auxs), torch.cat(labels)


def initial_weights(seed=1):
    """Starting point for training: Xavier-uniform weights, biases uniform in
    [0, 0.01], and the final 16 -> 1 layer's weights non-negative so that the
    output ReLU starts alive (with a dead output unit no gradient flows)."""
    from .weights import layout
    w = xavier_weights(seed, bias_range=(0.0, 0.01))
    off = 0
    for name, n in layout():
        if name == "LX12W":
            w[off:off + n] = np.abs(w[off:off + n])
        off += n
    return w


class Trainer:
    """fp32 master weights + Adam on the device (mr_trainer_*). precision
    "fp32" runs every layer on the CUDA cores; "bf16" runs the head's GEMMs
    (forward, input and weight gradients) on the tensor cores."""

    def __init__(self, weights, precision="fp32"):
        w = np.ascontiguousarray(weights, np.float32)
        h = C.c_void_p()
        check(_lib.load().mr_trainer_create(w.ctypes.data, w.size, C.byref(h)))
        self.handle = h
        if precision != "fp32":
            check(_lib.load().mr_trainer_set_precision(h, {"bf16": _lib.PREC_BF16}[precision]))

    def step(self, desc, aux, label, lr):
        loss = C.c_float()
        check(_lib.load().mr_trainer_step(self.handle, _ptr(desc), _ptr(aux), _ptr(label), len(label), lr,
                                          C.byref(loss), None))
        return loss.value

    def gradient(self, desc, aux, label):
        g = np.zeros(_lib.WEIGHT_TOTAL, np.float32)
        loss = C.c_float()
        check(_lib.load().mr_trainer_gradient(self.handle, _ptr(desc), _ptr(aux), _ptr(label), len(label),
                                              g.ctypes.data, C.byref(loss), None))
        return g, loss.value

    def weights(self):
        w = np.zeros(_lib.WEIGHT_TOTAL, np.float32)
        check(_lib.load().mr_trainer_weights(self.handle, w.ctypes.data, w.size))
        return w

    def close(self):
        if self.handle:
            _lib.load().mr_trainer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fit(desc, aux, label, weights, epochs, batch, lr, seed=0, log=None, precision="fp32"):
    """Adam over shuffled mini-batches; returns (weights, per-epoch mean
    losses)."""
    import torch
    tr = Trainer(weights, precision)
    n = len(label)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    history = []
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=gen)
        tot, cnt = 0.0, 0
        for b0 in range(0, n - batch + 1 if n >= batch else 1, batch):
            idx = perm[b0:b0 + batch]
            l = tr.step(desc[idx].contiguous(), aux[idx].contiguous(), label[idx].contiguous(), lr)
            tot += l
            cnt += 1
        history.append(tot / max(cnt, 1))
        if log:
            log("epoch %d loss %.5f" % (ep, history[-1]))
    w = tr.weights()
    tr.close()
    return w, history


def predict_x(weights, desc, aux, stencil=None):
    """Network output X (= log(1 + radiance / srp)) through the fp32
    inference kernel."""
    import torch
    net = Network(weights, builtin_stencil() if stencil is None else stencil)
    out = torch.empty(len(desc), 3, device="cuda")
    check(_lib.load().mr_radiance_predict(net.handle, _lib.PREC_FP32, _ptr(desc), _ptr(aux), len(desc), _ptr(out),
                                          None))
    torch.cuda.synchronize()
    net.close()
    srp = aux[:, 2]
    return torch.log1p(out[:, 0] / srp)


def targets(aux, label):
    import torch
    return torch.log1p(torch.clamp(label, min=0) / aux[:, 2])


def run(configs=32, samples=5_000_000, spp=4096, bounces=512, epochs=20, batch=65536, lr=1e-3, holdout=0.05,
        seed=0, log=None, precision="fp32"):
    """The whole learned part: generate the rows, train from initial_weights(1)
    and evaluate on a held-out share. Returns (weights, report); the report
    holds the row count, the held-out RMSE of X = log(1 + L / srp) with the
    trained network and with no network (X = 0: single scattering only), and
    the label / training throughput."""
    import torch
    t0 = time.time()
    cfgs = scene_configs(configs, seed)
    desc, aux, label = generate(cfgs, math.ceil(samples / configs), spp, bounces, seed)
    torch.cuda.synchronize()
    t1 = time.time()
    # one untimed step on a throwaway trainer: the kernels' first launches
    # (module loading, attribute setup) stay out of the training time
    warm = Trainer(initial_weights(1), precision)
    m = min(batch, len(label))
    warm.step(desc[:m].contiguous(), aux[:m].contiguous(), label[:m].contiguous(), lr)
    warm.close()
    torch.cuda.synchronize()
    tw = time.time()
    n = len(label)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    perm = torch.randperm(n, device="cuda", generator=gen)
    nh = max(1, int(n * holdout))
    hold, trn = perm[:nh], perm[nh:]
    w0 = initial_weights(1)
    w, hist = fit(desc[trn], aux[trn], label[trn], w0, epochs, batch, lr, seed, log=log, precision=precision)
    torch.cuda.synchronize()
    t2 = time.time()
    T = targets(aux[hold], label[hold])
    dh, ah = desc[hold].contiguous(), aux[hold].contiguous()
    rmse = float(torch.sqrt(torch.mean((predict_x(w, dh, ah) - T) ** 2)))
    rmse_init = float(torch.sqrt(torch.mean((predict_x(w0, dh, ah) - T) ** 2)))
    rmse0 = float(torch.sqrt(torch.mean(T ** 2)))
    rows_trained = (n - nh) * epochs
    return w, {"rows": n, "configs": configs, "spp": spp, "bounces": bounces, "epochs": epochs, "batch": batch,
               "lr": lr, "precision": precision, "holdout_rmse_log": rmse, "untrained_rmse_log": rmse_init, "no_network_rmse_log": rmse0,
               "generate_s": t1 - t0, "train_s": t2 - tw, "labels_per_s": n / (t1 - t0),
               "label_paths_per_s": n * spp / (t1 - t0), "train_rows_per_s": rows_trained / (t2 - tw),
               "loss_history": hist}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--configs", type=int, default=32)
    ap.add_argument("--samples", type=int, default=5_000_000, help="total training rows")
    ap.add_argument("--spp", type=int, default=4096)
    ap.add_argument("--bounces", type=int, default=512)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--holdout", type=float, default=0.05)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default="mrpnn_trained.npy")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "bf16"],
                    help="bf16: the head's GEMMs on the tensor cores (BF16 operands, FP32 accumulation)")
    args = ap.parse_args()
    w, rep = run(args.configs, args.samples, args.spp, args.bounces, args.epochs, args.batch, args.lr, args.holdout,
                 args.seed, log=print, precision=args.precision)
    np.save(args.out, w)
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
