"""Learned warm start for the DFSPH constant-density loop (host side).

The network and its training run in libsphgpu.so (sph_mlp.cu: BF16
tensor-core forward/backward kernels, Adam on FP32 master weights).  This
module wraps the handle and holds the training recipe:

  1. record (features, converged stiffness) pairs from plain DFSPH runs of the
     same kind of scene with different jitter seeds (sphgpu_attach_warm_start
     mode 2);
  2. normalise features and labels (mean / std from the recorded set);
  3. train with Adam (lr 1e-3, 20 epochs by default) on the GPU;
  4. attach to a scene in mode 1: every step predicts the stiffness, applies it
     once, and the unmodified Jacobi loop runs to the same tolerance.

Parameter layout: W1[16][64] b1[64] W2[64][64] b2[64] W3[64] b3 (FP32).
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import SphGpuError

NPARAM = _lib.MLP_NPARAM
NIN = _lib.MLP_IN


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class WarmStartNet:
    def __init__(self, device=0, dataset_cap=4_000_000, seed=0):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.sphgpu_mlp_create(int(device), int(dataset_cap), int(seed), C.byref(h))
        if rc:
            raise SphGpuError(rc, "sphgpu_mlp_create")
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.sphgpu_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what):
        if rc < 0:
            raise SphGpuError(rc, what)
        return rc

    # parameters
    def params(self):
        out = np.zeros(NPARAM, np.float32)
        self._chk(self.lib.sphgpu_mlp_get_params(self.h, _fp(out)), "get_params")
        return out

    def set_params(self, w):
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == NPARAM
        self._chk(self.lib.sphgpu_mlp_set_params(self.h, _fp(w)), "set_params")

    def norm(self):
        out = np.zeros(2 * NIN + 2, np.float32)
        self._chk(self.lib.sphgpu_mlp_get_norm(self.h, _fp(out)), "get_norm")
        return out

    def set_norm(self, nrm):
        nrm = np.ascontiguousarray(nrm, np.float32)
        self._chk(self.lib.sphgpu_mlp_set_norm(self.h, _fp(nrm)), "set_norm")

    # dataset
    def dataset_size(self):
        return self._chk(self.lib.sphgpu_mlp_dataset_size(self.h), "dataset_size")

    def set_dataset(self, X, y):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        self._chk(self.lib.sphgpu_mlp_dataset_set(self.h, _fp(X), _fp(y), len(y)), "dataset_set")

    def dataset(self, max_n=None):
        n = self.dataset_size() if max_n is None else min(max_n, self.dataset_size())
        X = np.zeros((max(n, 1), NIN), np.float32)
        y = np.zeros(max(n, 1), np.float32)
        m = self._chk(self.lib.sphgpu_mlp_dataset_get(self.h, _fp(X), _fp(y), n), "dataset_get")
        return X[:m], y[:m]

    def clear_dataset(self):
        self.set_dataset(np.zeros((0, NIN), np.float32), np.zeros(0, np.float32))

    def shuffle(self, seed=0):
        self._chk(self.lib.sphgpu_mlp_dataset_shuffle(self.h, int(seed)), "shuffle")

    def fit_normalisation(self, sample=200_000):
        """Feature / label mean and 1/std from (a sample of) the dataset."""
        X, y = self.dataset(sample)
        mu = X.mean(0)
        sd = X.std(0)
        inv = np.where(sd > 1e-6, 1.0 / np.maximum(sd, 1e-6), 1.0)
        mu = np.where(sd > 1e-6, mu, 0.0)  # constant inputs pass through
        ym, ys = float(y.mean()), float(y.std())
        nrm = np.concatenate([mu, inv, [ym, 1.0 / max(ys, 1e-6)]]).astype(np.float32)
        self.set_norm(nrm)
        return nrm

    def train(self, epochs=20, batch=8192, lr=1e-3):
        loss = np.zeros(max(epochs, 1), np.float32)
        self._chk(self.lib.sphgpu_mlp_train(self.h, int(epochs), int(batch), float(lr), _fp(loss)), "train")
        return loss[:epochs]

    def gradient(self, X, y):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(NPARAM, np.float32)
        loss = np.zeros(1, np.float32)
        self._chk(self.lib.sphgpu_mlp_gradient(self.h, _fp(X), _fp(y), len(y), _fp(g), _fp(loss)), "gradient")
        return g, float(loss[0])

    def predict(self, X):
        X = np.ascontiguousarray(X, np.float32)
        y = np.zeros(max(len(X), 1), np.float32)
        self._chk(self.lib.sphgpu_mlp_predict(self.h, _fp(X), _fp(y), len(X)), "predict")
        return y[:len(X)]

    # persistence
    def save(self, path):
        np.savez(path, params=self.params(), norm=self.norm())

    def load(self, path):
        z = np.load(path)
        self.set_params(z["params"])
        self.set_norm(z["norm"])


def attach(scene, net, mode, record_every=10):
    """mode 0 detach, 1 warm start, 2 record training data."""
    lib = _lib.load()
    rc = lib.sphgpu_attach_warm_start(scene.h, net.h if net is not None else None, int(mode), int(record_every))
    if rc:
        raise SphGpuError(rc, "attach_warm_start")


def record(scene, net, steps, every=10):
    """Run `steps` plain DFSPH steps on `scene`, appending (features, label)
    of every `every`-th particle per step to the network's dataset."""
    attach(scene, net, 2, every)
    try:
        st = scene.step("dfsph", steps)
    finally:
        attach(scene, None, 0)
    return st


def train_for_scenes(make_scene, seeds, settle, record_steps, every, epochs=20, lr=1e-3, batch=8192, device=0,
                     dataset_cap=4_000_000, **solver_kw):
    """Record from plain runs of make_scene(seed) for each seed, then train."""
    from .sph import scene_to_gpu
    net = WarmStartNet(device=device, dataset_cap=dataset_cap, seed=1234)
    for sd in seeds:
        sc = make_scene(sd)
        g = scene_to_gpu(sc, device=device, **solver_kw)
        if settle:
            g.step("dfsph", settle)
        record(g, net, record_steps, every)
        g.close()
    net.shuffle(7)
    net.fit_normalisation()
    losses = net.train(epochs=epochs, batch=batch, lr=lr)
    return net, losses
