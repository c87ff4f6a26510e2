"""The learned schedule's network on the GPU (``bfm_mlp_*`` in
include/pscbfm_b200.h): in -> 128 -> 128 -> out with ReLU, products on the
tcgen05 tensor cores (bf16 operands, fp32 accumulators in tensor memory),
fp32 masters and Adam; training runs many steps per launch."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native


class MLP:
    def __init__(self, n_in: int = 6, n_hidden: int = 128, n_out: int = 4, seed: int = 0, gpu: int = 0):
        self._lib = _native.lib()
        h = ctypes.c_void_p()
        st = self._lib.bfm_mlp_create(int(gpu), int(n_in), int(n_hidden), int(n_out), int(seed), ctypes.byref(h))
        if st != _native.BFM_OK:
            raise (ValueError if st == _native.BFM_EINVAL else RuntimeError)(f"bfm_mlp_create failed with status {st}")
        self._h = h
        self.shape = (int(n_in), int(n_hidden), int(n_out))
        n = ctypes.c_size_t()
        self._check(self._lib.bfm_mlp_num_params(self._h, ctypes.byref(n)))
        self.n_params = n.value

    def _check(self, st):
        if st == _native.BFM_OK:
            return
        msg = (self._lib.bfm_mlp_last_error(self._h) or b"").decode()
        raise (ValueError if st == _native.BFM_EINVAL else RuntimeError)(f"status {st}: {msg}")

    @staticmethod
    def _f32(a, cols=None):
        a = np.ascontiguousarray(a, dtype=np.float32)
        if cols is not None and (a.ndim != 2 or a.shape[1] != cols):
            raise ValueError(f"expected an array of shape (batch, {cols})")
        return a

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        self._check(self._lib.bfm_mlp_get_params(self._h, out.ctypes.data, out.size))
        return out

    def set_params(self, p):
        p = self._f32(p).ravel()
        self._check(self._lib.bfm_mlp_set_params(self._h, p.ctypes.data, p.size))

    def forward(self, x) -> np.ndarray:
        x = self._f32(x, self.shape[0])
        y = np.empty((x.shape[0], self.shape[2]), np.float32)
        self._check(self._lib.bfm_mlp_forward(self._h, x.ctypes.data, x.shape[0], y.ctypes.data))
        return y

    def gradients(self, x, t, w=None):
        x, t = self._f32(x, self.shape[0]), self._f32(t, self.shape[2])
        wv = None if w is None else self._f32(w)
        g = np.empty(self.n_params, np.float32)
        loss = ctypes.c_float()
        self._check(self._lib.bfm_mlp_gradients(self._h, x.ctypes.data, t.ctypes.data, None if wv is None else wv.ctypes.data,
                                                x.shape[0], g.ctypes.data, g.size, ctypes.byref(loss)))
        return loss.value, g

    def train_step(self, x, t, w=None, lr: float = 1e-3) -> float:
        x, t = self._f32(x, self.shape[0]), self._f32(t, self.shape[2])
        wv = None if w is None else self._f32(w)
        loss = ctypes.c_float()
        self._check(self._lib.bfm_mlp_train_step(self._h, x.ctypes.data, t.ctypes.data, None if wv is None else wv.ctypes.data,
                                                 x.shape[0], float(lr), ctypes.byref(loss)))
        return loss.value

    def train_steps(self, x, t, row_index, step_rows, w=None, lr: float = 1e-3) -> np.ndarray:
        """Adam steps in one launch: step s uses the next step_rows[s] rows of
        row_index; returns the loss of every step (before its update)"""
        x, t = self._f32(x, self.shape[0]), self._f32(t, self.shape[2])
        idx = np.ascontiguousarray(row_index, dtype=np.uint32)
        rows = np.ascontiguousarray(step_rows, dtype=np.uint32)
        if int(rows.sum()) != idx.size:
            raise ValueError("step_rows must add up to the length of row_index")
        wv = None if w is None else self._f32(w)
        losses = np.empty(rows.size, np.float32)
        self._check(self._lib.bfm_mlp_train_steps(self._h, x.ctypes.data, t.ctypes.data, None if wv is None else wv.ctypes.data,
                                                  x.shape[0], idx.ctypes.data, rows.ctypes.data, rows.size, float(lr),
                                                  losses.ctypes.data))
        return losses

    def last_ms(self) -> float:
        ms = ctypes.c_double()
        self._check(self._lib.bfm_mlp_last_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def fit(self, x, t, w=None, epochs: int = 200, batch: int = 256, lr: float = 1e-3, seed: int = 0):
        """mini-batch Adam over shuffled data, every epoch's steps in one
        launch; returns the loss per epoch"""
        x, t = self._f32(x, self.shape[0]), self._f32(t, self.shape[2])
        rng = np.random.default_rng(seed)
        n = len(x)
        idx = np.concatenate([rng.permutation(n) for _ in range(epochs)]).astype(np.uint32)
        per = [min(batch, n - b0) for b0 in range(0, n, batch)]
        losses = self.train_steps(x, t, idx, per * epochs, w, lr)
        wts = np.array(per * epochs, np.float64).reshape(epochs, len(per))
        return list((losses.reshape(epochs, len(per)) * wts).sum(1) / n)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bfm_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def main(argv=None):
    """time training steps of the schedule network on a synthetic batch"""
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description="train-step timing of the schedule network")
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--hidden", type=int, default=128)
    ap.add_argument("--steps", type=int, default=50)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(0)
    x = rng.normal(size=(a.batch, 6)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]), x[:, 1] * x[:, 2], np.cos(x[:, 3]), x[:, 4] - x[:, 5]], 1).astype(np.float32)
    m = MLP(6, a.hidden, 4, seed=1)
    first = m.train_step(x, t, lr=1e-3)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        last = m.train_step(x, t, lr=1e-3)
    dt = (time.perf_counter() - t0) / a.steps
    one_ms = m.last_ms()
    # the same steps in one launch
    idx = np.tile(np.arange(a.batch, dtype=np.uint32), a.steps)
    losses = m.train_steps(x, t, idx, [a.batch] * a.steps, lr=1e-3)
    fused_ms = m.last_ms() / a.steps
    flops = 3 * 2 * a.batch * (6 * a.hidden + a.hidden * a.hidden + a.hidden * 4)
    print(json.dumps({"batch": a.batch, "hidden": a.hidden, "ms_per_step_host": dt * 1e3, "ms_one_step_launch": one_ms,
                      "ms_per_step_fused": fused_ms, "loss_first": first, "loss_last": float(losses[-1]),
                      "tflops_per_s_fused": flops / (fused_ms / 1e3) / 1e12}))


if __name__ == "__main__":
    main()
