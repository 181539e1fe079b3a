"""The surrogate of the parameter sweeps: an ensemble of MLP heads (include/sph_mlp.h,
trained and evaluated by the engine's own tensor-core kernels) that maps the six sweep
inputs (sph_ensemble.FEATURES) to the four time-averaged observables of a box
(sph_b200.OBSERVABLES), with the batched solver as the fallback wherever the heads
disagree.

PyTorch only holds device memory here (datasets, batches, outputs); every operation of the
network runs in libsph_b200.so.
"""
import ctypes

import numpy as np

import sph_b200

IN, HID, OUT = 6, 256, 4
PF = ctypes.POINTER(ctypes.c_float)


def _lib():
    L = sph_b200.lib()
    if not getattr(L, "_mlp_bound", False):
        L.sph_mlp_num_params.restype = ctypes.c_int
        L.sph_mlp_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]
        L.sph_mlp_destroy.argtypes = [ctypes.c_void_p]
        L.sph_mlp_destroy.restype = None
        L.sph_mlp_get_params.argtypes = [ctypes.c_void_p, PF]
        L.sph_mlp_set_params.argtypes = [ctypes.c_void_p, PF]
        L.sph_mlp_train_step.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_int, ctypes.c_float, PF]
        L.sph_mlp_gradients.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int, PF, PF]
        L.sph_mlp_predict.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_void_p]
        L.sph_mlp_synchronize.argtypes = [ctypes.c_void_p]
        L._mlp_bound = True
    return L


def _ok(st, what):
    if st != 0:
        raise sph_b200.SphError(st, what)


def _dev(t):
    import torch

    assert t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
    return ctypes.c_void_p(t.data_ptr())


class MLP:
    """`heads` independent networks IN -> 256 -> 256 -> 256 -> OUT (GELU) on the GPU."""

    def __init__(self, heads=5, max_batch=1024, seed=0, device=0):
        L = _lib()
        self.heads, self.max_batch = heads, max_batch
        self.nparams = L.sph_mlp_num_params()
        h = ctypes.c_void_p()
        _ok(L.sph_mlp_create(heads, max_batch, seed, device, ctypes.byref(h)), "sph_mlp_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib().sph_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        p = np.zeros(self.heads * self.nparams, dtype=np.float32)
        _ok(_lib().sph_mlp_get_params(self._h, p.ctypes.data_as(PF)), "get_params")
        return p.reshape(self.heads, self.nparams)

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32).reshape(-1)
        assert p.size == self.heads * self.nparams
        _ok(_lib().sph_mlp_set_params(self._h, p.ctypes.data_as(PF)), "set_params")

    def gradients(self, x, y):
        """(loss per head, gradients heads x nparams) on one batch, no update."""
        g = np.zeros(self.heads * self.nparams, dtype=np.float32)
        loss = np.zeros(self.heads, dtype=np.float32)
        _ok(_lib().sph_mlp_gradients(self._h, _dev(x), _dev(y), x.shape[0], g.ctypes.data_as(PF),
                                     loss.ctypes.data_as(PF)), "gradients")
        return loss, g.reshape(self.heads, self.nparams)

    def train_step(self, x, y, lr=1e-3, want_loss=False):
        loss = np.zeros(self.heads, dtype=np.float32) if want_loss else None
        _ok(_lib().sph_mlp_train_step(self._h, _dev(x), _dev(y), x.shape[0], lr,
                                      loss.ctypes.data_as(PF) if want_loss else None), "train_step")
        return loss

    def synchronize(self):
        _ok(_lib().sph_mlp_synchronize(self._h), "synchronize")

    def predict(self, x):
        """heads x n x OUT outputs (a torch tensor on the GPU); n is padded to 128."""
        import torch

        n = x.shape[0]
        npad = (n + 127) // 128 * 128
        if npad != n:
            x = torch.cat([x, torch.zeros(npad - n, IN, device=x.device, dtype=x.dtype)])
        out = torch.empty(self.heads, npad, OUT, device=x.device, dtype=torch.float32)
        _ok(_lib().sph_mlp_predict(self._h, _dev(x.contiguous()), npad, _dev(out)), "predict")
        return out[:, :n]


class Normalizer:
    """Feature / target scaling: log10 of the log-uniform inputs, then zero mean and unit
    variance per column (statistics of the training set)."""

    LOG_FEATURES = (0, 1)  # Weissenberg number, omega tau

    def __init__(self, X, Y):
        Xl = self._log(X)
        self.xm, self.xs = Xl.mean(0), Xl.std(0) + 1e-12
        self.ym, self.ys = Y.mean(0), Y.std(0) + 1e-30

    def _log(self, X):
        X = np.array(X, dtype=np.float64, copy=True)
        for k in self.LOG_FEATURES:
            X[:, k] = np.log10(X[:, k])
        return X

    def x(self, X):
        return ((self._log(X) - self.xm) / self.xs).astype(np.float32)

    def y(self, Y):
        return ((np.asarray(Y, dtype=np.float64) - self.ym) / self.ys).astype(np.float32)

    def y_inv(self, Yn):
        return np.asarray(Yn, dtype=np.float64) * self.ys + self.ym


class Surrogate:
    """Heads trained on (features, observables) of solved sweep points; `route` sends the
    points on which the heads' wall-shear-stress predictions spread by more than `tol`
    (relative to their mean) back to the solver."""

    def __init__(self, heads=5, seed=0, batch=1024, device=0):
        self.mlp = MLP(heads=heads, max_batch=batch, seed=seed, device=device)
        self.batch = batch
        self.device = device
        self.norm = None

    def fit(self, X, Y, steps=3000, lr=1e-3, seed=0, log_every=0):
        import torch

        self.norm = Normalizer(X, Y)
        dev = "cuda:%d" % self.device
        Xn = torch.tensor(self.norm.x(X), device=dev)
        Yn = torch.tensor(self.norm.y(Y), device=dev)
        g = torch.Generator(device=dev).manual_seed(seed)
        n = Xn.shape[0]
        history = []
        for s in range(steps):
            idx = torch.randint(0, n, (self.batch,), device=dev, generator=g)
            xb, yb = Xn[idx].contiguous(), Yn[idx].contiguous()
            want = log_every and (s % log_every == 0 or s == steps - 1)
            loss = self.mlp.train_step(xb, yb, lr, want_loss=bool(want))
            if want:
                history.append((s, loss.tolist()))
        self.mlp.synchronize()
        return history

    def predict_heads(self, X):
        import torch

        xn = torch.tensor(self.norm.x(X), device="cuda:%d" % self.device)
        out = self.mlp.predict(xn).cpu().numpy()
        return np.stack([self.norm.y_inv(out[h]) for h in range(out.shape[0])])

    def predict(self, X, tol=0.02, target=0):
        """(mean over heads, mask of points to re-solve)."""
        P = self.predict_heads(X)
        mean = P.mean(0)
        spread = P[:, :, target].max(0) - P[:, :, target].min(0)
        scale = np.maximum(np.abs(mean[:, target]), 1e-12)
        return mean, spread / scale > tol


# ---- sweeps: the solver as data source and fallback ----

def solve_points(points, nsteps, precision="mixed", device=0, batch=512, observe_every=20,
                 warm_frac=0.25):
    """Observables (n x 4) of sweep points from the batched solver, `batch` boxes per
    context; the averages skip the first warm_frac of the steps.  Returns (Y, seconds of
    context creation + stepping)."""
    import os
    import tempfile
    import time

    import sph_ensemble

    Y = np.zeros((len(points), OUT))
    secs = 0.0
    for c0 in range(0, len(points), batch):
        chunk = points[c0:c0 + batch]
        with tempfile.TemporaryDirectory() as wd:
            paths, _ = sph_ensemble.write_inputs(chunk, os.path.join(wd, "in"), nsteps=nsteps)
            t0 = time.perf_counter()
            s = sph_b200.System(paths, precision=precision, device=device)
            obs, _ = sph_ensemble.run_sweep(s, nsteps, observe_every,
                                            warm=int(warm_frac * nsteps))
            s.close()
            secs += time.perf_counter() - t0
        Y[c0:c0 + len(chunk)] = obs
    return Y, secs


def features_of(points):
    import sph_ensemble

    return np.stack([sph_ensemble.features(p, sph_ensemble.box_spec(p)) for p in points])


def relative_error(pred, true):
    """Wall-stress error measure: mean |pred - true| over mean |true| (normalised MAE)."""
    return float(np.mean(np.abs(pred - true)) / max(np.mean(np.abs(true)), 1e-300))
