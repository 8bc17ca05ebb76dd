"""The learned BDF predictor: network binding, training data and training.

The network (include/zerork_b200_predictor.h, csrc/mlp.cu) maps one
reactor's state and step to the state one step later:

  inputs  log10(max(Y_k, 1e-30)) for every species, (T - 1500 K) / 1000 K,
          log10(P / 1 bar), log10(h / 1 s)
  targets log10(max(Y'_k, 1e-30)) - log10(max(Y_k, 1e-30)), (T' - T) / 100 K

both standardised per column with the training set's mean and standard
deviation.  Training pairs come from the integrator itself: reactors from
seeded initial states are advanced through the cfd_plugin API by intervals
drawn log-uniformly, and every (state, interval, next state) is a sample.
The network is trained on the GPU by the library's own forward, backward and
Adam kernels.
"""
import ctypes as C

import numpy as np

from . import check, lib

_bound = False
YMIN = 1e-30


def _lib():
    global _bound
    L = lib()
    if not _bound:
        vp, i, f = C.c_void_p, C.c_int, C.c_float
        L.zrk_mlp_create.argtypes = [i, i, i, i, C.c_ulonglong, C.POINTER(vp)]
        L.zrk_mlp_free.argtypes = [vp]
        L.zrk_mlp_sizes.argtypes = [vp, C.POINTER(C.c_long), C.POINTER(C.c_long)]
        L.zrk_mlp_get_params.argtypes = [vp, vp, vp]
        L.zrk_mlp_set_params.argtypes = [vp, vp, vp]
        L.zrk_mlp_get_grads.argtypes = [vp, vp, vp]
        L.zrk_mlp_forward.argtypes = [vp, i, vp, vp, vp]
        L.zrk_mlp_gradients.argtypes = [vp, i, vp, vp, vp, vp]
        L.zrk_mlp_adam.argtypes = [vp, f, f, f, f, vp]
        _bound = True
    return L


class Mlp:
    """n_in -> layers x hidden (SiLU) -> n_out on the current CUDA device."""

    def __init__(self, n_in, n_out, hidden=256, layers=3, seed=0):
        self.L = _lib()
        h = C.c_void_p()
        check(self.L.zrk_mlp_create(n_in, hidden, layers, n_out, seed, C.byref(h)))
        self.h = h
        self.n_in, self.n_out, self.hidden, self.layers = n_in, n_out, hidden, layers
        nw, nb = C.c_long(), C.c_long()
        check(self.L.zrk_mlp_sizes(self.h, C.byref(nw), C.byref(nb)))
        self.nw, self.nb = nw.value, nb.value

    def close(self):
        if getattr(self, "h", None):
            self.L.zrk_mlp_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        w, b = np.zeros(self.nw, np.float32), np.zeros(self.nb, np.float32)
        check(self.L.zrk_mlp_get_params(self.h, w.ctypes.data, b.ctypes.data))
        return w, b

    def set_params(self, w, b):
        w = np.ascontiguousarray(w, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        check(self.L.zrk_mlp_set_params(self.h, w.ctypes.data, b.ctypes.data))

    def grads(self):
        w, b = np.zeros(self.nw, np.float32), np.zeros(self.nb, np.float32)
        check(self.L.zrk_mlp_get_grads(self.h, w.ctypes.data, b.ctypes.data))
        return w, b

    def forward(self, x, y=None, stream=None):
        """x: float32 CUDA tensor [n, n_in]; returns y [n, n_out]."""
        import torch
        if y is None:
            y = torch.empty((x.shape[0], self.n_out), dtype=torch.float32, device=x.device)
        check(self.L.zrk_mlp_forward(self.h, x.shape[0], x.data_ptr(), y.data_ptr(), stream))
        return y

    def gradients(self, x, t, loss_dev, stream=None):
        check(self.L.zrk_mlp_gradients(self.h, x.shape[0], x.data_ptr(), t.data_ptr(),
                                       loss_dev.data_ptr(), stream))

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        check(self.L.zrk_mlp_adam(self.h, lr, beta1, beta2, eps, stream))


def features(T, P, Y, h):
    """Raw network inputs [n, nsp + 3] (float64) for states and steps."""
    ly = np.log10(np.maximum(Y, YMIN))
    return np.concatenate([ly, ((T - 1500.0) / 1000.0)[:, None], np.log10(P / 1e5)[:, None],
                           np.log10(h)[:, None]], axis=1)


def targets(T, Y, T2, Y2):
    """Raw network targets [n, nsp + 1]."""
    d = np.log10(np.maximum(Y2, YMIN)) - np.log10(np.maximum(Y, YMIN))
    return np.concatenate([d, ((T2 - T) / 100.0)[:, None]], axis=1)


def generate_pairs(mech, therm, T0, P0, Y0, rounds, dt_range=(1e-10, 1e-4), seed=0, **plugin_opts):
    """Advance the reactors (T0, P0, Y0) through the cfd_plugin API for
    `rounds` intervals drawn log-uniformly from dt_range (one draw per round
    for all reactors); returns raw (features, targets) of every successful
    (state, interval, next state) pair."""
    from .plugin import Plugin
    rng = np.random.default_rng(seed)
    p = Plugin(mech, therm, **plugin_opts)
    n = T0.shape[0]
    cost = p.set_aux_field("COST", np.zeros(n))
    T, P, Y = T0.copy(), P0.copy(), np.ascontiguousarray(Y0.copy())
    xs, ts = [], []
    for _ in range(rounds):
        dt = float(np.exp(rng.uniform(np.log(dt_range[0]), np.log(dt_range[1]))))
        T1, P1, Y1 = T.copy(), P.copy(), Y.copy()
        p.solve(dt, T1, P1, Y1, raise_on_fail=False)
        ok = cost >= 0
        xs.append(features(T[ok], P[ok], Y[ok], np.full(ok.sum(), dt)))
        ts.append(targets(T[ok], Y[ok], T1[ok], Y1[ok]))
        T[ok], P[ok], Y[ok] = T1[ok], P1[ok], Y1[ok]
    p.close()
    return np.concatenate(xs), np.concatenate(ts)


class Standardizer:
    def __init__(self, a):
        self.mu = a.mean(axis=0)
        self.sd = np.maximum(a.std(axis=0), 1e-6)

    def fwd(self, a):
        return (a - self.mu) / self.sd

    def inv(self, a):
        return a * self.sd + self.mu


def train(x_raw, t_raw, hidden=256, layers=3, epochs=4, batch=4096, lr=1e-3, seed=0, device="cuda"):
    """Train a network on raw pairs; returns (net, x_scaler, t_scaler,
    per-epoch mean losses)."""
    import torch
    xs, ts = Standardizer(x_raw), Standardizer(t_raw)
    X = torch.from_numpy(xs.fwd(x_raw).astype(np.float32)).to(device)
    Tt = torch.from_numpy(ts.fwd(t_raw).astype(np.float32)).to(device)
    net = Mlp(X.shape[1], Tt.shape[1], hidden, layers, seed)
    loss = torch.zeros(1, dtype=torch.float32, device=device)
    g = torch.Generator(device="cpu").manual_seed(seed)
    n = X.shape[0] // batch * batch
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(X.shape[0], generator=g)[:n].to(device)
        tot = 0.0
        for i in range(0, n, batch):
            idx = perm[i:i + batch]
            xb, tb = X[idx].contiguous(), Tt[idx].contiguous()
            net.gradients(xb, tb, loss)
            net.adam(lr)
            tot += float(loss.item())
        hist.append(tot / (n * Tt.shape[1]))
    return net, xs, ts, hist
