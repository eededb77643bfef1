"""Learned warm start of the saturation adjustment (C4).

A 4 -> 64 -> 64 -> 1 tanh network (canoe_mlp_* in the C ABI) maps a cell's
(density, specific internal energy, total H2O, total NH3) to the temperature
the plain Newton saturation adjustment converges to, as a correction to
the all-vapour temperature T_vapour = e / cv(all water as vapour) (the
latent heating, 0 for cells that stay unsaturated).  Training pairs come
from the plain solver itself on perturbed states of the moist LES column;
training runs on the GPU with the library's own forward / backward and Adam
kernels.  The network never changes the answer: the saturation adjustment
still iterates to its tolerance from the better of the cold start and the
guess, with the bracketed fallback unchanged; the gated start uses the
guess only where it predicts more than 0.05 K of latent heating, so cells
that stay unsaturated keep the cold start that is exact in one step.

The NH3 input is 0 for the H2O-only thermodynamics of the LES
configuration; the channel is kept so the same network shape serves an
H2O + NH3 atmosphere.
"""
import ctypes

import numpy as np

from . import problems, thermo
from ._abi import SatOpts, check, load

NPARAMS = 64 * 4 + 64 + 64 * 64 + 64 + 64 + 1


def _dev(a, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


class WarmStartNet:
    """The warm-start network (device parameters + normalisation)."""

    def __init__(self, seed=1234):
        self.lib = load()
        h = ctypes.c_void_p()
        check(self.lib.canoe_mlp_create(seed, ctypes.byref(h)), "canoe_mlp_create")
        self.h = h

    def close(self):
        if self.h:
            self.lib.canoe_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # parameters --------------------------------------------------------
    def params(self):
        p = np.zeros(NPARAMS, dtype=np.float32)
        check(self.lib.canoe_mlp_get_params(self.h, p.ctypes.data), "get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == NPARAMS
        check(self.lib.canoe_mlp_set_params(self.h, p.ctypes.data), "set_params")

    def set_normalization(self, in_mean, in_std, out_mean, out_std):
        a = np.ascontiguousarray(in_mean, dtype=np.float32)
        b = np.ascontiguousarray(in_std, dtype=np.float32)
        check(self.lib.canoe_mlp_set_normalization(self.h, a.ctypes.data, b.ctypes.data,
                                                   float(out_mean), float(out_std)))

    def normalization(self):
        a = np.zeros(4, dtype=np.float32)
        b = np.zeros(4, dtype=np.float32)
        om, os_ = ctypes.c_float(), ctypes.c_float()
        check(self.lib.canoe_mlp_get_normalization(self.h, a.ctypes.data, b.ctypes.data,
                                                   ctypes.byref(om), ctypes.byref(os_)))
        return a, b, om.value, os_.value

    def save(self, path):
        a, b, om, os_ = self.normalization()
        np.savez(path, params=self.params(), in_mean=a, in_std=b, out_mean=om, out_std=os_)

    @classmethod
    def load(cls, path):
        d = np.load(path)
        net = cls()
        net.set_params(d["params"])
        net.set_normalization(d["in_mean"], d["in_std"], float(d["out_mean"]),
                              float(d["out_std"]))
        return net

    # compute -------------------------------------------------------------
    def loss_grad(self, xn, yn):
        """MSE of normalised data and its gradient (device FP32 kernels)."""
        import torch
        dx, dy = _dev(xn, np.float32), _dev(yn, np.float32)
        g = torch.zeros(NPARAMS, dtype=torch.float32, device="cuda")
        loss = ctypes.c_float()
        torch.cuda.synchronize()
        check(self.lib.canoe_mlp_loss_grad(self.h, dx.data_ptr(), dy.data_ptr(), len(yn),
                                           g.data_ptr(), ctypes.byref(loss), None))
        return loss.value, g.cpu().numpy()

    def forward(self, xn, tensor_core=True):
        import torch
        dx = _dev(xn, np.float32)
        y = torch.zeros(len(xn), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        check(self.lib.canoe_mlp_forward(self.h, dx.data_ptr(), y.data_ptr(), len(xn),
                                         1 if tensor_core else 0, None))
        torch.cuda.synchronize()
        return y.cpu().numpy()

    def fit(self, x, T, th, epochs=20, batch=8192, lr=3e-3, lr_final=1e-4, seed=0, log=None):
        """Normalise (x, T - T_vapour), then Adam on the GPU; returns the
        final loss."""
        import torch
        x = np.asarray(x, dtype=np.float64)
        T = np.asarray(T, dtype=np.float64) - t_vapour(th, x)
        in_mean = x.mean(axis=0)
        in_std = x.std(axis=0)
        in_std[in_std == 0] = 1.0
        out_mean, out_std = T.mean(), T.std()
        self.set_normalization(in_mean, in_std, out_mean, out_std)
        xn = torch.from_numpy(((x - in_mean) / in_std).astype(np.float32)).cuda()
        yn = torch.from_numpy(((T - out_mean) / out_std).astype(np.float32)).cuda()
        n = len(T)
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        nb = max(1, n // batch)
        total = epochs * nb
        loss = ctypes.c_float()
        step = 0
        for ep in range(epochs):
            perm = torch.randperm(n, device="cuda", generator=gen)
            for b in range(nb):
                idx = perm[b * batch:(b + 1) * batch]
                xb = xn[idx].contiguous()
                yb = yn[idx].contiguous()
                cur = lr * (lr_final / lr) ** (step / max(1, total - 1))
                want = (b == nb - 1)
                check(self.lib.canoe_mlp_loss_grad(self.h, xb.data_ptr(), yb.data_ptr(),
                                                   len(idx), None,
                                                   ctypes.byref(loss) if want else None,
                                                   None))
                check(self.lib.canoe_mlp_adam_step(self.h, cur, 0.9, 0.999, 1e-8, None))
                step += 1
            if log:
                log(f"epoch {ep}: loss {loss.value:.3e}")
        torch.cuda.synchronize()
        return loss.value


def perturbed_states(th, n, seed, dT=10.0, dq=0.2, zmax=16.0e3):
    """n seeded cells of the LES column: temperature +-dT, total water
    x (1 +- dq), all water as vapour (so the adjustment has work to do);
    returns conserved cells (NV, n)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    zl = np.linspace(0.0, zmax, 257)[1:] - zmax / 512
    T0, p0, q0 = problems.moist_profile(th, zl)
    lev = rng.integers(0, len(zl), n)
    T = T0[lev] + rng.uniform(-dT, dT, n)
    p = p0[lev]
    qt = q0[lev] * (1.0 + rng.uniform(-dq, dq, n))
    ny = th.ny
    w = np.zeros((5 + ny, n))
    w[1] = qt
    feps = thermo.feps_of(th, w[1:1 + ny])
    w[0] = p / (th.rd * feps * T)
    w[1 + ny:4 + ny] = rng.uniform(-5.0, 5.0, (3, n))
    w[4 + ny] = p
    return thermo.prim_to_cons(th, w)


def t_vapour(th, x):
    """all-vapour temperature of feature rows x (n, 4)"""
    cvs = 1.0 + x[:, 2] * th.cv_ratio_m1[0]
    if th.nvapor > 1:
        cvs = cvs + x[:, 3] * th.cv_ratio_m1[1]
    return x[:, 1] / (th.rd / (th.gammad - 1.0) * cvs)


def predict(net, th, x):
    """the network's temperature guess for feature rows x (tensor cores)"""
    a, b, om, os_ = net.normalization()
    yn = net.forward(((x - a) / b).astype(np.float32), tensor_core=True)
    return t_vapour(th, x) + yn * os_ + om


def features(th, u):
    """network inputs (n, 4) of conserved cells u (NV, n)."""
    ny = th.ny
    rho = u[:1 + ny].sum(axis=0)
    ke = 0.5 * (u[1 + ny] ** 2 + u[2 + ny] ** 2 + u[3 + ny] ** 2) / rho
    e = (u[4 + ny] - ke) / rho
    fam = []
    for v in range(2):
        if v < th.nvapor:
            s = u[1 + v].copy()
            for sl in (th.liq_slot[v], th.ice_slot[v]):
                if sl > 0:
                    s += u[sl]
            fam.append(s / rho)
        else:
            fam.append(np.zeros_like(rho))
    return np.stack([rho, e, fam[0], fam[1]], axis=1)


def satadj_gpu(th, u, mode=0, net=None, tol=1e-8, max_iter=30):
    """Run the CUDA saturation adjustment on cells u (NV, n) (copied);
    returns (u_adjusted, T, evaluations, stats[cells, evals, fallbacks,
    non-converged], guesses or None)."""
    import torch
    lib = load()
    n = u.shape[1]
    d = _dev(u, np.float64)
    t = torch.zeros(n, dtype=torch.float64, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = torch.zeros(4, dtype=torch.int64, device="cuda")
    o = SatOpts(tol, max_iter, mode)
    torch.cuda.synchronize()
    guess = None
    if net is None:
        check(lib.canoe_saturation_adjust(ctypes.byref(th), ctypes.byref(o), d.data_ptr(), n,
                                          None, t.data_ptr(), it.data_ptr(), st.data_ptr(),
                                          None), "saturation_adjust")
    else:
        gq = torch.zeros(n, dtype=torch.float64, device="cuda")
        check(lib.canoe_saturation_adjust_learned(ctypes.byref(th), ctypes.byref(o), net.h,
                                                  d.data_ptr(), n, t.data_ptr(), it.data_ptr(),
                                                  st.data_ptr(), gq.data_ptr(), None),
              "saturation_adjust_learned")
        guess = gq
    torch.cuda.synchronize()
    return (d.cpu().numpy(), t.cpu().numpy(), it.cpu().numpy(), st.cpu().numpy(),
            None if guess is None else guess.cpu().numpy())


def training_pairs(th, n, seed=7):
    """(features, converged T) from the plain (cold-start) GPU solver."""
    u = perturbed_states(th, n, seed)
    _, T, _, _, _ = satadj_gpu(th, u, mode=0)
    return features(th, u), T


def default_net():
    """The committed network (canoe_b200/data/warm_start_c2.npz), or one
    trained now when the file is missing."""
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                        "warm_start_c2.npz")
    if os.path.exists(path):
        return WarmStartNet.load(path)
    return train_warm_start()


def train_warm_start(th=None, n=1 << 21, seed=7, epochs=20, batch=8192, log=None):
    th = th or thermo.earth_moist()
    x, T = training_pairs(th, n, seed)
    net = WarmStartNet(seed=seed)
    net.fit(x, T, th, epochs=epochs, batch=batch, log=log)
    return net
