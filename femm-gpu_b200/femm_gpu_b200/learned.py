"""Learned warm start: a reduced basis of A whose coefficients an MLP predicts.

Pipeline (every solve, projection, training step and prediction runs in libfemmgpu):

1. ``generate``: FP64 Newton solves of seeded samples with the plain method (the data the
   network learns from), projected on the basis as they are produced;
2. ``pod_basis``: proper orthogonal decomposition of a subset of those solutions (method of
   snapshots: eigenvectors of the snapshot Gram matrix), ``rank`` orthonormal modes;
3. ``Mlp.train``: features -> normalised coefficients, Adam, the library's own FP32 kernels;
4. ``LearnedWarmStart.solve``: fg_solve_batch_learned -- predicted warm start, guarded by
   the equation residual, Newton to the unchanged tolerances.

Features of a sample: its circuit currents divided by ``current_scale`` and the cosine and
sine of its magnet angle (constant for a model without a magnet).
"""
import ctypes as C
import math

import numpy as np

from .capi import FgError, FgItemInfo, Plan, SolveResult, _p, lib, production_options


def features(currents, current_scale, angle_deg=0.0):
    """[k, C + 2] float32: currents / current_scale, cos and sin of the magnet angle."""
    cur = np.atleast_2d(np.asarray(currents, np.float64))
    k = cur.shape[0]
    ang = np.broadcast_to(np.asarray(angle_deg, np.float64), (k,))
    rad = np.deg2rad(ang)
    f = np.concatenate([cur / current_scale, np.cos(rad)[:, None], np.sin(rad)[:, None]], axis=1)
    return np.ascontiguousarray(f, np.float32)


class Mlp:
    """fg_mlp: inputs -> hidden -> hidden -> outputs with GELU, FP32, on the GPU."""

    def __init__(self, inputs, hidden, outputs, seed=0):
        self._h = C.c_void_p()
        st = lib().fg_mlp_create(C.c_int32(inputs), C.c_int32(hidden), C.c_int32(outputs),
                                 C.c_uint64(seed), C.byref(self._h))
        if st:
            self._h = None
            raise FgError(st, "fg_mlp_create")
        self.inputs, self.hidden, self.outputs = inputs, hidden, outputs

    def close(self):
        if getattr(self, "_h", None):
            lib().fg_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def parameter_count(self):
        return int(lib().fg_mlp_parameter_count(self._h))

    def get_parameters(self):
        p = np.zeros(self.parameter_count, np.float32)
        st = lib().fg_mlp_get_parameters(self._h, _p(p))
        if st:
            raise FgError(st, "fg_mlp_get_parameters")
        return p

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.parameter_count
        st = lib().fg_mlp_set_parameters(self._h, _p(p))
        if st:
            raise FgError(st, "fg_mlp_set_parameters")

    def forward(self, x):
        x = np.ascontiguousarray(np.atleast_2d(x), np.float32)
        y = np.zeros((x.shape[0], self.outputs), np.float32)
        st = lib().fg_mlp_forward(self._h, C.c_int32(x.shape[0]), _p(x), _p(y))
        if st:
            raise FgError(st, "fg_mlp_forward")
        return y

    def loss_gradient(self, x, t):
        x = np.ascontiguousarray(np.atleast_2d(x), np.float32)
        t = np.ascontiguousarray(np.atleast_2d(t), np.float32)
        g = np.zeros(self.parameter_count, np.float32)
        loss = C.c_float(0.0)
        st = lib().fg_mlp_loss_gradient(self._h, C.c_int32(x.shape[0]), _p(x), _p(t),
                                        C.byref(loss), _p(g))
        if st:
            raise FgError(st, "fg_mlp_loss_gradient")
        return loss.value, g

    def train(self, x, t, epochs, batch=256, lr=1e-3, seed=0):
        x = np.ascontiguousarray(np.atleast_2d(x), np.float32)
        t = np.ascontiguousarray(np.atleast_2d(t), np.float32)
        loss = C.c_float(0.0)
        st = lib().fg_mlp_train(self._h, C.c_int32(x.shape[0]), _p(x), _p(t), C.c_int32(epochs),
                                C.c_int32(batch), C.c_float(lr), C.c_uint64(seed), C.byref(loss))
        if st:
            raise FgError(st, "fg_mlp_train")
        return loss.value


class WarmModel:
    """fg_warm: reduced basis (+ optional network) bound to a plan's node numbering."""

    def __init__(self, plan: Plan, mean, basis, mlp: Mlp = None, feature_shift=None,
                 feature_scale=None, coeff_shift=None, coeff_scale=None):
        self.mean = np.ascontiguousarray(mean, np.float64)
        self.basis = np.ascontiguousarray(basis, np.float64)
        self.rank = self.basis.shape[0]
        self.mlp = mlp
        arrs = [None if a is None else np.ascontiguousarray(a, dt) for a, dt in
                ((feature_shift, np.float32), (feature_scale, np.float32),
                 (coeff_shift, np.float64), (coeff_scale, np.float64))]
        self._keep = arrs
        self._h = C.c_void_p()
        st = lib().fg_warm_create(plan._h, C.c_int32(self.rank), _p(self.mean), _p(self.basis),
                                  mlp._h if mlp is not None else None, *[_p(a) for a in arrs],
                                  C.byref(self._h))
        if st:
            self._h = None
            raise FgError(st, "fg_warm_create")
        self.N = self.mean.size

    def close(self):
        if getattr(self, "_h", None):
            lib().fg_warm_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def project(self, a):
        a = np.ascontiguousarray(np.atleast_2d(a), np.float64)
        c = np.zeros((a.shape[0], self.rank))
        st = lib().fg_warm_project(self._h, C.c_int32(a.shape[0]), _p(a), _p(c))
        if st:
            raise FgError(st, "fg_warm_project")
        return c

    def predict(self, feats):
        f = np.ascontiguousarray(np.atleast_2d(feats), np.float32)
        a = np.zeros((f.shape[0], self.N))
        st = lib().fg_warm_predict(self._h, C.c_int32(f.shape[0]), _p(f), _p(a))
        if st:
            raise FgError(st, "fg_warm_predict")
        return a


def pod_basis(snapshots, rank):
    """Mean and `rank` orthonormal POD modes of snapshots [m, N] (method of snapshots)."""
    S = np.asarray(snapshots, np.float64)
    mean = S.mean(axis=0)
    D = S - mean
    G = D @ D.T
    w, V = np.linalg.eigh(G)
    order = np.argsort(w)[::-1]
    w, V = w[order], V[:, order]
    r = min(rank, int(np.sum(w > w[0] * 1e-24)))
    basis = (V[:, :r].T @ D) / np.sqrt(w[:r])[:, None]
    # re-orthonormalise (modified Gram-Schmidt) against rounding
    for i in range(r):
        for j in range(i):
            basis[i] -= np.dot(basis[i], basis[j]) * basis[j]
        basis[i] /= np.linalg.norm(basis[i])
    energy = w[:r].sum() / max(w.sum(), 1e-300)
    return mean, basis, energy


class LearnedWarmStart:
    """Train once on solves of the plain method, then solve from predicted warm starts."""

    def __init__(self, plan: Plan, current_scale, rank=64, hidden=256, seed=0):
        self.plan, self.current_scale = plan, float(current_scale)
        self.rank, self.hidden, self.seed = rank, hidden, seed
        self.warm = None
        self.mlp = None
        self.stats = {}

    def fit(self, currents, angles=0.0, pod_samples=256, epochs=200, batch=256, lr=2e-3,
            options=None, block=1024):
        """Solve every training sample (FP64, zero start), build the basis from the first
        `pod_samples` solutions, project all of them and train the network.  The samples
        are solved `block` at a time (a wide batch advances its chunks of 32 together)."""
        currents = np.atleast_2d(np.asarray(currents, np.float64))
        n = currents.shape[0]
        opts = options if options is not None else production_options()
        m = min(pod_samples, n)
        first = self.plan.solve(currents[:m], options=opts, outputs="a")
        if any(s != 0 for s in first.status):
            raise RuntimeError("training solve did not converge")
        mean, basis, energy = pod_basis(first.a, self.rank)
        self.rank = basis.shape[0]
        proj = WarmModel(self.plan, mean, basis)
        coeffs = [proj.project(first.a)]
        for s0 in range(m, n, block):
            r = self.plan.solve(currents[s0:s0 + block], options=opts, outputs="a")
            if any(s != 0 for s in r.status):
                raise RuntimeError("training solve did not converge")
            coeffs.append(proj.project(r.a))
        proj.close()
        coeffs = np.concatenate(coeffs)
        feats = features(currents, self.current_scale, angles)
        fshift = feats.mean(axis=0)
        fscale = feats.std(axis=0)
        fscale[fscale == 0] = 1.0
        # Each coefficient scaled by its own spread: the small, oscillatory modes are then
        # learned to the same relative accuracy as the dominant ones, which keeps the
        # residual K(A) A - b of the prediction small (a common scale leaves their
        # absolute error at the dominant mode's level, and K amplifies it).
        cshift = coeffs.mean(axis=0)
        cscale = coeffs.std(axis=0)
        cscale = np.maximum(cscale, 1e-9 * max(float(cscale.max()), 1e-300))
        x = (feats - fshift) / fscale
        t = ((coeffs - cshift) / cscale).astype(np.float32)
        self.mlp = Mlp(feats.shape[1], self.hidden, self.rank, seed=self.seed)
        loss = self.mlp.train(x, t, epochs=epochs, batch=batch, lr=lr, seed=self.seed + 1)
        self.warm = WarmModel(self.plan, mean, basis, self.mlp, fshift, fscale, cshift, cscale)
        self.stats = {"samples": n, "pod_samples": m, "rank": self.rank, "pod_energy": energy,
                      "final_loss": loss}
        return self

    def solve(self, currents, angles=0.0, hc_scale=None, options=None, outputs=True):
        cur = np.ascontiguousarray(np.atleast_2d(np.asarray(currents, np.float64)))
        k = cur.shape[0]
        feats = features(cur, self.current_scale, angles)
        opts = options if options is not None else production_options()
        p = self.plan
        a = np.zeros((k, p.N)) if outputs else None
        b1 = np.zeros((k, p.E)) if outputs is True else None
        b2 = np.zeros((k, p.E)) if outputs is True else None
        flux = np.zeros((k, max(p.C, 1))) if outputs else None
        hc = None if hc_scale is None else np.ascontiguousarray(hc_scale, np.float64)
        info = (FgItemInfo * k)()
        st = lib().fg_solve_batch_learned(p._h, self.warm._h, C.c_int32(k), _p(cur), _p(hc),
                                          _p(feats), C.byref(opts), _p(a), _p(b1), _p(b2),
                                          _p(flux), info)
        if st:
            raise FgError(st, "fg_solve_batch_learned")
        return SolveResult(a, b1, b2, None if flux is None else flux[:, : p.C],
                           [info[i] for i in range(k)])
