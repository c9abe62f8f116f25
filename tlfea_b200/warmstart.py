"""Learned warm start: PCA of solver-generated displacements plus an MLP that
maps load / material parameters to the PCA coefficients (new; the reference
has no counterpart).

Pipeline (one fixed mesh, many load and material cases):
  1. snapshots   -- the batched linear-static solver solves N training cases;
  2. PCA         -- displacements normalised by the linear-elastic scaling
                    |F| / E, centred, reduced to k modes through the eigen-
                    decomposition of the FP64 Gram matrix (library linear
                    algebra on the GPU);
  3. MLP         -- WarmStartMLP (this library's tcgen05 kernels) learns the
                    standardised coefficients from the 6 case parameters;
  4. warm start  -- u0 = (|F| / E) (mean + modes^T c) per case, handed to the
                    batched solver as its initial guess; the residual
                    tolerance judges the result and a cold start is the
                    fallback (``predict`` is only a guess).

Case parameters (one row per case): E, nu, load direction (3), load magnitude.
The network sees them normalised to about [-1, 1]: log10 E, nu and the
magnitude mapped linearly from their ranges, the direction as is.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .api import BatchedLinearStaticSolver, WarmStartMLP, TYPE_T10
from . import mesh as M


@dataclass
class CaseRanges:
    E: tuple = (1e6, 1e8)
    nu: tuple = (0.2, 0.45)
    magnitude: tuple = (1.0, 200.0)


def sample_cases(n: int, seed: int, ranges: CaseRanges = CaseRanges()) -> np.ndarray:
    """(n, 6) case parameters: E log-uniform, nu uniform, direction uniform on
    the unit sphere, magnitude uniform."""
    r = np.random.default_rng(seed)
    E = np.exp(r.uniform(np.log(ranges.E[0]), np.log(ranges.E[1]), n))
    nu = r.uniform(ranges.nu[0], ranges.nu[1], n)
    d = r.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    mag = r.uniform(ranges.magnitude[0], ranges.magnitude[1], n)
    return np.column_stack([E, nu, d, mag])


def features(cases: np.ndarray, ranges: CaseRanges = CaseRanges()) -> np.ndarray:
    lo, hi = np.log10(ranges.E[0]), np.log10(ranges.E[1])
    f = np.empty((cases.shape[0], 6), np.float32)
    f[:, 0] = 2.0 * (np.log10(cases[:, 0]) - lo) / (hi - lo) - 1.0
    f[:, 1] = 2.0 * (cases[:, 1] - ranges.nu[0]) / (ranges.nu[1] - ranges.nu[0]) - 1.0
    f[:, 2:5] = cases[:, 2:5]
    f[:, 5] = 2.0 * (cases[:, 5] - ranges.magnitude[0]) / (ranges.magnitude[1] - ranges.magnitude[0]) - 1.0
    return f


class FixedMeshCases:
    """One cantilever mesh (x = 0 clamped, tip load spread over the x = max
    face) solved for many cases by the batched solver, `batch` cases per launch."""

    def __init__(self, nx=40, ny=8, nz=8, lx=1.0, ly=0.1, lz=0.1, batch=512):
        self.x, self.y, self.z, self.conn = M.box_mesh(nx, ny, nz, 10, lx, ly, lz)
        self.fixed, _, self.tip = M.cantilever_loads(self.x, self.y, self.z)
        self.N = len(self.x)
        self.batch = int(batch)
        self.solver = BatchedLinearStaticSolver([(self.x, self.y, self.z, self.conn)] * self.batch, TYPE_T10,
                                                shared=True)
        self.solver.SetNodalFixed([self.fixed] * self.batch)

    def loads(self, cases: np.ndarray) -> np.ndarray:
        """(n, 3N) external forces: the case's force vector split over the tip nodes."""
        F = cases[:, 2:5] * cases[:, 5:6]
        f = np.zeros((cases.shape[0], self.N, 3))
        f[:, self.tip, :] = F[:, None, :] / len(self.tip)
        return f.reshape(cases.shape[0], 3 * self.N)

    def _load(self, cases: np.ndarray):
        n = cases.shape[0]
        if n > self.batch:
            raise ValueError("more cases than the batch holds")
        pad = self.batch - n
        E = np.concatenate([cases[:, 0], np.full(pad, 1e7)])
        nu = np.concatenate([cases[:, 1], np.full(pad, 0.3)])
        f = np.concatenate([self.loads(cases), np.zeros((pad, 3 * self.N))])  # padding: zero load, solved at once
        self.solver.SetMaterial(E, nu)
        self.solver.SetExternalForce(f.ravel())

    def solve(self, cases: np.ndarray, tol=1e-6, max_iter=200000, u0: np.ndarray | int | None = None):
        """Solve up to `batch` cases in one launch; returns (u (n, 3N), iterations, rel. residual, status)."""
        n = cases.shape[0]
        self._load(cases)
        if u0 is None:
            self.solver.SetInitialGuess(None)
        elif isinstance(u0, int):
            # a raw device pointer must cover the whole batch
            if n != self.batch:
                raise ValueError("a device-pointer guess needs exactly `batch` cases; pass a tensor instead")
            self.solver.SetInitialGuess(u0)
        elif hasattr(u0, "data_ptr"):
            import torch

            if tuple(u0.shape) != (n, 3 * self.N):
                raise ValueError("guess must be (cases, 3 * nodes)")
            g = torch.zeros(self.batch, 3 * self.N, dtype=torch.float64, device=u0.device)
            g[:n] = u0
            # the solver copies on its own stream: the guess must be complete first
            torch.cuda.synchronize()
            self.solver.SetInitialGuess(int(g.data_ptr()))
        else:
            g = np.zeros((self.batch, 3 * self.N))
            g[:n] = u0
            self.solver.SetInitialGuess(g.ravel())
        self.solver.Solve(tol, max_iter)
        it, res, st = self.solver.GetResults()
        u = self.solver.RetrieveDisplacement(split=False).reshape(self.batch, 3 * self.N)[:n]
        return u, it[:n], res[:n], st[:n]

    def destroy(self):
        self.solver.Destroy()


class PCA:
    """k-mode PCA of normalised snapshots via the FP64 Gram matrix (torch / cuSOLVER)."""

    def __init__(self, k: int = 64, coef_scale: str = "mode"):
        """coef_scale "mode": every coefficient standardised to unit variance;
        "global": one scale for all (the largest mode's), so a squared
        coefficient error is the squared displacement error."""
        self.k = k
        self.coef_scale = coef_scale

    def fit(self, W):
        """W: snapshots (n, dof), numpy or a torch tensor on the GPU."""
        import torch

        Wd = torch.as_tensor(W, dtype=torch.float64, device="cuda")
        self.mean = Wd.mean(0)
        Wc = Wd - self.mean
        G = Wc @ Wc.T
        evals, evecs = torch.linalg.eigh(G)
        order = torch.argsort(evals, descending=True)[: self.k]
        lam = evals[order].clamp_min(1e-300)
        V = evecs[:, order]
        self.modes = (Wc.T @ V) / torch.sqrt(lam)  # (n, k), orthonormal columns
        self.energy = (lam.sum() / evals.clamp_min(0).sum()).item()
        C = Wc @ self.modes
        self.c_mean = C.mean(0)
        self.c_std = C.std(0).clamp_min(1e-300)
        if self.coef_scale == "global":
            self.c_std = self.c_std.max().expand_as(self.c_std).clone()
        return ((C - self.c_mean) / self.c_std).cpu().numpy()

    def coefficients(self, W) -> np.ndarray:
        import torch

        Wd = torch.as_tensor(W, dtype=torch.float64, device="cuda")
        return (((Wd - self.mean) @ self.modes - self.c_mean) / self.c_std).cpu().numpy()

    def coefficients_t(self, Wd):
        """Standardised coefficients of device rows (torch, FP64), kept on the GPU."""
        return ((Wd - self.mean) @ self.modes - self.c_mean) / self.c_std

    def reconstruct(self, Cstd):
        """Standardised coefficients (n, k) -> normalised displacements (n, dof), on the GPU."""
        import torch

        C = torch.as_tensor(Cstd, dtype=torch.float64, device="cuda") * self.c_std + self.c_mean
        return self.mean + C @ self.modes.T


class LearnedWarmStart:
    """PCA + WarmStartMLP on one fixed mesh."""

    def __init__(self, hidden=(256, 256, 256), k=64, max_batch=512, seed=0, coef_scale="mode"):
        import torch

        self.pca = PCA(k, coef_scale)
        self.dims = [6, *hidden, k]
        self.net = WarmStartMLP(self.dims, max_batch=max_batch, seed=seed)
        self.max_batch = max_batch
        # torch work that feeds the network runs on the network's stream, so the
        # kernels see finished inputs without host synchronisation
        self.stream = torch.cuda.ExternalStream(self.net.GetStream())

    @staticmethod
    def normalise(u: np.ndarray, cases: np.ndarray) -> np.ndarray:
        return u * (cases[:, 0] / cases[:, 5])[:, None]

    def fit(self, cases: np.ndarray, u: np.ndarray, epochs=400, batch=512, lr=1e-3, lr_final=1e-5,
            weight_decay=0.0, seed=0, log=None):
        """PCA of the normalised snapshots, then MLP training on the GPU (AdamW,
        cosine learning-rate decay).  Returns the per-epoch mean training loss."""
        import torch

        target = self.pca.fit(self.normalise(u, cases)).astype(np.float32)
        torch.cuda.synchronize()
        n = cases.shape[0] - cases.shape[0] % batch
        r = np.random.default_rng(seed)
        hist = []
        steps = epochs * (n // batch)
        k = 0
        with torch.cuda.stream(self.stream):
            X = torch.as_tensor(features(cases), device="cuda")
            Y = torch.as_tensor(target, device="cuda")
            for ep in range(epochs):
                perm = torch.as_tensor(r.permutation(X.shape[0])[:n], device="cuda")
                Xs, Ys = X[perm].contiguous(), Y[perm].contiguous()
                tot = 0.0
                for b in range(n // batch):
                    a = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / max(steps, 1)))
                    want = (b == n // batch - 1)
                    l = self.net.TrainStep(Xs[b * batch:(b + 1) * batch].data_ptr(),
                                           Ys[b * batch:(b + 1) * batch].data_ptr(), batch, lr=float(a),
                                           weight_decay=weight_decay, want_loss=want)
                    if want:
                        tot = l
                    k += 1
                hist.append(tot)
                if log and (ep % 50 == 0 or ep == epochs - 1):
                    log(f"epoch {ep}: loss {tot:.3e}")
        self.stream.synchronize()
        return hist

    def predict_normalised(self, cases: np.ndarray):
        import torch

        with torch.cuda.stream(self.stream):
            X = torch.as_tensor(features(cases), device="cuda")
            out = torch.empty(X.shape[0], self.dims[-1], device="cuda")
            for b in range(0, X.shape[0], self.max_batch):
                m = min(self.max_batch, X.shape[0] - b)
                self.net.Forward(X[b:b + m].data_ptr(), m, out[b:b + m].data_ptr())
            w = self.pca.reconstruct(out.double())
        return w

    def predict(self, cases: np.ndarray):
        """Warm-start displacements (n, dof) on the GPU (FP64 torch tensor),
        complete when this returns."""
        import torch

        with torch.cuda.stream(self.stream):
            s = torch.as_tensor(cases[:, 5] / cases[:, 0], dtype=torch.float64, device="cuda")
            u = self.predict_normalised(cases) * s[:, None]
        self.stream.synchronize()
        return u

    def destroy(self):
        self.net.Destroy()


def lame(E, nu):
    """Lame parameters as SetSVK computes them (FEAT10Data.cuh:399-409)."""
    E, nu = np.asarray(E, np.float64), np.asarray(nu, np.float64)
    return E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), E / (2.0 * (1.0 + nu))


class GalerkinWarmStart:
    """Warm start from the learned basis alone, no network: the Galerkin
    (Rayleigh-Ritz) solution in span{PCA mean, PCA modes},
        (B^T K_i B) c = B^T f_i,   u0 = B c,
    with K_i = lambda_i K_lambda + mu_i K_mu for the fixed mesh (fixed DOFs
    eliminated; the basis is zero there).  B^T K_lambda B and B^T K_mu B are
    formed once from two batched products K B; each case then costs one small
    dense solve.  FP64 throughout (library linear algebra on the GPU)."""

    def __init__(self, pca: PCA, fm: FixedMeshCases, materials=((1e7, 0.3), (1e7, 0.45))):
        import torch

        B = torch.cat([pca.mean[None, :], pca.modes.T], 0)  # (k+1, dof)
        k1, n = B.shape
        if k1 > fm.batch:
            raise ValueError("the basis has more vectors than the batch holds")
        self.B = B.contiguous()
        X = torch.zeros(fm.batch, n, dtype=torch.float64, device="cuda")
        X[:k1] = B
        A = []
        for E, nu in materials:
            fm.solver.SetMaterial(np.full(fm.batch, E), np.full(fm.batch, nu))
            Y = torch.empty_like(X)
            torch.cuda.synchronize()
            fm.solver.Apply(int(X.data_ptr()), int(Y.data_ptr()))
            A.append(B @ Y[:k1].T)  # B^T K B
        l1, m1 = lame(*materials[0])
        l2, m2 = lame(*materials[1])
        det = l1 * m2 - l2 * m1
        self.A_lam = (m2 * A[0] - m1 * A[1]) / float(det)
        self.A_mu = (l1 * A[1] - l2 * A[0]) / float(det)
        self.fm = fm

    def predict(self, cases: np.ndarray):
        """Warm-start displacements (n, dof) on the GPU (FP64 torch tensor)."""
        import torch

        lam, mu = lame(cases[:, 0], cases[:, 1])
        lam = torch.as_tensor(lam, device="cuda")[:, None, None]
        mu = torch.as_tensor(mu, device="cuda")[:, None, None]
        A = lam * self.A_lam[None] + mu * self.A_mu[None]
        F = torch.as_tensor(self.fm.loads(cases), device="cuda")
        rhs = F @ self.B.T  # (n, k+1)
        c = torch.linalg.solve(A, rhs[:, :, None])[:, :, 0]
        u = c @ self.B
        torch.cuda.synchronize()
        return u


# ---------------------------------------------------------------- time stepping

class DeviceArray:
    """A raw device pointer seen as a CUDA array (``__cuda_array_interface__``), so
    torch can view the library's state without a copy."""

    def __init__(self, ptr: int, shape, typestr: str = "<f8"):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_view(ptr: int, shape, dtype="float64"):
    import torch

    return torch.as_tensor(DeviceArray(ptr, shape, "<f8" if dtype == "float64" else "<f4"), device="cuda")


class StepPredictor:
    """Learned step predictor for batched time-stepping sequences (new): the next
    step's velocity as the linear extrapolation of the last two plus a learned
    correction,

        v_(n+1) ~ 2 v_n - v_(n-1) + dv,   dv = mean + modes (c_std * MLP(features)),

    where the modes are a PCA basis of the corrections the solver itself produced
    on training sequences (its converged steps), and the MLP (WarmStartMLP: this
    library's BF16 tcgen05 kernels, FP32 accumulation) maps per-sequence features
    to the standardised coefficients.  Features: the coefficients of v_n, v_(n-1)
    and the displacement u_n in PCA bases of the velocity and displacement
    snapshots, the load factor at the last, this and the next step end times, and
    the material (log10 E and nu, scaled to about [-1, 1]).  The guess only starts
    the step's Nesterov iteration: the residual tolerance decides the answer."""

    def __init__(self, k_in=16, k_out=32, hidden=(256, 256), max_batch=128, seed=0, E_range=(1e6, 1e8),
                 nu_range=(0.2, 0.45)):
        import torch

        self.k_in, self.k_out = k_in, k_out
        self.E_range, self.nu_range = E_range, nu_range
        self.pca_v = PCA(k_in)
        self.pca_u = PCA(k_in)
        self.pca_d = PCA(k_out)
        self.n_feat = 3 * k_in + 5
        self.dims = [self.n_feat, *hidden, k_out]
        self.net = WarmStartMLP(self.dims, max_batch=max_batch, seed=seed)
        self.max_batch = max_batch
        self.stream = torch.cuda.ExternalStream(self.net.GetStream())

    def material_features(self, E, nu):
        lo, hi = np.log10(self.E_range[0]), np.log10(self.E_range[1])
        fe = 2.0 * (np.log10(E) - lo) / (hi - lo) - 1.0
        fn = 2.0 * (np.asarray(nu) - self.nu_range[0]) / (self.nu_range[1] - self.nu_range[0]) - 1.0
        return np.column_stack([fe, fn])

    def _features(self, v_n, v_nm1, u_n, loads, mat):
        """torch (B, n_feat) FP32 from FP64 device tensors (B, dof) and host arrays."""
        import torch

        a = torch.as_tensor(self.pca_v.coefficients_t(v_n))
        b = torch.as_tensor(self.pca_v.coefficients_t(v_nm1))
        c = torch.as_tensor(self.pca_u.coefficients_t(u_n))
        extra = torch.as_tensor(np.column_stack([loads, mat]), dtype=torch.float64, device="cuda")
        return torch.cat([a, b, c, extra], 1).float().contiguous()

    def fit(self, V, U, loads, mats, epochs=600, batch=128, lr=1e-3, lr_final=1e-5, seed=0):
        """V: (S, T, dof) velocities after steps 1..T of S training sequences (v_0 = 0),
        U: (S, T, dof) displacements, loads: (T, 3) load factors at (t_(n-1), t_n, t_(n+1))
        of the sample predicting step n+1, mats: (S, 2) material features.  Samples are the
        steps n = 1..T-1 (v_(n-1) = 0 for n = 1).  Returns the training-loss history."""
        import torch

        S, Tn, dof = V.shape
        Vd = torch.as_tensor(V, device="cuda")
        Ud = torch.as_tensor(U, device="cuda")
        Vprev = torch.cat([torch.zeros_like(Vd[:, :1]), Vd[:, :-1]], 1)
        self.pca_v.fit(Vd.reshape(-1, dof))
        self.pca_u.fit(Ud.reshape(-1, dof))
        vn, vnm1, un = Vd[:, :-1], Vprev[:, :-1], Ud[:, :-1]
        d = Vd[:, 1:] - 2.0 * vn + vnm1  # the correction to the linear extrapolation
        Y = torch.as_tensor(self.pca_d.fit(d.reshape(-1, dof)), dtype=torch.float32, device="cuda")
        L = np.repeat(loads[None, :-1], S, 0).reshape(-1, loads.shape[1])
        Mt = np.repeat(mats[:, None, :], Tn - 1, 1).reshape(-1, mats.shape[1])
        X = self._features(vn.reshape(-1, dof), vnm1.reshape(-1, dof), un.reshape(-1, dof), L, Mt)
        n = X.shape[0] - X.shape[0] % batch
        if n == 0:
            raise ValueError("fewer training samples than one batch")
        r = np.random.default_rng(seed)
        hist, steps, k = [], epochs * (n // batch), 0
        torch.cuda.synchronize()
        with torch.cuda.stream(self.stream):
            for ep in range(epochs):
                perm = torch.as_tensor(r.permutation(X.shape[0])[:n], device="cuda")
                Xs, Ys = X[perm].contiguous(), Y[perm].contiguous()
                tot = 0.0
                for b in range(n // batch):
                    a = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / max(steps, 1)))
                    want = (b == n // batch - 1)
                    l = self.net.TrainStep(Xs[b * batch:(b + 1) * batch].data_ptr(),
                                           Ys[b * batch:(b + 1) * batch].data_ptr(), batch, lr=float(a),
                                           want_loss=want)
                    if want:
                        tot = l
                    k += 1
                hist.append(tot)
        self.stream.synchronize()
        return hist

    def predict(self, v_n, v_nm1, u_n, loads, mat):
        """Velocity guesses (B, dof) FP64 on the GPU for the next step, complete on return."""
        import torch

        with torch.cuda.stream(self.stream):
            X = self._features(v_n, v_nm1, u_n, loads, mat)
            out = torch.empty(X.shape[0], self.k_out, device="cuda")
            for b in range(0, X.shape[0], self.max_batch):
                m = min(self.max_batch, X.shape[0] - b)
                self.net.Forward(X[b:b + m].data_ptr(), m, out[b:b + m].data_ptr())
            g = 2.0 * v_n - v_nm1 + self.pca_d.reconstruct(out.double())
        self.stream.synchronize()
        return g.contiguous()

    def destroy(self):
        self.net.Destroy()
