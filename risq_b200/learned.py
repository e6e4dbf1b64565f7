"""Learned correction of the Davidson diagonal preconditioner.

The reference's Davidson uses DPR, t = r / (lambda - H_ii)
(src/var/eigenvalues/algorithms/davidson.rs:391-408).  Here a small network gives
each determinant a factor f in [0.25, 4] and the step becomes f * r / (lambda - H_ii);
DPR stays the fallback whenever the residual stalls (risq_b200/csrc/davidson.cu).

Target.  DPR replaces H - lambda by its diagonal.  The second-order (Epstein-Nesbet)
resolvent keeps the couplings of each determinant to first order:
1 / (E - H_ii - S_i) with S_i = sum_j H_ij^2 / (E - H_jj) (risqgpu_self_energy).  The
target factor of determinant i is f_i = sqrt((H_ii - E) / (H_ii - E + |S_i|)),
clipped to [0.25, 4], at E = the converged energy of an FP64 DPR Davidson run on a
training system.  The network sees E only through the feature H_ii - E, and during a
solve E is the current Ritz value, so every training system contributes the same
targets under features taken at the Ritz values its own FP64 DPR trajectory visits:
the network learns the factor that suits the converged state from where the solver
stands.  Inference averages the network over the determinant and its spin-flipped
partner (alpha and beta occupations exchanged), so the factors keep the spin-flip
symmetry of the Hamiltonian.  Training runs on the device with this library's
forward / backward kernels (log-space squared error).

Features (the inference kernel computes the same, mlp.cu): 2n occupations as +1/-1
(alpha orbitals, then beta), (H_ii - E - mu_e) * s_e and
(sum of occupied h_pp - mu_h) * s_h.

Orbital-count-independent networks.  A network of the native layout is tied to one
orbital count n.  The universal layout gives every spin NMAX = 32 slots, slot k
holding the orbital with the k-th lowest h_pp (absent orbitals read 0), and replaces
the sum of occupied h_pp by its mean over the electrons.  A universal network trained
on systems of one or several orbital counts is turned, for a given system, into the
exactly equivalent native network (`adapt`: W1's occupation columns gathered by
orbital rank, the normalisation of the h_pp feature rescaled by the electron count),
so the device kernels serve both.  Slots no training system had stay at weight 0.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

from . import _capi as A
from .fcidump import Integrals, dets_to_ints

HIDDEN = 128
NMAX = 32  # orbital slots per spin of the universal layout
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


@dataclasses.dataclass
class PrecondMLP:
    norb: int
    hidden: int
    params: np.ndarray   # packed float32 [W1, b1, W2, b2, W3, b3]
    fnorm: np.ndarray    # float32 [mu_e, s_e, mu_h, s_h]

    @property
    def n_in(self):
        return 2 * self.norb + 2

    @classmethod
    def init(cls, norb, hidden=HIDDEN, seed=0, fnorm=None):
        n_in = 2 * norb + 2
        rng = np.random.default_rng(seed)
        W1 = rng.standard_normal((hidden, n_in)) * np.sqrt(2.0 / n_in)
        W2 = rng.standard_normal((hidden, hidden)) * np.sqrt(2.0 / hidden)
        W3 = rng.standard_normal(hidden) * np.sqrt(1.0 / hidden) * 0.1
        p = np.concatenate([W1.ravel(), np.zeros(hidden), W2.ravel(), np.zeros(hidden), W3, [0.0]]).astype(np.float32)
        fn = np.asarray(fnorm if fnorm is not None else [0.0, 1.0, 0.0, 1.0], dtype=np.float32)
        return cls(norb, hidden, p, fn)

    def split(self):
        H, n = self.hidden, self.n_in
        p = self.params
        o = 0
        W1 = p[o:o + H * n].reshape(H, n); o += H * n
        b1 = p[o:o + H]; o += H
        W2 = p[o:o + H * H].reshape(H, H); o += H * H
        b2 = p[o:o + H]; o += H
        W3 = p[o:o + H]; o += H
        b3 = p[o:o + 1]
        return W1, b1, W2, b2, W3, b3

    def save(self, path):
        np.savez(path, norb=self.norb, hidden=self.hidden, params=self.params, fnorm=self.fnorm)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(int(z["norb"]), int(z["hidden"]), z["params"].astype(np.float32), z["fnorm"].astype(np.float32))

    @staticmethod
    def pack(W1, b1, W2, b2, W3, b3):
        return np.concatenate([np.ravel(W1), b1, np.ravel(W2), b2, W3, np.ravel(b3)]).astype(np.float32)


def default_model_path(norb):
    return os.path.join(DATA_DIR, f"precond_mlp_n{norb}.npz")


def universal_model_path():
    return os.path.join(DATA_DIR, f"precond_mlp_u{NMAX}.npz")


def load_default(norb):
    path = default_model_path(norb)
    return PrecondMLP.load(path) if os.path.exists(path) else None


def install(gpu, model: PrecondMLP):
    """Load the network into a GpuHam handle (risqgpu_set_precond_mlp)."""
    W1, b1, W2, b2, W3, b3 = (np.ascontiguousarray(a, dtype=np.float32) for a in model.split())
    fn = np.ascontiguousarray(model.fnorm, dtype=np.float32)
    A.check(A.lib().risqgpu_set_precond_mlp(gpu._h, model.n_in, model.hidden, A.ptr(W1, A._fp), A.ptr(b1, A._fp),
                                            A.ptr(W2, A._fp), A.ptr(b2, A._fp), A.ptr(W3, A._fp), A.ptr(b3, A._fp),
                                            A.ptr(fn, A._fp)), gpu._h)


def device_factors(gpu, energy):
    out = np.zeros(gpu.n, dtype=np.float32)
    A.check(A.lib().risqgpu_precond_factors(gpu._h, energy, A.ptr(out, A._fp)), gpu._h)
    return out


def raw_features(dets, diag, energy, ints: Integrals):
    """(N, 2n+2) float32 features before normalisation of the last two columns."""
    n = ints.norb
    d = np.asarray(dets, dtype=np.uint64)
    N = d.shape[0]
    hpp = np.array([ints.h(k, k) for k in range(n)], dtype=np.float32)
    out = np.empty((N, 2 * n + 2), dtype=np.float32)
    up = np.zeros((N, n), dtype=bool)
    dn = np.zeros((N, n), dtype=bool)
    for k in range(n):
        word, bit = k // 64, np.uint64(k % 64)
        up[:, k] = ((d[:, word] >> bit) & np.uint64(1)).astype(bool)
        dn[:, k] = ((d[:, 2 + word] >> bit) & np.uint64(1)).astype(bool)
    out[:, :n] = np.where(up, 1.0, -1.0)
    out[:, n:2 * n] = np.where(dn, 1.0, -1.0)
    out[:, 2 * n] = (np.asarray(diag, dtype=np.float64) - energy).astype(np.float32)
    out[:, 2 * n + 1] = (up.astype(np.float32) @ hpp) + (dn.astype(np.float32) @ hpp)
    return out


def orbital_ranks(ints: Integrals):
    """rank[o]: position of orbital o in ascending h_pp order (ties by index)."""
    hpp = np.array([ints.h(k, k) for k in range(ints.norb)], dtype=np.float64)
    order = np.argsort(hpp, kind="stable")
    rank = np.empty(ints.norb, dtype=np.int64)
    rank[order] = np.arange(ints.norb)
    return rank


def n_electrons(dets):
    d = np.asarray(dets[:1], dtype=np.uint64)
    return int(sum(bin(int(w)).count("1") for w in d[0]))


def universal_features(dets, diag, energy, ints: Integrals):
    """(N, 2 NMAX + 2) float32 features of the universal layout before normalisation:
    occupations by orbital rank, H_ii - E, mean occupied h_pp."""
    n = ints.norb
    if n > NMAX:
        raise ValueError(f"the universal layout holds at most {NMAX} orbitals")
    raw = raw_features(dets, diag, energy, ints)
    rank = orbital_ranks(ints)
    out = np.zeros((raw.shape[0], 2 * NMAX + 2), dtype=np.float32)
    out[:, rank] = raw[:, :n]
    out[:, NMAX + rank] = raw[:, n:2 * n]
    out[:, 2 * NMAX] = raw[:, 2 * n]
    out[:, 2 * NMAX + 1] = raw[:, 2 * n + 1] / n_electrons(dets)
    return out


def adapt(model: PrecondMLP, ints: Integrals, nel: int) -> PrecondMLP:
    """The native network for a system of ints.norb orbitals and nel electrons that
    computes exactly what the universal network computes on its universal features."""
    if model.norb != NMAX:
        raise ValueError("adapt takes a network of the universal layout")
    n = ints.norb
    rank = orbital_ranks(ints)
    W1u, b1, W2, b2, W3, b3 = model.split()
    W1 = np.zeros((model.hidden, 2 * n + 2), dtype=np.float32)
    W1[:, :n] = W1u[:, rank]
    W1[:, n:2 * n] = W1u[:, NMAX + rank]
    W1[:, 2 * n:] = W1u[:, 2 * NMAX:]
    fn = model.fnorm.astype(np.float64)
    fnorm = np.array([fn[0], fn[1], fn[2] * nel, fn[3] / nel], dtype=np.float32)
    return PrecondMLP(n, model.hidden, PrecondMLP.pack(W1, b1, W2, b2, W3, b3), fnorm)


def normalise(feats, fnorm):
    f = feats.copy()
    n2 = f.shape[1] - 2
    f[:, n2] = (f[:, n2] - fnorm[0]) * fnorm[1]
    f[:, n2 + 1] = (f[:, n2 + 1] - fnorm[2]) * fnorm[3]
    return f


def dpr_trajectory(sigma, diag, tol=1e-4, etol=1e-8, max_iter=1000, record=None):
    """DPR Davidson (the reference's algorithm, one root, default start with identity
    columns 0 and 1) in FP64 numpy with a device sigma; record(k, lam, x, r) is called
    at every iteration with the normalised Ritz vector and residual."""
    N = len(diag)
    mss = min(11, N)
    V = np.zeros((N, mss))
    V[0, 0] = 1.0
    V[1, 1] = 1.0
    dim = 2
    HV = np.zeros((N, mss))
    for c in range(dim):
        HV[:, c] = sigma(V[:, c])
    last = 0.0
    for it in range(max_iter):
        P = V[:, :dim].T @ HV[:, :dim]
        P = (P + P.T) / 2
        w, Y = np.linalg.eigh(P)
        lam, y = w[0], Y[:, 0]
        x = V[:, :dim] @ y
        hx = HV[:, :dim] @ y
        r = hx - lam * x
        if record is not None:
            record(it, lam, x, r)
        if np.linalg.norm(r) < tol and abs(lam - last) < etol:
            return lam, x, it + 1
        last = lam
        if dim + 1 <= mss:
            t = r / (lam - diag)
            for _ in range(2):
                t -= V[:, :dim] @ (V[:, :dim].T @ t)
            t /= np.linalg.norm(t)
            V[:, dim] = t
            HV[:, dim] = sigma(t)
            dim += 1
        else:
            V[:, 0] = x / np.linalg.norm(x)
            HV[:, 0] = hx / np.linalg.norm(x)
            dim = 1
    return lam, x, max_iter


def self_energy(gpu, energy, gmin=1e-3):
    """S_i = -sum_j H_ij^2 / max(H_jj - E, gmin) over the built matrix (risqgpu_self_energy)."""
    out = np.zeros(gpu.n)
    A.check(A.lib().risqgpu_self_energy(gpu._h, float(energy), float(gmin), A.ptr(out, A._dp)), gpu._h)
    return out


def target_factors(diag, S, energy):
    """f_i = sqrt((H_ii - E) / (H_ii - E + S_i)) clipped to [0.25, 4] (S_i <= 0); 1 where
    H_ii <= E.  The denominator is held at >= (H_ii - E) / 16, the clip's upper end."""
    gap = np.asarray(diag, dtype=np.float64) - energy
    with np.errstate(divide="ignore", invalid="ignore"):
        den = np.maximum(gap + S, gap / 16.0)
        f = np.sqrt(gap / den)
    return np.where(gap > 0, np.clip(f, 0.25, 4.0), 1.0).astype(np.float32)


def training_samples(gpu, dets, diag, ints, n_energies=12, per_energy=50000, rng=None, max_iter=2000,
                     universal=False):
    """(features, targets, weights) of one training system with a built FP64 matrix."""
    rng = rng or np.random.default_rng(0)
    lams = []
    lam_star, _, iters = dpr_trajectory(gpu.matrix_vector_prod, diag, tol=1e-4, etol=1e-8, max_iter=max_iter,
                                        record=lambda k, lam, x, r: lams.append(float(lam)))
    f = target_factors(diag, self_energy(gpu, lam_star), lam_star)
    pick = np.asarray(lams)[np.unique(np.linspace(0, len(lams) - 1, n_energies).astype(int))]
    N = len(diag)
    feats, targets = [], []
    for E in pick:
        idx = np.sort(rng.choice(N, size=min(per_energy, N), replace=False))
        feats.append((universal_features if universal else raw_features)(dets[idx], diag[idx], E, ints))
        targets.append(f[idx])
    F = np.concatenate(feats)
    return F, np.concatenate(targets), np.ones(len(F), dtype=np.float32), dict(energy=lam_star, iters=iters)


def grad(model: PrecondMLP, feats, target, weight, device=0):
    """Loss and gradient of one batch on the device (risqgpu_mlp_grad)."""
    X = np.ascontiguousarray(feats, dtype=np.float32)
    t = np.ascontiguousarray(target, dtype=np.float32)
    w = np.ascontiguousarray(weight, dtype=np.float32)
    p = np.ascontiguousarray(model.params, dtype=np.float32)
    g = np.zeros_like(p)
    loss = C.c_float()
    A.check(A.lib().risqgpu_mlp_grad(device, model.n_in, model.hidden, A.ptr(p, A._fp), A.ptr(X, A._fp),
                                     A.ptr(t, A._fp), A.ptr(w, A._fp), X.shape[0], C.byref(loss), A.ptr(g, A._fp)))
    return loss.value, g


def train(model: PrecondMLP, feats, target, weight, epochs=20, batch=4096, lr=1e-3, seed=0, device=0):
    """Adam on the device (risqgpu_mlp_train); returns the per-epoch loss."""
    X = np.ascontiguousarray(feats, dtype=np.float32)
    t = np.ascontiguousarray(target, dtype=np.float32)
    w = np.ascontiguousarray(weight, dtype=np.float32)
    p = np.ascontiguousarray(model.params, dtype=np.float32).copy()
    hist = np.zeros(epochs, dtype=np.float32)
    A.check(A.lib().risqgpu_mlp_train(device, model.n_in, model.hidden, A.ptr(p, A._fp), A.ptr(X, A._fp),
                                      A.ptr(t, A._fp), A.ptr(w, A._fp), X.shape[0], epochs, batch, lr, seed,
                                      A.ptr(hist, A._fp)))
    model.params = p
    return hist


def train_from_systems(systems, norb, epochs=30, batch=4096, lr=1e-3, seed=0, device=0, n_energies=12,
                       per_energy=50000, log=print, universal=False):
    """systems: list of (ints, dets, diag).  Builds the samples (FP64 matrix and FP64
    DPR Davidson per system), fits the feature normalisation and trains a fresh network
    (universal: of the universal layout, norb ignored)."""
    from .gpu import GpuHam
    F, T, Wt = [], [], []
    rng = np.random.default_rng(seed)
    for k, (ints, dets, diag) in enumerate(systems):
        with GpuHam(ints, device) as g:
            g.set_dets(dets, 0, diag)
            g.build(A.FP64)
            f, t, w, info = training_samples(g, dets, diag, ints, n_energies=n_energies, per_energy=per_energy,
                                             rng=rng, universal=universal)
        F.append(f); T.append(t); Wt.append(w)
        log(f"# training system {k}: {len(dets)} dets, E = {info['energy']:.8f} after {info['iters']} DPR "
            f"iterations, {len(t)} samples, target factor median {np.median(t):.3f}")
    raw = np.concatenate(F)
    n2 = raw.shape[1] - 2
    mu_e, sd_e = float(raw[:, n2].mean()), float(raw[:, n2].std() + 1e-6)
    mu_h, sd_h = float(raw[:, n2 + 1].mean()), float(raw[:, n2 + 1].std() + 1e-6)
    model = PrecondMLP.init(NMAX if universal else norb, seed=seed, fnorm=[mu_e, 1.0 / sd_e, mu_h, 1.0 / sd_h])
    if universal:
        # slots that no training system fills keep weight 0, so that they add nothing
        # for larger systems
        W1, b1, W2, b2, W3, b3 = model.split()
        nmax_seen = max(ints.norb for ints, _, _ in systems)
        W1 = W1.copy()
        W1[:, nmax_seen:NMAX] = 0.0
        W1[:, NMAX + nmax_seen:2 * NMAX] = 0.0
        model.params = PrecondMLP.pack(W1, b1, W2, b2, W3, b3)
    feats = normalise(raw, model.fnorm)
    hist = train(model, feats, np.concatenate(T), np.concatenate(Wt), epochs=epochs, batch=batch, lr=lr, seed=seed,
                 device=device)
    return model, hist


__all__ = ["PrecondMLP", "install", "device_factors", "raw_features", "normalise", "dpr_trajectory",
           "NMAX", "orbital_ranks", "universal_features", "adapt", "n_electrons",
           "self_energy", "target_factors", "training_samples", "grad", "train", "train_from_systems",
           "load_default", "default_model_path", "universal_model_path", "dets_to_ints"]
