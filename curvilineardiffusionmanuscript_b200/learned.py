"""Learned initial guess: host side of include/cdm_net.h.

The network, its training step (features → forward → loss → backward →
Adam) and its prediction run in the library's CUDA kernels; this module only
holds handles, generates training trajectories with the APT solver itself,
samples crops and drives the optimisation loop.

No counterpart in the reference: the reference starts each step from
u = Tⁿ (src/pseudo_transient/PseudoTransientSolver.jl:229).  The guess
replaces that start only; the APT iteration still runs to the stopping
point of the plain start (see cdm_apt_set_guess_net).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib as L
from .solver import APTError, PseudoTransientSolver, step


def log_jmean(mesh) -> float:
    """log of the mean cell Jacobian over the domain (the network's J reference)."""
    h = mesh.nhalo
    J = mesh.cell_J[h:h + mesh.nj, h:h + mesh.ni]
    return float(math.log(float(J.double().mean())))


class GuessNet:
    """cdm_net handle: a 4-level bf16 U-Net (32 channels) on one GPU."""

    def __init__(self, seed: int = 0, device: int = 0, stream: Optional[int] = None):
        self._lib = L.load()
        h = C.c_void_p()
        rc = self._lib.cdm_net_create(device, seed, stream, C.byref(h))
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())
        self._h = h
        n = C.c_int64(0)
        self._lib.cdm_net_num_params(h, C.byref(n))
        self.nparams = n.value
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cdm_net_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())

    @property
    def handle(self):
        return self._h

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.nparams, dtype=np.float32)
        self._ck(self._lib.cdm_net_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        self._ck(self._lib.cdm_net_set_params(self._h, p.ctypes.data))

    def get_grads(self) -> np.ndarray:
        g = np.zeros(self.nparams, dtype=np.float32)
        self._ck(self._lib.cdm_net_get_grads(self._h, g.ctypes.data))
        return g

    def save(self, path):
        np.savez_compressed(path, params=self.get_params())

    def load(self, path):
        self.set_params(np.load(path)["params"])

    def forward(self, x_bf16: torch.Tensor) -> torch.Tensor:
        """x: [B, H, W, 16] torch.bfloat16 on the GPU → y [B, H, W, 16] float32."""
        assert x_bf16.dtype == torch.bfloat16 and x_bf16.is_cuda and x_bf16.is_contiguous()
        B, H, W, c = x_bf16.shape
        assert c == 16
        y = torch.empty((B, H, W, 16), dtype=torch.float32, device=x_bf16.device)
        torch.cuda.current_stream(x_bf16.device).synchronize()
        self._ck(self._lib.cdm_net_forward(self._h, x_bf16.data_ptr(), B, H, W, y.data_ptr()))
        return y

    def backward(self, target: torch.Tensor) -> float:
        """Mean squared error of channel 0 of the last forward against target [B, H, W]."""
        target = target.contiguous().float()
        torch.cuda.current_stream(target.device).synchronize()
        loss = C.c_float(0.0)
        self._ck(self._lib.cdm_net_backward(self._h, target.data_ptr(), C.byref(loss)))
        return loss.value

    def set_smoothing(self, passes: int):
        """3x3 binomial passes applied to the predicted correction (default 8)."""
        self._ck(self._lib.cdm_net_set_guess_smoothing(self._h, int(passes)))

    def train_step(self, frames: Sequence[torch.Tensor], idx: Sequence[int], ox: Sequence[int],
                   oy: Sequence[int], crop: int, mesh, k0: float, kn: float, lr: float, ljm: float,
                   dt: float = 0.0, rho_cp: float = 1.0) -> float:
        """One Adam step on crops: sample b uses frames[idx[b] − 1, idx[b], idx[b] + 1].
        dt > 0 weights each pixel's error by 1 + κΔt/(16ρcₚJ)."""
        n = len(idx)
        torch.cuda.current_stream(frames[0].device).synchronize()
        P = C.c_void_p * n
        tp = P(*[frames[i - 1].data_ptr() for i in idx])
        tc = P(*[frames[i].data_ptr() for i in idx])
        tn = P(*[frames[i + 1].data_ptr() for i in idx])
        ax = (C.c_int * n)(*[int(v) for v in ox])
        ay = (C.c_int * n)(*[int(v) for v in oy])
        b = L.NetBatch(n, C.cast(tp, C.POINTER(C.c_void_p)), C.cast(tc, C.POINTER(C.c_void_p)),
                       C.cast(tn, C.POINTER(C.c_void_p)), mesh.cell_J.data_ptr(),
                       C.cast(ax, C.POINTER(C.c_int)), C.cast(ay, C.POINTER(C.c_int)),
                       crop, mesh.ni, mesh.nj, mesh.nhalo, k0, kn, ljm, dt, rho_cp)
        loss = C.c_float(0.0)
        self._ck(self._lib.cdm_net_train_step(self._h, C.byref(b), lr, C.byref(loss)))
        return loss.value

    def predict(self, tprev: torch.Tensor, tcur: torch.Tensor, mesh, k0: float, kn: float,
                ljm: float) -> torch.Tensor:
        """Guess for the step after tcur (full array)."""
        torch.cuda.current_stream(tcur.device).synchronize()
        u0 = torch.empty_like(tcur)
        self._ck(self._lib.cdm_net_predict(self._h, tprev.data_ptr(), tcur.data_ptr(), mesh.cell_J.data_ptr(),
                                           mesh.ni, mesh.nj, mesh.nhalo, k0, kn, ljm, u0.data_ptr()))
        return u0


def attach(solver: PseudoTransientSolver, net: Optional[GuessNet], mesh=None):
    """Let `solver` start steps run with guess=CDM_GUESS_LEARNED from the network."""
    ljm = log_jmean(mesh or solver.mesh)
    rc = solver._lib.cdm_apt_set_guess_net(solver._h, net.handle if net is not None else None, ljm)
    if rc != L.CDM_OK:
        raise APTError(rc, L.last_error())


def generate_trajectories(make_problem, seeds: Sequence[int], nsteps: int, precision: str = "fp64",
                          rtol: float = 1e-8, atol: float = 1e-8, max_iter: int = 100000,
                          skipped: Optional[list] = None) -> List[List[torch.Tensor]]:
    """APT trajectories (nsteps + 1 frames, full arrays on the GPU) of the problems
    make_problem(seed) for each seed, advanced by the library's own solver.  A
    seed whose APT iteration fails (the pseudo-transient iteration itself can
    diverge on steep initial states, as the reference's does) is left out and
    appended to `skipped`."""
    out = []
    for seed in seeds:
        pr = make_problem(seed)
        g = PseudoTransientSolver(pr.mesh, pr.bcs, precision=precision)
        T = pr.T0.clone()
        frames = [T.clone()]
        try:
            for _ in range(nsteps):
                step(g, pr.mesh, T, pr.rho, pr.cp, pr.kappa, pr.dt, rtol=rtol, atol=atol, max_iter=max_iter)
                frames.append(T.clone())
        except APTError:
            if skipped is not None:
                skipped.append(seed)
            continue
        finally:
            g.close()
        out.append(frames)
    return out


def train(net: GuessNet, trajs: List[List[torch.Tensor]], mesh, k0: float, kn: float, steps: int,
          batch: int = 16, crop: int = 128, lr: float = 1e-3, seed: int = 0, log_every: int = 0,
          dt: float = 0.0, rho_cp: float = 1.0) -> List[float]:
    """Adam on random crops of random (Tⁿ⁻¹, Tⁿ, Tⁿ⁺¹) triples; cosine learning-rate decay.
    dt > 0 weights the loss by the local diffusion number (see cdm_net_batch)."""
    rng = np.random.default_rng(seed)
    ljm = log_jmean(mesh)
    triples = [(t, i) for t, fr in enumerate(trajs) for i in range(1, len(fr) - 1)]
    crop = min(crop, mesh.ni - mesh.ni % 8, mesh.nj - mesh.nj % 8)
    losses = []
    for s in range(steps):
        pick = rng.integers(0, len(triples), size=batch)
        frames, idx = [], []
        for k in pick:
            t, i = triples[k]
            base = len(frames)
            frames += [trajs[t][i - 1], trajs[t][i], trajs[t][i + 1]]
            idx.append(base + 1)
        ox = rng.integers(0, mesh.ni - crop + 1, size=batch)
        oy = rng.integers(0, mesh.nj - crop + 1, size=batch)
        a = lr * 0.5 * (1.0 + math.cos(math.pi * s / max(1, steps)))
        losses.append(net.train_step(frames, idx, ox, oy, crop, mesh, k0, kn, a, ljm, dt, rho_cp))
        if log_every and (s % log_every == 0 or s == steps - 1):
            print(f"[train] step {s} loss {losses[-1]:.4e} lr {a:.2e}", flush=True)
    return losses
