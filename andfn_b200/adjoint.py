"""Differentiable DFN solve: gradients with respect to log-transmissivity.

``DFNModel`` keeps one network resident on a GPU.  ``model.solve(logt)``
solves it at transmissivities ``exp(logt)`` (natural log, one value per
fracture) and returns the solved state as torch tensors:

    coef  float64 [ne, MAX_NCOEF, 2]   element coefficients (re, im)
    q     float64 [ne]                 discharges (intersections, constant-head
                                       lines, wells; 0 for the other types)
    C     float64 [nf]                 fracture constants

``model.heads(coef, q, C, logt, frac, z)`` evaluates heads Re Omega_f(z)/t_f
(andfn/hpc/hpc_fracture.py:205-252) at device-resident points.  Both are
``torch.autograd.Function``s: ``J.backward()`` of any objective built from
them runs the library's adjoint (a GMRES solve whose operator is one
transposed sweep of the solve, no stored iterates; include/andfn_b200.h) and
the transposed head evaluation, and leaves dJ/dlogt in ``logt.grad``.

The reference has no derivatives; its solve is what is differentiated
(hpc_solve.solve, andfn/hpc/hpc_solve.py:55-257, with the transmissivities
entering through the intersection update, the 1/t of the intersection rows
and phi = t * head of constant-head lines and wells).  Coefficients must not
grow during the solve (MAX_NCOEF = ncoef).

The library runs on its own CUDA stream; this module synchronises torch's
current stream before every library call and the library synchronises its
own stream before returning, so tensors pass safely both ways.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _ffi
from .records import AndfnAdjointStats
from .solver import Solver


def _ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


class DFNModel:
    def __init__(self, fractures: np.ndarray, elements: np.ndarray, constants, discharge_int: int = 50,
                 device: int = 0, adjoint_tol: float = 1e-10, adjoint_max_iterations: int = 5000):
        self.device = torch.device("cuda", device)
        self.solver = Solver(fractures, elements, discharge_int, device=device)
        self.constants = constants
        self.ne, self.nf = len(elements), len(fractures)
        self.mc = elements.dtype["coef"].shape[0]
        self.adjoint_tol = adjoint_tol
        self.adjoint_max_iterations = adjoint_max_iterations
        self.version = 0  # bumped by every solve; backward passes check it
        self.stats: dict = {}
        self.adjoint_stats: dict = {}

    def close(self):
        self.solver.close()

    def _sync(self):
        torch.cuda.current_stream(self.device).synchronize()

    def _lib(self):
        return _ffi.lib()

    # -- forward pieces ----------------------------------------------------
    def _solve_raw(self, logt: torch.Tensor):
        t = np.exp(logt.detach().to("cpu", torch.float64).numpy())
        t = np.ascontiguousarray(t)
        _ffi.check(self._lib().andfn_b200_set_transmissivity(self.solver._h, t.ctypes.data_as(ctypes.c_void_p)))
        self.stats = self.solver.run(self.constants)
        self.version += 1
        coef = torch.empty((self.ne, self.mc, 2), dtype=torch.float64, device=self.device)
        q = torch.empty(self.ne, dtype=torch.float64, device=self.device)
        C = torch.empty(self.nf, dtype=torch.float64, device=self.device)
        self._sync()
        _ffi.check(self._lib().andfn_b200_state_device(self.solver._h, _ptr(coef), self.mc, _ptr(q), _ptr(C)))
        return coef, q, C

    def solve(self, logt: torch.Tensor):
        """(coef, q, C) of the solve at t = exp(logt); differentiable in logt."""
        return _SolveFn.apply(logt, self)

    def heads(self, coef, q, C, logt, frac: torch.Tensor, z: torch.Tensor):
        """Heads at points z (complex128, device) of fractures frac (int64,
        device) for the state returned by the latest solve()."""
        return _HeadsFn.apply(coef, q, C, logt, self, frac, z)

    def adjoint(self, gcoef: torch.Tensor, gq: torch.Tensor, gC: torch.Tensor) -> torch.Tensor:
        """dJ/dlogt through the latest solve, given dJ/d(coef, q, C)."""
        glogt = torch.empty(self.nf, dtype=torch.float64, device=self.device)
        gcoef = gcoef.detach().to(torch.float64).contiguous()
        gq = gq.detach().to(torch.float64).contiguous()
        gC = gC.detach().to(torch.float64).contiguous()
        st = AndfnAdjointStats()
        self._sync()
        rc = self._lib().andfn_b200_adjoint(self.solver._h, _ptr(gcoef), gcoef.shape[1], _ptr(gq), _ptr(gC),
                                            float(self.adjoint_tol), int(self.adjoint_max_iterations),
                                            _ptr(glogt), ctypes.byref(st))
        self.adjoint_stats = st.as_dict()
        _ffi.check(rc, ok=(0, 1))
        return glogt


class _SolveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, logt, model):
        coef, q, C = model._solve_raw(logt)
        ctx.model = model
        ctx.version = model.version
        return coef, q, C

    @staticmethod
    def backward(ctx, gcoef, gq, gC):
        m = ctx.model
        if m.version != ctx.version:
            raise RuntimeError("the network was solved again after this forward; the adjoint needs the "
                               "converged state of the solve it differentiates")
        z = lambda shape: torch.zeros(shape, dtype=torch.float64, device=m.device)
        gcoef = z((m.ne, m.mc, 2)) if gcoef is None else gcoef
        gq = z(m.ne) if gq is None else gq
        gC = z(m.nf) if gC is None else gC
        return m.adjoint(gcoef, gq, gC), None


class _HeadsFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coef, q, C, logt, model, frac, z):
        frac = frac.to(device=model.device, dtype=torch.int64).contiguous()
        z = z.to(device=model.device, dtype=torch.complex128).contiguous()
        if frac.ndim != 1 or frac.shape != z.shape:
            raise ValueError(f"frac and z must be 1-d tensors of one length (got {tuple(frac.shape)} and "
                             f"{tuple(z.shape)})")
        out = torch.empty(len(frac), dtype=torch.float64, device=model.device)
        model._sync()
        _ffi.check(model._lib().andfn_b200_heads_device(model.solver._h, _ptr(frac), _ptr(z), len(frac),
                                                         _ptr(out)))
        ctx.model = model
        ctx.version = model.version
        ctx.save_for_backward(frac, z)
        return out

    @staticmethod
    def backward(ctx, gh):
        m = ctx.model
        if m.version != ctx.version:
            raise RuntimeError("the network was solved again after this forward")
        frac, z = ctx.saved_tensors
        gh = gh.to(torch.float64).contiguous()
        zeros = lambda shape: torch.zeros(shape, dtype=torch.float64, device=m.device)
        gcoef, gq, gC, glogt = zeros((m.ne, m.mc, 2)), zeros(m.ne), zeros(m.nf), zeros(m.nf)
        m._sync()
        _ffi.check(m._lib().andfn_b200_heads_vjp(m.solver._h, _ptr(frac), _ptr(z), len(frac), _ptr(gh),
                                                  _ptr(gcoef), m.mc, _ptr(gq), _ptr(gC), _ptr(glogt)))
        return gcoef, gq, gC, glogt, None, None, None
