"""The solver-interface route of the reference (README.md:56-70): LinearSolve.jl's
`LHLFactorization` consumes a `SciMLOperators.WOperator`, the split W = J - M/gamma an implicit
ODE solver builds, and moves the shift with `update_gamma!`, reusing the reduction of J.

Here the same use on the device, host side only: the reduction is done once, `update_gamma`
loads the shift (sigma, tau) = (-m/gamma, 1) for a mass matrix M = m I, and `solve` is
lhl_ldiv! followed by refinement to a tolerance.  LinearSolve.jl and SciMLOperators.jl are not
in the reference tree and their versions are not pinned: the semantics follow the README's
description (W = J - M/gamma), and parity with those packages is unpinned.  Only a scalar mass
matrix fits the algorithm's sigma I + tau J form; any other M is an ArgumentError."""
from __future__ import annotations

import torch

from . import (LHL_PREC_FP64, LHL_PREC_MIXED, ArgumentError, LHLShift, lhl, lhl_ldiv_, lhl_refine_gmres_,
               lhl_refine_tol_, lhl_shift_)


class LHLFactorization:
    """``init(LinearProblem(W, b), LHLFactorization())`` for ``W = WOperator(M, gamma, J)``,
    M = m I: one reduction of J, a new shift per ``update_gamma``, solves refined to ``tol``
    (fixed-point for the plain form, GMRES-IR for the mixed one)."""

    def __init__(self, J: torch.Tensor, gamma: float, mass_matrix=1.0, precision: int = LHL_PREC_FP64,
                 tol: float = 1e-10, max_steps: int = 8):
        if isinstance(mass_matrix, torch.Tensor):
            if mass_matrix.numel() != 1:
                raise ArgumentError("the mass matrix must be a multiple of the identity (sigma I + tau J form)")
            mass_matrix = float(mass_matrix.item())
        self.m = float(mass_matrix)
        self.J = J
        self.ws = lhl(J, precision=precision)
        self.tol = float(tol)
        self.max_steps = int(max_steps)
        self.precision = precision
        self.gamma = None
        self.update_gamma(gamma)

    def update_gamma(self, gamma: float) -> "LHLFactorization":
        """``update_gamma!(cache, gamma)``: W = J - (m / gamma) I, O(n^2); the reduction stays."""
        gamma = float(gamma)
        if gamma == 0.0:
            raise ArgumentError("gamma must be nonzero")
        self.gamma = gamma
        lhl_shift_(self.ws, -self.m / gamma, 1.0)
        return self

    @property
    def sigma_tau(self):
        return -self.m / self.gamma, 1.0

    def solve(self, b: torch.Tensor) -> torch.Tensor:
        """``solve!(cache).u``: x with ||b - W x|| / ||b|| <= tol (as far as FP64 allows)."""
        x = lhl_ldiv_(b.clone(), self.ws)
        if self.precision == LHL_PREC_MIXED:
            lhl_refine_gmres_(x, self.J, b, self.ws.shift, self.ws, tol=self.tol, max_cycles=self.max_steps)
        else:
            lhl_refine_tol_(x, self.J, b, self.ws.shift, self.ws, tol=self.tol, max_steps=self.max_steps)
        return x
