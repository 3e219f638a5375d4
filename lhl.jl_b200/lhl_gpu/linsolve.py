"""The solver-interface route of the reference (README.md:56-70): LinearSolve.jl's
`LHLFactorization` consumes a `SciMLOperators.WOperator`, the split W = J - M/gamma an implicit
ODE solver builds, and moves the shift with `update_gamma!`, reusing the reduction of J.

Here the same use on the device, host side only: the reduction is done once, `update_gamma`
loads the shift (sigma, tau) = (-m/gamma, 1), and `solve` is lhl_ldiv! followed by refinement to
a tolerance.  For a mass matrix M = m I that shift factorises W exactly.  Any other M (a diagonal
given as a vector, or a matrix) is handled as the reference's lhl_refine! allows, with the
caller's system matrix: the shift uses m = the mean of M's diagonal, W = J - M/gamma is formed on
the device, and GMRES-IR with W itself (lhl_refine_system_gmres) takes the solve to the
tolerance; that works while M/gamma stays close enough to (m/gamma) I relative to W.
LinearSolve.jl and SciMLOperators.jl are not in the reference tree and their versions are not
pinned: the semantics follow the README's description (W = J - M/gamma), and parity with those
packages is unpinned."""
from __future__ import annotations

import torch

from . import (LHL_PREC_FP64, LHL_PREC_MIXED, ArgumentError, DimensionMismatch, LHLShift, lhl, lhl_ldiv_,
               lhl_refine_gmres_, lhl_refine_system_, lhl_refine_tol_, lhl_shift_)


class LHLFactorization:
    """``init(LinearProblem(W, b), LHLFactorization())`` for ``W = WOperator(M, gamma, J)``: one
    reduction of J, a new shift per ``update_gamma``, solves refined to ``tol`` (for M = m I:
    fixed-point for the plain form, GMRES-IR for the mixed one; for any other M: GMRES-IR with W
    itself)."""

    def __init__(self, J: torch.Tensor, gamma: float, mass_matrix=1.0, precision: int = LHL_PREC_FP64,
                 tol: float = 1e-10, max_steps: int = 8):
        n = J.shape[0]
        self.M = None  # a mass matrix other than m I, as a dense device matrix
        if isinstance(mass_matrix, torch.Tensor) and mass_matrix.numel() != 1:
            Md = mass_matrix.to(device=J.device, dtype=J.dtype)
            if Md.dim() == 1:
                if Md.shape[0] != n:
                    raise DimensionMismatch(f"the mass matrix diagonal has length {Md.shape[0]}, J is {n}x{n}")
                Md = torch.diag(Md)
            elif tuple(Md.shape) != (n, n):
                raise DimensionMismatch(f"the mass matrix is {tuple(Md.shape)}, J is {n}x{n}")
            self.M = Md
            mass_matrix = float(torch.diagonal(Md).mean().real.item())
            if mass_matrix == 0.0:
                raise ArgumentError("the mass matrix's diagonal averages to zero: no shift approximates W")
        elif isinstance(mass_matrix, torch.Tensor):
            mass_matrix = float(mass_matrix.item())
        self.m = float(mass_matrix)
        self.W = None
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
        if self.M is not None:
            self.W = self.J - self.M / gamma
        return self

    @property
    def sigma_tau(self):
        return -self.m / self.gamma, 1.0

    def solve(self, b: torch.Tensor) -> torch.Tensor:
        """``solve!(cache).u``: x with ||b - W x|| / ||b|| <= tol (as far as FP64 allows)."""
        x = lhl_ldiv_(b.clone(), self.ws)
        if self.M is not None:
            lhl_refine_system_(x, self.W, b, self.ws, self.max_steps, tol=self.tol, gmres=True)
        elif self.precision == LHL_PREC_MIXED:
            lhl_refine_gmres_(x, self.J, b, self.ws.shift, self.ws, tol=self.tol, max_cycles=self.max_steps)
        else:
            lhl_refine_tol_(x, self.J, b, self.ws.shift, self.ws, tol=self.tol, max_steps=self.max_steps)
        return x
