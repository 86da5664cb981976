"""The linearised nonlinear term as a linear operator for Krylov methods.

SFEMaNS's stability and adjoint analyses go through LightKrylov linear
operators (SOURCES/LIGHTKRYLOV_OBJECTS/exponential_propagator.F90:61-62:
``exptA_linop`` with ``matvec`` and ``rmatvec``, the latter bound to the
forward map because the reference has no adjoint).  This module exposes the
Jacobian of the dealiased product N(u, w) = u x w about a base state as such an
operator, with ``matvec`` = the JVP (du, dw) -> du x w + u x dw and ``rmatvec``
= its exact transpose (the VJP), both on the GPU through the C-ABI:

* :class:`CrossJacobian` acts on CUDA tensors in the Fortran coefficient
  layout, one tangent or a batch of k tangents per call;
* :meth:`CrossJacobian.as_linear_operator` wraps it as a
  ``scipy.sparse.linalg.LinearOperator`` on flat float64 vectors, so that SciPy's
  Krylov routines (``svds``, ``lsqr``, ``gmres`` on normal equations ...) drive it
  as LightKrylov's ``svds`` / ``lsqr`` drive ``abstract_linop_rdp``; the Fortran
  counterpart is ``sfemans_b200/fortran/nl_linop.F90``.

The operator is rectangular (12 coefficient slots in, 6 out per point and
mode): ``eigs`` of a stability operator additionally needs the linearised time
stepper (the FEM solve), which is the caller's.
"""
from __future__ import annotations


class CrossJacobian:
    """J(du, dw) = du x w + u x dw about (u, w), both (np, 6, m) CUDA tensors in Fortran order."""

    def __init__(self, u, w, m_max_pad: int | None = None):
        from . import fortran_empty

        if u.shape != w.shape or u.dim() != 3 or u.shape[1] != 6:
            raise ValueError("u and w must be (np, 6, m) tensors of the same shape")
        self.u, self.w = u, w
        self.np, _, self.m = u.shape
        self.pad = m_max_pad or max(1, 3 * self.m // 2)
        self._empty = fortran_empty

    @property
    def shape(self):
        """(rows, columns) of the operator on flattened coefficient arrays."""
        return (self.np * 6 * self.m, self.np * 12 * self.m)

    def matvec(self, tan, out=None):
        """JVP: tan (np, 12, m[, k]) = (du, dw) -> (np, 6, m[, k])."""
        from . import cross_jvp

        return cross_jvp(self.u, self.w, tan, m_max_pad=self.pad, out=out)

    def rmatvec(self, cot, out=None):
        """VJP, the transpose of :meth:`matvec` for the Euclidean inner product of the arrays:
        cot (np, 6, m[, k]) -> (np, 12, m[, k])."""
        from . import cross_vjp

        return cross_vjp(self.u, self.w, cot, m_max_pad=self.pad, out=out)

    def as_linear_operator(self):
        """A ``scipy.sparse.linalg.LinearOperator`` on flat float64 vectors (Fortran order of the arrays);
        each product copies the vector to the device and the result back."""
        import numpy as np
        import torch
        from scipy.sparse.linalg import LinearOperator

        npts, m, dev = self.np, self.m, self.u.device

        def to_dev(v, nslot):
            a = np.asarray(v, dtype=np.float64).reshape((npts, nslot, m), order="F")
            t = torch.from_numpy(np.ascontiguousarray(a.T)).to(dev)
            return t.permute(2, 1, 0)

        def to_flat(t):  # Fortran order of (np, nslot, m[, 1])
            return t.permute(*reversed(range(t.dim()))).contiguous().cpu().numpy().ravel()

        def mv(v):
            return to_flat(self.matvec(to_dev(v, 12)))

        def rmv(c):
            return to_flat(self.rmatvec(to_dev(c, 6)))

        return LinearOperator(self.shape, matvec=mv, rmatvec=rmv, dtype=np.float64)
