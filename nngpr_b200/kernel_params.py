"""Reduction of a kernel tree to ``White + const + rbf_level * S(length_scale)``.

The GPU path evaluates one kernel family: sums and products of ``WhiteKernel``,
``ConstantKernel`` and one stationary kernel ``S``, either the ``RBF`` the reference
accelerates on CUDA (``nngpr/cuda_kernel_accelerators.py:169-194``) or a ``Matern`` with
nu = 1/2, 3/2 or 5/2 that the reference evaluates on its generic path
(``nngpr/batched_kernels.py:1070-1131``).  This module walks a scikit-learn kernel tree (the
reference's ``nngpr.batched_kernels`` classes subclass the scikit-learn ones, so both are
accepted) and returns

* the parameter values (``extract``; rules of ``RbfAccelerator.get_kernel_params``,
  ``cuda_kernel_accelerators.py:520-581``), and
* the position of each free hyperparameter in ``kernel.theta`` (``theta_map``; rules of
  ``get_kernel_theta_mapping``, ``:583-649``: clone the kernel with known theta values
  and find which ``exp(theta_k)`` each parameter equals).

Any other tree raises ``NotImplementedError("Cannot accelerate this kernel")``, the
reference's error for the same case (``cuda_kernel_accelerators.py:114-115``).  There
is no generic fallback.
"""

from __future__ import annotations

import dataclasses
import numbers

import numpy as np
from sklearn.gaussian_process import kernels as skk


@dataclasses.dataclass
class RbfParams:
    """Parameter values and theta positions of a ``White + const + rbf_level * RBF`` kernel.

    ``idx_*`` are positions in ``kernel.theta`` (``-1``: fixed or absent).  The
    length-scale positions are ``idx_ls, idx_ls + 1, ...`` (one per ARD dimension).
    """

    rbf_level: float = 0.0
    const_value: float = 0.0
    noise_level: float = 0.0
    length_scale: object = None  # None (no RBF), float, or 1-D float64 array
    family: int = 0  # stationary part: 0 RBF, 1/2/3 Matern nu = 1/2, 3/2, 5/2 (NNGP_FAMILY_*)
    idx_rbf_level: int = -1
    idx_const: int = -1
    idx_noise: int = -1
    idx_ls: int = -1
    n_theta: int = 0

    @property
    def ard(self) -> bool:
        return self.length_scale is not None and np.ndim(self.length_scale) > 0

    @property
    def n_ls(self) -> int:
        if self.length_scale is None:
            return 0
        return int(np.size(self.length_scale))

    def ls_vector(self, d: int) -> np.ndarray:
        """Length scale per feature (``1`` everywhere when the kernel has no RBF part)."""
        if self.length_scale is None:
            return np.ones(d)
        ls = np.asarray(self.length_scale, dtype=np.float64).reshape(-1)
        if ls.size == 1:
            return np.full(d, float(ls[0]))
        if ls.size != d:
            raise ValueError(f"length_scale has {ls.size} entries for {d} features")
        return ls


# nngp_kernel.family of the Matern smoothness values (include/nngp_b200.h, NNGP_FAMILY_*)
MATERN_FAMILY = {0.5: 1, 1.5: 2, 2.5: 3}


def _unsupported(msg: str):
    return NotImplementedError("Cannot accelerate this kernel: " + msg)


def _values(kernel) -> dict:
    """Parameter dictionary of a kernel tree (keys ``noise_level``, ``constant_value``,
    ``length_scale``, ``rbf_level``)."""
    if isinstance(kernel, skk.WhiteKernel):
        return {'noise_level': float(kernel.noise_level)}
    if isinstance(kernel, skk.ConstantKernel):
        return {'constant_value': float(kernel.constant_value)}
    if isinstance(kernel, skk.Matern):
        # Matern subclasses RBF in scikit-learn (and in nngpr.batched_kernels), so it is tested
        # first; the reference's generic path evaluates nu = 1/2, 3/2, 5/2 and inf
        # (batched_kernels.py:1070-1131), nu = inf being the RBF
        nu = float(kernel.nu)
        family = 0 if np.isinf(nu) else MATERN_FAMILY.get(nu)
        if family is None:
            raise _unsupported(f"Matern with nu = {nu} (only 0.5, 1.5, 2.5 and inf)")
        ls = kernel.length_scale
        if isinstance(ls, numbers.Number) or np.ndim(ls) == 0:
            return {'length_scale': float(ls), 'family': family}
        return {'length_scale': np.asarray(ls, dtype=np.float64).reshape(-1).copy(), 'family': family}
    if isinstance(kernel, skk.RBF):
        ls = kernel.length_scale
        if isinstance(ls, numbers.Number) or np.ndim(ls) == 0:
            return {'length_scale': float(ls)}
        return {'length_scale': np.asarray(ls, dtype=np.float64).reshape(-1).copy()}
    if isinstance(kernel, skk.Sum):
        a, b = _values(kernel.k1), _values(kernel.k2)
        a_rbf = bool(set(a) - {'noise_level', 'constant_value'})
        b_rbf = bool(set(b) - {'noise_level', 'constant_value'})
        if a_rbf and b_rbf:
            raise _unsupported("a sum of two stationary (RBF / Matern) kernels")
        if a_rbf:
            a, b = b, a
        # a has no RBF part: fold its white/constant terms into b
        for key in ('noise_level', 'constant_value'):
            if key in a or key in b:
                b[key] = a.get(key, 0.0) + b.get(key, 0.0)
        return b
    if isinstance(kernel, skk.Product):
        a, b = _values(kernel.k1), _values(kernel.k2)
        a_const = not (set(a) - {'constant_value'})
        b_const = not (set(b) - {'constant_value'})
        if not a_const and not b_const:
            raise _unsupported("a product whose factors are both non-constant")
        if b_const:
            a, b = b, a
        c = a['constant_value']
        if 'noise_level' in b:
            b['noise_level'] = c * b['noise_level']
        if 'constant_value' in b:
            b['constant_value'] = c * b['constant_value']
        if 'rbf_level' in b or 'length_scale' in b:
            b['rbf_level'] = c * b.get('rbf_level', 1.0)
        return b
    raise _unsupported(f"kernel type {type(kernel).__name__}")


def _base_kernel(kernel):
    """Unwrap the reference's ``BatchedKernelWrapper`` (``batched_kernels.py:41-108``)."""
    return getattr(kernel, 'base_kernel', kernel)


def theta_map(kernel) -> dict:
    """Position of each parameter in ``kernel.theta``.

    Same rule as ``get_kernel_theta_mapping`` (``cuda_kernel_accelerators.py:583-649``):
    clone the kernel with known theta values and find, for every parameter, the one
    position ``k`` whose ``exp(theta_k)`` it equals (within a relative 1e-15); products
    and sums of free parameters match nothing and make the kernel unsupported.  The
    reference probes with ``theta = 0, 1, 2, ...``, so a *fixed* parameter equal to
    ``exp(k)`` (for instance ``ConstantKernel(1.0, constant_value_bounds='fixed')``, the
    reference's default kernel) collides with position ``k`` and its mapping fails with an
    AssertionError.  Here two probes ``theta_k = a (k + 1) + b`` with incommensurate
    ``a, b`` are used and a parameter is mapped only where both agree, which keeps the rule
    and removes the collision.
    """
    kernel = _base_kernel(kernel)
    n = len(kernel.theta)
    eps = 1e-15
    maps = []
    for a_, b_ in ((0.5, 0.1 * np.sqrt(2.0)), (0.3 * np.sqrt(3.0), -0.2 * np.sqrt(5.0))):
        probe_theta = a_ * np.arange(1, n + 1, dtype=np.float64) + b_
        expected = np.exp(probe_theta)
        vals = _values(kernel.clone_with_theta(probe_theta))

        def hits(v):
            return np.flatnonzero((v < expected * (1 + eps)) & (v > expected * (1 - eps)))

        out = {}
        for key, v in vals.items():
            if key == 'length_scale' and np.ndim(v) > 0:
                found = []
                for comp in np.asarray(v).reshape(-1):
                    h = hits(comp)
                    if h.size == 1:
                        found.append(int(h[0]))
                if not found:
                    continue
                found = sorted(set(found))
                if len(found) > np.size(v):
                    raise _unsupported("ambiguous theta mapping for length_scale")
                if len(found) != np.size(v) or (len(found) > 1 and set(np.diff(found)) != {1}):
                    raise _unsupported("length_scale entries are not adjacent free hyperparameters")
                out[key] = found
            else:
                h = hits(v)
                if h.size > 1:
                    raise _unsupported(f"ambiguous theta mapping for {key}")
                if h.size == 1:
                    out[key] = int(h[0])
        maps.append(out)
    out = {k: v for k, v in maps[0].items() if maps[1].get(k) == v}
    found = sum(len(v) if isinstance(v, list) else 1 for v in out.values())
    if found != n:
        raise _unsupported("cannot map every kernel hyperparameter to theta")
    return out


def extract(kernel) -> RbfParams:
    """Parameter values plus theta map of a supported kernel; raises ``NotImplementedError``
    for every other kernel."""
    kernel = _base_kernel(kernel)
    vals = _values(kernel)
    tmap = theta_map(kernel)
    p = RbfParams()
    p.noise_level = float(vals.get('noise_level', 0.0))
    p.const_value = float(vals.get('constant_value', 0.0))
    if 'length_scale' in vals:
        p.length_scale = vals['length_scale']
        p.rbf_level = float(vals.get('rbf_level', 1.0))
        p.family = int(vals.get('family', 0))
    else:
        p.length_scale = None
        p.rbf_level = 0.0
    p.idx_noise = tmap.get('noise_level', -1)
    p.idx_const = tmap.get('constant_value', -1)
    p.idx_rbf_level = tmap.get('rbf_level', -1)
    ls_idx = tmap.get('length_scale', -1)
    p.idx_ls = ls_idx[0] if isinstance(ls_idx, list) else ls_idx
    p.n_theta = len(kernel.theta)
    return p


def params_from_theta(template: RbfParams, theta) -> RbfParams:
    """The parameters of ``template``'s kernel at log-hyperparameters ``theta`` (the values a
    ``kernel.clone_with_theta(theta)`` would hold): every free hyperparameter is ``exp`` of its
    theta entry, fixed ones keep the template's value."""
    th = np.asarray(theta, dtype=np.float64).reshape(-1)
    if th.size != template.n_theta:
        raise ValueError(f'theta has {th.size} entries, the kernel {template.n_theta}')
    p = dataclasses.replace(template)
    if template.idx_rbf_level >= 0:
        p.rbf_level = float(np.exp(th[template.idx_rbf_level]))
    if template.idx_const >= 0:
        p.const_value = float(np.exp(th[template.idx_const]))
    if template.idx_noise >= 0:
        p.noise_level = float(np.exp(th[template.idx_noise]))
    if template.idx_ls >= 0 and template.length_scale is not None:
        if template.ard:
            p.length_scale = np.exp(th[template.idx_ls:template.idx_ls + template.n_ls])
        else:
            p.length_scale = float(np.exp(th[template.idx_ls]))
    return p
