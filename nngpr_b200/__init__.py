"""nngpr_b200 — the NNGP fit/predict hot path of stavoltafunzia/nngpr on one NVIDIA B200.

* ``B200Nngpr``: scikit-learn estimator, drop-in for the reference ``NumpyNngpr``/``TorchNngpr``.
* ``ops``: torch-facing calls of the C ABI (``include/nngp_b200.h``, ``libnngp_b200.so``).
* ``kernel_params``: reduction of a kernel tree to ``White + const + rbf_level * RBF``.
* ``autograd``: the log-likelihood as a ``torch.autograd.Function`` and an L-BFGS fit on it.
* ``plain``: the plain FP32 GPU form (the benchmark's comparator).
"""

from .kernel_params import RbfParams, extract  # noqa: F401

__all__ = ['B200Nngpr', 'RbfParams', 'extract', 'ops']


def __getattr__(name):
    # torch-dependent modules are imported lazily so that CPU-only tooling can import the package
    import importlib
    if name == 'B200Nngpr':
        return importlib.import_module('.estimator', __name__).B200Nngpr
    if name in ('ops', 'estimator', 'autograd', 'plain'):
        return importlib.import_module('.' + name, __name__)
    raise AttributeError(name)
