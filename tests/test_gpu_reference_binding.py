"""The reference-side binding (nngpr_b200.reference_binding.b200_backed) run through the
reference's own known-answer tests.

The reference's estimator class (NumpyNngpr, imported from the installed reference under
baseline/_ref) gets its fit-step log-likelihood and only-train predict from this library; the
reference's NngprTester (nngpr/test/nngpr_base_tester.py:118-257) then checks, with its own
tolerances (1e-10 against scikit-learn's exact GP at num_nn = n):
  * test_same_lkl: log-likelihood and gradient, y_dim 1 and 100 (:174-192);
  * test_same_fit_results: the fitted hyperparameters of scikit-learn's L-BFGS-B loop driving the
    binding's log-likelihood (:194-205);
  * test_predict_same_results: posterior mean / std for 'only-train' (the binding) and, through
    the reference's own code, 'full' and 'full-double-nn' (:228-257);
  * test_prior_predict_same_results: the unfitted prior (:207-226, the reference's code).
The reference's worker pools are replaced by its 'sequential' distribution: a pool forked after
the first CUDA call is not safe.
"""
import os
import sys
import unittest

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, 'baseline', '_ref')

pytestmark = pytest.mark.gpu


def _tester_class(calls):
    if not os.path.isdir(os.path.join(REF, 'nngpr', 'test')):
        pytest.skip('the reference is not installed under baseline/_ref')
    if REF not in sys.path:
        sys.path.insert(0, REF)
    from nngpr.numpy_nngpr import NumpyNngpr
    from nngpr.test.nngpr_base_tester import NngprTester

    from nngpr_b200.reference_binding import b200_backed

    Backed = b200_backed(NumpyNngpr)

    class Counted(Backed):
        def log_marginal_likelihood(self, theta=None, eval_gradient=False, clone_kernel=True):
            if theta is not None:
                calls['lml'] += 1
            return super().log_marginal_likelihood(theta, eval_gradient, clone_kernel)

        def predict(self, X, return_std=False, return_cov=False, conditioning_method=None):
            if not return_cov and conditioning_method in (None, 'only-train') and hasattr(self, 'X_train_'):
                calls['predict'] += 1
            return super().predict(X, return_std=return_std, return_cov=return_cov,
                                   conditioning_method=conditioning_method)

    class TestB200Backed(NngprTester, unittest.TestCase):
        def get_gpr(self, fixed_bounds=False, kernel=None, num_nn=8, **kwargs):
            if kernel is None:
                kernel = self.get_kern(fixed_bounds=fixed_bounds)
            kwargs['batch_size'] = kwargs.get('batch_size', 7)
            kwargs['distribute_method'] = 'sequential'
            return Counted(kernel=kernel, num_nn=num_nn, **kwargs)

    return TestB200Backed


@pytest.mark.parametrize('method', ['test_same_lkl', 'test_same_fit_results', 'test_predict_same_results',
                                    'test_prior_predict_same_results'])
def test_reference_known_answers_through_the_binding(method):
    calls = {'lml': 0, 'predict': 0}
    T = _tester_class(calls)
    result = unittest.TestResult()
    T(method).run(result)
    problems = [f'{t}: {tb}' for t, tb in result.failures + result.errors]
    assert result.wasSuccessful() and not problems, '\n'.join(problems)
    if method in ('test_same_lkl', 'test_same_fit_results'):
        assert calls['lml'] > 0  # the binding's log-likelihood ran, not the reference's
    if method == 'test_predict_same_results':
        assert calls['predict'] > 0 and calls['lml'] > 0
