"""Generate the golden vectors in ``tests/golden/*.npz`` by running the reference nngpr.

Run in a container that has the reference source (stavoltafunzia/nngpr 0.1.1)::

    python tests/golden/make_golden.py --ref <path of the reference checkout>

(or with the path in the environment variable NNGPR_REFERENCE).

Every value stored here comes from the reference's own ``NumpyNngpr`` (FP64,
``allow_downcast_f32='no'``, ``distribute_method='sequential'``) or from
scikit-learn's exact ``GaussianProcessRegressor`` on the reference's own test
fixture (``nngpr/test/nngpr_base_tester.py:121-131``).  The inputs are stored
beside the outputs, so the tests never need the reference or the RNG streams.
"""

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _import_reference(path):
    sys.path.insert(0, path)
    from nngpr.numpy_nngpr import NumpyNngpr, NumpyWorker  # noqa: E402
    from nngpr import batched_kernels as bk  # noqa: E402
    return NumpyNngpr, NumpyWorker, bk


def _ref_fit_neighbours(gpr, worker, x, kernel, m):
    """Neighbour lists exactly as ``_log_likelihood_worker`` builds them for one chunk
    starting at 0 (``base_nngpr.py:530-535``), without the self column."""
    return np.asarray(gpr._find_nearest_neighbors_wrapper(
        worker, x, x, kernel, min(m, x.shape[0] - 1), ref_cut_index=0))


def _ref_predict_neighbours(gpr, worker, xt, xq, kernel, m):
    """Neighbour lists of ``_find_nn_indices_for_train_and_eval`` (only-train branch,
    ``base_nngpr.py:1454-1459``), without the self column."""
    return np.asarray(gpr._find_nearest_neighbors_wrapper(
        worker, xt, xq, kernel, min(m, xt.shape[0]), ref_cut_index=None))


def case(name, NumpyNngpr, NumpyWorker, kernel_fn, x, y, xq, m, theta_eval=None, normalize_y=False, alpha=1e-10):
    out = {'x': x, 'y': y, 'xq': xq, 'num_nn': np.int64(m), 'alpha': np.float64(alpha),
           'normalize_y': np.bool_(normalize_y)}
    # FP64 everywhere: the reference's most precise configuration
    gpr = NumpyNngpr(kernel=kernel_fn(), num_nn=m, optimizer=None, alpha=alpha, normalize_y=normalize_y,
                     allow_downcast_f32='no', distribute_method='sequential', num_workers=1)
    gpr.fit(x, y)
    theta = gpr.kernel_.theta.copy() if theta_eval is None else np.asarray(theta_eval, dtype=np.float64)
    lml, grad = gpr.log_marginal_likelihood(theta, eval_gradient=True)
    out['theta'] = theta
    out['theta_pred'] = gpr.kernel_.theta.copy()  # predict uses the fitted kernel
    out['lml'] = np.float64(lml)
    out['grad'] = np.asarray(grad, dtype=np.float64)
    mean, std = gpr.predict(xq, return_std=True)
    out['pred_mean'] = np.asarray(mean)
    out['pred_std'] = np.asarray(std)
    worker = NumpyWorker()
    kern = gpr.kernel_.clone_with_theta(theta)
    out['nbr_fit_f64'] = _ref_fit_neighbours(gpr, worker, x, kern, m)
    out['nbr_pred_f64'] = _ref_predict_neighbours(gpr, worker, x, xq, kern, m)
    # default precision of the search ('only-nn': float32 kernel-space search)
    gpr32 = NumpyNngpr(kernel=kernel_fn(), num_nn=m, optimizer=None, alpha=alpha, normalize_y=normalize_y,
                       distribute_method='sequential', num_workers=1)
    out['nbr_fit_f32'] = _ref_fit_neighbours(gpr32, worker, x, kern, m)
    np.savez_compressed(os.path.join(HERE, name + '.npz'), **out)
    print(name, 'lml', lml, 'grad', grad)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=os.environ.get('NNGPR_REFERENCE'),
                    help='directory holding the reference package nngpr (default: $NNGPR_REFERENCE)')
    ap.add_argument('--only', default='', help='comma-separated case groups to (re)generate: rbf,matern')
    args = ap.parse_args()
    if not args.ref:
        ap.error('give the reference checkout with --ref or NNGPR_REFERENCE')
    NumpyNngpr, NumpyWorker, bk = _import_reference(args.ref)
    only = set(filter(None, args.only.split(',')))
    if 'full' in only:
        return full_cases(NumpyNngpr, NumpyWorker, bk)
    if 'wide' in only:
        return wide_case(NumpyNngpr, NumpyWorker, bk)
    if only and 'rbf' not in only:
        return matern_cases(NumpyNngpr, NumpyWorker, bk)

    # 1. CPU-oracle workload: n=2000, x~U[0,1]^3, y=sin(2 pi x1)+cos(2 pi x2) x3+N(0,0.1^2), m=16,
    #    C(1.0)*RBF(0.3)+White(0.01), 500 test points, seed 0
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 1, (2000, 3))
    y = np.sin(2 * np.pi * x[:, 0]) + np.cos(2 * np.pi * x[:, 1]) * x[:, 2] + rng.normal(0, 0.1, 2000)
    xq = rng.uniform(0, 1, (500, 3))
    case('cpu_n2000_d3_m16', NumpyNngpr, NumpyWorker,
         lambda: bk.ConstantKernel(1.0) * bk.RBF(0.3) + bk.WhiteKernel(0.01), x, y, xq, 16)

    # 2. the reference's own test fixture (nngpr_base_tester.py:121-131), num_nn = n so NNGP == exact GP
    r = np.random.RandomState(234058)
    xs = r.rand(150, 4)
    xe = r.rand(50, 4)
    beta = r.rand(4, 3)
    beta[:, -1] += 1
    ys = xs @ beta + r.rand(150, 3)
    ys[:, 0] *= 10
    for ydim in (1, 3):
        case(f'reftest_n150_y{ydim}', NumpyNngpr, NumpyWorker,
             lambda: bk.ConstantKernel(1) * bk.RBF(length_scale=1) + bk.WhiteKernel(1),
             xs, ys[:, :ydim] if ydim > 1 else ys[:, 0], xe, 150, theta_eval=np.full(3, 0.5), normalize_y=True)
    # exact-GP values from scikit-learn for the same fixture (nngpr_base_tester.py:174-192)
    from sklearn import gaussian_process as skgp
    from sklearn.gaussian_process import kernels as skk
    sk = {}
    for ydim in (1, 3):
        gp = skgp.GaussianProcessRegressor(kernel=skk.ConstantKernel(1) * skk.RBF(1) + skk.WhiteKernel(1),
                                           normalize_y=True, optimizer=None)
        gp.fit(xs, ys[:, :ydim] if ydim > 1 else ys[:, 0])
        lml, grad = gp.log_marginal_likelihood(np.full(3, 0.5), eval_gradient=True)
        sk[f'lml_y{ydim}'] = np.float64(lml)
        sk[f'grad_y{ydim}'] = grad
        mean, std = gp.predict(xe, return_std=True)
        sk[f'mean_y{ydim}'] = mean
        sk[f'std_y{ydim}'] = std
    np.savez_compressed(os.path.join(HERE, 'reftest_sklearn.npz'), **sk)

    # 3. ARD length scales, two outputs
    rng = np.random.default_rng(1)
    x = rng.uniform(0, 1, (400, 5))
    y = np.stack([np.sin(3 * x[:, 0]) + x[:, 1] ** 2, np.cos(2 * x[:, 2]) * x[:, 3]], 1) + rng.normal(0, 0.05, (400, 2))
    xq = rng.uniform(0, 1, (100, 5))
    case('ard_n400_d5_m12_y2', NumpyNngpr, NumpyWorker,
         lambda: bk.ConstantKernel(0.7) * bk.RBF(np.array([0.3, 0.5, 0.8, 1.2, 2.0])) + bk.WhiteKernel(0.05),
         x, y, xq, 12)

    # 4. an additive constant term (gradient w.r.t. the constant), non-default alpha
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, (300, 2))
    y = np.sin(2 * x[:, 0]) * np.cos(x[:, 1]) + rng.normal(0, 0.1, 300)
    xq = rng.uniform(-1, 1, (80, 2))
    case('const_n300_d2_m10', NumpyNngpr, NumpyWorker,
         lambda: bk.ConstantKernel(0.5) + bk.ConstantKernel(1.3) * bk.RBF(0.4) + bk.WhiteKernel(0.02),
         x, y, xq, 10, alpha=1e-6)
    if not only or 'matern' in only:
        matern_cases(NumpyNngpr, NumpyWorker, bk)


def full_cases(NumpyNngpr, NumpyWorker, bk):
    """predict(conditioning_method='full') of the reference (the sequential algorithm,
    base_nngpr.py:896-1030) on three of the cases above, and sample_y(conditioning_method='full',
    n_samples=4, random_state=11) on the first 60 query points (:691-750) and predict with
    return_cov on the first 80 (full and only-train); the same for 'full-double-nn' (samples with
    random_state=12); on the first case also 'full' with num_nn=48.  Written to
    full_<case>.npz with the neighbour lists they used (indices into [x_train; x_query])."""
    specs = {
        'cpu_n2000_d3_m16': lambda: bk.ConstantKernel(1.0) * bk.RBF(0.3) + bk.WhiteKernel(0.01),
        'ard_n400_d5_m12_y2': lambda: bk.ConstantKernel(0.7) * bk.RBF(np.array([0.3, 0.5, 0.8, 1.2, 2.0]))
        + bk.WhiteKernel(0.05),
        'matern52_n400_d2_m10': lambda: bk.ConstantKernel(1.0) * bk.Matern(0.6, nu=2.5) + bk.WhiteKernel(0.005),
    }
    for name, kernel_fn in specs.items():
        g = dict(np.load(os.path.join(HERE, name + '.npz')))
        m = int(g['num_nn'])
        gpr = NumpyNngpr(kernel=kernel_fn(), num_nn=m, optimizer=None, alpha=float(g['alpha']),
                         normalize_y=bool(g['normalize_y']), allow_downcast_f32='no', distribute_method='sequential',
                         num_workers=1)
        gpr.fit(g['x'], g['y'])
        xq = g['xq']
        mean, std = gpr.predict(xq, return_std=True, conditioning_method='full')
        mean_only = gpr.predict(xq, return_std=False, conditioning_method='full')
        worker = NumpyWorker()
        nn, _ = gpr._find_nn_indices_for_train_and_eval(worker, gpr.kernel_, gpr.X_train_, xq, condition_on_eval=True,
                                                         double_nn=False)
        _, cov_full = gpr.predict(xq[:80], return_cov=True, conditioning_method='full')
        _, cov_train = gpr.predict(xq[:80], return_cov=True, conditioning_method='only-train')
        nn80, _ = gpr._find_nn_indices_for_train_and_eval(worker, gpr.kernel_, gpr.X_train_, xq[:80],
                                                           condition_on_eval=True, double_nn=False)
        samples = gpr.sample_y(xq[:60], n_samples=4, random_state=11, conditioning_method='full')
        nn60, _ = gpr._find_nn_indices_for_train_and_eval(worker, gpr.kernel_, gpr.X_train_, xq[:60],
                                                           condition_on_eval=True, double_nn=False)
        # 'full-double-nn': num_nn neighbours from the training set plus num_nn from the earlier
        # queries (base_nngpr.py:1418-1449)
        dn_mean, dn_std = gpr.predict(xq, return_std=True, conditioning_method='full-double-nn')
        dn_nn, _ = gpr._find_nn_indices_for_train_and_eval(worker, gpr.kernel_, gpr.X_train_, xq,
                                                            condition_on_eval=True, double_nn=True)
        _, dn_cov = gpr.predict(xq[:80], return_cov=True, conditioning_method='full-double-nn')
        dn_samples = gpr.sample_y(xq[:60], n_samples=4, random_state=12, conditioning_method='full-double-nn')
        extra = {}
        if name == 'cpu_n2000_d3_m16':
            # 'full' with 48 neighbours (more than one warp's 32 slots) on the first 150 queries
            gpr48 = NumpyNngpr(kernel=kernel_fn(), num_nn=48, optimizer=None, alpha=float(g['alpha']),
                               normalize_y=bool(g['normalize_y']), allow_downcast_f32='no',
                               distribute_method='sequential', num_workers=1)
            gpr48.fit(g['x'], g['y'])
            f48_mean, f48_std = gpr48.predict(xq[:150], return_std=True, conditioning_method='full')
            f48_nn, _ = gpr48._find_nn_indices_for_train_and_eval(worker, gpr48.kernel_, gpr48.X_train_, xq[:150],
                                                                   condition_on_eval=True, double_nn=False)
            extra = dict(f48_mean=np.asarray(f48_mean), f48_std=np.asarray(f48_std),
                         f48_nbr=np.asarray(f48_nn)[:, 1:])
        np.savez_compressed(os.path.join(HERE, 'full_' + name + '.npz'), mean=np.asarray(mean), std=np.asarray(std),
                            mean_only=np.asarray(mean_only), nbr=np.asarray(nn)[:, 1:],
                            samples60=np.asarray(samples), nbr60=np.asarray(nn60)[:, 1:],
                            cov80_full=np.asarray(cov_full), cov80_train=np.asarray(cov_train),
                            nbr80=np.asarray(nn80)[:, 1:], dn_mean=np.asarray(dn_mean), dn_std=np.asarray(dn_std),
                            dn_nbr=np.asarray(dn_nn)[:, 1:], dn_cov80=np.asarray(dn_cov),
                            dn_samples60=np.asarray(dn_samples), **extra)
        print('full', name, np.asarray(mean).ravel()[:3], np.asarray(std).ravel()[:3])


def wide_case(NumpyNngpr, NumpyWorker, bk):
    """8. One hundred outputs (normalize_y): every output column is its own right-hand side of
    each local system and the log-likelihood sums over the columns (base_nngpr.py:578-584).
    The reference's own known-answer test asks for y_dim = 100 (nngpr_base_tester.py:179) but
    slices a 150 x 3 array with [:, :100], i.e. runs 3 columns (the reftest_n150_y3 case); this
    case has 100 genuine columns."""
    rng = np.random.default_rng(8)
    x = rng.uniform(0, 1, (300, 3))
    w = rng.normal(size=(3, 100))
    y = np.sin(2 * x @ w) + 0.3 * np.arange(100)[None, :] + rng.normal(0, 0.05, (300, 100))
    xq = rng.uniform(0, 1, (60, 3))
    case('wide_n300_d3_m16_y100', NumpyNngpr, NumpyWorker,
         lambda: bk.ConstantKernel(1.0) * bk.RBF(0.4) + bk.WhiteKernel(0.02), x, y, xq, 16, normalize_y=True)


def matern_cases(NumpyNngpr, NumpyWorker, bk):
    """5-7. Matern nu = 1/2, 3/2, 5/2 (isotropic; the last with normalised y), evaluated
    by the reference's generic path (batched_kernels.py:1070-1131)."""
    rng = np.random.default_rng(5)
    x = rng.uniform(0, 1, (500, 3))
    y = np.sin(4 * x[:, 0]) + x[:, 1] * x[:, 2] + rng.normal(0, 0.05, 500)
    xq = rng.uniform(0, 1, (120, 3))
    case('matern12_n500_d3_m16', NumpyNngpr, NumpyWorker,
         lambda: bk.ConstantKernel(0.9) * bk.Matern(0.4, nu=0.5) + bk.WhiteKernel(0.01), x, y, xq, 16)
    rng = np.random.default_rng(6)
    x = rng.uniform(-1, 1, (450, 4))
    y = np.cos(2 * x[:, 0]) * x[:, 1] + 0.5 * x[:, 2] ** 2 + rng.normal(0, 0.05, 450)
    xq = rng.uniform(-1, 1, (90, 4))
    # isotropic: the reference's batched Matern checks an ARD length scale against the
    # neighbour axis of its (batch, k, d) input (batched_kernels.py:1033) and raises
    case('matern32_n450_d4_m12', NumpyNngpr, NumpyWorker,
         lambda: bk.ConstantKernel(1.2) * bk.Matern(0.7, nu=1.5) + bk.WhiteKernel(0.02), x, y, xq, 12)
    rng = np.random.default_rng(7)
    x = rng.uniform(0, 2, (400, 2))
    y = 3.0 + np.sin(3 * x[:, 0]) * np.exp(-x[:, 1]) + rng.normal(0, 0.05, 400)
    xq = rng.uniform(0, 2, (100, 2))
    case('matern52_n400_d2_m10', NumpyNngpr, NumpyWorker,
         lambda: bk.ConstantKernel(1.0) * bk.Matern(0.6, nu=2.5) + bk.WhiteKernel(0.005), x, y, xq, 10,
         normalize_y=True)


if __name__ == '__main__':
    main()
