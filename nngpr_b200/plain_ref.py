"""The reference's own CUDA kernels, compiled from the installed reference, as the plain FP32 GPU
comparator of the benchmark.

The reference accelerates its CUDA backends with two kernels kept as source strings in
``nngpr/cuda_kernel_accelerators.py`` and JIT-compiled through cupy (NVRTC): ``calc_nn`` (one
thread per query, insertion into a sorted top-m list, ``:663-743``; launched by ``:196-381``) and
``fill_nn_kernel`` (one thread per point writing K and dK to global memory, ``:748-863``; launched by
``:383-518``).  cupy is not installed here, so this module reads those two strings from the
reference's source file (``ast``; the module itself cannot be imported without cupy), prepends the
``#define`` header that the reference's launchers build for the same arguments, compiles with NVRTC
for sm_100a with NVRTC's default options (as cupy does) and launches them with the CUDA driver API
on torch's current stream.  The local systems then follow the reference's worker arithmetic on
batched torch tensors (``nngpr_b200.plain.plain_loglik``).

Comparator only: nothing of the product path imports this module.
"""
from __future__ import annotations

import ast
import ctypes
import os

import numpy as np

_SOURCES = None
_CACHE = {}


def available(ref_root: str) -> bool:
    """Whether the reference's kernel sources are under ``ref_root`` (the directory holding the
    installed package ``nngpr``)."""
    return os.path.isfile(os.path.join(ref_root, 'nngpr', 'cuda_kernel_accelerators.py'))


def _sources(ref_root: str) -> dict:
    global _SOURCES
    if _SOURCES is None:
        path = os.path.join(ref_root, 'nngpr', 'cuda_kernel_accelerators.py')
        tree = ast.parse(open(path).read())
        found = {}
        for node in tree.body:
            if isinstance(node, ast.Assign) and len(node.targets) == 1 and isinstance(node.targets[0], ast.Name):
                name = node.targets[0].id
                if name in ('_calc_nn_rbf_kernel_text', '_fill_nn_RBF_kernel_text'):
                    found[name] = ast.literal_eval(node.value)
        if len(found) != 2:
            raise RuntimeError(f'kernel sources not found in {path}')
        _SOURCES = found
    return _SOURCES


def _check(res, what):
    """The value of a cuda-python call returning ``(status, value...)``; raises on a bad status."""
    err, rest = (res[0], res[1:]) if isinstance(res, tuple) else (res, ())
    if int(err) != 0:
        raise RuntimeError(f'{what} failed: {err}')
    if len(rest) == 1:
        return rest[0]
    return rest or None


def _function(src: str, name: str, dyn_smem: int = 0):
    """Compile ``src`` with NVRTC (sm_100a, default options) once and return the driver function."""
    from cuda.bindings import driver, nvrtc
    key = (src, name)
    if key in _CACHE:
        return _CACHE[key]
    prog = _check(nvrtc.nvrtcCreateProgram(src.encode(), (name + '.cu').encode(), 0, [], []), 'nvrtcCreateProgram')
    opts = [b'--gpu-architecture=sm_100a']
    err = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)[0]
    if int(err) != 0:
        log_size = _check(nvrtc.nvrtcGetProgramLogSize(prog), 'nvrtcGetProgramLogSize')
        log = b' ' * log_size
        nvrtc.nvrtcGetProgramLog(prog, log)
        raise RuntimeError('NVRTC: ' + log.decode(errors='replace'))
    size = _check(nvrtc.nvrtcGetCUBINSize(prog), 'nvrtcGetCUBINSize')
    cubin = b' ' * size
    _check(nvrtc.nvrtcGetCUBIN(prog, cubin), 'nvrtcGetCUBIN')
    module = _check(driver.cuModuleLoadData(cubin), 'cuModuleLoadData')
    fn = _check(driver.cuModuleGetFunction(module, name.encode()), 'cuModuleGetFunction')
    if dyn_smem:
        _check(driver.cuFuncSetAttribute(fn, driver.CUfunction_attribute.CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                                         dyn_smem), 'cuFuncSetAttribute')
    _CACHE[key] = (module, fn)
    return module, fn


def _launch(fn, grid, block, smem, args):
    import torch
    from cuda.bindings import driver
    stream = driver.CUstream(torch.cuda.current_stream().cuda_stream)
    vals = tuple(a[0] for a in args)
    types = tuple(a[1] for a in args)
    _check(driver.cuLaunchKernel(fn, grid, 1, 1, block, 1, 1, smem, stream, (vals, types), 0), 'cuLaunchKernel')


def calc_nn(ref_root: str, ref, query, num_nn: int, ref_cut_index, length_scale):
    """The reference's ``calc_nn`` on torch FP32 CUDA tensors ``ref (n, d)``, ``query (nq, d)``:
    int32 ``(nq, num_nn)``.  Scaling, layout and defines as its launcher
    (``cuda_kernel_accelerators.py:235-381``) for FP32 inputs."""
    import torch
    src = _sources(ref_root)['_calc_nn_rbf_kernel_text']
    ref = ref.to(torch.float32)
    query = query.to(torch.float32)
    if length_scale is not None:
        ls = torch.as_tensor(np.broadcast_to(np.asarray(length_scale, dtype=np.float32), (ref.shape[1],)).copy(),
                             device=ref.device)
        ref, query = ref / ls, query / ls
    n_ref, d = ref.shape
    nq = query.shape[0]
    block = 256
    index_t, size_t = 'int', 'int'
    big = max(nq * d, n_ref * d, num_nn * block)
    if big > np.iinfo(np.int32).max:
        size_t = 'long long'
    smem = num_nn * block * (4 + 4)
    defines = {'DATA_TYPE': 'float', 'INFINITY': '__int_as_float(0x7f800000)',
               'NEG_INFINITY': '__int_as_float(0xff800000)', 'INDEX_TYPE': index_t, 'N_QUERY': nq, 'N_REF': n_ref,
               'NUM_K': num_nn, 'NUM_FEATURE': d, 'SIZE_TYPE': size_t}
    if smem <= 49152:
        defines['USE_STATIC_SHARED_MEM_CACHE'] = 'true'
        dyn = 0
    elif smem <= 98304 * 0.9:
        defines['USE_DYNAMIC_SHARED_MEM_CACHE'] = 'true'
        dyn = smem
    else:
        raise NotImplementedError('num_nn too large for the shared-memory list of calc_nn')
    defines['REF_PITCH_FEATURE'] = '* ' + str(n_ref)
    defines['REF_PITCH_POINT'] = ''
    index = torch.empty((num_nn, nq), dtype=torch.int32, device=ref.device)
    if ref_cut_index is None:
        defines['MAX_SEARCH_POINT'] = defines['N_REF']
    else:
        defines['MAX_SEARCH_POINT'] = '(i_query + ' + str(int(ref_cut_index)) + ')'
        index[:, :max(0, num_nn - int(ref_cut_index))] = -1
    defines.update({'BLOCK_DIM': block, 'QUERY_PITCH': nq, 'NUM_K_FOR_CACHE': num_nn, 'INDEX_PITCH': nq})
    header = '\n'.join(f'#define {k} {v}' for k, v in defines.items()) + '\n\n'
    _, fn = _function(header + src, 'calc_nn', dyn)
    ref_t = ref.t().contiguous()
    q_t = query.t().contiguous()
    _launch(fn, (nq + block - 1) // block, block, dyn,
            [(ref_t.data_ptr(), ctypes.c_void_p), (q_t.data_ptr(), ctypes.c_void_p),
             (index.data_ptr(), ctypes.c_void_p)])
    return index.t().contiguous()


def fill_nn_kernel(ref_root: str, x, nn_indices, p, eval_gradient: bool):
    """The reference's ``fill_nn_kernel`` on FP32: ``x (n, d)``, ``nn_indices (b, k)`` int32 (the
    point itself in column 0, -1 for missing).  Returns ``K (b, k, k)`` and ``dK (b, k, k, n_theta)``
    (or None), as its launcher (``cuda_kernel_accelerators.py:409-518``)."""
    import torch
    src = _sources(ref_root)['_fill_nn_RBF_kernel_text']
    x = x.to(torch.float32).contiguous()
    nn_t = nn_indices.to(torch.int32).t().contiguous()  # (k, b)
    k, b = nn_t.shape
    n_theta = p.n_theta if eval_gradient else 0
    K = torch.zeros((k, k, b), dtype=torch.float32, device=x.device)
    G = torch.zeros((k, k, n_theta, b) if eval_gradient else (0, 0, 0, 0), dtype=torch.float32, device=x.device)
    ard = p.length_scale is not None and np.size(p.length_scale) > 1
    ls = torch.as_tensor(np.asarray(1.0 if p.length_scale is None else p.length_scale, dtype=np.float32).reshape(-1),
                         device=x.device)
    big = max(K.numel(), G.numel())
    big_t = 'int' if big <= np.iinfo(np.int32).max else 'long long'
    defines = {'BLOCK_DIM': 64, 'EXP': 'expf', 'NUM_REF_POINTS': b, 'NUM_NN': k, 'NUM_FEATURES': x.shape[1],
               'NUM_THETA': n_theta, 'PITCH_NN_POINTS': b, 'PITCH_DATA_POINTS': x.shape[1], 'PITCH_NN_KERNEL': b,
               'PITCH_NN_KERNEL_GRAD': b * n_theta if eval_gradient else 0, 'THETA_PITCH': b if eval_gradient else 0,
               'DATA_TYPE': 'float', 'INDEX_TYPE': 'int', 'NN_IND_DTYPE': 'int', 'BIG_INDEX_TYPE': big_t,
               'WHITE_NOISE_INDEX': p.idx_noise if eval_gradient else -1,
               'CONSTANT_LEVEL_INDEX': p.idx_const if eval_gradient else -1,
               'RBF_LEVEL_INDEX': p.idx_rbf_level if eval_gradient else -1,
               'RBF_SCALE_INDEX': p.idx_ls if eval_gradient and not ard else -1,
               'RBF_SCALE_VEC_INDEX_0': p.idx_ls if eval_gradient and ard else -1,
               'RBF_SCALE_VEC_INDEX_1': p.idx_ls + np.size(p.length_scale) if eval_gradient and ard else -1}
    if ard:
        defines['IS_VEC_RBF_SCALE'] = 1
    header = '\n'.join(f'#define {kk} {v}' for kk, v in defines.items()) + '\n\n'
    _, fn = _function(header + src, 'fill_nn_kernel')
    rbf = p.rbf_level if p.length_scale is not None else 0.0
    _launch(fn, (b + 63) // 64, 64, 0,
            [(x.data_ptr(), ctypes.c_void_p), (nn_t.data_ptr(), ctypes.c_void_p), (ls.data_ptr(), ctypes.c_void_p),
             (K.data_ptr(), ctypes.c_void_p), (G.data_ptr(), ctypes.c_void_p),
             (float(p.const_value), ctypes.c_float), (float(p.noise_level), ctypes.c_float),
             (float(rbf), ctypes.c_float)])
    K = K.permute(2, 0, 1)
    G = G.permute(3, 0, 1, 2) if eval_gradient else None
    return K, G
