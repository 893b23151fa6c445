"""The allocation-free prediction entry point against the workspace one.

fmlb_kernel_predict_f64_noalloc serves callers that cannot allocate device
memory while they run (all device memory reserved up front by their own arena,
or a host framework that hands over only input and output buffers). It keeps
its scratch in a fixed array inside the library, so this test checks, through
the C ABI, that two calls in a row give the results of fmlb_kernel_predict_f64
(1e-12 relative, the FP64 kernel tolerance of the parity tests) — the second
call smaller than the first, so stale scratch from the first would show — and
that a call larger than the fixed scratch is refused.

This file is collected last on purpose; it passes alone in a fresh process and
after the other tests.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problem(rng, nq, nt, d, nsig):
    Xq = torch.from_numpy(rng.standard_normal((nq, d)) * 3.0).cuda()
    Xt = torch.from_numpy(rng.standard_normal((nt, d)) * 3.0).cuda()
    alpha = torch.from_numpy(rng.standard_normal((nsig, nt))).cuda()
    return Xq, Xt, alpha


def _predict(name, kind, Xq, Xt, alpha, sigmas, workspace):
    from fml_b200 import _lib
    nq, d = Xq.shape
    nt = Xt.shape[0]
    nsig = len(sigmas)
    y = torch.full((nsig, nq), float("nan"), dtype=torch.float64, device="cuda")
    sp, keep = _lib.host_doubles(sigmas)
    args = [kind, _lib.ptr(Xq), nq, d, _lib.ptr(Xt), nt, d, d, sp, nsig, _lib.ptr(alpha), nt,
            _lib.ptr(y), nq]
    if workspace:
        lib = _lib.load()
        ws = torch.empty(lib.fmlb_kernel_predict_workspace_bytes(nq, nt, nsig),
                         dtype=torch.uint8, device="cuda")
        args += [_lib.ptr(ws), ws.numel()]
    args.append(_lib.stream_handle())
    _lib.call(name, *args)
    torch.cuda.synchronize()
    del keep
    return y.cpu().numpy()


@pytest.mark.parametrize("kind", [0, 1])
def test_noalloc_matches_workspace_entry_point_twice(kind):
    rng = np.random.default_rng(11 + kind)
    sigmas = [3.0, 7.5, 20.0]
    # first call larger than the second
    for nq, nt, d in [(777, 2500, 45), (130, 1100, 45)]:
        Xq, Xt, alpha = _problem(rng, nq, nt, d, len(sigmas))
        ref = _predict("fmlb_kernel_predict_f64", kind, Xq, Xt, alpha, sigmas, True)
        out = _predict("fmlb_kernel_predict_f64_noalloc", kind, Xq, Xt, alpha, sigmas, False)
        assert np.isfinite(out).all()
        np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-300)


def test_noalloc_rejects_oversize_call():
    rng = np.random.default_rng(5)
    # ceil(4097 / 1024) = 5 splits * 8 sigmas * 26215 queries > 2**20 doubles
    nq, nt, d = 26215, 4097, 2
    Xq, Xt, alpha = _problem(rng, nq, nt, d, 8)
    with pytest.raises(ValueError, match="fixed scratch"):
        _predict("fmlb_kernel_predict_f64_noalloc", 0, Xq, Xt, alpha, [1.0] * 8, False)
