"""The evaluation entry point that allocates nothing: cco_energy_grad_noalloc.

Some callers of this library cannot allocate device memory while they call
it: code running while a CUDA stream is captured into a graph (cudaMalloc is
not allowed there), processes that reserve all device memory up front in
their own pool, and latency-critical loops that cannot afford an allocator
round trip. For them cco_energy_grad_noalloc carves its scratch out of one
fixed device array compiled into libcco.so instead of allocating per call.

These tests call it through the C ABI and compare it with the allocating
entry point cco_energy_grad on two calls in a row: the fixed array keeps the
previous call's contents, so a second call with different inputs must not
see any of the first. This file is collected last on purpose.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from xla_cco import _native
from xla_cco.box import cubic_box
from xla_cco.energy import make_stealthy_energy
from xla_cco.kvectors import enumerate_kvectors, k_outer_from_ka, ka_from_chi

pytestmark = pytest.mark.gpu

RTOL_E = 1e-12  # energy tolerance used by the kernel parity tests
RTOL_F = 1e-10  # gradient tolerance (relative to max |g|)


def _energy(n: int, d: int, chi: float):
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, 0.05, d), 0.05, d))
    return make_stealthy_energy(box, ks)


def _call(fn, handle, s, phi, grad, stream):
    lib = _native.load()
    if fn == "cco_energy_grad":
        return lib.cco_energy_grad(handle, stream, s.shape[0], s.data_ptr(), phi.data_ptr(),
                                   grad.data_ptr(), None, None)  # fmt: skip
    return lib.cco_energy_grad_noalloc(handle, stream, s.shape[0], s.data_ptr(), phi.data_ptr(),
                                       grad.data_ptr())  # fmt: skip


@pytest.mark.parametrize("n,d,chi,b", [(1000, 2, 0.40, 8), (300, 3, 0.25, 5), (500, 1, 0.3, 4)])
def test_noalloc_matches_allocating_entry_point_two_calls(n, d, chi, b):
    import torch

    en = _energy(n, d, chi)
    dev = torch.cuda.current_device()
    handle = en.problem_handle(dev, n)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(n + d)
    inputs = [torch.from_numpy(rng.uniform(size=(b, n, d))).cuda() for _ in range(2)]
    for s in inputs:  # two calls in a row on the shared fixed scratch
        phi_ref = torch.empty(b, dtype=torch.float64, device="cuda")
        g_ref = torch.empty_like(s)
        assert _call("cco_energy_grad", handle, s, phi_ref, g_ref, stream) == _native.CCO_OK
        phi = torch.full((b,), float("nan"), dtype=torch.float64, device="cuda")
        g = torch.full_like(s, float("nan"))
        code = _call("cco_energy_grad_noalloc", handle, s, phi, g, stream)
        assert code == _native.CCO_OK, _native.load().cco_last_error()
        torch.cuda.synchronize()
        pr, gr = phi_ref.cpu().numpy(), g_ref.cpu().numpy()
        np.testing.assert_allclose(phi.cpu().numpy(), pr, rtol=RTOL_E)
        np.testing.assert_allclose(g.cpu().numpy(), gr, rtol=RTOL_F, atol=RTOL_F * np.abs(gr).max())


def test_noalloc_rejects_batch_beyond_fixed_scratch():
    import torch

    n, d = 1000, 2
    en = _energy(n, d, 0.40)
    handle = en.problem_handle(torch.cuda.current_device(), n)
    s = torch.zeros((1, n, d), dtype=torch.float64, device="cuda")
    phi = torch.zeros(1, dtype=torch.float64, device="cuda")
    lib = _native.load()
    # the size check happens before anything is launched, so these small
    # buffers are never touched for the oversized batch
    code = lib.cco_energy_grad_noalloc(handle, None, 100_000, s.data_ptr(), phi.data_ptr(), None)
    assert code == _native.CCO_ERR_ARG
    assert b"split the batch" in lib.cco_last_error()
    assert float(phi.cpu()[0]) == 0.0
    assert ctypes.c_uint(16 << 20).value == 16777216  # CCO_NOALLOC_SCRATCH_BYTES, 16 MiB
