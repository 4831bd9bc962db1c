"""The allocation-free exact potential (mms_potential_direct_noalloc).

Some callers cannot allocate device memory: a host whose own pool allocator
owns the GPU memory, code that runs while a CUDA graph is being captured, or a
loop that must not take the driver's allocation lock.  For them the library
exports a variant of the direct sum whose scratch table sits in a fixed array
inside the library.  This file checks, through the C ABI, that it returns what
the context-based entry point (mms_potential_dev with the direct solver)
returns, within the direct sum's tolerance (rel-L2 <= 2e-6), on two calls in a
row with different grids, that it allocates nothing, and that sizes beyond its
fixed table are refused.  A wide-row case checks both entry points against the
FP64 oracle after a context of another row length has set the sum kernel's
shared-memory limit (the limit is per kernel, shared by both entry points).
It runs last (file name) and passes alone or after the other tests.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _noalloc(lib, rho, phi, dims, d, stream):
    X, Y, Z = dims
    return lib.mms_potential_direct_noalloc(ctypes.c_void_p(rho.data_ptr()), ctypes.c_void_p(phi.data_ptr()),
                                            X, Y, Z, d[0], d[1], d[2], ctypes.c_void_p(stream))


def test_noalloc_matches_context_entry_point_twice(cuda, lib):
    import mmsb200
    torch = cuda
    stream = torch.cuda.current_stream().cuda_stream
    cases = [((64, 48, 3), (5e-9, 5e-9, 5e-9), 1), ((37, 90, 4), (4e-9, 5e-9, 6e-9), 2)]
    free_after_first = None
    for n, (dims, d, seed) in enumerate(cases):
        X, Y, Z = dims
        rng = np.random.default_rng(seed)
        rho_h = rng.standard_normal((Z, Y, X)).astype(np.float32) * 1e14
        rho = torch.from_numpy(rho_h).cuda()
        phi_ref = torch.empty_like(rho)
        with mmsb200.Context(mmsb200.Grid(X, Y, Z, *d), mmsb200.make_params(),
                             mmsb200.make_solver(mmsb200.SOLVER_DIRECT), stream=stream) as ctx:
            ctx.potential_dev(rho, phi_ref)
            ctx.sync()
        torch.cuda.synchronize()
        phi = torch.full_like(rho, float("nan"))
        if n == 1:
            free_before = torch.cuda.mem_get_info()[0]
        st = _noalloc(lib, rho, phi, dims, d, stream)
        assert st == mmsb200.MMS_OK, lib.mms_last_error()
        torch.cuda.synchronize()
        if n == 1:
            # the second call allocates nothing on the device
            assert torch.cuda.mem_get_info()[0] == free_before
        assert torch.isfinite(phi).all()
        assert rel_l2(phi.cpu().numpy(), phi_ref.cpu().numpy()) <= 2e-6


def test_noalloc_rejects_sizes_beyond_its_table(cuda, lib):
    import mmsb200
    torch = cuda
    rho = torch.zeros(16, device="cuda")
    phi = torch.zeros(16, device="cuda")
    st = _noalloc(lib, rho, phi, (1024, 1024, 2), (5e-9, 5e-9, 5e-9), 0)
    assert st == mmsb200.MMS_ERR_ARG
    assert b"exceeds" in lib.mms_last_error()


def test_noalloc_wide_rows_after_a_context_of_another_width(cuda, lib, oracle_mod):
    """A context whose rows need more than 48 KB of shared memory (xdim 900)
    sets the sum kernel's limit; an allocation-free call with wider rows
    (xdim 1100) must still launch, and both results must match the FP64 sum."""
    import mmsb200
    torch = cuda
    stream = torch.cuda.current_stream().cuda_stream
    d = (5e-9, 5e-9, 5e-9)
    results = []
    for dims, seed, use_ctx in (((900, 4, 2), 11, True), ((1100, 8, 3), 12, False)):
        X, Y, Z = dims
        rng = np.random.default_rng(seed)
        rho_h = (rng.standard_normal((Z, Y, X)) * 1e14).astype(np.float32)
        rho = torch.from_numpy(rho_h).cuda()
        phi = torch.full_like(rho, float("nan"))
        if use_ctx:
            with mmsb200.Context(mmsb200.Grid(X, Y, Z, *d), mmsb200.make_params(),
                                 mmsb200.make_solver(mmsb200.SOLVER_DIRECT), stream=stream) as ctx:
                ctx.potential_dev(rho, phi)
                ctx.sync()
        else:
            st = _noalloc(lib, rho, phi, dims, d, stream)
            assert st == mmsb200.MMS_OK, lib.mms_last_error()
        torch.cuda.synchronize()
        ref = oracle_mod.potential_direct(oracle_mod.Grid(X, Y, Z, *d), rho_h.astype(np.float64))
        results.append(rel_l2(phi.cpu().numpy(), ref))
    assert results[0] <= 2e-6, results
    assert results[1] <= 2e-6, results
