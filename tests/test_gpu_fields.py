"""GPU parity: field operators and the exact potential through the C ABI vs the
oracle (FP64) and the reference's own outputs (golden fixtures).

Tolerances:
  * FP32 stencils (divergence, gradient, exchange): bit-exact vs the reference.
  * direct potential (FP32 table + compensated sums): rel-L2 <= 2e-6 vs the
    FP64 oracle, <= 5e-6 vs the reference's FP32 sum.
"""
import numpy as np
import pytest

from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu


def mkctx(mmsb200, dims, d, solver=None, **pk):
    g = mmsb200.Grid(*dims, *d)
    return mmsb200.Context(g, mmsb200.make_params(**pk), solver or mmsb200.make_solver())


def dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def dims_of(z):
    return tuple(int(v) for v in z["dims"]), tuple(float(v) for v in z["d"])


def test_stencils_bit_exact(cuda, lib):
    import mmsb200
    torch = cuda
    z = golden("stencils_16x16x3.npz")
    dims, d = dims_of(z)
    mu0 = float(np.float32(4e-7 * np.pi))
    with mkctx(mmsb200, dims, d, mu0=mu0) as ctx:
        M = dev(torch, z["M"])
        S = dev(torch, z["S"])
        rho = torch.empty(dims[::-1], dtype=torch.float32, device="cuda")
        H = torch.zeros(dims[::-1] + (3,), dtype=torch.float32, device="cuda")
        E = torch.zeros_like(H)
        ctx.divergence_dev(M, rho)
        ctx.gradient_dev(S, 1 / (4 * np.pi), H)
        ctx.exchange_dev(M, E)
        ctx.sync()
        assert np.array_equal(rho.cpu().numpy(), z["div"])
        assert np.array_equal(H.cpu().numpy(), z["grad"])
        assert np.array_equal(E.cpu().numpy(), z["exch"])


@pytest.mark.parametrize("name", ["potential_16x16x3.npz", "potential_24x10x3.npz", "potential_32x32x3.npz"])
def test_direct_vs_reference_and_oracle(cuda, lib, oracle_mod, name):
    import mmsb200
    z = golden(name)
    dims, d = dims_of(z)
    g = oracle_mod.Grid(*dims, *d)
    exact = oracle_mod.potential_direct(g, z["rho"])
    with mkctx(mmsb200, dims, d) as ctx:
        phi = ctx.potential_host(z["rho"])
    assert rel_l2(phi, exact) < 2e-6
    assert rel_l2(phi, z["phi_direct"]) < 5e-6


@pytest.mark.parametrize("dims", [(64, 64, 3), (37, 23, 4), (300, 5, 3), (8, 8, 1), (1, 1, 3), (513, 3, 2)])
def test_direct_sizes(cuda, lib, oracle_mod, dims):
    """ragged rows (not multiples of 8), rows longer than one warp segment,
    a single layer, a single column"""
    import mmsb200
    rng = np.random.default_rng(sum(dims))
    X, Y, Z = dims
    d = (5e-9, 4e-9, 6e-9)
    rho = rng.standard_normal((Z, Y, X)).astype(np.float32) * 1e14
    rho[rng.random((Z, Y, X)) < 0.3] = 0  # masked cells: zero charge
    g = oracle_mod.Grid(X, Y, Z, *d)
    exact = oracle_mod.potential_direct(g, rho)
    with mkctx(mmsb200, dims, d) as ctx:
        phi = ctx.potential_host(rho)
    assert rel_l2(phi, exact) < 2e-6


def test_direct_deterministic_and_empty(cuda, lib):
    import mmsb200
    torch = cuda
    dims, d = (96, 80, 3), (5e-9, 5e-9, 5e-9)
    rng = np.random.default_rng(7)
    rho = dev(torch, rng.standard_normal(dims[::-1]).astype(np.float32))
    with mkctx(mmsb200, dims, d) as ctx:
        a = torch.empty_like(rho)
        b = torch.empty_like(rho)
        ctx.potential_dev(rho, a)
        ctx.potential_dev(rho, b)
        ctx.sync()
        assert torch.equal(a, b)
        zero = torch.zeros_like(rho)
        ctx.potential_dev(zero, a)
        ctx.sync()
        assert float(a.abs().max()) == 0.0


def test_hfield_vs_reference(cuda, lib):
    import mmsb200
    z = golden("hfield_16x16x3.npz")
    dims, d = dims_of(z)
    mu0 = float(np.float32(4e-7 * np.pi))
    for ext in (0, 1):
        with mkctx(mmsb200, dims, d, mu0=mu0, external=bool(ext)) as ctx:
            H, q, phi = ctx.hfield_host(z["M"], t=float(z[f"t_ext{ext}"]))
        assert np.array_equal(q, z[f"charge_ext{ext}"])  # divergence is bit-exact
        assert rel_l2(phi, z[f"phi_ext{ext}"]) < 5e-6
        assert rel_l2(H, z[f"H_ext{ext}"]) < 5e-6


def test_hfield_dev_matches_host(cuda, lib):
    import mmsb200
    torch = cuda
    z = golden("hfield_16x16x3.npz")
    dims, d = dims_of(z)
    with mkctx(mmsb200, dims, d) as ctx:
        Hh, qh, ph = ctx.hfield_host(z["M"])
        M = dev(torch, z["M"])
        H = torch.empty_like(M)
        q = torch.empty(dims[::-1], dtype=torch.float32, device="cuda")
        p = torch.empty_like(q)
        ctx.hfield_dev(M, H, q, p, 0.0)
        ctx.sync()
        assert np.array_equal(H.cpu().numpy(), Hh)
        assert np.array_equal(p.cpu().numpy(), ph)


def test_invalid_arguments_raise(cuda, lib):
    import mmsb200
    with pytest.raises(mmsb200.MmsError):
        mkctx(mmsb200, (0, 4, 3), (5e-9, 5e-9, 5e-9))
    with pytest.raises(mmsb200.MmsError):
        mkctx(mmsb200, (4, 4, 3), (5e-9, -1.0, 5e-9))
    with mkctx(mmsb200, (4, 4, 3), (5e-9, 5e-9, 5e-9)) as ctx:
        with pytest.raises(mmsb200.MmsError) as e:
            ctx.run_fixed(1e-13, 1)  # no state yet
        assert e.value.status == mmsb200.MMS_ERR_NOT_READY
