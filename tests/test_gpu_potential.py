"""Gaussian impurity potentials built on the device (itp2d_add_gaussian_impurities)
against the oracle's restatement of the reference's host loop
(GaussianImpurities::add_noise, noise.cpp:24-40, once per impurity in list order
on the cell-centred grid of datalayout.cpp:21-35), which tests/test_oracle.py pins
to the compiled reference."""
import numpy as np
import pytest

from itp2d_b200 import capi
from oracle import itp_oracle as O

pytestmark = pytest.mark.gpu


def _host_loop(V0, sx, sy, dx, imp):
    return O.gaussian_impurities(O.Grid(sx, sy, dx), imp, V0)


@pytest.mark.parametrize("sx,sy,n", [(96, 80, 300), (512, 512, 400)])
def test_gaussian_impurities_match_host_loop(sx, sy, n):
    import torch
    dx = 16.0 / sx
    rng = np.random.default_rng(sx + n)
    imp = np.column_stack([rng.uniform(-6, 6, n), rng.uniform(-5, 5, n), rng.uniform(0.8, 1.2, n),
                           rng.uniform(0.1, 0.3, n)])
    x = (2 * np.arange(sx) + 1 - sx) * dx / 2
    y = (2 * np.arange(sy) + 1 - sy) * dx / 2
    V0 = 0.5 * (x[None, :] ** 2 + y[:, None] ** 2)  # harmonic(1) base potential
    ref = _host_loop(V0, sx, sy, dx, imp)
    Vd = torch.tensor(V0, dtype=torch.float64, device="cuda")
    impd = torch.tensor(imp, dtype=torch.float64, device="cuda")
    capi.add_gaussian_impurities(sx, sy, dx, impd.data_ptr(), n, Vd.data_ptr())
    torch.cuda.synchronize()
    got = Vd.cpu().numpy()
    # each term differs from the host loop only through exp() (a few ulps)
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    print(f"impurities {sx}x{sy} n={n}: max relative difference {err:.2e}")
    assert err < 1e-14
    # adding the same list again doubles the impurity part
    capi.add_gaussian_impurities(sx, sy, dx, impd.data_ptr(), n, Vd.data_ptr())
    torch.cuda.synchronize()
    assert np.max(np.abs(Vd.cpu().numpy() - _host_loop(ref, sx, sy, dx, imp))) < 1e-14 * np.max(np.abs(ref)) * 2


def test_gaussian_impurities_argument_checks():
    import torch
    V = torch.zeros(16 * 16, dtype=torch.float64, device="cuda")
    imp = torch.tensor([[0.0, 0.0, 1.0, 0.2]], dtype=torch.float64, device="cuda")
    capi.add_gaussian_impurities(16, 16, 0.5, imp.data_ptr(), 0, V.data_ptr())  # n = 0: nothing to add
    torch.cuda.synchronize()
    assert float(V.abs().max()) == 0.0
    host = np.zeros(16 * 16)
    with pytest.raises(capi.ITP2DError):  # host memory is rejected before any launch
        capi.add_gaussian_impurities(16, 16, 0.5, imp.data_ptr(), 1, host.ctypes.data)
    with pytest.raises(capi.ITP2DError):
        capi.add_gaussian_impurities(16, 16, -0.5, imp.data_ptr(), 1, V.data_ptr())
