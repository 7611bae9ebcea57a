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
    # each term differs from the host loop only through exp() (a few ulps);
    # the impurity part alone is compared (the harmonic base, up to 64 at the
    # corners, would hide errors in the O(1) impurity terms)
    part, ref_part = got - V0, ref - V0
    err = np.max(np.abs(part - ref_part)) / np.max(np.abs(ref_part))
    print(f"impurities {sx}x{sy} n={n}: max difference relative to the impurity part {err:.2e}")
    assert err < 4e-15
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


# every type of the reference's potential library, with defaults and with
# explicit parameters
LIBRARY = ["harmonic", "harmonic(2,0.5,-0.25)", "elliptic", "elliptic(1,3)", "prettyhardsquare",
           "prettyhardsquare(6)", "softpentagon", "henonheiles", "henon(1,-1)", "gaussian", "gaussianblob(2,0.7,1,-1)",
           "quartic", "quarticoscillator(0.2)", "squareoscillator", "squareoscillator(3)", "power",
           "poweroscillator(3,2)", "ring", "ringpotential(3,1,2,0.5,1)", "cosh", "coshpotential(2,3)",
           "softstadium", "softstadium(1.5,3,50,2,5)", "powerstadium", "powerstadium(1.5,3,6)"]


@pytest.mark.parametrize("desc", LIBRARY)
def test_potential_library_matches_reference(desc):
    """itp2d_evaluate_potential against the reference's own potential table
    (Potential built from parse_potential_description, compiled from the
    reference sources): the same operations in the same order, so values
    differ only through the math library's exp / pow / trigonometric /
    hypot / cosh roundings (a few units in the last place); the purely
    polynomial types agree exactly."""
    import ctypes as C

    import torch
    from oracle import refkit as R
    if not R.available():
        pytest.fail("oracle/_ref/libitp2d_ref.so missing: build it with make -C oracle")
    sx, sy, L = 96, 80, 10.0
    dx = L / sx
    ref = R.RefKit(sx, sy, L, 0, 0.0, 1, 0.1, 1, potential=desc, threads=1).potential()
    V = torch.full((sy, sx), np.nan, dtype=torch.float64, device="cuda")
    f = capi.lib().itp2d_evaluate_potential
    f.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]
    assert f(desc.encode(), sx, sy, dx, C.c_void_p(V.data_ptr()), None) == capi.OK
    torch.cuda.synchronize()
    got = V.cpu().numpy()
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    print(f"{desc}: max |dV| / max |V| = {err:.2e}")
    if desc.split("(")[0] in ("harmonic", "elliptic", "quartic", "quarticoscillator"):
        assert np.array_equal(got, ref)
    assert err < 1e-14


@pytest.mark.parametrize("shape,p0,p1", [(1, 1.0, 0.3), (1, 2.5, 1.0), (2, 2.0, 0.6), (3, 0.0, 0.0)])
def test_impurity_shapes_match_reference(shape, p0, p1):
    """itp2d_add_impurities against the reference's CoulombImpurities,
    HemisphereImpurities and DeltaImpurities::add_noise (noise.cpp:42-87),
    in list order on a harmonic base potential; delta impurities include two
    that land on the same grid point."""
    import ctypes as C

    import torch
    from oracle import refkit as R
    sx, sy, L = 96, 80, 12.0
    dx = L / sx
    rng = np.random.default_rng(shape + 7)
    n = 40
    pos = np.column_stack([rng.uniform(-5, 5, n), rng.uniform(-4, 4, n)])
    if shape == 3:
        pos[1] = pos[0] + 0.1 * dx  # same nearest grid point
        rows = np.column_stack([pos, rng.uniform(0.5, 1.5, n)])
    else:
        rows = pos
    x = (2 * np.arange(sx) + 1 - sx) * dx / 2
    y = (2 * np.arange(sy) + 1 - sy) * dx / 2
    V0 = 0.5 * (x[None, :] ** 2 + y[:, None] ** 2)
    ref = R.add_impurities(shape, sx, sy, dx, rows, p0, p1, V0)
    Vd = torch.tensor(V0, dtype=torch.float64, device="cuda")
    rd = torch.tensor(np.ascontiguousarray(rows), dtype=torch.float64, device="cuda")
    f = capi.lib().itp2d_add_impurities
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p, C.c_double, C.c_double,
                  C.c_void_p, C.c_void_p]
    assert f(shape, sx, sy, dx, n, C.c_void_p(rd.data_ptr()), p0, p1, C.c_void_p(Vd.data_ptr()), None) == capi.OK
    torch.cuda.synchronize()
    got = Vd.cpu().numpy()
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    print(f"impurity shape {shape}: max |dV| / max |V| = {err:.2e}")
    if shape == 3:
        assert np.array_equal(got, ref)
    assert err < 1e-14


def test_driver_uses_the_device_library():
    """The native driver takes every potential type through the device kernel:
    a system set up with "ring(2,1,2,0.5,1)" propagates states like the
    compiled reference's MultiProductSplit with that potential (one step,
    through the system's own context)."""
    import ctypes as C

    from itp2d_b200 import system
    from oracle import refkit as R
    g = O.Grid.from_length(64, 64, 10.0)
    psi = O.gaussian_states(g, 3, 21)
    desc = "ring(2,1,2,0.5,1)"
    p = system.Parameters(sx=64, sy=64, length=10.0, halforder=2, num_states=3, wanted=1, eps=[0.05],
                          potential=desc, max_steps=1)
    s = system.ITPSystem(p, init_states=psi)
    ctx = C.c_void_p(s.context_handle())
    L = capi.lib()
    a = np.ascontiguousarray(psi)
    assert L.itp2d_upload_states(ctx, a.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))) == capi.OK
    assert L.itp2d_propagate(ctx) == capi.OK
    out = np.empty_like(a)
    assert L.itp2d_download_states(ctx, out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))) == capi.OK
    kit = R.RefKit(64, 64, 10.0, 0, 0.0, 2, 0.05, 3, potential=desc, threads=1)
    kit.set_states(psi)
    kit.propagate()
    ref = kit.states()
    assert np.max(np.abs(out - ref)) / np.max(np.abs(ref)) < 1e-12
    s.close()
