"""GPU parity at the grid sizes the benchmark and the configurations run.

The register-FFT passes (``row_reg`` / ``col_reg`` / ``energy_*_reg`` in
csrc/rfft.cu) are one template instantiation per line length: 32, 64, 128,
256, 512 and 1024 points, each with its own split of the line over threads
and its own register footprint, in FP64 and FP32. Every one of them is
reached here by one propagation step, one Hamiltonian application and the
energies, compared with the oracle (and at the magnetic-dot and bumpy-dot
grids with the compiled reference itself):

* FP64: per state max|dpsi| / max|psi_ref| <= 1e-12, as for the small grids;
* FP32 form: the same quantity against the FP64 oracle within a bound derived
  from single precision (stated beside each assertion).

Reference: ExpKinetic (expkinetic.cpp:79-107,158-172), MultiProductSplit
(multiproductsplit.cpp:23-59), Kinetic (kinetic.cpp:99-142),
Operator::mean_and_standard_deviation (operators.cpp:40-50).
"""
import numpy as np
import pytest

from oracle import itp_oracle as O

pytestmark = pytest.mark.gpu

# sx, sy, L, boundary, B, halforder, eps, bumps; comments name the register
# instantiations <A,B> (line = A * B points over B threads) the grid reaches.
SIZES = [
    (128, 128, 12.0, O.PERIODIC, 0.0, 1, 0.02, 0),    # rows/cols <16,8>, B = 0 kinetic
    (128, 128, 12.0, O.DIRICHLET, 0.0, 1, 0.02, 0),   # configuration C1's grid (DST-II/III lines)
    (256, 256, 14.0, O.PERIODIC, 1.0, 2, 0.05, 0),    # magnetic dot: <16,16>
    (512, 512, 16.0, O.PERIODIC, 0.5, 3, 0.05, 20),   # bumpy dot: <32,16>
    (1024, 64, 16.0, O.PERIODIC, 0.3, 2, 0.05, 5),    # rows <32,32>, columns <8,8>
    (64, 1024, 16.0, O.PERIODIC, 0.3, 2, 0.05, 5),    # rows <8,8>, columns <32,32>
    (256, 128, 12.0, O.PERIODIC, 0.0, 2, 0.05, 3),    # B = 0 on a rectangle: rows <16,16>, cols <16,8>
    (32, 512, 16.0, O.PERIODIC, 0.0, 3, 0.05, 3),     # rows <8,4>, columns <32,16>, B = 0
]
IDS = [f"{s[0]}x{s[1]}_{'dir' if s[3] else 'per'}_B{s[4]}_m{s[5]}" for s in SIZES]
K = 3


@pytest.fixture(scope="module")
def capi():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import capi as C
    C.lib()
    return C


def per_state_rel(a, b):
    return float(np.max(np.max(np.abs(a - b), axis=(-2, -1)) / np.max(np.abs(b), axis=(-2, -1))))


def setup(cfg):
    sx, sy, L, bt, B, m, eps, nb = cfg
    g = O.Grid.from_length(sx, sy, L)
    V = O.harmonic(g) + (O.bumpy_potential(g, nb, 7, extent=L / 3) if nb else 0.0)
    psi = O.gaussian_states(g, K, sx + 3 * sy)
    return g, V, psi, bt, B, m, eps


_cache = {}


def oracle_outputs(cfg):
    """Propagated states, H psi of the input, and energies of the normalised
    propagated states, from the numpy restatement (cached per grid)."""
    if cfg not in _cache:
        g, V, psi, bt, B, m, eps = setup(cfg)
        prop = O.MultiProductSplit(g, V, bt, B, m, eps).apply(psi)
        H = O.Hamiltonian(g, V, bt, B)
        hpsi = H.apply(psi)
        nrm = np.sqrt(np.sum(np.abs(prop) ** 2, axis=(1, 2))) * g.dx
        pn = prop / nrm[:, None, None]
        mean, sd = O.energies(H, pn)
        hp = H.apply(pn)
        res = np.sqrt(np.sum(np.abs(hp - mean.real[:, None, None] * pn) ** 2, axis=(1, 2))) * g.dx
        _cache[cfg] = (prop, hpsi, pn, mean.real, sd.real, res)
    return _cache[cfg]


@pytest.mark.parametrize("cfg", SIZES, ids=IDS)
def test_fp64_step_matches_oracle(capi, cfg):
    g, V, psi, bt, B, m, eps = setup(cfg)
    prop, hpsi, pn, E_ref, sd_ref, res_ref = oracle_outputs(cfg)
    c = capi.Context(g.sx, g.sy, g.dx, K, bt, B, m)
    c.set_column_variant(capi.COL_SMEM)
    c.set_potential(V)
    c.set_time_step(eps)
    c.upload(psi)
    c.propagate()
    assert per_state_rel(c.download(), prop) < 1e-12
    c.upload(psi)
    c.apply_hamiltonian()
    assert per_state_rel(c.download(), hpsi) < 1e-12
    c.upload(pn)
    E, sig, res, Ei = c.energies()
    assert np.max(np.abs(E - E_ref) / np.abs(E_ref)) < 1e-12
    # sigma through <H^2> - <H>^2 is bounded by its FP64 cancellation floor
    assert np.max(np.abs(sig - sd_ref)) < 1e-10 * np.max(np.abs(E_ref))
    # residual ||H psi - E psi|| of normalised states. The first call shifts by
    # the previous energies held in the context (none yet), so it is
    # ||H psi||^2 - E^2 under one square root; the second shifts by these
    # energies and has no cancellation.
    assert np.max(np.abs(res - res_ref) / res_ref) < 1e-8
    E2, sig2, res2, _ = c.energies()
    assert np.max(np.abs(res2 - res_ref) / res_ref) < 1e-11
    assert np.array_equal(E, E2)


@pytest.mark.parametrize("cfg", SIZES, ids=IDS)
def test_fp32_form_step_matches_fp64_oracle(capi, cfg):
    """The FP32 sweep kernels against the FP64 oracle. A line FFT of N points
    in single precision has an error of a few 2^-24 * log2(N) relative to the
    line's largest value; a step chains 2 m(m+2) such passes and the
    multi-product sum (coefficients up to 81/40 in absolute value at m = 3)
    adds them, so 2e-5 of max|psi| per state bounds a step. Energies are
    Rayleigh quotients accumulated in FP64 from FP32 products: 2e-6 relative."""
    g, V, psi, bt, B, m, eps = setup(cfg)
    prop, hpsi, pn, E_ref, sd_ref, res_ref = oracle_outputs(cfg)
    c = capi.Context(g.sx, g.sy, g.dx, K, bt, B, m, capi.FP32)
    c.set_column_variant(capi.COL_SMEM)
    c.set_potential(V)
    c.set_time_step(eps)
    c.upload(psi)
    c.propagate()
    err = per_state_rel(c.download(), prop)
    assert err < 2e-5, err
    c.upload(psi)
    c.apply_hamiltonian()
    err_h = per_state_rel(c.download(), hpsi)
    assert err_h < 2e-5, err_h
    c.upload(pn)
    E, sig, res, Ei = c.energies()
    assert np.max(np.abs(E - E_ref) / np.abs(E_ref)) < 2e-6
    # the residual of an FP32 state is accurate to the FP32 rounding of H psi
    assert np.max(np.abs(res - res_ref) / res_ref) < 1e-4


@pytest.mark.parametrize("cfg", [SIZES[2], SIZES[3]], ids=["magnetic_dot_256", "bumpy_dot_512"])
def test_fp64_step_matches_compiled_reference(capi, cfg):
    """The magnetic-dot and bumpy-dot grids against the reference's own
    MultiProductSplit and Hamiltonian (oracle/_ref, compiled from the
    reference sources) on the same states and potential."""
    from oracle import refkit as R
    if not R.available():
        pytest.fail("oracle/_ref/libitp2d_ref.so missing: build it with make -C oracle")
    g, V, psi, bt, B, m, eps = setup(cfg)
    nb = cfg[7]
    bumps = O.bumpy_potential(g, nb, 7, extent=g.lenx / 3) if nb else None
    kit = R.RefKit(g.sx, g.sy, g.lenx, bt, B, m, eps, K, potential="harmonic(1)", extra_potential=bumps,
                   threads=4)
    V = kit.potential()  # the reference's own table, fed to both codes
    kit.set_states(psi)
    kit.propagate()
    prop = kit.states()
    kit.set_states(psi)
    kit.apply_hamiltonian()
    hpsi = kit.states()
    c = capi.Context(g.sx, g.sy, g.dx, K, bt, B, m)
    c.set_potential(V)
    c.set_time_step(eps)
    c.upload(psi)
    c.propagate()
    assert per_state_rel(c.download(), prop) < 1e-12
    c.upload(psi)
    c.apply_hamiltonian()
    assert per_state_rel(c.download(), hpsi) < 1e-12


# the grids whose column lines take the TMA pass (256 and 512 points, periodic)
TMA_SIZES = [c for c in SIZES if c[3] == O.PERIODIC and c[1] in (256, 512)]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("cfg", TMA_SIZES, ids=[f"{c[0]}x{c[1]}_B{c[4]}_m{c[5]}" for c in TMA_SIZES])
def test_tma_column_pass_matches_staged_pass(capi, cfg, precision):
    """The TMA column pass (tiles moved by cp.async.bulk.tensor through a
    three-slot ring) gives the same step as the register-staged pass, bit for
    bit: both run the same line transforms on the same values. Checked on the
    propagation (mode 0 passes with the kinetic tables) and on the
    Hamiltonian, with k = 37 states (ragged last tiles of a CTA's ring)."""
    g, V, psi, bt, B, m, eps = setup(cfg)
    rng = np.random.default_rng(5)
    psi = np.concatenate([psi] * 13)[:37] * (1 + 0.1 * rng.standard_normal((37, 1, 1)))
    out = {}
    for variant in (capi.COL_SMEM, capi.COL_TMA):
        c = capi.Context(g.sx, g.sy, g.dx, 37, bt, B, m, capi.FP64 if precision == "fp64" else capi.FP32)
        c.set_column_variant(variant)
        assert c.column_variant == variant
        c.set_potential(V)
        c.set_time_step(eps)
        c.upload(psi)
        c.propagate()
        a = c.download()
        c.apply_hamiltonian()
        out[variant] = (a, c.download(), c.energies()[0])
        c.close()
    for x, y in zip(out[capi.COL_SMEM], out[capi.COL_TMA]):
        assert np.array_equal(x, y)
    # and the TMA step against the oracle
    prop = O.MultiProductSplit(g, V, bt, B, m, eps).apply(psi)
    tol = 1e-12 if precision == "fp64" else 2e-5
    assert per_state_rel(out[capi.COL_TMA][0], prop) < tol


def test_column_variant_is_tuned_at_the_first_time_step(capi):
    """The first time step of a precision times the column passes at the
    bumpy-dot grid and keeps one of them; -1 restores the tuned choice after a
    forced one; out-of-range variants are refused."""
    g, V, psi, bt, B, m, eps = setup(SIZES[3])
    c = capi.Context(g.sx, g.sy, g.dx, 64, bt, B, m, capi.FP32)
    c.set_potential(V)
    c.set_time_step(eps)
    tuned = c.column_variant
    assert tuned in (capi.COL_SMEM, capi.COL_TMA)
    c.set_column_variant(1 - tuned)
    assert c.column_variant == 1 - tuned
    c.set_column_variant(-1)
    assert c.column_variant == tuned
    with pytest.raises(capi.ITP2DError):
        c.set_column_variant(2)
    print(f"bumpy-dot grid, FP32: column variant {tuned}")
