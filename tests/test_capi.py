"""CPU-side checks of the C ABI library: it loads, and it exports every
entry point declared in include/itp2d_gpu.h. No device calls."""
import ctypes

from itp2d_b200 import capi


def test_library_exports_header_symbols():
    L = capi.lib()
    names = capi.header_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings():
    L = capi.lib()
    for code in range(9):
        s = L.itp2d_status_string(code)
        assert s and s != b"unknown status"
    assert L.itp2d_status_string(99) == b"unknown status"


def test_invalid_arguments_rejected_before_device_use():
    L = capi.lib()
    out = ctypes.c_void_p()
    # sizes and enums are validated before any CUDA call
    assert L.itp2d_ctx_create(1, 16, 0.1, 4, 0, 0.0, 1, 0, None, ctypes.byref(out)) == capi.E_INVALID
    assert L.itp2d_ctx_create(16, 16, 0.1, 4, 7, 0.0, 1, 0, None, ctypes.byref(out)) == capi.E_INVALID
    assert L.itp2d_ctx_create(22, 16, 0.1, 4, 0, 0.0, 1, 0, None, ctypes.byref(out)) == capi.E_UNSUPPORTED
    assert L.itp2d_ctx_create(8192, 16, 0.1, 4, 1, 1.0, 1, 0, None, ctypes.byref(out)) == capi.E_UNSUPPORTED
    assert L.itp2d_propagate(None) == capi.E_INVALID


def test_impurity_arguments_rejected_before_device_use():
    L = capi.lib()
    V = ctypes.c_void_p(1)  # never dereferenced: every case below returns before a CUDA call
    imp = ctypes.c_void_p(1)
    add = L.itp2d_add_gaussian_impurities
    assert add(0, 16, 0.1, 1, imp, V, None) == capi.E_INVALID       # empty grid
    assert add(16, 16, 0.0, 1, imp, V, None) == capi.E_INVALID      # dx <= 0
    assert add(16, 16, 0.1, -1, imp, V, None) == capi.E_INVALID     # negative count
    assert add(16, 16, 0.1, 1, None, V, None) == capi.E_INVALID     # no impurity list
    assert add(16, 16, 0.1, 1, imp, None, None) == capi.E_INVALID   # no potential
    assert add(16, 16, 0.1, 0, None, V, None) == capi.OK            # nothing to add


def test_library_exports_host_header_symbols():
    """Every function of include/itp2d_host.h (the native driver and the
    serving loop) is exported too."""
    import os
    import re
    L = capi.lib()
    txt = open(os.path.join(capi.ROOT, "include", "itp2d_host.h")).read()
    names = sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*\**\s+\**(itp2d_[a-z0-9_]+)\s*\(",
                                  txt, flags=re.M)))
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_footprint_estimate():
    """itp2d_ctx_footprint counts the state buffers (two, three for
    halforder >= 3 or Dirichlet with a field) and the tensor-core scratch,
    and grows with k and N; it computes without a device."""
    fp = capi.lib().itp2d_ctx_footprint
    fp.restype = ctypes.c_longlong
    fp.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int]
    a = fp(256, 256, 500, 0, 1.0, 2)
    assert a >= 2 * 256 * 256 * 500 * 16
    assert fp(256, 256, 500, 0, 1.0, 3) >= 3 * 256 * 256 * 500 * 16
    assert fp(256, 256, 500, 1, 0.7, 2) >= 3 * 256 * 256 * 500 * 16
    assert fp(256, 256, 1000, 0, 1.0, 2) > a and fp(512, 512, 500, 0, 1.0, 2) > a
    # the state buffers (2 x 16 bytes per complex) and the FP32 form's pre-split
    # tensor-core operands (2 x 12 bytes) dominate
    assert a < 1.15 * (2 * 16 + 2 * 12) * 256 * 256 * 500
    assert fp(1, 16, 4, 0, 0.0, 1) == -1


def test_server_refuses_before_device_use():
    """The serving loop validates and admits on the host: a request larger
    than the whole budget is refused at submission, before any device call."""
    from itp2d_b200 import system
    with system.Server(2, 1e6) as srv:
        p = system.Parameters(sx=64, sy=64, num_states=16, wanted=8, halforder=2, eps=[0.1])
        try:
            srv.submit(p)
        except capi.ITP2DError as e:
            assert e.status == capi.E_OOM
        else:
            raise AssertionError("oversized request admitted")
        assert srv.stats()["queued"] == 0 and srv.stats()["completed"] == 0
    L = capi.lib()
    out = ctypes.c_void_p()
    assert L.itp2d_server_create(0, 1e9, ctypes.byref(out)) == capi.E_INVALID
    assert L.itp2d_server_create(2, 0.0, ctypes.byref(out)) == capi.E_INVALID


def test_potential_descriptions_checked_like_the_reference():
    """itp2d_potential_check applies the reference's names, parameter counts
    and value checks (potentialtypes.cpp:56-500) without a device."""
    L = capi.lib()
    f = L.itp2d_potential_check
    f.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    good = ["zero", "harmonic", "harmonic(2)", "harmonic(1,0.5,-0.5)", "elliptic(1,2)", "prettyhardsquare(6)",
            "softpentagon", "henonheiles", "henon(1,-1)", "gaussian(1,2)", "gaussianblob(1,2,0,1)",
            "quartic(0.1)", "quarticoscillator", "squareoscillator(4)", "power(3)", "poweroscillator(3,2)",
            "ring", "ring(3,1,2)", "ringpotential(3,1,2,0.5,1)", "cosh(1,2)", "coshpotential",
            "softstadium", "softstadium(1,2,100)", "softstadium(1,2,100,1,10)", "powerstadium(4)",
            "powerstadium(1,2,4)"]
    bad = ["nosuchpotential", "harmonic(1,2)", "harmonic(-1)", "elliptic(1)", "elliptic(-1,1)",
           "softpentagon(1)", "gaussian(1,0)", "gaussian(-1,1)", "quartic(-1)", "power(2,-1)", "ring(-1,1,2)",
           "ring(3,0,2)", "ring(3,1)", "cosh(0,1)", "cosh(1,0)", "softstadium(0,2,100)", "softstadium(1,2)",
           "powerstadium(1,0,4)", "powerstadium(1,2)", "zero(1)", "harmonic(1", "harmonic(a)"]
    for d in good:
        n = ctypes.c_int(-1)
        assert f(d.encode(), ctypes.byref(n)) == capi.OK, d
        assert n.value == (1 if d == "zero" else 0)
    for d in bad:
        assert f(d.encode(), None) == capi.E_INVALID, d
    # device entry points reject bad arguments before any device call
    ev = L.itp2d_evaluate_potential
    ev.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    assert ev(b"foo", 16, 16, 0.1, ctypes.c_void_p(1), None) == capi.E_INVALID
    assert ev(b"harmonic", 0, 16, 0.1, ctypes.c_void_p(1), None) == capi.E_INVALID
    add = L.itp2d_add_impurities
    add.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
                    ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    assert add(9, 16, 16, 0.1, 1, ctypes.c_void_p(1), 1.0, 1.0, ctypes.c_void_p(1), None) == capi.E_INVALID
    assert add(1, 16, 16, 0.1, 0, None, 1.0, 1.0, ctypes.c_void_p(1), None) == capi.OK


def test_parameter_defaults_match_the_reference_and_leave_extensions_off():
    """itp2d_parameters_default gives the reference's defaults
    (parameters.cpp:25-55) and leaves every extension off: canonical
    orthonormalisation every step, Lowdin between (unused), no Rayleigh-Ritz
    step at the switch, the default switch-rule span."""
    from itp2d_b200 import system
    p = system._Params()
    system._lib().itp2d_parameters_default(ctypes.byref(p))
    assert (p.halforder, p.num_states, p.wanted, p.max_steps) == (5, 25, 16, 50)
    assert p.eps_divisor == 5.0 and p.min_eps == 1e-9
    assert p.precision == capi.FP64 and p.fp32_switch == 0.0
    assert p.fp32_canonical_every == 0 and p.fp32_between == capi.BETWEEN_LOWDIN
    assert p.switch_rayleigh_ritz == 0 and p.fp32_switch_span == 0 and p.fp32_eig_sweeps == 0
    assert p.fp64_engine == 0 and p.fp32_canonical_delay == 0
    assert p.timestep_test == b"relstdev(1e-3,1e-4)" and p.final_test == b"relstdev(1e-3,0)"


def test_signal_flags_are_process_wide_ints():
    """The abort and save flags the handlers raise are two distinct
    sig_atomic_t (int) objects owned by the library, lowered at load."""
    from itp2d_b200 import system
    a, s = system.abort_flag(), system.save_flag()
    assert ctypes.addressof(a.contents) != ctypes.addressof(s.contents)
    assert a[0] in (0, 1) and s[0] in (0, 1)
