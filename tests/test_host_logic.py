"""CPU tests of the host-side logic: libdipcu.so loads and exports every symbol include/dipcu.h
declares; boundary-condition strings, kernel-weight construction and the closed-form boundary
extension used by the kernels (diplib_b200/csrc/dipcu_common.cuh, compiled for the host by
tests/native/host_logic_shim.cpp) agree with the oracle."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from tests.conftest import HOSTLOGIC, ROOT

HEADER = os.path.join(ROOT, "include", "dipcu.h")
BCS = list(oracle.BC_CODES)


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dipcu_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from diplib_b200 import _abi
    lib = _abi.lib()
    syms = declared_symbols()
    assert "dipcu_gauss_fir" in syms
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) <= set(_abi.SIGNATURES), set(syms) - set(_abi.SIGNATURES)
    assert b"sm_100a" in lib.dipcu_version()


def test_bc_strings_match_reference_parser():
    from diplib_b200 import _abi
    lib = _abi.lib()
    for s in BCS:
        assert lib.dipcu_bc_from_string(s.encode()) == oracle.BC_CODES[s], s
        if oracle.ref_available():
            assert oracle.ref_lib().dipref_string_to_bc(s.encode()) == oracle.BC_CODES[s], s
    assert lib.dipcu_bc_from_string(b"symmetric mirror") == -1
    assert _abi.last_error() == "Boundary condition not recognized: symmetric mirror"
    if oracle.ref_available():
        assert oracle.ref_lib().dipref_string_to_bc(b"symmetric mirror") == -1


def test_boundary_parsing_errors_python():
    import diplib_b200 as dipcu
    with pytest.raises(dipcu.ParameterError, match="Boundary condition not recognized: bogus"):
        dipcu.BoundaryConditionFromString("bogus")


def _hl():
    l = ctypes.CDLL(HOSTLOGIC)
    l.hl_extend_f32.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p]
    l.hl_half_gaussian_length.restype = ctypes.c_int64
    l.hl_half_gaussian_length.argtypes = [ctypes.c_double, ctypes.c_uint32, ctypes.c_double, ctypes.c_int]
    l.hl_make_half_gaussian.argtypes = [ctypes.c_double, ctypes.c_uint32, ctypes.c_int64, ctypes.c_void_p,
                                        ctypes.c_void_p]
    return l


def host_half_gaussian(sigma, order, trunc, dt_double, with_derivative=False, lib=None):
    l = lib or _hl()
    n = l.hl_half_gaussian_length(sigma, order, trunc, int(dt_double))
    w = np.zeros(n)
    dw = np.zeros(n)
    l.hl_make_half_gaussian(sigma, order, n, w.ctypes.data, dw.ctypes.data if with_derivative else None)
    return (w, dw) if with_derivative else w


@pytest.mark.parametrize("dt_double", [False, True])
def test_weights_match_oracle(dt_double):
    from diplib_b200 import _abi
    for sigma in [0.3, 0.5, 0.8, 1.0, 1.5, 2.0, 3.0, 4.0, 7.3, 8.0, 20.0]:
        for order in range(4):
            for trunc in [0.0, 1.0, 3.0, 4.5, 10.0]:
                ref = oracle.half_gaussian(sigma, order, trunc, dt_double)[::-1]  # centre first
                got = host_half_gaussian(sigma, order, trunc, dt_double)
                assert got.shape == ref.shape, (sigma, order, trunc)
                np.testing.assert_array_equal(got, ref)
                assert _abi.lib().dipcu_half_gaussian_length(sigma, order, trunc, int(dt_double)) == ref.size
    assert _abi.lib().dipcu_half_gaussian_length(1.0, 4, 3.0, 0) == -1


def test_exp_rn_is_correctly_rounded():
    """exp_rn (the device weights' exp) against exp evaluated to 60 digits and rounded to double,
    over the argument range the weights use and beyond (normal results)."""
    from decimal import Decimal, getcontext
    getcontext().prec = 60
    l = ctypes.CDLL(HOSTLOGIC)
    l.hl_exp_rn.restype = ctypes.c_double
    l.hl_exp_rn.argtypes = [ctypes.c_double]
    rng = np.random.default_rng(7)
    xs = np.concatenate([rng.uniform(-60.0, 0.0, 4000), rng.uniform(-708.0, 709.0, 1000), -rng.random(500) * 1e-6,
                         [0.0, -0.5, -1.0, -4.5, -18.0, -0.34657359027997264, 0.34657359027997264]])
    for x in xs:
        got = l.hl_exp_rn(float(x))
        exact = Decimal(float(x)).exp()
        # the nearest double: no double beside `got` is closer to the exact value
        err = abs(Decimal(got) - exact)
        for nb in (np.nextafter(got, np.inf), np.nextafter(got, -np.inf)):
            assert err <= abs(Decimal(float(nb)) - exact), x


def test_device_weight_arithmetic_matches_reference_in_float():
    """The device weights (K0) compute with exp_rn instead of the C library's exp, which rounds a few
    arguments differently in the last double bit.  After the cast to float the taps must be the
    reference's bit for bit: the host build of the same arithmetic (libhostlogic_rn) against the
    reference's MakeHalfGaussian over a grid of sigmas, all orders and truncations."""
    lrn = ctypes.CDLL(HOSTLOGIC.replace("libhostlogic.so", "libhostlogic_rn.so"))
    lrn.hl_half_gaussian_length.restype = ctypes.c_int64
    lrn.hl_half_gaussian_length.argtypes = [ctypes.c_double, ctypes.c_uint32, ctypes.c_double, ctypes.c_int]
    lrn.hl_make_half_gaussian.argtypes = [ctypes.c_double, ctypes.c_uint32, ctypes.c_int64, ctypes.c_void_p,
                                          ctypes.c_void_p]
    rng = np.random.default_rng(3)
    sigmas = list(np.round(rng.uniform(0.3, 30.0, 300), 3)) + [0.8, 1.0, 1.5, 2.0, 3.0, 4.0, 8.0, 11.0]
    for sigma in sigmas:
        for order in range(4):
            for trunc in (3.0, 4.5):
                ref = oracle.half_gaussian(float(sigma), order, trunc, False)[::-1].astype(np.float32)
                got = host_half_gaussian(float(sigma), order, trunc, False, lib=lrn).astype(np.float32)
                np.testing.assert_array_equal(got, ref, err_msg=f"sigma {sigma} order {order} trunc {trunc}")


@pytest.mark.parametrize("order", [0, 1, 2, 3])
def test_sigma_derivative_of_weights(order):
    for sigma in [0.9, 1.5, 3.0, 6.0]:
        w, dw = host_half_gaussian(sigma, order, 3.0, False, with_derivative=True)
        n = w.size
        h = 1e-6
        l = _hl()
        wp = np.zeros(n)
        wm = np.zeros(n)
        l.hl_make_half_gaussian(sigma + h, order, n, wp.ctypes.data, None)
        l.hl_make_half_gaussian(sigma - h, order, n, wm.ctypes.data, None)
        fd = (wp - wm) / (2 * h)
        np.testing.assert_allclose(dw, fd, rtol=1e-5, atol=1e-8 * np.abs(fd).max())


def test_boundary_closed_forms_match_expand_buffer():
    l = _hl()
    rng = np.random.default_rng(7)
    for bc in BCS:
        code = oracle.BC_CODES[bc]
        if code == 12:
            continue
        for n in [1, 2, 3, 4, 7, 10]:
            for border in [1, 2, 5, 9, 23]:
                line = (rng.random(n) * 10 - 3).astype(np.float32)
                ref = oracle.expand_buffer(line, border, border, bc)
                got = np.zeros(n + 2 * border, np.float32)
                l.hl_extend_f32(line.ctypes.data, n, border, code, got.ctypes.data)
                if bc in ("antisym reflect",):
                    # Multiple reflections: the reference rounds each stored value before
                    # deriving the next offset; the closed form rounds once.
                    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-5)
                else:
                    assert np.array_equal(got, ref), (bc, n, border)


@pytest.mark.skipif(not oracle.ref_available(), reason="the compiled reference (oracle/_ref) is not built")
def test_read_pixel_known_answers_of_the_reference():
    """The reference's own check of ReadPixelWithBoundaryCondition (src/library/boundary.cpp:331-381):
    a 15 x 10 sfloat image of uniform noise in [0.5, 3.8), read at coordinates just outside the
    image and around the turn into the second reflection or period, for every boundary condition
    it lists.  Here the kernels' closed-form extension, applied separably (rows along x, then
    columns along y), must give the reference's value exactly."""
    l = _hl()
    rng = np.random.default_rng(11)
    img = rng.uniform(0.5, 3.8, size=(10, 15)).astype(np.float32)   # DIPlib sizes {15, 10}
    coords = [(0, 0), (-1, 0), (0, -1), (-1, -1), (20, 14), (19, 15), (20, 15), (28, -9), (29, -9), (28, -10),
              (29, -10), (30, -10), (29, -11), (30, -11)]
    bx, by = 20, 16

    def ext(line, border, code):
        line = np.ascontiguousarray(line, np.float32)
        out = np.zeros(line.size + 2 * border, np.float32)
        l.hl_extend_f32(line.ctypes.data, line.size, border, code, out.ctypes.data)
        return out

    for bc in ["mirror", "asym mirror", "periodic", "asym periodic", "add zeros", "add max", "add min", "zero order"]:
        code = oracle.BC_CODES[bc]
        rows = np.stack([ext(img[y], bx, code) for y in range(img.shape[0])])
        full = np.stack([ext(rows[:, c], by, code) for c in range(rows.shape[1])], axis=1)
        for x, y in coords:
            assert full[y + by, x + bx] == oracle.ref_read_pixel_bc(img, [x, y], [code, code]), (bc, x, y)
