"""Test infrastructure only: Python access to the two CPU checkers of the Gaussian FIR path.

* ``liboracle_gauss.so`` -- the plain-C restatement in ``gauss_oracle.c`` (always built).
* ``_ref/libdipref.so`` -- the unmodified DIPlib sources compiled by ``oracle/Makefile``, reached
  through ``ref_shim.cpp`` (only where the reference tree was present at build time).

Nothing in the product imports this package; ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg use it as the checker.

Arrays are numpy arrays in numpy axis order (slowest first).  Like PyDIP
(pydip/src/image.cpp:25-33,148-151) the DIPlib axis order is the reverse, and per-axis
parameters (sigmas, orders, boundary conditions) are listed x first.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle_gauss.so")
REF_LIB = os.path.join(HERE, "_ref", "libdipref.so")

DTYPE_CODES = {
    np.dtype(np.bool_): 0, np.dtype(np.uint8): 1, np.dtype(np.uint16): 2, np.dtype(np.uint32): 3,
    np.dtype(np.uint64): 4, np.dtype(np.int8): 5, np.dtype(np.int16): 6, np.dtype(np.int32): 7,
    np.dtype(np.int64): 8, np.dtype(np.float32): 9, np.dtype(np.float64): 10,
}
CODE_DTYPES = {v: k for k, v in DTYPE_CODES.items()}

# dip::BoundaryCondition enumerators and their strings (include/diplib/boundary.h:65-109,
# include/diplib/library/stringparams.h:259-272).
BC_CODES = {
    "": 0, "default": 0, "mirror": 0, "asym mirror": 1, "antisym reflect": 2, "periodic": 3,
    "asym periodic": 4, "add zeros": 5, "add max": 6, "add min": 7, "zero order": 8,
    "first order": 9, "second order": 10, "third order": 11, "already expanded": 12,
}

_i64p = ctypes.POINTER(ctypes.c_int64)


def _load(path):
    if not os.path.exists(path):
        return None
    return ctypes.CDLL(path)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        _oracle = _load(ORACLE_LIB)
        if _oracle is None:
            raise RuntimeError(f"{ORACLE_LIB} is not built (run `make -C oracle`)")
        _oracle.or_gauss_fir.restype = ctypes.c_int
        _oracle.or_make_half_gaussian.restype = ctypes.c_int
        _oracle.or_make_half_gaussian.argtypes = [ctypes.c_double, ctypes.c_uint, ctypes.c_double, ctypes.c_int,
                                                  ctypes.c_void_p, ctypes.c_int]
        _oracle.or_half_gaussian_size.restype = ctypes.c_size_t
        _oracle.or_half_gaussian_size.argtypes = [ctypes.c_double, ctypes.c_uint, ctypes.c_double, ctypes.c_int]
        for fn in (_oracle.or_expand_buffer_f32, _oracle.or_expand_buffer_f64):
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_void_p, ctypes.c_ssize_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
                           ctypes.c_int]
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        _ref = _load(REF_LIB)
        if _ref is None:
            raise RuntimeError(f"{REF_LIB} is not built (run `make -C oracle ref` where the reference tree exists)")
        _ref.dipref_half_gaussian.argtypes = [ctypes.c_double, ctypes.c_uint32, ctypes.c_double, ctypes.c_int,
                                              ctypes.c_void_p, ctypes.c_int]
        _ref.dipref_expand_buffer.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64,
                                              ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int]
        _ref.dipref_max_gauss_truncation.restype = ctypes.c_double
        _ref.dipref_structure_tensor.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _i64p, ctypes.c_double,
                                                 ctypes.c_double, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                                                 ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                                 ctypes.POINTER(ctypes.c_int), ctypes.c_char_p,
                                                 ctypes.c_int]
        _ref.dipref_derivative_op.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _i64p,
                                              ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                              ctypes.c_char_p, ctypes.c_int]
    return _ref


def bc_code(bc: str) -> int:
    if bc not in BC_CODES:
        raise ValueError("Boundary condition not recognized: " + bc)
    return BC_CODES[bc]


def suggest_flex(dtype) -> np.dtype:
    """DataType::SuggestFlex (src/library/datatype.cpp:109-124) for real types."""
    dt = np.dtype(dtype)
    if dt in (np.dtype(np.uint32), np.dtype(np.int32), np.dtype(np.uint64), np.dtype(np.int64),
              np.dtype(np.float64)):
        return np.dtype(np.float64)
    return np.dtype(np.float32)


def _dip_geometry(a: np.ndarray):
    """DIPlib sizes/strides (x first, in samples) of a numpy array."""
    sizes = (ctypes.c_int64 * a.ndim)(*reversed(a.shape))
    strides = (ctypes.c_int64 * a.ndim)(*(s // a.itemsize for s in reversed(a.strides)))
    return sizes, strides


def _broadcast(values, nd, default):
    """ArrayUseParameter: 0 entries -> default, 1 entry -> broadcast, nd entries -> as is."""
    values = list(values) if values is not None else []
    if len(values) == 0:
        return [default] * nd
    if len(values) == 1:
        return values * nd
    if len(values) != nd:
        raise ValueError("Array parameter has the wrong number of elements")
    return values


# ------------------------------------------------------------------------------------------------
# The C restatement
# ------------------------------------------------------------------------------------------------

def half_gaussian(sigma: float, order: int, truncation: float = 3.0, dt_double: bool = False) -> np.ndarray:
    lib = oracle_lib()
    n = lib.or_make_half_gaussian(sigma, order, truncation, int(dt_double), None, 0)
    if n < 0:
        raise ValueError("Gaussian FIR filter not implemented for order > 3")
    out = np.zeros(n, np.float64)
    lib.or_make_half_gaussian(sigma, order, truncation, int(dt_double), out.ctypes.data, n)
    return out


def expand_buffer(line: np.ndarray, left: int, right: int, bc: str) -> np.ndarray:
    """Returns `line` extended by `left`/`right` samples with boundary condition `bc`."""
    line = np.ascontiguousarray(line)
    buf = np.zeros(left + line.size + right, line.dtype)
    buf[left:left + line.size] = line
    fn = oracle_lib().or_expand_buffer_f64 if line.dtype == np.float64 else oracle_lib().or_expand_buffer_f32
    ptr = buf.ctypes.data + left * buf.itemsize
    st = fn(ptr, 1, line.size, left, right, bc_code(bc))
    if st != 0:
        raise RuntimeError(f"or_expand_buffer failed ({st})")
    return buf


def gauss_fir(x: np.ndarray, sigmas: Sequence[float] = (1.0,), orders: Sequence[int] = (0,),
              bcs: Sequence[str] = (), truncation: float = 3.0, out_dtype=None) -> np.ndarray:
    """The restated dip::GaussFIR on a numpy array (parameters in DIPlib order, x first)."""
    nd = x.ndim
    sig = _broadcast(sigmas, nd, 1.0)
    ords = _broadcast(orders, nd, 0)
    bcl = _broadcast(bcs, nd, "mirror")
    out_dt = suggest_flex(x.dtype) if out_dtype is None else np.dtype(out_dtype)
    out = np.zeros(x.shape, out_dt)
    sizes, in_strides = _dip_geometry(x)
    _, out_strides = _dip_geometry(out)
    st = oracle_lib().or_gauss_fir(
        ctypes.c_void_p(x.ctypes.data), DTYPE_CODES[x.dtype], nd, sizes, in_strides,
        ctypes.c_void_p(out.ctypes.data), DTYPE_CODES[out_dt], out_strides,
        (ctypes.c_double * nd)(*sig), (ctypes.c_uint * nd)(*ords), (ctypes.c_int * nd)(*[bc_code(b) for b in bcl]),
        ctypes.c_double(truncation))
    if st == 1:
        raise ValueError("Gaussian FIR filter not implemented for order > 3")
    if st != 0:
        raise RuntimeError(f"or_gauss_fir failed ({st})")
    return out


def gauss_iir(x: np.ndarray, sigmas: Sequence[float] = (1.0,), orders: Sequence[int] = (0,),
              bcs: Sequence[str] = (), filter_orders: Sequence[int] | None = None,
              design: str = "discrete time fit", truncation: float = 3.0, out_dtype=None) -> np.ndarray:
    """The restated dip::GaussIIR on a numpy array (parameters in DIPlib order, x first)."""
    nd = x.ndim
    sig = _broadcast(sigmas, nd, 1.0)
    ords = _broadcast(orders, nd, 0)
    bcl = _broadcast(bcs, nd, "mirror")
    out_dt = suggest_flex(x.dtype) if out_dtype is None else np.dtype(out_dtype)
    out = np.zeros(x.shape, out_dt)
    sizes, in_strides = _dip_geometry(x)
    _, out_strides = _dip_geometry(out)
    fo = None if not filter_orders else (ctypes.c_uint * nd)(*_broadcast(filter_orders, nd, 3))
    if design not in ("discrete time fit", "forward backward"):
        raise ValueError("Invalid flag: " + design)
    lib = oracle_lib()
    lib.or_gauss_iir.restype = ctypes.c_int
    st = lib.or_gauss_iir(
        ctypes.c_void_p(x.ctypes.data), DTYPE_CODES[x.dtype], nd, sizes, in_strides,
        ctypes.c_void_p(out.ctypes.data), DTYPE_CODES[out_dt], out_strides,
        (ctypes.c_double * nd)(*sig), (ctypes.c_uint * nd)(*ords), (ctypes.c_int * nd)(*[bc_code(b) for b in bcl]),
        fo, int(design == "forward backward"), ctypes.c_double(truncation))
    if st != 0:
        raise RuntimeError(f"or_gauss_iir failed ({st})")
    return out


SYMMETRIES = {"": 0, "general": 0, "even": 1, "odd": 2, "conj": 1, "d-even": 3, "d-odd": 4, "d-conj": 3}


def _filter_arrays(filters):
    """(data pointers, lens, origins, symmetry codes, symmetry strings, keep-alive) of filters given as
    dicts {"filter": values, "origin": int (-1 centre), "symmetry": str} (dip::OneDimensionalFilter)."""
    n = len(filters)
    arrs = [np.ascontiguousarray(np.asarray(f["filter"], dtype=np.float64)) for f in filters]
    data = (ctypes.c_void_p * n)(*[a.ctypes.data for a in arrs])
    lens = (ctypes.c_int * n)(*[a.size for a in arrs])
    origins = (ctypes.c_long * n)(*[int(f.get("origin", -1)) for f in filters])
    syms = [str(f.get("symmetry", "general")) for f in filters]
    codes = (ctypes.c_int * n)(*[SYMMETRIES[s_] for s_ in syms])
    return data, lens, origins, codes, syms, arrs


def separable_convolution(x: np.ndarray, filters, bcs: Sequence[str] = (), process=None, out_dtype=None) -> np.ndarray:
    """The restated dip::SeparableConvolution (real filters) on a numpy array."""
    nd = x.ndim
    if len(filters) not in (1, nd):
        raise ValueError("Array parameter has the wrong number of elements")
    bcl = _broadcast(bcs, nd, "mirror")
    out_dt = suggest_flex(x.dtype) if out_dtype is None else np.dtype(out_dtype)
    out = np.zeros(x.shape, out_dt)
    sizes, in_strides = _dip_geometry(x)
    _, out_strides = _dip_geometry(out)
    data, lens, origins, codes, _, keep = _filter_arrays(filters)
    proc = None if process is None else (ctypes.c_int * nd)(*[int(bool(p)) for p in process])
    lib = oracle_lib()
    st = lib.or_separable_convolution(
        ctypes.c_void_p(x.ctypes.data), DTYPE_CODES[x.dtype], nd, sizes, in_strides,
        ctypes.c_void_p(out.ctypes.data), DTYPE_CODES[out_dt], out_strides, len(filters), data, lens, origins, codes,
        (ctypes.c_int * nd)(*[bc_code(b) for b in bcl]), proc)
    if st != 0:
        raise RuntimeError(f"or_separable_convolution failed ({st})")
    return out


def uniform(x: np.ndarray, sizes, bcs: Sequence[str] = (), out_dtype=None) -> np.ndarray:
    """The restated dip::Uniform with a rectangular kernel of per-axis `sizes` (DIPlib order)."""
    nd = x.ndim
    fs = _broadcast(sizes, nd, 7)
    bcl = _broadcast(bcs, nd, "mirror")
    out_dt = suggest_flex(x.dtype) if out_dtype is None else np.dtype(out_dtype)
    out = np.zeros(x.shape, out_dt)
    isz, in_strides = _dip_geometry(x)
    _, out_strides = _dip_geometry(out)
    st = oracle_lib().or_uniform_rect(
        ctypes.c_void_p(x.ctypes.data), DTYPE_CODES[x.dtype], nd, isz, in_strides,
        ctypes.c_void_p(out.ctypes.data), DTYPE_CODES[out_dt], out_strides,
        (ctypes.c_int64 * nd)(*[int(f) for f in fs]), (ctypes.c_int * nd)(*[bc_code(b) for b in bcl]))
    if st != 0:
        raise RuntimeError(f"or_uniform_rect failed ({st})")
    return out


def optimal_dft_size(n: int, max_factor: int = 5) -> int:
    """GetOptimalDFTSize(n, larger=true, maxFactor) (src/transform/dft_optimal_size.cpp:168-184): the
    smallest size >= n whose prime factors are all <= max_factor."""
    primes = [p_ for p_ in (2, 3, 5, 7, 11) if p_ <= max_factor]
    m = max(1, int(n))
    while True:
        r = m
        for p_ in primes:
            while r % p_ == 0:
                r //= p_
        if r == 1:
            return m
        m += 1


def window_origin(image_size: int, window_size: int) -> int:
    """GetWindowOrigin for CENTER (src/library/image_manip.cpp:557-566)."""
    return (image_size - window_size) // 2 + int((image_size % 2 == 0) and (window_size % 2 == 1))


def _gaussft_lut(n: int, sigma: float, order: int, truncation: float, dt_double: bool) -> np.ndarray:
    """GaussFTLineFilter's look-up table (src/linear/gauss.cpp:296-343) for one axis, centred
    coordinates (origin n // 2), in the computation precision."""
    ft = np.float64 if dt_double else np.float32
    ct = np.complex128 if dt_double else np.complex64
    lut = np.zeros(n, ct)
    origin = n // 2
    b = ft(2.0 * np.pi * sigma) / ft(n)
    b = -ft(0.5) * b * b
    if b == 0:
        nh = n
    else:
        nh = int(oracle_lib().or_half_gaussian_size(float(n) / (2.0 * np.pi * sigma), order, truncation, int(dt_double)))
    begin, end = max(0, origin - nh), min(n, origin + nh + 1)
    x = (np.arange(begin, end) - origin).astype(ft)
    if order > 0:
        a = ct(complex(0.0, float(ft(2.0 * np.pi) / ft(n)))) ** order
        val = a * (x.astype(ct) ** order)
        if b != 0:
            val = val * np.exp(b * x * x)
        lut[begin:end] = val
    else:
        lut[begin:end] = np.exp(b * x * x) if b != 0 else 1
    return lut


def gauss_ft(x: np.ndarray, sigmas: Sequence[float] = (1.0,), orders: Sequence[int] = (0,),
             truncation: float = 3.0, bcs: Sequence[str] | None = None, rdim: int | None = None) -> np.ndarray:
    """dip::GaussFT (src/linear/gauss.cpp:397-487) for real input, spatial in and out, restated with
    numpy's FFT in double precision: the input (extended by the boundary condition to an optimal DFT
    size when `bcs` is given, centred as ExtendImageToSize places it) is transformed, multiplied by
    each axis' Gaussian (derivative) look-up table at the centred frequency, transformed back (real
    part, scaled by 1/N) and cropped back to the input's sizes."""
    nd = x.ndim
    sig = [float(v) for v in _broadcast(sigmas, nd, 1.0)]     # DIPlib order (x first)
    ords = [int(v) for v in _broadcast(orders, nd, 0)]
    dims = list(reversed(x.shape))                             # DIPlib order
    for d in range(nd):
        if dims[d] == 1:
            sig[d], ords[d] = 0.0, 0
        elif sig[d] < 0:
            sig[d] = 0.0
    out_dt = suggest_flex(x.dtype)
    if not any(sig) and not any(ords):
        return x.astype(out_dt)
    dt_double = out_dt == np.float64
    img = x.astype(np.float64)
    origins = [0] * nd
    if bcs:
        bcl = _broadcast(bcs, nd, "mirror")
        new = []
        for d in range(nd):
            h = int(oracle_lib().or_half_gaussian_size(sig[d], ords[d], truncation, int(x.dtype == np.float64)))
            new.append(optimal_dft_size(dims[d] + 2 * h, 5))
        for d in range(nd):
            ax = nd - 1 - d
            o = window_origin(new[d], dims[d])
            origins[d] = o
            idx = np.arange(new[d]) - o
            src = np.array([_map_index(int(j), dims[d], bcl[d]) for j in idx])
            sgn = np.array([_map_sign(int(j), dims[d], bcl[d]) for j in idx], dtype=np.float64)
            img = np.take(img, np.where(src < 0, 0, src), axis=ax)
            shape = [1] * nd
            shape[ax] = new[d]
            img = img * np.where(src < 0, 0.0, sgn).reshape(shape)
    F = np.fft.fftn(np.fft.ifftshift(img))                   # spatial origin at index n // 2
    # The reference's real-to-complex transform (src/transform/fourier.cpp:86-96, 387-441) runs along
    # one dimension r (the first with more than 2 samples, all strides being normal); for an odd size
    # along r its half-line shift leaves the outermost frequency unconjugated, so that the spectrum it
    # produces holds the planes x_r = +M and x_r = -M (M = (N_r - 1) / 2) swapped.  Its inverse is a
    # complex-to-real transform that uses only the half x_r <= 0.  Both are restated here.
    sizes_dip = [img.shape[nd - 1 - d] for d in range(nd)]
    r = 0
    for d in range(1, nd):
        if sizes_dip[r] <= 2 and sizes_dip[d] > 2:
            r = d
    if rdim is not None:          # the axis the reference picks for an input with other strides
        r = rdim
    axr = nd - 1 - r
    nr = img.shape[axr]
    if nr % 2 == 1 and nr > 2:
        m = (nr - 1) // 2
        idx = [slice(None)] * nd
        idx[axr] = m
        pos = F[tuple(idx)].copy()
        idx2 = list(idx)
        idx2[axr] = nr - m                       # x_r = -M in the unshifted layout
        F[tuple(idx)] = F[tuple(idx2)]
        F[tuple(idx2)] = pos
    for d in range(nd):
        ax = nd - 1 - d
        n = img.shape[ax]
        lut_c = _gaussft_lut(n, sig[d], ords[d], truncation, dt_double).astype(np.complex128)
        k = np.arange(n)
        lut_u = lut_c[(k + n // 2) % n]
        shape = [1] * nd
        shape[ax] = n
        F = F * lut_u.reshape(shape)
    # Hermitian completion of the half x_r <= 0 (unshifted: 0 and nr - nr // 2 .. nr - 1)
    H = F.copy()
    for xr in range(1, (nr + 1) // 2):
        src = [slice(None)] * nd
        src[axr] = nr - xr
        part = np.conj(F[tuple(src)])
        # negate the other frequencies: index -k mod n along every other axis
        for ax in range(nd):
            if ax != axr:
                part = np.roll(np.flip(part, axis=ax if ax < axr else ax - 1), 1, axis=ax if ax < axr else ax - 1)
        dst = [slice(None)] * nd
        dst[axr] = xr
        H[tuple(dst)] = part
    res = np.fft.fftshift(np.real(np.fft.ifftn(H)))
    sl = tuple(slice(origins[nd - 1 - ax], origins[nd - 1 - ax] + x.shape[ax]) for ax in range(nd))
    return res[sl].astype(out_dt)


def _map_index(j: int, n: int, bc: str) -> int:
    """Source sample of extended position j (index-mapping conditions; -1: "add zeros")."""
    if 0 <= j < n:
        return j
    code = bc_code(bc)
    if code == 5:
        return -1
    if n == 1:
        return 0
    if code in (0, 1):
        p_ = n - 1
        k = -j if j < 0 else j - p_
        t = k % (2 * p_)
        if t > p_:
            t = 2 * p_ - t
        return t if j < 0 else p_ - t
    if code in (3, 4):
        return j % n
    if code == 8:
        return 0 if j < 0 else n - 1
    raise ValueError("boundary condition not supported by the FT restatement: " + bc)


def _map_sign(j: int, n: int, bc: str) -> float:
    if 0 <= j < n:
        return 1.0
    code = bc_code(bc)
    if n == 1:
        return -1.0 if code in (1, 4) else 1.0
    if code == 1:
        p_ = n - 1
        k = -j if j < 0 else j - p_
        return -1.0 if ((k - 1) // p_) % 2 == 0 else 1.0
    if code == 4:
        k = -j if j < 0 else j - (n - 1)
        return -1.0 if ((k - 1) // n) % 2 == 0 else 1.0
    return 1.0


def separable_fir(x: np.ndarray, taps, odd, bcs, out_dtype=None) -> np.ndarray:
    """The restated dip::SeparableConvolution with given EVEN/ODD half kernels, centre tap first
    (per axis, DIPlib order; None leaves an axis unfiltered)."""
    nd = x.ndim
    out_dt = suggest_flex(x.dtype) if out_dtype is None else np.dtype(out_dtype)
    out = np.zeros(x.shape, out_dt)
    sizes, in_strides = _dip_geometry(x)
    _, out_strides = _dip_geometry(out)
    keep = [None if t is None else np.ascontiguousarray(t, np.float64) for t in taps]
    ptrs = (ctypes.c_void_p * nd)(*[None if t is None else t.ctypes.data for t in keep])
    lens = (ctypes.c_int * nd)(*[0 if t is None else t.size for t in keep])
    bcl = _broadcast(bcs, nd, "mirror")
    st = oracle_lib().or_separable_fir(
        ctypes.c_void_p(x.ctypes.data), DTYPE_CODES[x.dtype], nd, sizes, in_strides,
        ctypes.c_void_p(out.ctypes.data), DTYPE_CODES[out_dt], out_strides, ptrs, lens,
        (ctypes.c_int * nd)(*[int(o) for o in odd]), (ctypes.c_int * nd)(*[bc_code(b) for b in bcl]))
    if st != 0:
        raise RuntimeError(f"or_separable_fir failed ({st})")
    return out


def symmetric_pairs(m: int) -> list:
    """Index pairs of DIPlib's symmetric-matrix storage (include/diplib/library/tensor.h:100-110):
    the diagonal first, then the elements above it column by column."""
    return [(i, i) for i in range(m)] + [(i, j) for j in range(1, m) for i in range(j)]


def derivative_dims(shape, sigmas, process=None) -> list:
    """FindGradientDimensions (src/linear/derivative.cpp:120-138) for the Gaussian methods: the
    DIPlib axes (x first) with process set, size > 1 and sigma > 0."""
    nd = len(shape)
    pr = _broadcast(process, nd, True)
    return [d for d in range(nd) if pr[d] and shape[nd - 1 - d] > 1 and sigmas[d] > 0]


def gradient(x: np.ndarray, sigmas, bcs=("mirror",), truncation: float = 3.0, process=None) -> np.ndarray:
    """dip::Gradient (src/linear/derivative.cpp:142-172): one first derivative per kept axis."""
    nd = x.ndim
    sg = _broadcast([sigmas] if np.isscalar(sigmas) else sigmas, nd, 1.0)
    out = []
    for d in derivative_dims(x.shape, sg, process):
        o = [0] * nd
        o[d] = 1
        out.append(gauss_fir(x, sg, o, list(bcs), truncation))
    return np.stack(out)


def hessian(x: np.ndarray, sigmas, bcs=("mirror",), truncation: float = 3.0, process=None) -> np.ndarray:
    """dip::Hessian (src/linear/derivative.cpp:330-372): second derivatives d_ii on the diagonal,
    mixed d_ij above it, in symmetric-matrix storage order."""
    nd = x.ndim
    sg = _broadcast([sigmas] if np.isscalar(sigmas) else sigmas, nd, 1.0)
    dims = derivative_dims(x.shape, sg, process)
    out = []
    for i, j in symmetric_pairs(len(dims)):
        o = [0] * nd
        o[dims[i]] += 1
        o[dims[j]] += 1
        out.append(gauss_fir(x, sg, o, list(bcs), truncation))
    return np.stack(out)


def laplace(x: np.ndarray, sigmas, bcs=("mirror",), truncation: float = 3.0, process=None) -> np.ndarray:
    """dip::Laplace, Gaussian methods (src/linear/derivative.cpp:374-418): the sum of the second
    derivatives along the kept axes, accumulated in the flex type."""
    nd = x.ndim
    sg = _broadcast([sigmas] if np.isscalar(sigmas) else sigmas, nd, 1.0)
    acc = None
    for d in derivative_dims(x.shape, sg, process):
        o = [0] * nd
        o[d] = 2
        t = gauss_fir(x, sg, o, list(bcs), truncation)
        acc = t if acc is None else (acc + t).astype(t.dtype)
    return acc


def structure_tensor(x: np.ndarray, grad_sigma, tensor_sigma, bc="mirror", truncation: float = 3.0) -> np.ndarray:
    """dip::StructureTensor (src/analysis/structure_tensor.cpp:33-59) built from the restated
    GaussFIR: the gradient along the axes FindGradientDimensions keeps (src/linear/derivative.cpp:120-138:
    size > 1 and sigma > 0), the products g_i g_j, and the smoothing of each product.  Sigmas and
    boundary conditions are scalars or per-axis lists in DIPlib order.  Returns an array of shape
    (ncomp,) + x.shape with DIPlib's symmetric-matrix component order (diagonal first, then the
    upper triangle column by column, include/diplib/library/tensor.h:100-110)."""
    nd = x.ndim
    gs = [float(grad_sigma)] * nd if np.isscalar(grad_sigma) else [float(s) for s in grad_sigma]
    ts = [float(tensor_sigma)] * nd if np.isscalar(tensor_sigma) else [float(s) for s in tensor_sigma]
    bcs = [bc] if isinstance(bc, str) else list(bc)
    dims = [d for d in range(nd) if x.shape[nd - 1 - d] > 1 and gs[d] > 0]
    grads = []
    for d in dims:
        o = [0] * nd
        o[d] = 1
        grads.append(gauss_fir(x, gs, o, bcs, truncation))
    m = len(dims)
    pairs = symmetric_pairs(m)
    comps = [gauss_fir((grads[i] * grads[j]).astype(grads[0].dtype), ts, [0] * nd, bcs, truncation)
             for i, j in pairs]
    return np.stack(comps)


# ------------------------------------------------------------------------------------------------
# The reference itself
# ------------------------------------------------------------------------------------------------

def ref_set_threads(n: int) -> int:
    return ref_lib().dipref_set_threads(n)


def ref_half_gaussian(sigma: float, order: int, truncation: float = 3.0, dt_double: bool = False) -> np.ndarray:
    lib = ref_lib()
    buf = np.zeros(4096, np.float64)
    n = lib.dipref_half_gaussian(sigma, order, truncation, int(dt_double), buf.ctypes.data, buf.size)
    if n < 0:
        raise ValueError("MakeHalfGaussian failed")
    return buf[:n].copy()


def ref_expand_buffer(line: np.ndarray, left: int, right: int, bc: str) -> np.ndarray:
    line = np.ascontiguousarray(line)
    buf = np.zeros(left + line.size + right, line.dtype)
    buf[left:left + line.size] = line
    st = ref_lib().dipref_expand_buffer(buf.ctypes.data + left * buf.itemsize, DTYPE_CODES[line.dtype], 1,
                                        line.size, left, right, bc_code(bc))
    if st != 0:
        raise RuntimeError("ExpandBuffer failed")
    return buf


def ref_gauss(x: np.ndarray, sigmas: Sequence[float] = (1.0,), orders: Sequence[int] = (0,),
              bcs: Sequence[str] | None = None, truncation: float = 3.0, method: str = "FIR",
              out_dtype=None, strides: Sequence[int] | None = None) -> np.ndarray:
    """dip::Gauss of the reference on a numpy array.  `bcs=None` passes an empty array.  With
    `out_dtype` the output is a protected image of that type (the reference's protected path)."""
    nd = x.ndim
    sizes, st = _dip_geometry(x)
    errbuf = ctypes.create_string_buffer(512)
    sig = list(sigmas)
    ords = list(orders)
    bc_str = "\n".join(bcs) if bcs else ""
    protect = out_dtype is not None
    res_dt = np.dtype(out_dtype) if protect else suggest_flex(x.dtype)
    out = np.zeros(x.shape, res_dt)
    code = ctypes.c_int(DTYPE_CODES[res_dt])
    rc = ref_lib().dipref_gauss(
        ctypes.c_void_p(x.ctypes.data), DTYPE_CODES[x.dtype], nd, sizes, st,
        (ctypes.c_double * max(1, len(sig)))(*sig), len(sig), (ctypes.c_uint32 * max(1, len(ords)))(*ords), len(ords),
        bc_str.encode(), int(bcs is not None and len(bcs) > 0), ctypes.c_double(truncation), method.encode(),
        ctypes.c_void_p(out.ctypes.data), ctypes.byref(code), int(protect), errbuf, 512)
    if rc != 0:
        raise RuntimeError(errbuf.value.decode())
    if not protect and code.value != DTYPE_CODES[res_dt]:
        raise RuntimeError(f"unexpected output type code {code.value}")
    return out


def ref_gauss_iir(x: np.ndarray, sigmas: Sequence[float] = (1.0,), orders: Sequence[int] = (0,),
                  bcs: Sequence[str] | None = None, filter_orders: Sequence[int] = (),
                  design: str = "discrete time fit", truncation: float = 3.0) -> np.ndarray:
    """dip::GaussIIR of the reference on a numpy array (`bcs=None`: an empty array)."""
    nd = x.ndim
    sizes, st = _dip_geometry(x)
    errbuf = ctypes.create_string_buffer(512)
    sig, ords, fo = list(sigmas), list(orders), list(filter_orders)
    out = np.zeros(x.shape, suggest_flex(x.dtype))
    code = ctypes.c_int(0)
    bc_str = "\n".join(bcs) if bcs else ""
    rc = ref_lib().dipref_gauss_iir(
        ctypes.c_void_p(x.ctypes.data), DTYPE_CODES[x.dtype], nd, sizes, st,
        (ctypes.c_double * max(1, len(sig)))(*sig), len(sig), (ctypes.c_uint32 * max(1, len(ords)))(*ords), len(ords),
        bc_str.encode(), int(bcs is not None and len(bcs) > 0), (ctypes.c_uint32 * max(1, len(fo)))(*fo), len(fo),
        design.encode(), ctypes.c_double(truncation), ctypes.c_void_p(out.ctypes.data), ctypes.byref(code), errbuf, 512)
    if rc != 0:
        raise RuntimeError(errbuf.value.decode())
    if code.value != DTYPE_CODES[out.dtype]:
        raise RuntimeError(f"unexpected output type code {code.value}")
    return out


def ref_separable_convolution(x: np.ndarray, filters, bcs: Sequence[str] | None = None, process=None) -> np.ndarray:
    """dip::SeparableConvolution of the reference (real filters given as dicts, see
    separable_convolution)."""
    nd = x.ndim
    sizes, st = _dip_geometry(x)
    out = np.zeros(x.shape, suggest_flex(x.dtype))
    code = ctypes.c_int(0)
    errbuf = ctypes.create_string_buffer(512)
    data, lens, origins, _, syms, keep = _filter_arrays(filters)
    proc = None if process is None else (ctypes.c_int * nd)(*[int(bool(p)) for p in process])
    rc = ref_lib().dipref_separable_convolution(
        ctypes.c_void_p(x.ctypes.data), DTYPE_CODES[x.dtype], nd, sizes, st, len(filters), data, lens, origins,
        "\n".join(syms).encode(), "\n".join(bcs or []).encode(), int(bool(bcs)), proc, ctypes.c_void_p(out.ctypes.data),
        ctypes.byref(code), errbuf, 512)
    if rc != 0:
        raise RuntimeError(errbuf.value.decode())
    return out


def ref_uniform(x: np.ndarray, sizes, bcs: Sequence[str] | None = None) -> np.ndarray:
    """dip::Uniform of the reference with a rectangular kernel of per-axis `sizes`."""
    nd = x.ndim
    isz, st = _dip_geometry(x)
    out = np.zeros(x.shape, suggest_flex(x.dtype))
    code = ctypes.c_int(0)
    errbuf = ctypes.create_string_buffer(512)
    fs = _broadcast(sizes, nd, 7)
    rc = ref_lib().dipref_uniform(
        ctypes.c_void_p(x.ctypes.data), DTYPE_CODES[x.dtype], nd, isz, st, (ctypes.c_double * nd)(*[float(f) for f in fs]),
        "\n".join(bcs or []).encode(), int(bool(bcs)), ctypes.c_void_p(out.ctypes.data), ctypes.byref(code), errbuf, 512)
    if rc != 0:
        raise RuntimeError(errbuf.value.decode())
    return out


def ref_structure_tensor(x: np.ndarray, grad_sigma: float, tensor_sigma: float, bc: str = "mirror",
                         truncation: float = 3.0, method: str = "gaussFIR") -> np.ndarray:
    """dip::StructureTensor of the reference; returns (ncomp,) + x.shape."""
    nd = x.ndim
    maxcomp = nd * (nd + 1) // 2
    sizes, _ = _dip_geometry(x)
    x = np.ascontiguousarray(x)
    res_dt = suggest_flex(x.dtype)
    out = np.zeros(x.size * maxcomp, res_dt)
    code = ctypes.c_int(0)
    ncomp = ctypes.c_int(0)
    errbuf = ctypes.create_string_buffer(512)
    rc = ref_lib().dipref_structure_tensor(x.ctypes.data, DTYPE_CODES[x.dtype], nd, sizes, grad_sigma, tensor_sigma,
                                           method.encode(), bc.encode(), truncation, out.ctypes.data,
                                           ctypes.byref(code), ctypes.byref(ncomp), errbuf, 512)
    if rc != 0:
        raise RuntimeError(errbuf.value.decode() or "StructureTensor failed")
    out = out[:x.size * ncomp.value].reshape(x.shape + (ncomp.value,))
    return np.moveaxis(out, -1, 0).copy()


def ref_derivative_op(which: str, x: np.ndarray, sigmas, bcs=("mirror",), truncation: float = 3.0,
                      method: str = "gaussFIR") -> np.ndarray:
    """dip::Gradient / GradientMagnitude / Hessian / Laplace of the reference
    (src/linear/derivative.cpp:142-418); returns (ncomp,) + x.shape, or x.shape for the scalar
    results (GradientMagnitude, Laplace)."""
    code_of = {"gradient": 0, "gradient_magnitude": 1, "hessian": 2, "laplace": 3}
    nd = x.ndim
    maxcomp = nd * (nd + 1) // 2
    sizes, _ = _dip_geometry(x)
    x = np.ascontiguousarray(x)
    sg = np.asarray([sigmas] if np.isscalar(sigmas) else list(sigmas), dtype=np.float64)
    bl = [bcs] if isinstance(bcs, str) else list(bcs)
    out = np.zeros(x.size * maxcomp, suggest_flex(x.dtype))
    code = ctypes.c_int(0)
    ncomp = ctypes.c_int(0)
    errbuf = ctypes.create_string_buffer(512)
    rc = ref_lib().dipref_derivative_op(code_of[which], x.ctypes.data, DTYPE_CODES[x.dtype], nd, sizes,
                                        sg.ctypes.data, len(sg), "\n".join(bl).encode(), int(len(bl) > 0),
                                        truncation, method.encode(), out.ctypes.data, maxcomp, ctypes.byref(code),
                                        ctypes.byref(ncomp), errbuf, 512)
    if rc != 0:
        raise RuntimeError(errbuf.value.decode() or which + " failed")
    n = ncomp.value
    out = out[:x.size * n].reshape(x.shape + (n,))
    return out[..., 0].copy() if which in ("gradient_magnitude", "laplace") else np.moveaxis(out, -1, 0).copy()


def ref_read_pixel_bc(img: np.ndarray, coords, bcs) -> float:
    """dip::ReadPixelWithBoundaryCondition of the reference (src/library/boundary.cpp:47-128) on a
    scalar sfloat image; `coords` (which may lie outside the image) and `bcs` (enumerator codes)
    in DIPlib order, x first."""
    img = np.ascontiguousarray(img, np.float32)
    nd = img.ndim
    sizes = (ctypes.c_int64 * nd)(*reversed(img.shape))
    c = (ctypes.c_int64 * nd)(*coords)
    b = (ctypes.c_int * nd)(*bcs)
    out = ctypes.c_float(0.0)
    rc = ref_lib().dipref_read_pixel_bc(ctypes.c_void_p(img.ctypes.data), ctypes.c_int(nd), sizes, c, b,
                                        ctypes.byref(out))
    if rc != 0:
        raise RuntimeError("ReadPixelWithBoundaryCondition failed")
    return float(out.value)
