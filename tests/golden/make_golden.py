"""Generates tests/golden/*.npz from the reference itself (oracle/_ref/libdipref.so, the
unmodified DIPlib sources compiled by oracle/Makefile).  Run where the reference tree exists:

    make -C oracle ref && python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py --iir-only                       # gauss_iir_ref.npz alone

The fixtures pin the C restatement (oracle/gauss_oracle.c) and the CUDA path on machines
without the reference tree.  Inputs are regenerated from the stored seeds and shapes.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

BCS = ["mirror", "asym mirror", "antisym reflect", "periodic", "asym periodic", "add zeros", "add max", "add min",
       "zero order", "first order", "second order", "third order"]


def make_input(seed: int, shape, dtype) -> np.ndarray:
    rng = np.random.default_rng(seed)
    dt = np.dtype(dtype)
    if dt.kind == "f":
        return rng.random(shape).astype(dt)
    if dt == np.bool_:
        return rng.random(shape) > 0.5
    info = np.iinfo(dt)
    hi = min(int(info.max), 4095)
    lo = max(int(info.min), -2048)
    return rng.integers(lo, hi + 1, size=shape).astype(dt)


# (name, seed, shape (numpy order), dtype, sigmas (x first), orders (x first), bc list, truncation)
CASES = [
    ("cfg1_small", 1, (48, 64), "float32", [2.0, 2.0], [0, 0], ["mirror"], 3.0),
    ("d1x_periodic", 2, (40, 52), "float32", [1.5, 2.5], [1, 0], ["periodic"], 3.0),
    ("d2y_addzeros", 3, (33, 47), "float32", [1.0, 3.0], [0, 2], ["add zeros"], 3.0),
    ("d3_asym", 4, (30, 41), "float32", [2.0, 1.2], [3, 1], ["asym mirror", "asym periodic"], 3.0),
    ("zero_order", 5, (37, 29), "float32", [2.2, 0.9], [0, 1], ["zero order"], 2.5),
    ("extrap", 6, (26, 35), "float32", [1.7, 1.3], [1, 0], ["first order", "third order"], 3.0),
    ("antisym_2nd", 7, (21, 18), "float32", [1.1, 2.0], [2, 0], ["antisym reflect", "second order"], 3.0),
    ("multi_reflect", 8, (5, 7), "float32", [3.0, 4.0], [0, 1], ["mirror", "periodic"], 3.0),
    ("u16_3d", 9, (12, 20, 24), "uint16", [1.5, 1.5, 3.0], [0, 0, 0], ["mirror"], 3.0),
    ("u16_3d_dx", 10, (12, 20, 24), "uint16", [1.5, 1.5, 3.0], [1, 0, 0], ["mirror"], 3.0),
    ("u8_2d", 11, (30, 30), "uint8", [2.0], [0], [], 3.0),
    ("s16_2d", 12, (25, 31), "int16", [1.0, 2.0], [0, 1], ["periodic"], 3.0),
    ("f64_3d", 13, (9, 11, 13), "float64", [1.0, 2.0, 1.5], [0, 1, 2], ["mirror"], 3.0),
    ("s32_2d", 14, (20, 22), "int32", [1.5], [1], ["add zeros"], 3.0),
    ("sigma0_axis", 15, (16, 20, 24), "float32", [2.0, 0.0, 1.0], [0, 0, 1], ["mirror"], 3.0),
    ("one_d", 16, (200,), "float32", [5.0], [2], ["mirror"], 4.0),
    ("add_max", 17, (20, 24), "float32", [1.0, 1.0], [0, 0], ["add max"], 3.0),
]


# dip::GaussIIR cases: (name, seed, shape, dtype, sigmas, orders, bc list, filter orders, design)
IIR_CASES = [
    ("iir_d0_dtf", 31, (60, 70), "float32", [12.0, 3.0], [0, 0], ["mirror"], [], "discrete time fit"),
    ("iir_d1_fb", 32, (45, 50), "uint16", [5.0, 11.0], [1, 0], ["periodic", "add zeros"], [], "forward backward"),
    ("iir_d2_3d", 33, (14, 18, 22), "float64", [2.0, 6.0, 4.0], [2, 0, 1], ["asym mirror", "zero order", "third order"],
     [], "discrete time fit"),
    ("iir_d3_orders", 34, (40, 33), "float32", [7.0, 2.5], [3, 4], ["first order", "second order"], [4, 3],
     "discrete time fit"),
    ("iir_short", 35, (9, 200), "int32", [15.0, 1.5], [0, 1], ["antisym reflect", "asym periodic"], [1, 2],
     "forward backward"),
]


def make_iir() -> None:
    """gauss_iir_ref.npz only (the other fixtures untouched)."""
    out = {}
    for name, seed, shape, dtype, sig, ords, bcs, fo, dm in IIR_CASES:
        x = make_input(seed, shape, dtype)
        out[name] = oracle.ref_gauss_iir(x, sig, ords, bcs, fo, dm)
    np.savez_compressed(os.path.join(HERE, "gauss_iir_ref.npz"), **out)


def main() -> None:
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libdipref.so is not built")
    if "--iir-only" in sys.argv:
        make_iir()
        print("written to", HERE)
        return
    make_iir()
    out = {}
    for name, seed, shape, dtype, sig, ords, bcs, trunc in CASES:
        x = make_input(seed, shape, dtype)
        y = oracle.ref_gauss(x, sig, ords, bcs, trunc)
        out[name] = y
    np.savez_compressed(os.path.join(HERE, "gauss_ref.npz"), **out)

    # Half-Gaussian tables (MakeHalfGaussian) for both precisions.
    tables = {}
    for s in [0.5, 0.8, 1.0, 1.5, 2.0, 3.0, 4.0, 8.0]:
        for o in range(4):
            for dt in (0, 1):
                tables[f"s{s}_o{o}_d{dt}"] = oracle.ref_half_gaussian(s, o, 3.0, bool(dt))
    np.savez_compressed(os.path.join(HERE, "half_gaussian_ref.npz"), **tables)

    # ExpandBuffer on float lines for every BC, including multiple reflections.
    ext = {}
    rng = np.random.default_rng(99)
    for bc in BCS:
        for n in (1, 2, 3, 7):
            for left, right in ((4, 5), (17, 13)):
                line = rng.random(n).astype(np.float32)
                ext[f"{bc}|{n}|{left}|{right}|in"] = line
                ext[f"{bc}|{n}|{left}|{right}|out"] = oracle.ref_expand_buffer(line, left, right, bc)
    np.savez_compressed(os.path.join(HERE, "expand_buffer_ref.npz"), **ext)

    # Structure tensor of a small volume.
    x = make_input(21, (10, 12, 14), "float32")
    np.savez_compressed(os.path.join(HERE, "structure_tensor_ref.npz"),
                        st=oracle.ref_structure_tensor(x, 1.0, 2.0, "mirror", 3.0))
    print("written to", HERE)


if __name__ == "__main__":
    main()
