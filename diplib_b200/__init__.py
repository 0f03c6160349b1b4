"""dipcu: DIPlib's Gaussian FIR filtering path (dip::Gauss "FIR" -> dip::GaussFIR ->
dip::SeparableConvolution -> dip::Framework::Separable) on NVIDIA B200 (sm_100a).

The Python API mirrors PyDIP's (``Gauss``, ``GaussFIR``, ``Derivative`` ...); all pixel work
runs in libdipcu.so's CUDA kernels through the C-ABI declared in include/dipcu.h.
"""
from .filtering import (BestGaussMethod, BoundaryConditionFromString, Derivative, Error, Gauss, GaussFIR, GaussFT,
                        GaussIIR, OneDimensionalFilter, ParameterError, RunTimeError, SeparableConvolution, Uniform,
                        flex_dtype, image_desc)
from .analysis import StructureTensor
from .derivatives import Gradient, GradientMagnitude, Hessian, Laplace

__all__ = ["BestGaussMethod", "BoundaryConditionFromString", "Derivative", "Error", "Gauss", "GaussFIR", "GaussFT", "GaussIIR", "Gradient",
           "GradientMagnitude", "Hessian", "Laplace", "OneDimensionalFilter", "ParameterError", "SeparableConvolution",
           "StructureTensor", "RunTimeError", "Uniform", "flex_dtype", "image_desc"]
