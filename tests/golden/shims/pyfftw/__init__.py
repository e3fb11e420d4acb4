"""pyfftw stand-in over numpy.fft (pocketfft), complex64 in and out.

FFTW.__call__ normalises the inverse transform by 1/(nx*nz), as pyfftw's
default normalise_idft=True does, so the scale matches the reference."""
import numpy as _np
from . import interfaces  # noqa: F401


class config:
    NUM_THREADS = 1


def empty_aligned(shape, dtype="complex128", n=None):
    return _np.empty(shape, dtype=dtype)


def zeros_aligned(shape, dtype="complex128", n=None):
    return _np.zeros(shape, dtype=dtype)


class FFTW:
    def __init__(self, input_array, output_array, axes=(-1,), direction="FFTW_FORWARD",
                 threads=1, flags=()):
        self.input_array = input_array
        self.output_array = output_array
        self.axes = tuple(axes)
        self.direction = direction

    def __call__(self, *args, **kwargs):
        if self.direction == "FFTW_FORWARD":
            res = _np.fft.fftn(self.input_array, axes=self.axes)
        else:
            res = _np.fft.ifftn(self.input_array, axes=self.axes)
        self.output_array[...] = res.astype(self.output_array.dtype)
        return self.output_array

    execute = __call__
