"""FFTW stand-in for timing the reference's Gaussian smoothing on the host.

NewGalFinder's gaussian_Smoothing (gsmooth.c:14-115) runs FFTW3 single
precision with threads: an r2c transform of the (nz, ny, nx) mesh, a
multiply by exp(-(pi RG/cellsize)^2 (k^2/nz^2 + j^2/ny^2 + i^2/nx^2)) with
RG/cellsize stored back into a float (gsmooth.c:67), a c2r transform and a
scale by 1/(nx ny nz).  FFTW is not installed here (and the reference does
not pin its version), so the benchmark's CPU legs time this arithmetic with
scipy.fft (pocketfft) in single precision on every host thread, which runs
at FFTW-like speed.  The oracle's accuracy reference for the smoothing is the
FP64 restatement in gf_oracle.c, not this module.
"""
from __future__ import annotations

import numpy as np


def gaussian_smoothing(den: np.ndarray, nx: int, ny: int, nz: int, cellsize: float, rg: float,
                       workers: int = -1) -> np.ndarray:
    """Smooths the padded r2c mesh den[i + mx (j + ny k)], mx = 2(nx/2+1), in
    place and returns it."""
    import scipy.fft as sf

    mx = 2 * (nx // 2 + 1)
    grid = den.reshape(nz, ny, mx)
    a = grid[:, :, :nx]
    rgc = float(np.float32(float(np.float32(rg)) / cellsize))  # gsmooth.c:67 (float RG)
    fac = (np.pi * rgc) ** 2
    kz = np.fft.fftfreq(nz) * nz
    ky = np.fft.fftfreq(ny) * ny
    kx = np.arange(nx // 2 + 1, dtype=np.float64)
    # exp of a sum = product of the per-axis exps
    fz = np.exp(-fac * kz ** 2 / nz ** 2).astype(np.float32)
    fy = np.exp(-fac * ky ** 2 / ny ** 2).astype(np.float32)
    fx = np.exp(-fac * kx ** 2 / nx ** 2).astype(np.float32)
    spec = sf.rfftn(a, axes=(0, 1, 2), workers=workers)
    spec *= fz[:, None, None]
    spec *= fy[None, :, None]
    spec *= fx[None, None, :]
    grid[:, :, :nx] = sf.irfftn(spec, s=(nz, ny, nx), axes=(0, 1, 2), workers=workers)
    return den
