"""The allocation-free smoothing entry point (gf_gaussian_smooth_noalloc),
for callers that cannot allocate device memory: its scratch is a fixed static
device array instead of context-owned cudaMalloc buffers.  Two calls in a row,
on different mesh sizes, must reproduce the context-based entry point
gf_gaussian_smooth on the same meshes, and the oracle's FP64 smoothing.  This file is collected last so a run
that stops at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest
import torch

from galaxyfinder_b200 import _lib, batch

pytestmark = pytest.mark.gpu


def _mesh(nx, ny, nz, seed):
    mx = 2 * (nx // 2 + 1)
    rng = np.random.default_rng(seed)
    den = np.zeros((nz, ny, mx), np.float32)
    den[:, :, :nx] = (rng.random((nz, ny, nx)) ** 6 * 1e3).astype(np.float32)
    return den.ravel()


def _logical(a, nx, ny, nz):
    mx = 2 * (nx // 2 + 1)
    return np.asarray(a).reshape(nz, ny, mx)[:, :, :nx]


def _with_context(den_host, nx, ny, nz, cell, rg):
    """The existing entry point: gf_gaussian_smooth on a context."""
    ctx = batch.Context(0)
    mesh = np.zeros(1, _lib.MESH_DTYPE)
    mesh["nx"], mesh["ny"], mesh["nz"] = nx, ny, nz
    mesh["ptype"] = _lib.TYPE_ALL
    mesh["cellsize"], mesh["rg"] = cell, rg
    mesh_dev = torch.from_numpy(mesh.view(np.uint8)).cuda()
    d = torch.from_numpy(den_host.copy()).cuda()
    _lib.check(_lib.lib().gf_gaussian_smooth(ctx.handle, 1, _lib.ptr(mesh), _lib.ptr(mesh_dev),
                                             _lib.ptr(d)))
    torch.cuda.synchronize()
    out = d.cpu().numpy()
    ctx.close()
    return out


def test_noalloc_smoothing_matches_context_entry_point(cuda_device, restatement):
    stream = torch.cuda.current_stream()
    cases = [((64, 48, 40), 0.004, 0.008), ((37, 64, 128), 0.005, 0.0075)]
    for i, ((nx, ny, nz), cell, rg) in enumerate(cases):
        den = _mesh(nx, ny, nz, 100 + i)
        d = torch.from_numpy(den.copy()).cuda()
        _lib.check(_lib.lib().gf_gaussian_smooth_noalloc(
            _lib.ptr(d), nx, ny, nz, cell, rg, ctypes.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize()
        got = _logical(d.cpu().numpy(), nx, ny, nz)
        ref = _logical(_with_context(den, nx, ny, nz, cell, rg), nx, ny, nz)
        assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max(), (nx, ny, nz)
        # and, independently of the context path, the FP64 spectral smoothing
        # of the oracle on the same mesh
        _, s64 = restatement.smooth(den, nx, ny, nz, cell, rg)
        want = _logical(s64, nx, ny, nz)
        assert np.abs(got - want).max() <= 2e-6 * np.abs(want).max(), (nx, ny, nz)


def test_noalloc_rejects_meshes_beyond_its_scratch(cuda_device):
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    status = _lib.lib().gf_gaussian_smooth_noalloc(_lib.ptr(d), 2048, 2, 2, 0.004, 0.008, None)
    assert status == _lib.GF_EINVAL
    assert b"1024" in _lib.lib().gf_last_error()
