"""The NFW tidal-radius table of the reference's OLD_TIDAL build
(NewGalFinder/mkRtidal.c): the table libgf builds on the GPU against the
table of the reference's own mkRtidal() (compiled from its source into
oracle/_ref), and nfw_rtidal's lookups, through the reference signatures
and the batched device entry point.  The table's arithmetic keeps the
reference's float/double types operation by operation (a host restatement
of it matches the reference bit for bit); on the GPU only the device
library's double log/log10/pow can move the last bits of an entry."""
import ctypes
from pathlib import Path

import numpy as np
import pytest
import torch

from galaxyfinder_b200 import _lib, batch

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libmkrtidal.so"


@pytest.fixture(scope="module")
def reference_table():
    if not REF.exists():
        pytest.fail(f"{REF} missing: build the oracle (make -C oracle ref)")
    lib = ctypes.CDLL(str(REF))
    lib.mkRtidal.restype = None
    lib.nfw_rtidal.restype = ctypes.c_float
    lib.nfw_rtidal.argtypes = [ctypes.c_float] * 3
    lib.mkRtidal()
    n = _lib.lib().gf_nfw_rtidal_cells()
    table = np.ctypeslib.as_array((ctypes.c_float * n).in_dll(lib, "tidal_den")).copy()
    return lib, table


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    m = (10.0 ** rng.uniform(-5, 1, n)).astype(np.float32)     # satellite / host mass
    d = (10.0 ** rng.uniform(-4, 1.5, n)).astype(np.float32)   # distance / host Rvir
    c = rng.uniform(0.5, 36, n).astype(np.float32)             # host concentration
    return m, d, c


def test_table_matches_reference(cuda_device, reference_table):
    _, ref = reference_table
    ctx = batch.Context(0)
    t = torch.empty(ref.size, dtype=torch.float32, device=cuda_device)
    _lib.check(_lib.lib().gf_nfw_rtidal_table(ctx.handle, _lib.ptr(t)))
    torch.cuda.synchronize()
    got = t.cpu().numpy()
    ctx.close()
    assert np.all(np.isfinite(got)) and np.all(got > 0)
    rel = np.abs(got.astype(np.float64) - ref) / np.abs(ref)
    exact = float(np.mean(got == ref))
    print(f"table: {exact:.6f} of {ref.size} entries bit-identical, max rel diff {rel.max():.3g}")
    assert rel.max() <= 1e-5
    assert exact >= 0.99


def test_dropin_lookups_match_reference(cuda_device, reference_table):
    reflib, ref = reference_table
    gf = _lib.lib()
    gf.mkRtidal()
    _lib.check_last()
    m, d, c = _inputs(20000, 1)
    got = np.array([gf.nfw_rtidal(float(a), float(b), float(e)) for a, b, e in zip(m, d, c)], np.float32)
    want = np.array([reflib.nfw_rtidal(float(a), float(b), float(e)) for a, b, e in zip(m, d, c)], np.float32)
    rel = np.abs(got.astype(np.float64) - want) / np.abs(want)
    assert rel.max() <= 1e-5
    # the cell index is computed with the host C library, as the reference's
    assert float(np.mean(got == want)) >= 0.99


def test_device_lookups_match_host(cuda_device, reference_table):
    gf = _lib.lib()
    gf.mkRtidal()
    ctx = batch.Context(0)
    t = torch.empty(gf.gf_nfw_rtidal_cells(), dtype=torch.float32, device=cuda_device)
    _lib.check(gf.gf_nfw_rtidal_table(ctx.handle, _lib.ptr(t)))
    m, d, c = _inputs(100000, 2)
    dm, dd, dc = (torch.from_numpy(a).to(cuda_device) for a in (m, d, c))
    out = torch.empty(m.size, dtype=torch.float32, device=cuda_device)
    _lib.check(gf.gf_nfw_rtidal_lookup(ctx.handle, m.size, _lib.ptr(dm), _lib.ptr(dd), _lib.ptr(dc),
                                       _lib.ptr(t), _lib.ptr(out)))
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    ctx.close()
    host = np.array([gf.nfw_rtidal(float(a), float(b), float(e)) for a, b, e in zip(m, d, c)], np.float32)
    # same table; the device's log10 can put an input sitting on a cell
    # boundary into the neighbouring cell
    assert float(np.mean(got == host)) >= 0.999
