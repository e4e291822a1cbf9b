"""The pipelined stage (halo chunks on their own streams and host threads)
gives the single-call stage's outputs: every halo is computed on its own, so
splitting the catalogue changes no bit of the kNN lists and SPH densities.
The mesh density (float atomic deposit) and the potential (node moments
accumulated with atomics, leaf order set by atomic scatter) depend on the
order in which atomics land, which varies from run to run, so they agree to
float rounding.
Both the device-resident run and the end-to-end run (pinned host inputs in,
host outputs back) are checked."""
import numpy as np
import pytest
import torch

from galaxyfinder_b200 import _lib, batch, synth

pytestmark = pytest.mark.gpu

K = 32


@pytest.fixture(scope="module")
def cat(cuda_device):
    hb = synth.catalogue(seed=synth.SEED_BASE + 11, nhalo=192, nmax=200_000)
    rule = batch.mesh_rule(mode=_lib.MESH_POW2, nmin=64, nmax=256, rg=2.0, rg_in_cells=True)
    cfg = batch.stage_config(mesh=rule, knn_k=K)
    ctx = batch.Context(0)
    db = batch.DeviceBatch.from_halobatch(hb)
    out = batch.stage_run(ctx, db, cfg)
    torch.cuda.synchronize()
    ref = {f: getattr(out, f).cpu().numpy() for f in ("nearindex", "dens_sph", "dens_mesh", "penergy")}
    ctx.close()
    return hb, cfg, ref


@pytest.mark.parametrize("nchunk", [1, 3, 5])
def test_pipelined_matches_single_call(cat, nchunk):
    hb, cfg, ref = cat
    pipe = batch.PipelinedStage(hb, cfg, nchunk=nchunk, k=K)
    try:
        assert sum(c["n"] for c in pipe.chunks) == hb.n
        # end to end: outputs land in the chunks' pinned host buffers
        for c in pipe.chunks:
            for t in c["hout"].values():
                t.fill_(0)
        pipe.run_e2e()
        torch.cuda.synchronize()
        got = {f: np.concatenate([c["hout"][f].numpy() for c in pipe.chunks]) for f in ref}
        for f in ("nearindex", "dens_sph"):
            np.testing.assert_array_equal(got[f], ref[f], err_msg=f)
        np.testing.assert_allclose(got["penergy"], ref["penergy"], rtol=1e-6, atol=0)
        scale = np.abs(ref["dens_mesh"]).max()
        assert np.abs(got["dens_mesh"] - ref["dens_mesh"]).max() < 1e-5 * scale
        # device-resident run into the chunks' device buffers
        for c in pipe.chunks:
            c["out"].dens_sph.fill_(0)
        pipe.run_resident()
        torch.cuda.synchronize()
        dev = np.concatenate([c["out"].dens_sph.cpu().numpy() for c in pipe.chunks])
        np.testing.assert_array_equal(dev, ref["dens_sph"])
    finally:
        pipe.close()
