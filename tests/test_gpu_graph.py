"""The stage captured as a CUDA graph (gf_stage_graph_*): replays against
eager gf_stage_run calls on the same inputs, after the inputs move within the
plan, and after they move out of it (re-plan)."""
import numpy as np
import pytest
import torch

from galaxyfinder_b200 import _lib, batch, synth

pytestmark = pytest.mark.gpu


def _outputs(out):
    torch.cuda.synchronize()
    return {f: getattr(out, f).cpu().numpy().copy() for f in ("nearindex", "dens_sph", "dens_mesh", "penergy", "phi")}


def _same(a, b):
    """Graph and eager outputs: the kNN rows and SPH densities are exact; the
    mesh density and potential differ only in the order of float atomics
    (mesh cells, node moments) and of the particles within an octant."""
    np.testing.assert_array_equal(a["nearindex"], b["nearindex"])
    np.testing.assert_array_equal(a["dens_sph"], b["dens_sph"])
    dm = np.abs(a["dens_mesh"] - b["dens_mesh"]).max() / np.abs(b["dens_mesh"]).max()
    assert dm <= 2e-6, dm
    rel = np.abs(a["phi"] - b["phi"]) / np.abs(b["phi"])
    assert rel.max() <= 1e-6, rel.max()


@pytest.fixture()
def setup(cuda_device):
    hb = synth.catalogue(seed=977, nhalo=48, nmin=60, nmax=60000, straddle_frac=0.2)
    ctx = batch.Context(0)
    db = batch.DeviceBatch.from_halobatch(hb)
    cfg = batch.stage_config()
    yield hb, ctx, db, cfg
    torch.cuda.synchronize()
    ctx.close()


def _eager(hb_db_cfg, db):
    ctx2 = batch.Context(0)
    try:
        out = batch.stage_run(ctx2, db, hb_db_cfg)
        return _outputs(out)
    finally:
        ctx2.close()


def test_replay_matches_eager(setup):
    hb, ctx, db, cfg = setup
    ref = _eager(cfg, db)
    out = batch.StageBuffers(hb.n, 32, db.x.device, keep_phi=True)
    g = batch.StageGraph(ctx, db, cfg, out)
    _same(_outputs(out), ref)  # the planning run
    for _ in range(3):
        out.nearindex.fill_(-7)
        out.dens_mesh.zero_()
        out.phi.zero_()
        torch.cuda.synchronize()  # the graph runs on the context's own stream
        g.launch()
        g.sync()
        _same(_outputs(out), ref)
    assert g.replans == 0
    g.close()


def _unwrapped(hb):
    """Per halo: positions unwrapped across the periodic box (numpy FP64)."""
    out = []
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        p = np.stack([hb.x[a:b], hb.y[a:b], hb.z[a:b]], 1).copy()
        for ax in range(3):
            c = p[:, ax]
            cs = np.where(c < 50.0, c + 100.0, c)
            if c.max() - c.min() > 50.0 and cs.max() - cs.min() < c.max() - c.min():
                p[:, ax] = cs
        out.append(p)
    return out


def _shapes(parts, cfg):
    ext = np.array([p.max(0) - p.min(0) for p in parts])
    mesh, _ = batch.plan_meshes(ext, cfg.mesh)
    return np.stack([mesh["nx"], mesh["ny"], mesh["nz"]], 1)


def _scaled(hb, cfg, factor, want_change):
    """Each halo scaled by `factor` about its first particle (in the unwrapped
    frame, then wrapped back into the box) where that keeps (want_change
    False) or changes (True) its planned mesh shape; returns the new x, y, z
    and the number of halos scaled."""
    parts = _unwrapped(hb)
    before = _shapes(parts, cfg)
    moved = [p[0] + factor * (p - p[0]) for p in parts]
    after = _shapes(moved, cfg)
    keep = (before != after).any(1) if want_change else (before == after).all(1)
    new = [m if k else p for p, m, k in zip(parts, moved, keep)]
    xyz = np.mod(np.concatenate(new), 100.0)
    return xyz, int(keep.sum())


def _write(db, xyz):
    for i, f in enumerate(("x", "y", "z")):
        getattr(db, f).copy_(torch.from_numpy(np.ascontiguousarray(xyz[:, i])))
    torch.cuda.synchronize()


def test_replay_follows_moved_particles(setup):
    hb, ctx, db, cfg = setup
    out = batch.StageBuffers(hb.n, 32, db.x.device, keep_phi=True)
    g = batch.StageGraph(ctx, db, cfg, out)
    # halos shrunk by 1 %: new positions, the same mesh shapes, a similar octree
    xyz, nmoved = _scaled(hb, cfg, 0.99, want_change=False)
    assert nmoved >= hb.nhalo // 2
    _write(db, xyz)
    ref = _eager(cfg, db)
    assert not g.run()  # replayed, no re-plan
    _same(_outputs(out), ref)
    g.close()


def test_replan_when_a_mesh_changes_shape(setup):
    hb, ctx, db, cfg = setup
    out = batch.StageBuffers(hb.n, 32, db.x.device, keep_phi=True)
    g = batch.StageGraph(ctx, db, cfg, out)
    # halos stretched 3x where that enlarges their mesh: the plan no longer fits
    xyz, nmoved = _scaled(hb, cfg, 3.0, want_change=True)
    assert nmoved >= 1
    _write(db, xyz)
    ref = _eager(cfg, db)
    g.launch()
    with pytest.raises(_lib.GFError) as e:
        g.sync()
    assert e.value.status == _lib.GF_ESTALE
    assert g.run()  # re-planned and re-captured; the eager run left the results
    assert g.replans == 1
    _same(_outputs(out), ref)
    out.nearindex.fill_(-7)
    torch.cuda.synchronize()
    assert not g.run()  # the new plan replays
    _same(_outputs(out), ref)
    g.close()


def test_graph_refuses_onchip_and_plain(setup):
    hb, ctx, db, cfg = setup
    out = batch.StageBuffers(hb.n, 32, db.x.device, keep_phi=True)
    for c in (batch.stage_config(mesh_onchip=True), batch.stage_config(plain_fp64=True)):
        with pytest.raises(_lib.GFError) as e:
            batch.StageGraph(ctx, db, c, out)
        assert e.value.status == _lib.GF_ENOTIMPL
