"""CPU checks of the C ABI: libgf.so loads, exports every entry point that
include/gf.h declares, and the host-only planner follows the reference's
mesh sizing rule.  No kernel is launched here."""
import ctypes
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in {"if", "for", "while", "return", "sizeof"}:
                names.add(name)
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol(gf):
    names = declared_functions()
    assert "assign_density_TSC" in names and "gf_plan_meshes" in names
    missing = [n for n in names if not hasattr(gf, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "galaxyfinder_b200/libgf.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    assert set(names) <= exported


def test_dropins_report_a_missing_device(gf):
    """Without a GPU a drop-in fails loudly: with GF_NOEXIT set it returns and
    leaves the status, without it the process exits with code 99 and names
    the function (the reference's callers have no status to read)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    gf.mkRtidal()
    assert gf.gf_last_status() != 0
    assert gf.nfw_rtidal(0.01, 0.5, 10.0) == 0.0  # no table was built
    code = "import ctypes, sys; ctypes.CDLL(sys.argv[1]).mkRtidal(); print('returned')"
    env = {k: v for k, v in os.environ.items() if k != "GF_NOEXIT"}
    r = subprocess.run([sys.executable, "-c", code, str(ROOT / "galaxyfinder_b200/libgf.so")], env=env,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 99 and "mkRtidal" in r.stderr and "returned" not in r.stdout


def test_status_strings(gf):
    from galaxyfinder_b200 import _lib
    assert gf.gf_status_string(_lib.GF_ERANGE) == b"particle outside mesh"
    assert gf.gf_status_string(0) == b"ok"


def test_struct_layouts_match_reference():
    from galaxyfinder_b200 import _lib
    assert _lib.BP_DTYPE.itemsize == 88                    # tree.h:155-162
    assert _lib.BP_DTYPE.fields["x"][1] == 16
    assert _lib.BP_DTYPE.fields["indx"][1] == 72
    assert _lib.VEC3_DTYPE.itemsize == 24                  # subhaloden.mod6.c:70
    assert _lib.MESH_DTYPE.itemsize == 64


def test_physics_matches_reference(golden, gf):
    """physical_parameters (gfind.c:842-890) and GetBGpotent (subhaloden.mod6.c:1093)
    at the default cosmology used by the golden fixtures."""
    from galaxyfinder_b200 import dropin
    g = golden("potential")
    ph = dropin.physics()
    assert ph["potentfact"] == pytest.approx(float(g["potentfact"]), rel=1e-12)
    assert ph["r1kineticfact"] == pytest.approx(float(g["r1kineticfact"]), rel=1e-7)
    assert dropin.bg_potent(1e12) == pytest.approx(float(g["bg_1e12"]), rel=1e-12)


def _reference_dims(ext, cell=0.004, nbuff=10):
    e = ext + ext * 0.0001
    return [int(v / cell + nbuff) for v in e]


def test_plan_reference_rule_matches_lagFindStellarCore():
    from galaxyfinder_b200 import batch
    rng = np.random.default_rng(5)
    ext = rng.uniform(0.01, 0.6, (50, 3))
    mesh, total = batch.plan_meshes(ext, batch.mesh_rule())
    for h in range(50):
        assert [mesh["nx"][h], mesh["ny"][h], mesh["nz"][h]] == _reference_dims(ext[h])
        assert mesh["xmin"][h] == 0.0 - 0.004 * 10 / 2.0
        assert mesh["off"][h] % 64 == 0
    last = mesh[-1]
    assert total >= last["off"] + 2 * (last["nx"] // 2 + 1) * last["ny"] * last["nz"]


def test_plan_pow2_rule():
    from galaxyfinder_b200 import _lib, batch
    ext = np.array([[0.05, 0.04, 0.03], [0.5, 0.2, 0.1], [3.0, 1.0, 1.0]])
    rule = batch.mesh_rule(mode=_lib.MESH_POW2, rg=2.0, rg_in_cells=True)
    mesh, _ = batch.plan_meshes(ext, rule)
    assert list(mesh["nx"]) == [64, 256, 256]
    assert mesh["cellsize"][0] == 0.004 and mesh["cellsize"][1] == 0.004
    assert mesh["cellsize"][2] == pytest.approx(3.0 * 1.0001 / 246)
    assert np.allclose(mesh["rg"], 2.0 * mesh["cellsize"])
    # every particle stencil stays inside its mesh
    assert np.all((ext * 1.0001 / mesh["cellsize"][:, None] + 5 + 1) < mesh["nx"][:, None])


def test_plan_rejects_bad_rule():
    from galaxyfinder_b200 import _lib, batch
    with pytest.raises(_lib.GFError):
        batch.plan_meshes(np.ones((1, 3)), batch.mesh_rule(nbuff=3))
