"""CPU: the autotuner's search space respects the kernels' compile-time limits,
and build.py turns tuned.json into -D flags."""
import json

from galaxyfinder_b200 import build as B
from galaxyfinder_b200 import tune as T


def _valid(p):
    assert p["GF_KNN_ALGO"] in (0, 1, 2)
    assert p["GF_KNNB_SEEDS"] >= 32 and p["GF_KNNB_SEEDS"] % 2 == 0
    assert 0 <= p["GF_KNNB_QUEUE"] <= 16
    assert p["GF_KNNB_LANECERT"] in (0, 1)
    assert p["GF_KNNB_BLOCK"] % 32 == 0 and p["GF_KNNB_BLOCK"] <= 512
    assert p["GF_KNN_BLOCK"] % 32 == 0 and p["GF_KNN_BLOCK"] <= 1024
    assert p["GF_BH_BLOCK"] % 32 == 0 and p["GF_BH_BLOCK"] <= 1024
    assert p["GF_FFT_PENCILS"] % 2 == 0 and (p["GF_FFT_PENCILS"] // 2) * 512 // 8 <= 1024
    assert p["GF_FFT_PENCILS_64"] in (32, 64, 128) and p["GF_FFT_PENCILS_128"] in (32, 64)
    assert 128 <= p["GF_TREE_BLOCK"] <= 1024
    assert p["GF_TSC_TILE"] == 0 or 1024 <= p["GF_TSC_TILE"] <= 12288
    assert p["GF_KNNB_WIN"] in (0, 8, 16, 32)
    assert p["GF_BH_TMA"] in (0, 1) and p["GF_BH_LEAF4"] in (0, 1)
    assert p["GF_KNNB_FILT"] in (0, 1) and p["GF_KNNB_HEAPF"] in (0, 1, 2, 3)
    for b, m in ((p["GF_KNN_BLOCK"], p["GF_KNN_MINB"]), (p["GF_BH_BLOCK"], p["GF_BH_MINB"]),
                 (p["GF_KNNB_BLOCK"], p["GF_KNNB_MINB"])):
        assert m >= 1 and b * m <= 2048  # resident threads per SM
    # the float-key kernel's shared memory per warp: heaps, node window, tile
    warp_bytes = 32 * 32 * 8 + p["GF_KNNB_WIN"] * 48 + 32 * 16 + 32 * 4 + 32 * p["GF_KNNB_QUEUE"] * 8
    if p["GF_KNN_ALGO"] == 2:
        assert p["GF_KNNB_MINB"] * (p["GF_KNNB_BLOCK"] // 32 * warp_bytes + 1024) <= 228 * 1024


def test_search_space_is_valid():
    # both kNN kernels: the warp-per-query stages open up when it wins
    for algo in (0, 1, 2):
        base = dict(T.DEFAULTS, GF_KNN_ALGO=algo)
        for g in T.GROUPS:
            nonempty = 0
            for stage_fn in T.stages(g):
                stage = stage_fn(base)
                nonempty += bool(stage)
                for ov in stage:
                    _valid(dict(base, **ov))
            assert nonempty >= 1
        assert len(T.stages("knn")[1](base)) == (5 if algo == 2 else 0)  # seed windows
        assert len(T.stages("knn")[2](base)) == (2 if algo == 2 else 0)  # lane or warp certification
        assert len(T.stages("knn")[3](base)) == (2 if algo == 2 else 0)  # work counter or grid-stride
        assert len(T.stages("knn")[4](base)) == (4 if algo == 2 else 0)  # node window x resident blocks
        assert len(T.stages("knn")[5](base)) == (4 if algo == 2 else 0)  # survivor queues
        assert len(T.stages("knn")[6](base)) == (8 if algo == 2 else 0)  # tile filter x heap order
        assert len(T.stages("knn")[7](base)) == (3 if algo == 0 else 0)


def test_tuned_params_become_flags(tmp_path, monkeypatch):
    f = tmp_path / "tuned.json"
    f.write_text(json.dumps({"params": {"GF_KNN_CHUNK": 16, "GF_BH_BLOCK": 64}}))
    monkeypatch.setattr(B, "TUNED", f)
    flags = B._flags("gf_knn.cu")
    assert "-DGF_KNN_CHUNK=16" in flags and "-DGF_BH_BLOCK=64" in flags and "--fmad=false" in flags
    assert B.tuned_params() == {"GF_KNN_CHUNK": 16, "GF_BH_BLOCK": 64}
    assert T.variant_name({"GF_KNN_CHUNK": 16}) == "knn_chunk16"


def test_library_reports_its_launch_parameters():
    """gf_tuning_value reports the parameters the loaded library was compiled
    with; build.py compiles with tuned.json's values."""
    from galaxyfinder_b200 import _lib
    params = B.tuned_params()
    for name in ("GF_KNN_ALGO", "GF_KNNB_BLOCK", "GF_KNNB_SEEDS", "GF_BH_BLOCK", "GF_FFT_PENCILS", "GF_KNNB_WIN",
                 "GF_KNNB_MINB", "GF_BH_DYN", "GF_KNNB_DYN"):
        assert _lib.tuning_value(name) == params.get(name, T.DEFAULTS[name]), name
    import pytest
    with pytest.raises(_lib.GFError):
        _lib.tuning_value("GF_NO_SUCH_PARAMETER")
