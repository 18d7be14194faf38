"""Curve exporters and full-state checkpoints on the GPU.

  * exportToBCC / exportToOBJ (io/fileExport.cpp:6-100) write, byte for byte, what the
    restatement in oracle/files.py writes for the same downloaded vertices;
  * a simulation saved with save_state and restored with load_state continues bit-identically
    to the one that never stopped (both precisions; detectionPeriod 3 exercises the contact
    lists carried across substeps without detection; a batch of scenes; the step counter).
"""
import numpy as np
import pytest

from oracle import files as ofiles
from yarnball_b200 import scenes
from yarnball_b200.sim import Sim

pytestmark = pytest.mark.gpu


def _batch_spec():
    return scenes.batched_spec(seed=5, num_scenes=6, cap=40000, max_yarns=6, min_len=64, max_len=1500)


@pytest.mark.parametrize("polyline", [False, True])
def test_export_bcc_matches_restatement(tmp_path, polyline):
    sim = scenes.build_readme()
    sim.advance(1 / 30)
    path = tmp_path / "readme.bcc"
    sim.exportToBCC(str(path), polyline)
    data = path.read_bytes()
    assert data == ofiles.bcc_bytes(sim.verts, polyline)
    parsed = ofiles.read_bcc(data)
    assert parsed["sign"] == b"BCC" and parsed["byteCount"] == 0x44 and parsed["end"] == len(data)
    assert parsed["curveType"] == (b"PL" if polyline else b"C0")
    assert parsed["curveCount"] == 2 and parsed["totalControlPointCount"] == sim.numVerts
    np.testing.assert_array_equal(np.concatenate(parsed["curves"]), sim.verts["pos"])
    sim.close()


def test_export_obj_matches_restatement(tmp_path):
    sim = scenes.build_readme()
    sim.advance(1 / 30)
    path = tmp_path / "readme.obj"
    sim.exportToOBJ(str(path))
    assert path.read_text() == ofiles.obj_text(sim.verts)
    sim.close()


def test_export_batch_writes_every_scene(tmp_path):
    spec = _batch_spec()
    sim, _ = scenes.build_batched(seed=5, spec=spec)
    sim.advance(1 / 30)
    sim.exportToBCC(str(tmp_path / "b.bcc"))
    sim.exportToOBJ(str(tmp_path / "b.obj"))
    data = (tmp_path / "b.bcc").read_bytes()
    assert data == ofiles.bcc_bytes(sim.verts)
    parsed = ofiles.read_bcc(data)
    assert parsed["curveCount"] == sum(spec[0])
    assert (tmp_path / "b.obj").read_text() == ofiles.obj_text(sim.verts)
    sim.close()


def test_export_unopenable_path_is_an_error():
    sim = scenes.build_readme()
    with pytest.raises(RuntimeError):
        sim.exportToBCC("/nonexistent-dir/x.bcc")
    sim.close()


def _exact_state(sim):
    pos, vel, q = sim.read_state_f64()
    return pos, vel, q


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("period", [1, 3])
def test_checkpoint_resumes_bit_identically(tmp_path, precision, period):
    sim = scenes.build_pile(seed=3, yarns=48, verts=160, precision=precision, meta={"detectionPeriod": period})
    sim.advance(1 / 30)
    path = tmp_path / "pile.ybck"
    sim.save_state(str(path))
    steps_at_save = sim.stepCount()
    sim.advance(1 / 30)
    sim.advance(1 / 30)
    want = _exact_state(sim)

    back = Sim.load_state(str(path))
    assert back.precision == precision and back.numVerts == sim.numVerts
    assert back.stepCount() == steps_at_save
    assert back.meta.detectionPeriod == period
    back.advance(1 / 30)
    back.advance(1 / 30)
    got = _exact_state(back)
    for a, b in zip(want, got):
        np.testing.assert_array_equal(a, b)
    assert back.stepCount() == sim.stepCount()
    sim.close()
    back.close()


def test_checkpoint_of_a_batch(tmp_path):
    spec = _batch_spec()
    sim, _ = scenes.build_batched(seed=5, spec=spec)
    sim.advance(1 / 30)
    sim.save_state(str(tmp_path / "batch.ybck"))
    sim.advance(1 / 30)
    want = _exact_state(sim)
    back = Sim.load_state(str(tmp_path / "batch.ybck"))
    assert back.numScenes == sim.numScenes
    np.testing.assert_array_equal(back.sceneOffsets, sim.sceneOffsets)
    back.advance(1 / 30)
    for a, b in zip(want, _exact_state(back)):
        np.testing.assert_array_equal(a, b)
    sim.close()
    back.close()


def test_load_state_rejects_a_foreign_file(tmp_path):
    p = tmp_path / "junk.ybck"
    p.write_bytes(b"not a checkpoint at all")
    with pytest.raises(RuntimeError):
        Sim.load_state(str(p))


def test_export_fiber_mesh_matches_restatement(tmp_path):
    from oracle import mesher
    sim = scenes.build_readme()
    sim.advance(1 / 30)
    path = tmp_path / "fibers.obj"
    sim.exportFiberMesh(str(path))
    got = mesher.parse_obj(path.read_text())
    m = sim.meta
    fv, fl, zv, zl = mesher.fiber_mesh(sim.verts["pos"], sim.qs, sim.verts["lRest"], sim.verts["flags"],
                                       m.radius, m.barrierThickness)
    assert list(got) == ["fiber", "fuzz"]
    gv, gl = got["fiber"]
    assert gv.shape == fv.shape and gl == fl
    assert len(fl) == 16  # 8 fibres x 2 yarns
    np.testing.assert_allclose(gv, fv, rtol=0, atol=2e-6)
    hv, hl = got["fuzz"]
    assert hv.shape == zv.shape and [tuple(x) for x in hl] == zl and len(zl) > 100
    np.testing.assert_allclose(hv, zv, rtol=0, atol=2e-6)
    with pytest.raises(RuntimeError):
        sim.exportFiberMesh("/nonexistent-dir/f.obj")
    sim.close()
