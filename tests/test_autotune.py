"""Row-tiling autotuner of the z-operator GEMMs (tg_autotune): the JSON cache
is written, read back and validated, and the fields do not depend on the
tiling (every tiling gives the same fields bit for bit)."""
import json
import math

import numpy as np
import pytest

import turbid_b200 as tb
from oracle import turbid_oracle as O

pytestmark = pytest.mark.gpu

CASE_KEYS = ("nx", "ny", "nz", "lx", "ly", "nphase", "mapping", "mapping_coef", "slope", "slope_direction", "dt",
             "output_based_on_step", "reynolds", "froude", "averaged_concentration", "specific_gravity",
             "affected_by_scalar", "bc_u", "bc_v", "bc_w", "bc_p", "force_type", "force_direction",
             "force_amplitude", "schmidt", "settling", "erosion_rate", "critical_shear", "scalar_bc")


def sediment_cfg(**kw):
    base = dict(nx=32, ny=24, nz=65, nphase=2, reynolds=800.0, froude=1.0, averaged_concentration=1e-3,
                specific_gravity=2.65, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4, schmidt=0.5,
                critical_shear=2e-4, erosion_rate=1e-4, dt=2 * math.pi / 2000)
    base.update(kw)
    return O.CaseConfig(**base)


def make_case(cfg, precision):
    uvw, p, phi = O.make_initial_state(cfg, seed=7, noise=0.05)
    gc = tb.ChannelCase(precision=precision, **{k: getattr(cfg, k) for k in CASE_KEYS})
    gc.upload_state(uvw, p, phi)
    return gc


def run(cfg, precision, nsteps, cache=None):
    gc = make_case(cfg, precision)
    tiling = gc.autotune(cache) if cache is not None else None
    feats = np.zeros(50)
    assert gc.run_steps(nsteps, features=feats) == nsteps
    out = gc.download_state()
    gc.close()
    return out, feats, tiling


def row_tiling(rows, pref):
    need = (rows + 7) // 8
    tiles = -(-need // pref)
    return -(-need // tiles), tiles


def test_autotune_writes_and_reads_cache(cuda, tmp_path):
    cfg = sediment_cfg()
    path = tmp_path / "tiling.json"
    gc = make_case(cfg, "mixed")
    t0 = gc.autotune(str(path))
    gc.close()
    cache = json.loads(path.read_text())
    assert len(cache) == 1
    (key, (pd, ps)), = cache.items()
    assert key.startswith(f"{cfg.nx}x{cfg.ny}x{cfg.nz}:mixed:sm")
    assert 1 <= pd <= 16 and 1 <= ps <= 6
    assert (t0["mt_dense"], t0["tiles_dense"]) == row_tiling(cfg.nz, pd)
    assert (t0["mt_folded"], t0["tiles_folded"]) == row_tiling((cfg.nz - 1) // 2 + 1, ps)
    text = path.read_text()
    # a second context on the same case takes the cached entry without timing
    gc = make_case(cfg, "mixed")
    assert gc.autotune(str(path)) == t0
    gc.close()
    assert path.read_text() == text
    # another precision is another entry; the first stays
    gc = make_case(cfg, "fp64")
    gc.autotune(str(path))
    gc.close()
    cache2 = json.loads(path.read_text())
    assert len(cache2) == 2 and cache2[key] == [pd, ps]
    # no cache: timed, nothing written
    gc = make_case(cfg, "mixed")
    t1 = gc.autotune(None)
    gc.close()
    assert t1["tiles_dense"] >= 1 and t1["tiles_folded"] >= 1


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fields_do_not_depend_on_tiling(cuda, tmp_path, precision):
    cfg = sediment_cfg()
    path = tmp_path / "tiling.json"
    gc = make_case(cfg, precision)
    gc.autotune(str(path))
    gc.close()
    (key, _), = json.loads(path.read_text()).items()
    (u0, p0, c0), f0, _ = run(cfg, precision, 3)   # built-in tiling
    for pd, ps in ((1, 1), (3, 2), (8, 4), (16, 6)):
        path.write_text(json.dumps({key: [pd, ps]}))
        (u1, p1, c1), f1, t = run(cfg, precision, 3, str(path))
        assert (t["mt_dense"], t["tiles_dense"]) == row_tiling(cfg.nz, pd)
        assert (t["mt_folded"], t["tiles_folded"]) == row_tiling((cfg.nz - 1) // 2 + 1, ps)
        assert np.array_equal(u0, u1) and np.array_equal(p0, p1) and np.array_equal(c0, c1), (pd, ps)
        assert np.array_equal(f0, f1)


def test_autotune_rejects_bad_cache(cuda, tmp_path):
    cfg = sediment_cfg(nz=33)
    path = tmp_path / "tiling.json"
    gc = make_case(cfg, "fp64")
    gc.autotune(str(path))
    (key, _), = json.loads(path.read_text()).items()
    path.write_text(json.dumps({key: [40, 2]}))
    with pytest.raises(tb.TgError, match="out of range") as e:
        gc.autotune(str(path))
    assert e.value.code == 3
    other = tmp_path / "notes.txt"
    other.write_text("not a cache\n")
    with pytest.raises(tb.TgError, match="not a tiling cache"):
        gc.autotune(str(other))
    assert other.read_text() == "not a cache\n"
    # the context still steps after the refusals
    assert gc.run_steps(1) == 1
    gc.close()
