"""Device tables written as .qttb files byte for byte as TravelTimeTable.Write lays them out, and
.qttb files read back into a resident table set (TravelTimeTable.Open)."""
import numpy as np
import pytest

from oracle import qttb as OQ
from tomostar_b200 import _lib as L
from tomostar_b200 import location as loc
from tomostar_b200 import qttb
from tomostar_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def test_write_then_load(solver, tmp_path):
    job = syn.relocation_small()
    with loc.Tables.build(solver, job.grid, job.slowness, job.table_source, job.table_phase) as t:
        tabs = t.copy()
        names = [f"S{i % 12:02d}" for i in range(len(tabs))]
        phases = ["P" if p == 0 else "S" for p in job.table_phase]
        keys = [qttb.model_key(job.grid, job.slowness[p]) for p in job.table_phase]
        heads = [qttb.header_json(nm, ph, *src, job.grid, key, "cuda fast sweeping")
                 for nm, ph, src, key in zip(names, phases, job.table_source, keys)]
        paths = [tmp_path / f"{nm}.{ph}.qttb" for nm, ph in zip(names, phases)]
        qttb.write(t, paths, heads)
    for k, p in enumerate(paths):
        data = p.read_bytes()
        assert data == OQ.write_bytes(heads[k], tabs[k].astype(np.float64))
        h, v = OQ.open_bytes(data)
        assert h == heads[k] and np.array_equal(v, tabs[k])
    assert not list(tmp_path.glob("*.tmp"))
    with qttb.load(solver, job.grid, paths) as back:
        assert np.array_equal(back.copy(), tabs)


def test_non_finite_values_and_refusals(solver, tmp_path):
    job = syn.relocation_small()
    g = job.grid
    tab = np.linspace(0, 9, g.count, dtype=np.float32)[None, :].repeat(2, axis=0)
    tab[0, 5], tab[0, 7], tab[1, 0] = np.nan, -np.inf, np.inf
    head = qttb.header_json("X", "P", 13.1, 43.1, 0.0, g)
    with loc.Tables.upload(solver, g, tab) as t:
        qttb.write(t, [tmp_path / "a.qttb", tmp_path / "b.qttb"], [head, head + b" "])
    a = (tmp_path / "a.qttb").read_bytes()
    assert a == OQ.write_bytes(head, tab[0].astype(np.float64))
    assert np.isposinf(OQ.open_bytes(a)[1][[5, 7]]).all()
    assert (tmp_path / "b.qttb").read_bytes() == OQ.write_bytes(head + b" ", tab[1].astype(np.float64))
    bad = tmp_path / "bad.qttb"
    bad.write_bytes(b"QTTX" + a[4:])
    with pytest.raises(L.TsError):
        qttb.load(solver, g, [bad])
    short = tmp_path / "short.qttb"
    short.write_bytes(a[:-4])
    with pytest.raises(L.TsError):
        qttb.load(solver, g, [tmp_path / "a.qttb", short])
    with pytest.raises(L.TsError):
        qttb.load(solver, g, [tmp_path / "missing.qttb"])
