"""Gauge configuration files through the C ABI (yg_gauge_save_cfg / yg_gauge_load_cfg,
yg_gauge_save_hirep / yg_gauge_load_hirep).

The file formats are those of gaugefield.cpp:44-161 (CFG: 256-byte header, native byte
order) and hirep.cpp:56-212 (big-endian); the oracle's reader and writer for them are pinned
bit-exactly to the reference's own save and load.  Here the engine writes files the oracle
reads back bit-exactly, and loads the oracle's files into the links the reference's load
gives (boundary conditions applied), with the represented field and clover term rebuilt."""
import numpy as np
import pytest

from oracle import yahmc_oracle as yo
from tests.helpers import make_pair, rel, source
from yahmc_b200 import fields

pytestmark = pytest.mark.gpu

NAMES = ["su3_fund_ap", "su3_fund_open", "su3_fund_sf", "su2_adj_ap", "su4_asym_ap", "su3_fund_ap_full"]


def _dims(name):
    return (8, 8, 8, 8) if name.startswith("su3") else (6, 4, 4, 8)


@pytest.mark.parametrize("name", NAMES)
def test_save_is_read_exactly(name, tmp_path):
    lat, O, rng = make_pair(name, _dims(name), seed=61)
    U = lat.get_links()
    p = tmp_path / "a.cfg"
    lat.gauge_field_save(p, num_cnfg=17, num_accept=11)
    c = yo.cfg_read(p, O.p.eo)
    assert c["ident"] == yo.CFG_IDENT and c["version"] == yo.CFG_VERSION
    assert c["dims"] == tuple(_dims(name)) and c["nc"] == O.nc and c["repr"] == yo.REPR_NAMES.index(O.p.rep)
    assert (c["num_cnfg"], c["num_accept"]) == (17, 11)
    assert c["plaquette"] == lat.plaquette()
    assert np.array_equal(c["U"], U)
    assert p.stat().st_size == 256 + O.V * 4 * 2 * O.nc * O.nc * 8
    h = tmp_path / "a.hirep"
    lat.gauge_field_save_hirep(h)
    hr = yo.hirep_read(h, O.p.eo)
    assert hr["nc"] == O.nc and hr["dims"] == tuple(_dims(name)) and hr["plaquette"] == lat.plaquette()
    assert np.array_equal(hr["U"], U)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("fmt", ["cfg", "hirep"])
def test_load_matches_reference_semantics(name, fmt, tmp_path):
    lat, O, rng = make_pair(name, _dims(name), seed=62)
    W = fields.haar_su(O.nc, O.V * 4, rng).reshape(O.V, 4, O.nc, O.nc)
    stored = 0.3125
    if fmt == "cfg":
        p = tmp_path / "b.cfg"
        yo.cfg_write(p, W, _dims(name), O.nc, yo.REPR_NAMES.index(O.p.rep), stored, 9, 4, O.p.eo)
        n, a, pd = lat.gauge_field_load(p)
        assert (n, a) == (9, 4)
    else:
        p = tmp_path / "run3_n42"
        yo.hirep_write(p, W, _dims(name), O.nc, stored, O.p.eo)
        n, pd = lat.gauge_field_load_hirep(p)
        assert n == 42
    O.fund = W.copy()
    O.bcs_on_gauge()
    # the SF boundary links diag exp(i v / L) come from libm here and numpy in the oracle:
    # equal to the last ulp; everything else is copied bit for bit
    assert np.abs(lat.get_links() - O.fund).max() <= (1e-15 if O.p.bc == "sf" else 0.0)
    O.set_links(O.fund)
    assert abs(pd - abs(stored - O.plaquette())) < 1e-13
    assert rel(lat.repr_links(), O.links) < 1e-13
    src = source(O, rng)
    for fn, mass in [("Dphi", -0.6), ("Hphi_sq", -0.6)]:
        d_dev, d2 = lat.field(), O.new_field()
        getattr(lat, fn)(mass, d_dev, lat.field(src))
        getattr(O, fn)(mass, d2, src.copy())
        assert rel(lat.download(d_dev), d2) < 1e-13, fn


def test_round_trip_and_errors(tmp_path):
    from yahmc_b200 import YGError
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=63)
    U = lat.get_links()
    p, h = tmp_path / "c.cfg", tmp_path / "c_n5"
    lat.gauge_field_save(p, 3, 2)
    lat.gauge_field_save_hirep(h)
    lat2, _, _ = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=64)
    assert lat2.gauge_field_load(p) == (3, 2, 0.0)
    assert np.array_equal(lat2.get_links(), U)
    lat3, _, _ = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=65)
    assert lat3.gauge_field_load_hirep(h) == (5, 0.0)
    assert np.array_equal(lat3.get_links(), U)
    # an inconsistent header, a short file and a missing file are errors
    other, _, _ = make_pair("su3_fund_ap", (8, 8, 8, 12), seed=66)
    with pytest.raises(YGError):
        other.gauge_field_load(p)
    with pytest.raises(YGError):
        other.gauge_field_load_hirep(h)
    adj, _, _ = make_pair("su3_adj_ap", (8, 8, 8, 8), seed=67)
    with pytest.raises(YGError):
        adj.gauge_field_load(p)                      # repr differs
    short = tmp_path / "short.cfg"
    short.write_bytes(p.read_bytes()[:4096])
    with pytest.raises(YGError):
        lat2.gauge_field_load(short)
    with pytest.raises(YGError):
        lat2.gauge_field_load(tmp_path / "missing.cfg")
    assert np.array_equal(lat2.get_links(), U)       # a failed load leaves the field alone
