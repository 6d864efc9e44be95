"""The .geo and .init readers and writers and the .params series reader
(adh_kraken_b200/deck.py) against the reference's own readers, sgrid_read,
smodel_super_read_init and sseries_read_allocate, run through the compiled harness
(oracle/_ref/); no GPU."""
import os

import numpy as np
import pytest

from adh_kraken_b200.deck import case_from_files, read_geo, read_init, write_geo, write_init
from adh_kraken_b200.mesh import flume_case, small_delaunay_case
from oracle.oracle import OracleModel
from oracle import refio
from oracle.refio import harness_available, run_harness
from adh_kraken_b200 import deck

needs_harness = pytest.mark.skipif(not harness_available(), reason="reference harness not built")
from fixtures import reference_src

_SRC = reference_src()
QA_GEO = os.path.join(os.path.dirname(_SRC), "qa", "flume", "test.geo") if _SRC else None


def cases():
    return [flume_case(nsteps=2, npx=21, npy=6), small_delaunay_case(n=12, seed=5, nsteps=2)]


def states(case, seed):
    rng = np.random.default_rng(seed)
    s = [case.sol0 + 0.01 * rng.standard_normal(case.sol0.size) for _ in range(3)]
    s[0][0::3] -= 1e-300          # values that need all 17 digits
    return s


@pytest.mark.parametrize("ci", [0, 1])
def test_geo_and_init_round_trip(tmp_path, ci):
    case = cases()[ci]
    geo, init = str(tmp_path / "g.geo"), str(tmp_path / "g.init")
    write_geo(geo, case.xyz, case.tri, case.seg, seg_bflag=case.seg_kind + 7)
    g = read_geo(geo)
    assert np.array_equal(g.xyz, case.xyz) and np.array_equal(g.tri, case.tri) and np.array_equal(g.seg, case.seg)
    assert np.array_equal(g.seg_bflag, case.seg_kind + 7) and np.all(g.tri_bflag == -1)
    s = states(case, ci)
    write_init(init, *s, nelems=case.ntri)
    r = read_init(init, case.nnodes)
    for a, b in zip(r, s):
        assert np.array_equal(a, b)


@needs_harness
@pytest.mark.parametrize("ci", [0, 1])
def test_geo_reader_matches_reference(tmp_path, ci):
    case = cases()[ci]
    geo = str(tmp_path / "g.geo")
    write_geo(geo, case.xyz, case.tri, case.seg)
    ref = run_harness("geo", in_path=geo)
    g = read_geo(geo)
    assert np.array_equal(ref["xyz"], g.xyz.ravel())
    assert np.array_equal(ref["tri"], g.tri.ravel()) and np.array_equal(ref["seg"], g.seg.ravel())
    assert np.array_equal(ref["djac"], OracleModel(case).tri_djac)


@needs_harness
@pytest.mark.skipif(QA_GEO is None or not os.path.exists(QA_GEO), reason="reference QA deck not present")
def test_geo_reader_on_the_reference_qa_grid():
    """The reference's own QA flume grid (comment lines, unordered cards, no materials
    on the element cards) read by both readers."""
    ref = run_harness("geo", in_path=QA_GEO)
    g = read_geo(QA_GEO)
    assert g.xyz.shape == (561, 3) and g.tri.shape == (1000, 3) and g.seg.shape == (120, 2)
    assert np.array_equal(ref["xyz"], g.xyz.ravel())
    assert np.array_equal(ref["tri"], g.tri.ravel()) and np.array_equal(ref["seg"], g.seg.ravel())


@needs_harness
@pytest.mark.parametrize("ci", [0, 1])
def test_init_reader_matches_reference(tmp_path, ci):
    case = cases()[ci]
    base = str(tmp_path / "state")
    s = states(case, 10 + ci)
    write_init(base + ".init", *s, nelems=case.ntri)
    ref = run_harness("init", case, extra=(base,))
    r = read_init(base + ".init", case.nnodes)
    for key, mine in zip(("sol", "sol_old", "sol_older"), r):
        assert np.array_equal(ref[key], mine)


@needs_harness
def test_init_reader_partial_file_matches_reference(tmp_path):
    """A file that sets only some levels and variables: the rest stays 0 in both."""
    case = cases()[1]
    base = str(tmp_path / "part")
    s = states(case, 3)
    write_init(base + ".init", *s, nelems=case.ntri)
    with open(base + ".init") as f:
        text = f.read()
    blocks = text.split("DATASET\n")[1:]
    keep = [b for b in blocks if "NAME DEPTH" in b or "NAME OLD DA_VELOCITY" in b]
    with open(base + ".init", "w") as f:
        f.write("".join("DATASET\n" + b for b in keep))
    ref = run_harness("init", case, extra=(base,))
    r = read_init(base + ".init", case.nnodes)
    for key, mine in zip(("sol", "sol_old", "sol_older"), r):
        assert np.array_equal(ref[key], mine)
    assert np.array_equal(r[0][0::3], s[0][0::3]) and not r[0][1::3].any()
    assert np.array_equal(r[1][1::3], s[1][1::3]) and not r[1][0::3].any() and not r[2].any()


def test_geo_card_order_comments_and_errors(tmp_path):
    case = cases()[0]
    geo = str(tmp_path / "g.geo")
    write_geo(geo, case.xyz, case.tri, case.seg)
    with open(geo) as f:
        lines = f.read().splitlines()
    nd = [ln for ln in lines if ln.startswith("ND ")]
    other = [ln for ln in lines if not ln.startswith("ND ")]
    shuffled = str(tmp_path / "s.geo")
    with open(shuffled, "w") as f:
        f.write("! a comment card\n" + "\n".join(other[:3] + nd[::-1] + ["", "! boundary"] + other[3:]) + "\n")
    g = read_geo(shuffled)
    assert np.array_equal(g.xyz, case.xyz) and np.array_equal(g.tri, case.tri)
    bad = str(tmp_path / "b.geo")
    with open(bad, "w") as f:
        f.write("\n".join(other[:3] + nd[1:] + other[3:]) + "\n")       # node 1 missing
    with pytest.raises(ValueError):
        read_geo(bad)
    with open(bad, "w") as f:
        f.write("\n".join(lines + ["QUAD 1 1 2 3 4 -1"]) + "\n")
    with pytest.raises(ValueError):
        read_geo(bad)


def test_init_errors(tmp_path):
    case = cases()[0]
    p = str(tmp_path / "e.init")
    write_init(p, *states(case, 1))
    with pytest.raises(ValueError):
        read_init(p, case.nnodes + 1)
    with open(p) as f:
        text = f.read()
    for old, new in (("NAME DEPTH", "NAME SALINITY"), ("DIM 2", "DIM 1")):
        with open(p, "w") as f:
            f.write(text.replace(old, new, 1))
        with pytest.raises(ValueError):
            read_init(p, case.nnodes)


def test_case_from_files_steps_like_the_original(tmp_path):
    case = cases()[1]
    geo, init = str(tmp_path / "c.geo"), str(tmp_path / "c.init")
    write_geo(geo, case.xyz, case.tri, case.seg, seg_bflag=case.seg_kind + 1)
    write_init(init, case.sol0, case.sol0, case.sol0)
    c2 = case_from_files("wetdry_from_files", geo, init, {1: 0, 2: 1}, case.dt, 2, case.series, t0=case.t0)
    a, ha = OracleModel(case).run(2)
    b, hb = OracleModel(c2).run(2)
    assert np.array_equal(a, b) and [h["newton_its"] for h in ha] == [h["newton_its"] for h in hb]


PARAMS_TEXT = """MODEL 1 SW2
# series in several time units, with tabs and blank lines
SERIES BC 1 3 0 0
0 2.0
3600\t2.5
7200 2.25

SERIES BC 3 4 2 0
0   0.1
0.5 0.2
1.25 0.35
2 0.1e-1
IP NTL 1e-6
SERIES BC 2 2 1 1
0 -0.125
90 3.3333333333333335
BC 3 SW2 NB VEL 1
"""


@pytest.mark.skipif(not refio.harness_available(), reason="reference harness not built")
def test_params_series_match_the_reference_reader(tmp_path):
    """The .params series pass reads what the reference's sseries_read_allocate reads,
    bit for bit: ids, times scaled by the input unit, values."""
    p = tmp_path / "deck.params"
    p.write_text(PARAMS_TEXT)
    files = [str(p)]
    src = reference_src()
    if src is not None:
        files += [os.path.join(os.path.dirname(src), "qa", "flume", f) for f in ("test_sm1.params", "test_sm2.params")]
    for f in files:
        ours = deck.read_params_series(f)
        ref = refio.run_params_series(f)
        assert list(ours) == list(ref), f
        for k in ours:
            assert np.array_equal(ours[k][0], ref[k][0]) and np.array_equal(ours[k][1], ref[k][1]), (f, k)
    ours = deck.read_params_series(str(p))
    assert sorted(ours) == [0, 1, 2]
    assert ours[2][0].tolist() == [0.0, 1800.0, 4500.0, 7200.0]      # hours
    assert ours[1][0].tolist() == [0.0, 5400.0]                       # minutes


def test_params_series_refuse_bad_units(tmp_path):
    p = tmp_path / "bad.params"
    p.write_text("SERIES BC 1 1 7 0\n0 1\n")
    with pytest.raises(ValueError):
        deck.read_params_series(str(p))


def test_case_from_a_params_file_steps_like_the_original(tmp_path):
    """The case's series written as SERIES BC cards and read back from the .params file
    give the same run (the cards' values are written with 17 significant digits)."""
    case = cases()[1]
    geo, init, params = str(tmp_path / "c.geo"), str(tmp_path / "c.init"), str(tmp_path / "c.params")
    write_geo(geo, case.xyz, case.tri, case.seg, seg_bflag=case.seg_kind + 1)
    write_init(init, case.sol0, case.sol0, case.sol0)
    with open(params, "w") as fh:
        fh.write("MODEL 1 SW2\n")
        for sid, (t, v) in sorted(case.series.items()):
            fh.write(f"SERIES BC {sid + 1} {len(t)} 0 0\n")
            for ti, vi in zip(t, v):
                fh.write(f"{ti:.17g} {vi:.17g}\n")
    c2 = case_from_files("wetdry_from_params", geo, init, {1: 0, 2: 1}, case.dt, 2, params, t0=case.t0)
    for sid in case.series:
        assert np.array_equal(c2.series[sid][0], case.series[sid][0])
        assert np.array_equal(c2.series[sid][1], case.series[sid][1])
    a, _ = OracleModel(case).run(2)
    b, _ = OracleModel(c2).run(2)
    assert np.array_equal(a, b)
