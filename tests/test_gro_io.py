"""The .gro reader and writer against the reference engine's own GromacsFileManager
(ENG/src/GromacsFileManager.cpp:7-124) built in oracle/_ref: values read, bytes
written, files without velocities and malformed files.  Host code only."""
import os

import numpy as np
import pytest

from oracle.refpath import reference_root

_REF = reference_root()
# the reference's own start configurations (read only when the tree is present)
REF_CONFS = [
    os.path.join(_REF or "", "shortRange.inhomo/template/confs/N00010000-T0.7-100x020x020.gro"),
    os.path.join(_REF or "", "shortRange.inhomo/template/confs/conf.16000.gro"),
]


def _synthetic(n, seed=0):
    rng = np.random.default_rng(seed)
    box = np.array([31.7, 20.25, 88.125])
    pos = rng.uniform(0, 1, (n, 3)) * box
    vel = rng.normal(0, 1.3, (n, 3))
    names = ["lj", "OW", "HW1", "SOL", "C", "NA+", "abcde"]
    rn = [names[i % len(names)] for i in range(n)]
    an = [names[(3 * i + 1) % len(names)] for i in range(n)]
    ri = (np.arange(n) // 3 + 1) % 100000
    ai = (np.arange(n) + 1) % 100000
    return box, pos, vel, rn, an, ri, ai


@pytest.fixture(scope="module")
def refgro(orc):
    if not orc.ref_available("libref_gro.so"):
        pytest.skip("reference GromacsFileManager not built (needs the reference tree at build time)")
    return orc


def test_read_matches_reference_reader(mdf, refgro, tmp_path):
    box, pos, vel, rn, an, ri, ai = _synthetic(1000)
    path = tmp_path / "a.gro"
    assert refgro.ref_gro_write(path, "synthetic", ri, rn, an, ai, pos, vel, box) == 0
    ref = refgro.ref_gro_read(path, 1000)
    conf = mdf.read_gro(path)
    assert conf.n == 1000 and conf.title == "synthetic"
    assert np.array_equal(conf.pos, ref["pos"].astype(np.float64))
    assert np.array_equal(conf.vel, ref["vel"].astype(np.float64))
    assert np.array_equal(conf.box, ref["box"].astype(np.float64))
    assert np.array_equal(conf.resd_index, ref["resd_index"])
    assert np.array_equal(conf.atom_index, ref["atom_index"])
    assert conf.resd_name == ref["resd_name"] and conf.atom_name == ref["atom_name"]
    assert conf.resd_name[:3] == rn[:3]


def test_write_is_byte_identical_to_reference_writer(mdf, refgro, tmp_path):
    box, pos, vel, rn, an, ri, ai = _synthetic(777, seed=1)
    p32, v32, b32 = pos.astype(np.float32), vel.astype(np.float32), box.astype(np.float32)
    title = "# at time = 12.500000, step = 2500"
    a, b = tmp_path / "ours.gro", tmp_path / "ref.gro"
    mdf.write_gro(a, mdf.GroConf(p32, b32, v32, ri, rn, an, ai), title)
    assert refgro.ref_gro_write(b, title, ri, rn, an, ai, p32, v32, b32) == 0
    assert a.read_bytes() == b.read_bytes()
    # binary32 passes through both ways: writing the FP64 values gives the same bytes
    mdf.write_gro(a, mdf.GroConf(p32.astype(np.float64), b32, v32, ri, rn, an, ai), title)
    assert a.read_bytes() == b.read_bytes()


def test_round_trip_is_idempotent(mdf, tmp_path):
    box, pos, vel, rn, an, ri, ai = _synthetic(300, seed=2)
    a, b = tmp_path / "a.gro", tmp_path / "b.gro"
    mdf.write_gro(a, mdf.GroConf(pos, box, vel, ri, rn, an, ai), "t")
    c1 = mdf.read_gro(a)
    assert np.abs(c1.pos - pos).max() <= 5e-4 + 1e-5 and np.abs(c1.vel - vel).max() <= 5e-5 + 1e-6
    mdf.write_gro(b, c1)
    assert a.read_bytes() == b.read_bytes()


def test_atom_lines_without_velocities(mdf, refgro, tmp_path):
    path = tmp_path / "nov.gro"
    path.write_text("no velocities\n2\n    1   lj   lj    1   1.000   2.000   3.000\n"
                    "    2   lj   lj    2   4.500   5.250  -0.125\n 10.0 11.0 12.0\n")
    conf = mdf.read_gro(path)
    ref = refgro.ref_gro_read(path, 2)
    assert np.array_equal(conf.pos, ref["pos"].astype(np.float64))
    assert np.all(conf.vel == 0) and np.all(ref["vel"] == 0)
    assert np.array_equal(conf.box, [10.0, 11.0, 12.0])


@pytest.mark.parametrize("text,why", [
    ("title\nnot-a-number\n", "count"),
    ("title\n2\n    1   lj   lj    1   1.000   2.000   3.000\n", "short"),
    ("title\n1\n    1   lj   lj    1   1.000   2.000\n 1 1 1\n", "fields"),
    ("title\n1\n    1   lj   lj    1   1.000   2.000   3.000\n 1 1\n", "box"),
])
def test_malformed_files_are_rejected_like_the_reference(mdf, refgro, tmp_path, text, why):
    path = tmp_path / f"bad_{why}.gro"
    path.write_text(text)
    with pytest.raises(mdf.MDExcptIO):
        mdf.read_gro(path)
    if why != "count":
        assert refgro.ref_gro_read(path, 2 if why == "short" else 1) is None


def test_missing_file(mdf, tmp_path):
    with pytest.raises(mdf.MDExcptIO):
        mdf.read_gro(tmp_path / "absent.gro")
    with pytest.raises(mdf.MDExcptIO):
        mdf.write_gro(tmp_path / "no_dir" / "x.gro", mdf.GroConf(np.zeros((1, 3)), np.ones(3)))


@pytest.mark.parametrize("path", REF_CONFS)
def test_reference_configurations(mdf, refgro, path):
    """The engine's own start configurations, read by both readers."""
    if not os.path.exists(path):
        pytest.skip("reference tree not present")
    conf = mdf.read_gro(path)
    ref = refgro.ref_gro_read(path, conf.n)
    assert np.array_equal(conf.pos, ref["pos"].astype(np.float64))
    assert np.array_equal(conf.vel, ref["vel"].astype(np.float64))
    assert np.array_equal(conf.box, ref["box"].astype(np.float64))
    assert conf.atom_name == ref["atom_name"]
