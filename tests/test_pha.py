"""FORBILD phantom files (.pha) and point sampling, on the CPU.

* the reader against values written in the reference's head phantom file
  (src/aprict/data/FORBILD/head/HeadPhantom.pha, parsed into
  tests/golden/forbild_head_shapes.npy by tests/golden/make_forbild_golden.py)
  and against a synthetic file covering the format's features;
* writer -> reader round trip;
* the FP64 point-sampling oracle against the reference's own sampling body
  (its _in_region, compiled for the CPU) on the head phantom and random
  clipped quadrics: only sample points within FP32 rounding of a surface may
  differ;
* FBVolume transforms.
"""

from __future__ import annotations

import math
import pathlib

import numpy as np
import pytest

from aprict_b200 import FBVolume, pha, phantoms
from aprict_b200 import _structs as S
from oracle import oracle as O

GOLDEN = pathlib.Path(__file__).parent / "golden" / "forbild_head_shapes.npy"


def head() -> np.ndarray:
    return np.load(GOLDEN)


def test_expressions() -> None:
    assert pha.evaluate("1.5") == 1.5
    assert pha.evaluate("0.5*cos(60)") == pytest.approx(0.25)
    assert pha.evaluate("-sin(30) + sqrt(4)") == pytest.approx(1.5)
    assert pha.evaluate("2*(3-1)/4") == 1.0
    with pytest.raises(ValueError):
        pha.evaluate("__import__('os')")


def test_preprocessor(tmp_path) -> None:
    (tmp_path / "inc").write_text("#define WATER 1.0 // comment\n#define TWICE(a) (2*(a))\n")
    text = '/* block */ #include "inc"\nx = WATER + TWICE(WATER + 1)\n'
    out = pha.preprocess(text, base_dir=tmp_path)
    assert pha.evaluate(out.split("=")[1]) == pytest.approx(5.0)


SYNTH = """
#define MAT(d) formel=H2O dichte=d
Detector{ whatever=1 }
{ "a" [Sphere: x=1mm y=-2 z=0.5 r=3 ] MAT(1.25) }
{ "b" [Ellipsoid_free: dx=1 dy=2 dz=3 a_x (1,0,0) a_y(0,cos(30),sin(30)) x>-1 r(1,1,0)<2] MAT(0.5) }
{ [Ellipt_Cyl: y=3.6 dx=1.2 dy=4.0 l=0.5*cos(15) achse(0,-cos(30),sin(30)) a_y(0,sin(30),cos(30))] rho=1.8 }
{ [Cone_z: z=-1 l=2 r1=1 r2=0.5 z < 0.3] rho=-0.2 }
"""


def test_reader_features() -> None:
    s = pha.parse_text(SYNTH)
    assert list(s["type"]) == [13, 11, 12, 5]
    assert (s[0]["x"], s[0]["y"], s[0]["z"], s[0]["r"], s[0]["rho"]) == (1.0, -2.0, 0.5, 3.0, 1.25)
    e = s[1]
    ax, ay, az = (np.array(e[k].tolist()) for k in ("a_x", "a_y", "a_z"))
    np.testing.assert_allclose(az, np.cross(ax, ay), atol=1e-7)  # the missing axis, right-handed
    assert e["cas1"]["mode"] == 2 and tuple(e["cas1"]["axis"].tolist()) == (1.0, 0.0, 0.0)
    assert e["cas1"]["dotprod"] == -1.0
    assert e["cas2"]["mode"] == 1 and e["cas2"]["dotprod"] == 2.0
    np.testing.assert_allclose(e["cas2"]["axis"].tolist(), [2**-0.5, 2**-0.5, 0], rtol=1e-6)
    c = s[2]
    np.testing.assert_allclose(c["axis"].tolist(), [0, -math.cos(math.pi / 6), 0.5], rtol=1e-6)
    np.testing.assert_allclose(c["a_x"].tolist(), np.cross(c["a_y"].tolist(), c["axis"].tolist()), atol=1e-6)
    assert c["l"] == np.float32(0.5 * math.cos(math.radians(15)))
    assert s[3]["cas1"]["mode"] == 1 and s[3]["cas1"]["dotprod"] == np.float32(0.3)


def test_head_phantom_values_from_the_file() -> None:
    s = head()
    assert s.dtype == S.forbild_shape and len(s) == 479
    # { "5" [Ellipsoid: dx=9.6 dy=12 dz=12.5 ] DTMAT(1.800) }
    assert s[0]["type"] == 10 and (s[0]["dx"], s[0]["dy"], s[0]["dz"], s[0]["rho"]) == (
        np.float32(9.6), 12.0, 12.5, np.float32(1.8))
    # { "1" [Sphere: x=-4.7 y= 4.3 z= 0.872 r=2.0] DTMAT(1.060) }
    assert s[4]["type"] == 13 and (s[4]["x"], s[4]["z"], s[4]["r"]) == (np.float32(-4.7), np.float32(0.872), 2.0)
    # { "14"[Ellipt_Cyl: y=3.6 dx=1.2 dy=4.0 l=0.5*cos(15) achse(0,-cos(30),sin(30)) a_y(0,sin(30),cos(30))] }
    e = s[8]
    assert e["type"] == 12 and e["y"] == np.float32(3.6)
    np.testing.assert_allclose(e["axis"].tolist(), [0, -math.sqrt(3) / 2, 0.5], rtol=1e-6)
    np.testing.assert_allclose(e["a_y"].tolist(), [0, 0.5, math.sqrt(3) / 2], rtol=1e-6)
    # { "8" [Ellipsoid_free: x=-1.9 y=5.4 dx=1.206483*cos(15) ... a_z(sin(15),0,cos(15)) ...] }
    f = s[10]
    assert f["type"] == 11 and f["dx"] == np.float32(1.206483 * math.cos(math.radians(15)))
    np.testing.assert_allclose(f["a_z"].tolist(), [math.sin(math.radians(15)), 0, math.cos(math.radians(15))], rtol=1e-6)
    assert np.bincount(s["type"], minlength=17)[[4, 10, 11, 12]].tolist() == [2, 149, 3, 4]


def test_writer_round_trip(tmp_path) -> None:
    s = head()
    fb = FBVolume(s)
    fb.save(tmp_path / "h.pha")
    back = FBVolume.load(tmp_path / "h.pha").shapes
    assert back.tobytes() == s.tobytes()
    rq = phantoms.random_quadric_phantom(5, n_ellipsoids=8, n_cylinders=6)
    assert pha.parse_text(pha.format_shapes(rq)).tobytes() == rq.tobytes()


def _grid(n: tuple[int, int, int], lo: float, hi: float, seed: int):
    # non-round, slightly irregular coordinates: no sample sits exactly on a face
    rng = np.random.default_rng(seed)
    return [np.sort(rng.uniform(lo, hi, k)).astype(np.float32) for k in n]


@pytest.mark.skipif(not O.have_ref(), reason="reference oracle not built")
@pytest.mark.parametrize("which", ["head", "random"])
def test_sampling_oracle_matches_reference_body(which: str) -> None:
    if which == "head":
        s, xs, ys, zs = head(), *_grid((40, 44, 24), -10.5, 10.5, 1)
    else:
        s = phantoms.random_quadric_phantom(7, n_ellipsoids=20, n_cylinders=15, radius=60)
        xs, ys, zs = _grid((36, 36, 36), -70, 70, 2)
    ours = O.forbild_sample(s, xs, ys, zs)
    ref = O.ref_forbild_sample(s, xs, ys, zs)
    assert np.abs(ours).max() > 0
    bad = np.abs(ours - ref) > 1e-5
    assert bad.mean() <= 2e-3, bad.mean()


def test_transforms() -> None:
    s = phantoms.random_quadric_phantom(3, n_ellipsoids=4, n_cylinders=3)
    fb = FBVolume(s.copy())
    fb.flip("y")
    fb.flip(1)
    assert fb.shapes.tolist() == s.tolist()  # (copies leave struct padding undefined: compare fields)
    fb.translate("x", 2.5)
    assert np.allclose(fb.shapes["x"], s["x"] + 2.5)
    fb.scale_len(2.0)
    assert np.allclose(fb.shapes["dx"], 2 * s["dx"]) and np.allclose(fb.shapes["cas1"]["dotprod"], 2 * (s["cas1"]["dotprod"] + 2.5 * s["cas1"]["axis"]["x"]))
    fb.multiply_attenuation(0.5)
    assert np.allclose(fb.shapes["rho"], 0.5 * s["rho"])
    # a translated phantom samples like the original on a shifted grid
    xs, ys, zs = _grid((20, 20, 20), -80, 80, 3)
    t = FBVolume(s.copy())
    t.translate("z", 7.0)
    np.testing.assert_array_equal(O.forbild_sample(t.shapes, xs, ys, zs + np.float32(7.0)) != 0,
                                  O.forbild_sample(s, xs, ys, zs) != 0)
