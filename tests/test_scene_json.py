"""Scene files in the reference's format (scene/SceneSerializer.java): the
scanner's rules and quirks, Float.parseFloat rounding, save/load round trips,
and the triangles and BVH built from a loaded file against those built from
the same scene described directly."""
from fractions import Fraction

import numpy as np
import pytest

from retrocam_b200 import scene_json as sj
from retrocam_b200 import scenes


def _dec(q: Fraction, digits=60) -> str:
    """Exact decimal text of a dyadic rational."""
    n, d = q.numerator, q.denominator
    ip = n // d
    rem = n - ip * d
    out = []
    while rem and len(out) < digits:
        rem *= 10
        out.append(str(rem // d))
        rem %= d
    assert rem == 0
    return f"{ip}." + ("".join(out) or "0")


def test_parse_float_rounds_the_decimal_text_once():
    f32 = lambda x: float(np.float32(x))   # noqa: E731
    one = Fraction(1)
    ulp = Fraction(1, 2 ** 23)
    # halfway between 1 and 1 + ulp: ties to even
    assert sj.java_parse_float(_dec(one + ulp / 2)) == 1.0
    # halfway between 1 + ulp and 1 + 2 ulp: ties to even (the upper one)
    assert sj.java_parse_float(_dec(one + 3 * ulp / 2)) == f32(1 + 2 * 2 ** -23)
    # a hair above halfway: rounds up, where double-then-float rounding lands
    # on the tie and goes down
    above = one + ulp / 2 + Fraction(1, 2 ** 60)
    assert float(np.float32(float(_dec(above)))) == 1.0
    assert sj.java_parse_float(_dec(above)) == f32(1 + 2 ** -23)
    rng = np.random.default_rng(1)
    for v in np.exp(rng.normal(0, 8, 2000)).astype(np.float32):
        for text in (repr(float(v)), f"{float(v):.9g}", f"{float(v):.3e}"):
            assert sj.java_parse_float(text) == f32(float(text))
    assert sj.java_parse_float("-0") == 0.0 and np.signbit(sj.java_parse_float("-0"))
    assert sj.java_parse_float("1e-50") == 0.0 and sj.java_parse_float("1e39") == float("inf")
    assert sj.java_parse_float(" 2.5f") == 2.5 and sj.java_parse_float("2.5D") == 2.5
    assert sj.java_parse_float("0x1.8p3") == 12.0 and sj.java_parse_float("-Infinity") == float("-inf")
    assert np.isnan(sj.java_parse_float("NaN"))
    for bad in ("", ".", "e5", "1e", "--1", "1.5.3", "0x1.8", "NaNf", "１"):
        with pytest.raises(ValueError):
            sj.java_parse_float(bad)
    assert sj.java_f2i(2.9) == 2 and sj.java_f2i(-2.9) == -2 and sj.java_f2i(1e30) == 2 ** 31 - 1


TEXT = r'''{
  "materials": [
    {"name": "White \"matte\"", "albedo": [0.73, 0.73, 0.73], "roughness": 0.5, "ior": 1.5},
    {"name": "Lamp", "albedo": [1, 0.95], "emission": [1.0, 0.95, 0.85], "emissionStrength": 15},
    {"albedo": [0.9, 0.9, 0.9], "metallic": 1, "roughness": 0.2, "ior": 0.001}
  ],
  "objects": [
    {"name": "Floor", "type": "BOX", "px": 0, "py": 0, "pz": 0, "sx": 5, "sy": 0.05, "sz": 5,
     "materialIndex": 0},
    {"name": "Ball", "type": "sphere", "px": 0, "py": 1.2, "pz": 1.5, "sx": 1.2,
     "stacks": 2, "slices": 40, "materialIndex": -3},
    {"name": "px", "type": "BOX", "px": 2.0, "py": 1, "pz": 1, "sx": 1, "sy": 1, "sz": 1,
     "ry": 30, "materialIndex": 2.7}
  ]
}'''


def test_scanner_rules_and_quirks():
    sf = sj.loads(TEXT)
    m0, m1, m2 = (e.material for e in sf.materials)
    assert sf.materials[0].name == 'White "matte"' and sf.materials[2].name == "Material"
    assert m0.albedo == (np.float32(0.73),) * 3 and m0.metallic == 0.0 and m0.transmission == 0.0
    assert m1.albedo == (0.8, 0.8, 0.8)                  # two entries: the default stays
    assert m1.emission == (1.0, float(np.float32(0.95)), float(np.float32(0.85)))
    assert m1.emission_strength == 15.0
    assert m1.roughness == 0.0                           # missing reads 0, not Material's 0.5
    assert m1.ior == 1.5 and m2.ior == 1.5               # missing or < 0.01
    assert m2.metallic == 1.0
    floor, ball, odd = sf.objects
    assert (floor.type, floor.sx, floor.sy) == ("BOX", 5.0, float(np.float32(0.05)))
    assert (ball.type, ball.stacks, ball.slices, ball.material_index) == ("SPHERE", 24, 40, 0)
    # the key "px" first occurs as the object's name, where no number follows
    assert odd.px == 0.0 and odd.py == 1.0 and odd.ry == 30.0 and odd.material_index == 2
    desc = sf.to_scene_desc()
    assert isinstance(desc.objects[1], scenes.Sphere) and desc.objects[1].radius == float(np.float32(1.2))
    assert desc.objects[2].rot == (0.0, 30.0, 0.0)
    assert sj.loads('{"objects": []}').materials == [] and sj.loads("{}").objects == []


def _mixed_scene():
    mats = [scenes.diffuse(0.73, 0.73, 0.73), scenes.emissive(1.0, 0.95, 0.85, 15.0),
            scenes.metal(0.95, 0.85, 0.55, 0.1), scenes.glass(1.5)]
    objs = [scenes.Box((0.0, 0.0, 0.0), (1.0, 0.05, 1.0), 0),
            scenes.Box((0.0, 2.0, 0.0), (0.25, 0.02, 0.25), 1),
            scenes.Box((-0.4, 0.6, -0.3), (0.2, 0.6, 0.2), 0, (0.0, 17.5, 0.0)),
            scenes.Box((0.45, 0.3, 0.2), (0.3, 0.3, 0.3), 2, (5.0, -33.0, 12.0)),
            scenes.Sphere((0.1, 0.35, 0.5), 0.3, 3, 20, 36),
            scenes.Sphere((-0.5, 0.25, 0.55), 0.22, 2, 12, 16, (0.0, 0.0, 45.0))]
    return scenes.SceneDesc(mats, objs)


def test_round_trip_through_text():
    desc = _mixed_scene()
    sf = sj.from_scene_desc(desc, names=[f"o{i}" for i in range(6)])
    text = sj.dumps(sf)
    back = sj.loads(text)
    assert sj.dumps(back) == text
    assert [o.name for o in back.objects] == [f"o{i}" for i in range(6)]
    with pytest.raises(sj.SceneFormatError):
        sj.from_scene_desc(scenes.export_frame_scene())   # its walls are triangle lists


def test_loaded_scene_builds_the_same_triangles_and_tree(product, tmp_path):
    """File -> SceneDesc -> tessellation, BVH and lights through the library's
    host code gives the same bits as the SceneDesc written directly."""
    desc = _mixed_scene()
    path = str(tmp_path / "scene.json")
    sj.save(sj.from_scene_desc(desc), path)
    a = product.build_scene(desc)
    b = product.build_scene(sj.load(path).to_scene_desc())
    for k in ("tris", "nodes", "mats", "lights"):
        assert a[k].tobytes() == b[k].tobytes(), k
    assert (a["light_count"], a["total_power"]) == (b["light_count"], b["total_power"])
    assert len(a["tris"]) == 4 * 12 + 20 * 36 * 2 - 2 * 36 + 12 * 16 * 2 - 2 * 16   # poles skipped
