"""Scene files: scene/SceneSerializer.java's JSON format, read and written.

The reference saves a SceneEditor as a flat JSON object with two arrays,
"materials" (name, albedo[3], metallic, emission[3], emissionStrength,
roughness, ior, transmission) and "objects" (name, type BOX|SPHERE, centre
px/py/pz, half extents or radius sx/sy/sz, Euler degrees rx/ry/rz, sphere
stacks/slices, materialIndex), and reads it back with a hand-written scanner
rather than a JSON parser.  `load`/`loads` follow that scanner, so a file the
reference reads gives the same scene here, quirks included:

* a key is found by the first occurrence of its quoted name anywhere in its
  object's text (SceneSerializer.java:161-215);
* a missing number reads as 0 -- not the Material/SceneObject default --
  and a missing or malformed albedo/emission (not exactly three entries)
  keeps the default; an ior below 0.01 becomes 1.5 (:84-95);
* type "SPHERE" in any case makes a sphere, anything else a box; stacks and
  slices apply only above 2 (else 24); a negative material index becomes 0
  (:100-120);
* numbers are rounded from their decimal text straight to float32, as
  Float.parseFloat does (correctly rounded, ties to even), not through a
  double.

`save`/`dumps` write the reference's layout (SceneSerializer.java:24-66),
each float as the shortest text that reads back to the same float32, so the
reference loads the files this module writes, and the other way round.
`SceneFile.to_scene_desc()` gives the scenes.SceneDesc the render path
builds (SceneEditor.buildScene: each object's Box or Sphere, rotated about
its centre when any angle is non-zero).
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np

from . import scenes


class SceneFormatError(ValueError):
    """Text the reference's scanner would also fail on (it throws)."""


# ---------------------------------------------------------------------------
# Float.parseFloat and the (int) cast
# ---------------------------------------------------------------------------
_F32_MAX = Fraction(int(np.finfo(np.float32).max))
_F32_HALF_ULP_TOP = Fraction(2) ** 103   # half an ulp above FLT_MAX (ulp 2^104)
_TRIM = "".join(chr(c) for c in range(33))   # String.trim(): chars <= ' '
_DEC = re.compile(r"([+-]?)((?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?)[fFdD]?")
_HEX = re.compile(r"([+-]?)0[xX]([0-9a-fA-F]*)(?:\.([0-9a-fA-F]*))?[pP]([+-]?[0-9]+)[fFdD]?")
_SPECIAL = re.compile(r"([+-]?)(NaN|Infinity)")


def _f32_nearest(q: Fraction) -> float:
    """The float32 nearest to the exact non-negative value q (ties to even),
    as a Python float."""
    if q == 0:
        return 0.0
    if q >= _F32_MAX + _F32_HALF_ULP_TOP:
        return float("inf")
    try:
        approx = np.float32(float(q))
    except OverflowError:
        return float("inf")
    f32 = np.float32
    cands = {float(approx), float(np.nextafter(approx, f32(0))), float(np.nextafter(approx, f32(np.inf)))}
    best, best_d, best_bits = None, None, None
    for c in sorted(cands):
        if c == float("inf"):
            continue
        d = abs(Fraction(c) - q)
        bits = int(np.float32(c).view(np.uint32))
        if best is None or d < best_d or (d == best_d and (bits & 1) == 0 and (best_bits & 1) == 1):
            best, best_d, best_bits = c, d, bits
    return best


def java_parse_float(text: str) -> float:
    """Float.parseFloat: the float32 value of `text` (returned as a Python
    float holding it); raises ValueError where Java throws
    NumberFormatException."""
    t = text.strip(_TRIM)
    m = _SPECIAL.fullmatch(t)
    if m:
        if m.group(2) == "NaN":
            return float("nan")
        return float("-inf") if m.group(1) == "-" else float("inf")
    m = _DEC.fullmatch(t)
    if m:
        q = Fraction(m.group(2))
    else:
        m = _HEX.fullmatch(t)
        if not m or (not m.group(2) and not m.group(3)):
            raise ValueError(f"not a float: {text!r}")
        digits = (m.group(2) or "") + (m.group(3) or "")
        q = Fraction(int(digits, 16)) * Fraction(2) ** (int(m.group(4)) - 4 * len(m.group(3) or ""))
    v = _f32_nearest(q)
    return -v if m.group(1) == "-" else v


def java_f2i(v: float) -> int:
    """The Java (int) cast of a float: NaN to 0, truncation toward zero,
    saturation at the int range."""
    if v != v:
        return 0
    if v >= 2147483647.0:
        return 2147483647
    if v <= -2147483648.0:
        return -2147483648
    return int(v)


def _short_f32(v: float) -> str:
    """Shortest decimal text that reads back as the same float32 (NaN and
    the infinities as Float.toString writes them)."""
    f = np.float32(v)
    if np.isnan(f):
        return "NaN"
    if np.isinf(f):
        return "Infinity" if f > 0 else "-Infinity"
    s = np.format_float_positional(f, unique=True, trim="0")
    return s if len(s) <= 16 else np.format_float_scientific(f, unique=True, trim="0")


# ---------------------------------------------------------------------------
# the reference's scanner (SceneSerializer.java:130-215), restated
# ---------------------------------------------------------------------------
def _array_body(text: str, key: str) -> str | None:
    token = f'"{key}"'
    ki = text.find(token)
    if ki < 0:
        return None
    start = text.find("[", ki + len(token))
    if start < 0:
        return None
    depth = 0
    for i in range(start, len(text)):
        c = text[i]
        if c == "[":
            depth += 1
        elif c == "]":
            depth -= 1
            if depth == 0:
                return text[start + 1:i]
    return None


def _split_objects(body: str) -> list[str]:
    out, depth, start = [], 0, -1
    for i, c in enumerate(body):
        if c == "{":
            if depth == 0:
                start = i
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0 and start >= 0:
                out.append(body[start:i + 1])
                start = -1
    return out


def _str_field(obj: str, key: str) -> str | None:
    token = f'"{key}"'
    ki = obj.find(token)
    if ki < 0:
        return None
    scan = ki + len(token)
    while scan < len(obj) and obj[scan] != '"':
        scan += 1
    if scan >= len(obj):
        return None
    close = scan + 1
    while close < len(obj):
        c = obj[close]
        if c == "\\":
            close += 2
            continue
        if c == '"':
            break
        close += 1
    if close > len(obj):
        raise SceneFormatError(f"unterminated string for {key!r}")
    return obj[scan + 1:close].replace('\\"', '"').replace("\\\\", "\\")


def _float_field(obj: str, key: str) -> float:
    token = f'"{key}"'
    ki = obj.find(token)
    if ki < 0:
        return 0.0
    i = ki + len(token)
    while i < len(obj) and obj[i] in ": \t\n\r":
        i += 1
    if i >= len(obj):
        return 0.0
    end = i
    while end < len(obj) and (obj[end].isdecimal() or obj[end] in ".-+eE"):
        end += 1
    if end <= i:
        return 0.0
    try:
        return java_parse_float(obj[i:end])
    except ValueError:
        return 0.0


def _float_arr(obj: str, key: str) -> list[float] | None:
    token = f'"{key}"'
    ki = obj.find(token)
    if ki < 0:
        return None
    start = obj.find("[", ki + len(token))
    end = obj.find("]", start if start > 0 else 0)
    if start < 0 or end < 0:
        return None
    if end < start + 1:
        raise SceneFormatError(f"malformed array for {key!r}")
    inner = obj[start + 1:end]
    parts = inner.split(",")
    if inner:   # String.split drops trailing empty parts (an empty string stays one part)
        while parts and parts[-1] == "":
            parts.pop()
    out = []
    for p in parts:
        try:
            out.append(java_parse_float(p))
        except ValueError:
            out.append(0.0)
    return out


# ---------------------------------------------------------------------------
# scene file <-> SceneDesc
# ---------------------------------------------------------------------------
@dataclass
class MaterialEntry:
    """A named material (scene/Material.java fields; defaults as there)."""
    name: str = "Material"
    material: scenes.MaterialDesc = field(default_factory=scenes.MaterialDesc)


@dataclass
class ObjectEntry:
    """scene/SceneObject.java: centre, half extents (a sphere's radius in
    sx), Euler degrees (XYZ), sphere stacks/slices, material index."""
    name: str = "Object"
    type: str = "BOX"          # "BOX" or "SPHERE"
    px: float = 0.0
    py: float = 0.0
    pz: float = 0.0
    sx: float = 1.0
    sy: float = 1.0
    sz: float = 1.0
    rx: float = 0.0
    ry: float = 0.0
    rz: float = 0.0
    stacks: int = 24
    slices: int = 24
    material_index: int = 0

    def primitive(self):
        """SceneObject.toPrimitive (SceneObject.java:82-90)."""
        rot = (self.rx, self.ry, self.rz)
        if self.type == "SPHERE":
            return scenes.Sphere((self.px, self.py, self.pz), self.sx, self.material_index, self.stacks,
                                 self.slices, rot)
        return scenes.Box((self.px, self.py, self.pz), (self.sx, self.sy, self.sz), self.material_index, rot)


@dataclass
class SceneFile:
    materials: list = field(default_factory=list)   # MaterialEntry
    objects: list = field(default_factory=list)     # ObjectEntry

    def to_scene_desc(self) -> scenes.SceneDesc:
        """SceneEditor.buildScene (SceneEditor.java:101-107): the materials in
        order and one primitive per object."""
        return scenes.SceneDesc([m.material for m in self.materials], [o.primitive() for o in self.objects])


def from_scene_desc(desc: scenes.SceneDesc, names=None) -> SceneFile:
    """The scene file of a SceneDesc made of boxes and spheres (the only
    primitives the format has); raises SceneFormatError otherwise."""
    out = SceneFile()
    for i, m in enumerate(desc.materials):
        out.materials.append(MaterialEntry(f"Material {i}", m))
    for i, o in enumerate(desc.objects):
        name = names[i] if names else f"Object {i}"
        if isinstance(o, scenes.Box):
            e = ObjectEntry(name, "BOX", *o.center, *o.half)
        elif isinstance(o, scenes.Sphere):
            e = ObjectEntry(name, "SPHERE", *o.center, o.radius, o.radius, o.radius)
            e.stacks, e.slices = o.stacks, o.slices
        else:
            raise SceneFormatError(f"{type(o).__name__} has no scene-file form (boxes and spheres only)")
        e.rx, e.ry, e.rz = o.rot
        e.material_index = int(o.mat)
        out.objects.append(e)
    return out


def loads(text: str) -> SceneFile:
    """SceneSerializer.load (SceneSerializer.java:72-124) on a string."""
    out = SceneFile()
    mats = _array_body(text, "materials")
    if mats is not None:
        for obj in _split_objects(mats):
            m = scenes.MaterialDesc()
            name = _str_field(obj, "name")
            alb, em = _float_arr(obj, "albedo"), _float_arr(obj, "emission")
            if alb is not None and len(alb) == 3:
                m.albedo = tuple(alb)
            if em is not None and len(em) == 3:
                m.emission = tuple(em)
            m.metallic = _float_field(obj, "metallic")
            m.emission_strength = _float_field(obj, "emissionStrength")
            m.roughness = _float_field(obj, "roughness")
            m.ior = _float_field(obj, "ior")
            if m.ior < np.float32(0.01):
                m.ior = 1.5
            m.transmission = _float_field(obj, "transmission")
            out.materials.append(MaterialEntry(name if name is not None else "Material", m))
    objs = _array_body(text, "objects")
    if objs is not None:
        for obj in _split_objects(objs):
            name, kind = _str_field(obj, "name"), _str_field(obj, "type")
            o = ObjectEntry(name if name is not None else "Object",
                            "SPHERE" if kind is not None and kind.upper() == "SPHERE" else "BOX",
                            *(_float_field(obj, k) for k in ("px", "py", "pz", "sx", "sy", "sz")))
            o.rx, o.ry, o.rz = (_float_field(obj, k) for k in ("rx", "ry", "rz"))
            stacks = java_f2i(_float_field(obj, "stacks"))
            slices = java_f2i(_float_field(obj, "slices"))
            o.material_index = max(0, java_f2i(_float_field(obj, "materialIndex")))
            if stacks > 2:
                o.stacks = stacks
            if slices > 2:
                o.slices = slices
            out.objects.append(o)
    return out


def load(path: str) -> SceneFile:
    with open(path, "r", encoding="utf-8") as f:
        return loads(f.read())


def _jstr(s: str) -> str:
    return '"' + s.replace("\\", "\\\\").replace('"', '\\"') + '"'


def dumps(sf: SceneFile) -> str:
    """SceneSerializer.save's layout (SceneSerializer.java:24-66)."""
    f = _short_f32
    lines = ["{", '  "materials": [']
    for i, e in enumerate(sf.materials):
        m = e.material
        lines += ["    {",
                  f'      "name": {_jstr(e.name)},',
                  f'      "albedo": [{", ".join(f(v) for v in m.albedo)}],',
                  f'      "metallic": {f(m.metallic)},',
                  f'      "emission": [{", ".join(f(v) for v in m.emission)}],',
                  f'      "emissionStrength": {f(m.emission_strength)},',
                  f'      "roughness": {f(m.roughness)},',
                  f'      "ior": {f(m.ior)},',
                  f'      "transmission": {f(m.transmission)}',
                  "    }" + ("," if i < len(sf.materials) - 1 else "")]
    lines += ["  ],", '  "objects": [']
    for i, o in enumerate(sf.objects):
        lines += ["    {",
                  f'      "name": {_jstr(o.name)},',
                  f'      "type": {_jstr(o.type)},',
                  f'      "px": {f(o.px)}, "py": {f(o.py)}, "pz": {f(o.pz)},',
                  f'      "sx": {f(o.sx)}, "sy": {f(o.sy)}, "sz": {f(o.sz)},',
                  f'      "rx": {f(o.rx)}, "ry": {f(o.ry)}, "rz": {f(o.rz)},',
                  f'      "stacks": {int(o.stacks)}, "slices": {int(o.slices)},',
                  f'      "materialIndex": {int(o.material_index)}',
                  "    }" + ("," if i < len(sf.objects) - 1 else "")]
    lines += ["  ]", "}"]
    return "\n".join(lines) + "\n"


def save(sf: SceneFile, path: str) -> None:
    with open(path, "w", encoding="utf-8") as f:
        f.write(dumps(sf))


def _main(argv=None) -> int:
    """Reads a scene file and prints what the render path gets from it."""
    import argparse
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("path")
    args = ap.parse_args(argv)
    sf = load(args.path)
    from . import api
    sc = api.build_scene(sf.to_scene_desc())
    print(f"{len(sf.materials)} materials, {len(sf.objects)} objects -> {len(sc['tris'])} triangles, "
          f"{len(sc['nodes'])} BVH nodes, {sc['light_count']} lights")
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
