"""Workload scenes, cameras and settings of the benchmark configurations.

A scene is described the way the reference's authoring API builds one
(scene/Scene.java: materials, then primitives tessellated in insertion
order; scene/SceneObject.java:80-88: Box/Sphere wrapped in a
TransformedPrimitive when rotated; Primitive.toTriangles as the extension
point for triangle lists).  `build_scene` turns a description into the four
SSBO arrays with any backend that offers tess_box / tess_sphere /
flat_triangles / build_bvh / build_lights: the product's C ABI
(retrocam_b200.api) or the oracle.

Configurations (sizes from the project brief; choices the brief leaves open
are fixed here and recorded in the design notes):
  cornell_small  256x256, 16 spp, 35 mm f/16, focus 2.5, 36 triangles
  export_frame   854x480, 128 spp, + glass and GGX spheres (32x64 UV,
                 3,968 triangles each), 28 mm f/2.8, focus 1.8, 6 blades,
                 LCA (-0.5%, 0, +0.5%) of focus, SPPM 2M photons x 16,
                 2^22 hash, r0 0.02, alpha 0.7, a-trous 5 passes
  bvh_stress     1,000,000 seeded random triangles + box + 4 lights, 32 spp
  keyframes      64 Catmull-Rom keyframed frames of export_frame's scene
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# ---- materials (scene/Material.java factories) ----


@dataclass
class MaterialDesc:
    albedo: tuple = (0.8, 0.8, 0.8)
    metallic: float = 0.0
    emission: tuple = (0.0, 0.0, 0.0)
    emission_strength: float = 0.0
    roughness: float = 0.5
    ior: float = 1.5
    transmission: float = 0.0


def diffuse(r, g, b):
    return MaterialDesc(albedo=(r, g, b))


def emissive(r, g, b, strength):
    return MaterialDesc(albedo=(r, g, b), emission=(r, g, b), emission_strength=strength)


def metal(r, g, b, roughness):
    return MaterialDesc(albedo=(r, g, b), metallic=1.0, roughness=roughness)


def glass(ior):
    return MaterialDesc(albedo=(1.0, 1.0, 1.0), transmission=1.0, roughness=0.0, ior=ior)


@dataclass
class Box:
    center: tuple
    half: tuple
    mat: int
    rot: tuple = (0.0, 0.0, 0.0)


@dataclass
class Sphere:
    center: tuple
    radius: float
    mat: int
    stacks: int = 24
    slices: int = 24
    rot: tuple = (0.0, 0.0, 0.0)


@dataclass
class TriangleList:
    positions: np.ndarray           # (n, 9) float32: v0, v1, v2
    mat: int | np.ndarray           # one index or one per triangle


@dataclass
class SceneDesc:
    materials: list = field(default_factory=list)
    objects: list = field(default_factory=list)


# ---- camera / lens (camera/OrbitCamera.java, ThinLensCamera.java,
#      core/RenderSettings.java defaults for fields a config leaves open) ----


@dataclass
class LensDesc:
    focal_length_mm: float = 35.0
    f_stop: float = 2.0
    focus_dist_m: float = 2.0
    blades: int = 5
    sa_strength: float = 0.04
    lca_delta: tuple = (0.0, 0.0, 0.0)


@dataclass
class OrbitDesc:
    theta: float
    phi: float
    radius: float
    target: tuple


@dataclass
class SppmDesc:
    photons: int = 2_000_000
    hash_size: int = 1 << 22
    r0: float = 0.02
    alpha: float = 0.7
    iterations: int = 16


@dataclass
class AtrousDesc:
    enabled: int = 1
    iterations: int = 5
    sigma_color: float = 1.0
    sigma_normal: float = 128.0
    sigma_depth: float = 1.0
    max_spp: int = 0
    exposure: float = 1.0


@dataclass
class Workload:
    name: str
    width: int
    height: int
    spp: int
    scene: SceneDesc
    orbit: OrbitDesc
    lens: LensDesc
    sppm: SppmDesc | None = None
    atrous: AtrousDesc | None = None
    nee_enabled: int = 1
    nee_firefly_clamp: float = 1.0


# ---- the Cornell box in [0,1]^3 ----

def _quad(a, b, c, d):
    """Two triangles (a,b,c), (a,c,d), the Box.addQuad split."""
    return [a + b + c, a + c + d]


def _quad_y(y, x0, x1, z0, z1, down):
    a, b, c, d = (x0, y, z0), (x1, y, z0), (x1, y, z1), (x0, y, z1)
    return _quad(a, b, c, d) if down else _quad(a, d, c, b)


def cornell_materials():
    # The brief's light (17, 12, 4) is emissive(1, 12/17, 4/17, 17): the
    # reference gives emitters their emission colour as albedo
    # (Material.java:32-38), which must stay <= 1.
    return [diffuse(0.73, 0.73, 0.73),            # 0 white
            diffuse(0.63, 0.065, 0.05),           # 1 red
            diffuse(0.14, 0.45, 0.09),            # 2 green
            emissive(1.0, 12.0 / 17.0, 4.0 / 17.0, 17.0)]  # 3 light


def cornell_walls_and_light(light_half=0.125, light_center=(0.5, 0.5)):
    """Five walls (open at z=0, facing the camera at z<0) as 10 triangles
    with inward normals, and a ceiling quad light at y=0.999 facing down.
    The camera looks along +z, so its right vector is -x: the red wall
    (image left) is the x=1 plane and the green wall the x=0 plane."""
    white = []
    white += _quad((0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 0, 0))        # floor, normal +y
    white += _quad((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1))        # ceiling, normal -y
    white += _quad((0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1))        # back, normal -z
    red = _quad((1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0))           # x=1, normal -x
    green = _quad((0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1))         # x=0, normal +x
    cx, cz = light_center
    light = _quad_y(0.999, cx - light_half, cx + light_half, cz - light_half, cz + light_half, down=True)
    f = lambda t: np.asarray(t, np.float32).reshape(-1, 9)  # noqa: E731
    return [TriangleList(f(white), 0), TriangleList(f(red), 1), TriangleList(f(green), 2),
            TriangleList(f(light), 3)]


TALL_BOX = Box(center=(0.66, 0.3, 0.62), half=(0.15, 0.3, 0.15), mat=0, rot=(0.0, 15.0, 0.0))
SHORT_BOX = Box(center=(0.34, 0.15, 0.35), half=(0.15, 0.15, 0.15), mat=0, rot=(0.0, -18.0, 0.0))

# Camera: eye (0.5, 0.5, -1.4) looking at the box centre, expressed in the
# reference's orbit parameters (theta = -pi/2, phi = pi/2, radius 1.9).
CORNELL_ORBIT = OrbitDesc(theta=-math.pi / 2, phi=math.pi / 2, radius=1.9, target=(0.5, 0.5, 0.5))


def cornell_small() -> Workload:
    sc = SceneDesc(cornell_materials(), cornell_walls_and_light() + [TALL_BOX, SHORT_BOX])
    return Workload("cornell_small", 256, 256, 16, sc, CORNELL_ORBIT,
                    LensDesc(focal_length_mm=35.0, f_stop=16.0, focus_dist_m=2.5))


def cornell_variant(seed: int, width: int = 854, height: int = 480, spp: int = 16) -> Workload:
    """A randomised Cornell box for the learned denoiser's data: wall
    colours, box poses, light size and lens drawn from a seeded generator.
    Same geometry as the small box (walls, ceiling light, two boxes)."""
    rng = np.random.default_rng(seed)
    u = lambda lo, hi, n=None: rng.uniform(lo, hi, n)  # noqa: E731
    grey = float(u(0.45, 0.85))
    half = float(u(0.06, 0.2))
    # the emitted power of the reference light (17 x 0.25^2) for any size
    mats = [diffuse(grey, grey, grey), diffuse(*u(0.05, 0.85, 3)), diffuse(*u(0.05, 0.85, 3)),
            emissive(1.0, 12.0 / 17.0, 4.0 / 17.0, 17.0 * (0.125 / half) ** 2)]
    th, ts = u(0.18, 0.34), u(0.12, 0.2)
    tall = Box(center=(float(u(0.5, 0.8)), float(th), float(u(0.45, 0.8))), half=(0.15, float(th), 0.15), mat=0,
               rot=(0.0, float(u(-45.0, 45.0)), 0.0))
    short = Box(center=(float(u(0.2, 0.45)), float(ts), float(u(0.2, 0.45))), half=(float(ts), float(ts), float(ts)),
                mat=0, rot=(0.0, float(u(-45.0, 45.0)), 0.0))
    sc = SceneDesc(mats, cornell_walls_and_light(light_half=half) + [tall, short])
    lens = LensDesc(focal_length_mm=float(u(24.0, 50.0)), f_stop=float(u(2.8, 16.0)),
                    focus_dist_m=float(u(1.5, 2.5)))
    return Workload(f"cornell_variant_{seed}", width, height, spp, sc, CORNELL_ORBIT, lens)


def export_frame_scene() -> SceneDesc:
    mats = cornell_materials() + [glass(1.5), metal(0.95, 0.85, 0.55, 0.2)]
    objs = cornell_walls_and_light() + [TALL_BOX, SHORT_BOX,
                                        Sphere((0.34, 0.45, 0.35), 0.15, 4, stacks=32, slices=64),
                                        Sphere((0.72, 0.15, 0.22), 0.15, 5, stacks=32, slices=64)]
    return SceneDesc(mats, objs)


def export_frame() -> Workload:
    focus = 1.8
    lca = (-0.005 * focus, 0.0, 0.005 * focus)
    return Workload("export_frame", 854, 480, 128, export_frame_scene(), CORNELL_ORBIT,
                    LensDesc(focal_length_mm=28.0, f_stop=2.8, focus_dist_m=focus, blades=6, lca_delta=lca),
                    sppm=SppmDesc(), atrous=AtrousDesc())


@dataclass
class KeyTrack:
    """A keyframe track (keyframe/KeyframeTrack.java): times in [0, 1],
    values, and per-key interpolation (0 STEP, 1 LINEAR, 2 BEZIER)."""
    times: tuple
    values: tuple
    interp: tuple = (2, 2, 2, 2)


# The keyframed orbit of the batched export: azimuth sweep of 90 degrees
# centred on the front view, lens zoom, aperture and focus pulls.
KEYFRAME_TRACKS = {
    "azimuth_deg": KeyTrack((0.0, 1 / 3, 2 / 3, 1.0), (0.0, 30.0, 60.0, 90.0)),
    "focal_mm": KeyTrack((0.0, 1 / 3, 2 / 3, 1.0), (20.0, 35.0, 50.0, 80.0)),
    "f_stop": KeyTrack((0.0, 1 / 3, 2 / 3, 1.0), (1.8, 4.0, 8.0, 16.0)),
    "focus_m": KeyTrack((0.0, 1 / 3, 2 / 3, 1.0), (1.0, 2.5, 1.5, 4.0)),
}


def keyframe_batch(backend, n_frames: int = 64, seed: int = 1):
    """Frames of the batched keyframe export: (camera dict, spp, SPPM
    iterations) per frame.  Cameras from the Catmull-Rom tracks above at
    t = f / (n - 1) (orbit theta = front view - 45 deg + azimuth); spp drawn
    from U{8..128} and SPPM iterations from U{4..16} (capped at spp) with an
    MT19937 generator seeded `seed`; LCA offsets +-0.5% of the focus
    distance, 6 blades, as in the export frame."""
    rng = np.random.Generator(np.random.MT19937(seed))
    spp = rng.integers(8, 129, n_frames)
    iters = rng.integers(4, 17, n_frames)
    frames = []
    for f in range(n_frames):
        t = f / max(1, n_frames - 1)
        ev = {k: backend.keyframe(tr.times, tr.values, tr.interp, t) for k, tr in KEYFRAME_TRACKS.items()}
        orbit = OrbitDesc(theta=CORNELL_ORBIT.theta + math.radians(ev["azimuth_deg"] - 45.0), phi=CORNELL_ORBIT.phi,
                          radius=CORNELL_ORBIT.radius, target=CORNELL_ORBIT.target)
        focus = ev["focus_m"]
        lens = LensDesc(focal_length_mm=ev["focal_mm"], f_stop=ev["f_stop"], focus_dist_m=focus, blades=6,
                        lca_delta=(-0.005 * focus, 0.0, 0.005 * focus))
        frames.append((camera(orbit, lens, backend), int(spp[f]), int(min(iters[f], spp[f]))))
    return frames


def bvh_stress(n_tris: int = 1_000_000, seed: int = 1) -> Workload:
    """Seeded random triangles (numpy PCG64): centres U[0,1]^3, two edge
    lengths log-uniform in [1e-3, 5e-2] along random unit directions;
    per-triangle materials 40% Lambertian U(0.2,0.9), 30% GGX metal with
    roughness U(0,0.5), 30% glass with IOR U(1.3,1.7); four ceiling quad
    lights with side U(0.05, 0.2)."""
    rng = np.random.default_rng(seed)
    c = rng.random((n_tris, 3))
    lens = np.exp(rng.uniform(math.log(1e-3), math.log(5e-2), (n_tris, 2)))
    d = rng.normal(size=(n_tris, 2, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    e1 = d[:, 0] * lens[:, :1]
    e2 = d[:, 1] * lens[:, 1:]
    v0 = c - (e1 + e2) / 3.0
    pos = np.concatenate([v0, v0 + e1, v0 + e2], axis=1).astype(np.float32)
    kind = rng.random(n_tris)
    u = rng.random(n_tris).astype(np.float32)
    base = cornell_materials()
    nb = len(base)
    n = nb + n_tris
    table = {"albedo": np.zeros((n, 3), np.float32), "metallic": np.zeros(n, np.float32),
             "emission": np.zeros((n, 3), np.float32), "emission_strength": np.zeros(n, np.float32),
             "roughness": np.full(n, 0.5, np.float32), "ior": np.full(n, 1.5, np.float32),
             "transmission": np.zeros(n, np.float32)}
    for i, m in enumerate(base):
        for k in table:
            table[k][i] = getattr(m, k)
    lam, met, gls = kind < 0.4, (kind >= 0.4) & (kind < 0.7), kind >= 0.7
    sl = slice(nb, n)
    a = (0.2 + 0.7 * u).astype(np.float32)
    table["albedo"][sl][lam] = a[lam, None]
    table["albedo"][sl][met] = (0.95, 0.85, 0.55)
    table["metallic"][sl][met] = 1.0
    table["roughness"][sl][met] = 0.5 * u[met]
    table["albedo"][sl][gls] = 1.0
    table["transmission"][sl][gls] = 1.0
    table["roughness"][sl][gls] = 0.0
    table["ior"][sl][gls] = 1.3 + 0.4 * u[gls]
    mats = table
    mat_idx = np.arange(nb, n, dtype=np.int32)
    objs = cornell_walls_and_light()[:3]
    sides = rng.uniform(0.05, 0.2, 4)
    centers = [(0.3, 0.3), (0.7, 0.3), (0.3, 0.7), (0.7, 0.7)]
    light_pos = []
    for s, (lx, lz) in zip(sides, centers):
        light_pos += _quad_y(0.999, lx - s / 2, lx + s / 2, lz - s / 2, lz + s / 2, down=True)
    objs.append(TriangleList(np.asarray(light_pos, np.float32).reshape(-1, 9), 3))
    objs.append(TriangleList(pos, mat_idx))
    return Workload("bvh_stress", 854, 480, 32, SceneDesc(mats, objs), CORNELL_ORBIT, LensDesc())


WORKLOADS = {"cornell_small": cornell_small, "export_frame": export_frame, "bvh_stress": bvh_stress}


# ---- building ----

def material_array(mats, dtype):
    if isinstance(mats, dict):
        a = np.zeros(len(mats["metallic"]), dtype)
        for k, v in mats.items():
            a[k] = v
        a["albedo_tex"] = -1
        return a
    a = np.zeros(len(mats), dtype)
    for i, m in enumerate(mats):
        a[i]["albedo"] = m.albedo
        a[i]["metallic"] = m.metallic
        a[i]["emission"] = m.emission
        a[i]["emission_strength"] = m.emission_strength
        a[i]["roughness"] = m.roughness
        a[i]["ior"] = m.ior
        a[i]["transmission"] = m.transmission
        a[i]["albedo_tex"] = -1
    return a


def tessellate(desc: SceneDesc, backend) -> np.ndarray:
    """Scene.build(): primitives' triangles concatenated in insertion order."""
    parts = []
    for o in desc.objects:
        if isinstance(o, Box):
            parts.append(backend.tess_box(o.center, o.half, o.mat, o.rot))
        elif isinstance(o, Sphere):
            parts.append(backend.tess_sphere(o.center, o.radius, o.mat, o.stacks, o.slices, o.rot))
        elif isinstance(o, TriangleList):
            t = backend.flat_triangles(o.positions, 0 if not np.isscalar(o.mat) else int(o.mat))
            if not np.isscalar(o.mat):
                t["mat_index"] = o.mat
            parts.append(t)
        else:
            raise TypeError(type(o))
    return np.concatenate(parts)


def build_scene(desc: SceneDesc, backend, mat_dtype) -> dict:
    """SceneUploader.upload() up to the device copy: tessellate, build the
    BVH (reordering triangles), build the light list."""
    tris = tessellate(desc, backend)
    mats = material_array(desc.materials, mat_dtype)
    tris, nodes = backend.build_bvh(tris)
    lights, total = backend.build_lights(tris, mats)
    light_count = len(lights)
    if light_count == 0:
        lights = np.zeros(1, lights.dtype)
    return {"tris": tris, "nodes": nodes, "mats": mats, "lights": lights,
            "light_count": light_count, "total_power": total}


def camera(orbit: OrbitDesc, lens: LensDesc, backend) -> dict:
    """ThinLensCamera.uploadTo: orbit basis + lens uniforms; focal_dist is
    the focus distance (no auto-focus lag)."""
    b = backend.orbit_basis(orbit.theta, orbit.phi, orbit.radius, orbit.target)
    lr, th = backend.thin_lens(lens.focal_length_mm, lens.f_stop)
    return {"cam_pos": b[0:3], "cam_forward": b[3:6], "cam_right": b[6:9], "cam_up": b[9:12],
            "focal_dist": lens.focus_dist_m, "lens_radius": lr, "fov_tan_half": th,
            "aperture_blades": lens.blades, "sa_strength": lens.sa_strength, "lca_delta": lens.lca_delta}
