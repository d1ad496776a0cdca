"""Scene model of the offline path tracer and the procedural workloads.

Mirrors the reference's scene layer (include/minirender/scene/scene.hpp): a ``SceneDocument``
with materials, meshes, objects (mesh + material + ``Transform``), directional lights,
a constant environment and homogeneous medium regions. ``SceneDocument.snapshot()`` resolves it
into the flat C descriptor (``mr_scene_desc``) that both the CUDA library and the CPU oracle read,
exactly as ``make_snapshot`` (src/scene/scene.cpp:364-405) resolves a document into a
``SceneSnapshot``.

The procedural generators at the bottom build the benchmark scenes (Cornell box, displaced
icosphere fields, uneven job tables). All inputs are synthetic and seeded; nothing is loaded.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi

F32 = np.float32


# ---- transforms ------------------------------------------------------------------------------

def _rotate(m: np.ndarray, angle: np.float32, axis) -> np.ndarray:
    """glm::rotate(m, angle, axis) in float (right-handed, column-major m[c][r])."""
    a = F32(angle)
    c = F32(math.cos(float(a)))
    s = F32(math.sin(float(a)))
    axis = np.asarray(axis, dtype=F32)
    axis = axis * F32(1.0 / math.sqrt(float(np.dot(axis, axis))))
    temp = (F32(1) - c) * axis
    r = np.zeros((3, 3), dtype=F32)
    r[0, 0] = c + temp[0] * axis[0]
    r[0, 1] = temp[0] * axis[1] + s * axis[2]
    r[0, 2] = temp[0] * axis[2] - s * axis[1]
    r[1, 0] = temp[1] * axis[0] - s * axis[2]
    r[1, 1] = c + temp[1] * axis[1]
    r[1, 2] = temp[1] * axis[2] + s * axis[0]
    r[2, 0] = temp[2] * axis[0] + s * axis[1]
    r[2, 1] = temp[2] * axis[1] - s * axis[0]
    r[2, 2] = c + temp[2] * axis[2]
    out = m.copy()
    for col in range(3):
        out[col] = (m[0] * r[col, 0] + m[1] * r[col, 1]) + m[2] * r[col, 2]
    out[3] = m[3]
    return out


@dataclass
class Transform:
    """T * Rz * Ry * Rx * S (include/minirender/scene/scene.hpp:70-81)."""

    translation: tuple = (0.0, 0.0, 0.0)
    rotation_degrees: tuple = (0.0, 0.0, 0.0)
    scale: tuple = (1.0, 1.0, 1.0)

    def validate(self):  # src/scene/scene.cpp:119-124
        values = np.asarray([*self.translation, *self.rotation_degrees, *self.scale], dtype=F32)
        if not np.all(np.isfinite(values)):
            raise ValueError("Transform must be finite")
        if not all(abs(F32(s)) > F32(1e-6) for s in self.scale):
            raise ValueError("Transform scale must be invertible")

    def matrix(self) -> np.ndarray:
        """Column-major 4x4 float32 (m[c][r]), src/scene/scene.cpp:126-133."""
        self.validate()
        m = np.eye(4, dtype=F32)
        t = np.asarray(self.translation, dtype=F32)
        m[3] = ((m[0] * t[0] + m[1] * t[1]) + m[2] * t[2]) + m[3]
        radians = np.asarray(self.rotation_degrees, dtype=F32) * F32(0.017453292519943295)
        m = _rotate(m, radians[2], (0, 0, 1))
        m = _rotate(m, radians[1], (0, 1, 0))
        m = _rotate(m, radians[0], (1, 0, 0))
        s = np.asarray(self.scale, dtype=F32)
        m[0] = m[0] * s[0]
        m[1] = m[1] * s[1]
        m[2] = m[2] * s[2]
        return m

    def normal_matrix(self) -> np.ndarray:
        """Inverse transpose of the linear part in double, stored as float
        (src/scene/scene.cpp:135-139). Column-major 3x3."""
        m = self.matrix().astype(np.float64)
        linear = m[:3, :3].T  # row-major linear map
        inverse_transpose = np.linalg.inv(linear).T
        return inverse_transpose.T.astype(F32)  # back to column-major


# ---- scene document ----------------------------------------------------------------------------

@dataclass
class Material:
    """Material (include/minirender/scene/scene.hpp:113-136). Textures are indices into
    SceneDocument.textures (None: no texture)."""

    kind: str = "diffuse"
    base_color: tuple = (0.7, 0.7, 0.7)
    emission: tuple = (0.0, 0.0, 0.0)
    roughness: float = 0.35
    ior: float = 1.5
    double_sided: bool = True
    base_color_texture: int | None = None
    texture_filter: str = "trilinear"
    normal_texture: int | None = None
    normal_scale: float = 1.0
    normal_flip_y: bool = False


@dataclass
class TextureData:
    """A decoded texture: (height, width, 3) float32 linear RGB, row 0 at the top
    (TextureAsset's data, include/minirender/scene/scene.hpp:148-154). `linear` records the source
    encoding (normal maps must come from linear textures)."""

    rgb: np.ndarray
    linear: bool = True


@dataclass
class MeshData:
    """MeshData (include/minirender/scene/scene.hpp:45-50) as arrays.

    positions: (P, 3) float32; corner_positions: (T, 3) uint32; corner_normals: (T, 3, 3)
    float32; corner_uvs: (T, 3, 2) float32."""

    positions: np.ndarray
    corner_positions: np.ndarray
    corner_normals: np.ndarray
    corner_uvs: np.ndarray | None = None

    @property
    def triangle_count(self) -> int:
        return int(self.corner_positions.shape[0])

    def validate(self):  # src/scene/scene.cpp:38-66
        if self.positions.shape[0] == 0 or self.corner_positions.shape[0] == 0:
            raise ValueError("Mesh must contain positions and triangles")
        if not np.all(np.isfinite(self.positions)):
            raise ValueError("Mesh position must be finite")
        if self.corner_positions.max() >= self.positions.shape[0]:
            raise ValueError("Mesh position index is out of range")
        n = self.corner_normals
        if not np.all(np.isfinite(n)) or np.any(np.einsum("tci,tci->tc", n, n) <= 1e-12):
            raise ValueError("Mesh normal must be finite and nonzero")
        p = self.positions[self.corner_positions]
        area = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
        if np.any(np.einsum("ti,ti->t", area, area) <= 1e-20):
            raise ValueError("Degenerate mesh triangle")

    def corners_array(self) -> np.ndarray:
        """Packs the corners as mr_mesh_corner records (24 bytes each)."""
        t = self.triangle_count
        rec = np.zeros((t, 3), dtype=np.dtype([("position", "<u4"), ("normal", "<f4", 3),
                                                ("uv", "<f4", 2)]))
        rec["position"] = self.corner_positions
        rec["normal"] = self.corner_normals
        if self.corner_uvs is not None:
            rec["uv"] = self.corner_uvs
        return rec.reshape(-1)


@dataclass
class SceneObject:
    mesh: int
    material: int
    transform: Transform = field(default_factory=Transform)
    visible: bool = True


@dataclass
class DirectionalLight:
    direction: tuple = (-1.0, -2.0, -1.0)
    color: tuple = (1.0, 1.0, 1.0)
    intensity: float = 3.0


@dataclass
class MediumRegion:
    minimum: tuple = (-1.0, -1.0, -1.0)
    maximum: tuple = (1.0, 1.0, 1.0)
    absorption: tuple = (0.0, 0.0, 0.0)
    scattering: tuple = (0.0, 0.0, 0.0)
    anisotropy: float = 0.0
    enabled: bool = True


@dataclass
class Camera:
    position: tuple = (0.0, 1.5, 4.0)
    target: tuple = (0.0, 0.5, 0.0)
    up: tuple = (0.0, 1.0, 0.0)
    vertical_fov_degrees: float = 45.0
    near_plane: float = 0.05
    far_plane: float = 100.0
    aperture_radius: float = 0.0
    focus_distance: float = 4.0


@dataclass
class SceneDocument:
    """SceneDocument (include/minirender/scene/scene.hpp:185-198)."""

    camera: Camera = field(default_factory=Camera)
    environment: tuple = (0.03, 0.03, 0.03)
    materials: list = field(default_factory=list)
    meshes: list = field(default_factory=list)
    objects: list = field(default_factory=list)
    directional_lights: list = field(default_factory=list)
    media: list = field(default_factory=list)
    textures: list = field(default_factory=list)  # TextureData
    environment_texture: int | None = None        # EnvironmentMap (scene.hpp:178-183)
    environment_strength: float = 1.0
    environment_rotation_degrees: float = 0.0

    @property
    def triangle_count(self) -> int:
        return sum(self.meshes[o.mesh].triangle_count for o in self.objects if o.visible)

    def snapshot(self) -> "Snapshot":
        return Snapshot(self)


class Snapshot:
    """The resolved, immutable scene as an ``mr_scene_desc`` plus the buffers it points into."""

    def __init__(self, document: SceneDocument):
        self.document = document
        self._keep = []
        desc = _abi.SceneDesc()
        cam = document.camera
        desc.camera = _abi.Camera(
            _abi.f3(*cam.position), _abi.f3(*cam.target), _abi.f3(*cam.up),
            cam.vertical_fov_degrees, cam.near_plane, cam.far_plane, cam.aperture_radius,
            cam.focus_distance)
        desc.environment = _abi.f3(*document.environment)

        meshes = (_abi.Mesh * max(1, len(document.meshes)))()
        for i, mesh in enumerate(document.meshes):
            positions = np.ascontiguousarray(mesh.positions, dtype=F32).reshape(-1)
            corners = np.ascontiguousarray(mesh.corners_array())
            self._keep += [positions, corners]
            meshes[i].positions = positions.ctypes.data_as(C.POINTER(C.c_float))
            meshes[i].position_count = mesh.positions.shape[0]
            meshes[i].corners = C.cast(corners.ctypes.data, C.POINTER(_abi.MeshCorner))
            meshes[i].triangle_count = mesh.triangle_count
        desc.meshes = meshes
        desc.mesh_count = len(document.meshes)

        def one_based(index):
            return 0 if index is None else int(index) + 1

        materials = (_abi.Material * max(1, len(document.materials)))()
        for i, m in enumerate(document.materials):
            materials[i] = _abi.Material(_abi.MATERIAL_KINDS[m.kind], _abi.f3(*m.base_color),
                                         _abi.f3(*m.emission), m.roughness, m.ior,
                                         1 if m.double_sided else 0,
                                         one_based(m.base_color_texture),
                                         _abi.TEXTURE_FILTERS[m.texture_filter],
                                         one_based(m.normal_texture), m.normal_scale,
                                         1 if m.normal_flip_y else 0)
        desc.materials = materials

        textures = (_abi.Texture * max(1, len(document.textures)))()
        for i, t in enumerate(document.textures):
            rgb = np.ascontiguousarray(t.rgb, dtype=F32)
            if rgb.ndim != 3 or rgb.shape[2] != 3:
                raise ValueError("Texture data must be (height, width, 3)")
            self._keep.append(rgb)
            textures[i] = _abi.Texture(rgb.ctypes.data_as(C.POINTER(C.c_float)), rgb.shape[1],
                                       rgb.shape[0])
        desc.textures = textures
        desc.texture_count = len(document.textures)
        desc.environment_texture = one_based(document.environment_texture)
        desc.environment_strength = document.environment_strength
        desc.environment_rotation_degrees = document.environment_rotation_degrees
        desc.material_count = len(document.materials)

        visible = [o for o in document.objects if o.visible]
        instances = (_abi.Instance * max(1, len(visible)))()
        self.matrices = []
        for i, o in enumerate(visible):
            m = o.transform.matrix()
            n = o.transform.normal_matrix()
            self.matrices.append((m, n))
            instances[i].mesh = o.mesh
            instances[i].material = o.material
            instances[i].object_to_world = (C.c_float * 16)(*m.reshape(-1).tolist())
            instances[i].normal_to_world = (C.c_float * 9)(*n.reshape(-1).tolist())
        desc.instances = instances
        desc.instance_count = len(visible)

        lights = (_abi.DirectionalLight * max(1, len(document.directional_lights)))()
        for i, l in enumerate(document.directional_lights):
            lights[i] = _abi.DirectionalLight(_abi.f3(*l.direction), _abi.f3(*l.color),
                                              l.intensity)
        desc.directional_lights = lights
        desc.directional_light_count = len(document.directional_lights)

        media = (_abi.MediumRegion * max(1, len(document.media)))()
        for i, r in enumerate(document.media):
            media[i] = _abi.MediumRegion(_abi.d3(*r.minimum), _abi.d3(*r.maximum),
                                         _abi.d3(*r.absorption), _abi.d3(*r.scattering),
                                         r.anisotropy, 1 if r.enabled else 0)
        desc.media = media
        desc.medium_count = len(document.media)
        self._keep += [meshes, materials, instances, lights, media, textures]
        self.desc = desc
        self.triangle_count = sum(document.meshes[o.mesh].triangle_count for o in visible)

    def desc_pointer(self):
        return C.pointer(self.desc)

    def world_triangles(self) -> np.ndarray:
        """World-space float32 vertices (N, 3, 3) in primitive order, computed like
        SceneBvh's constructor (src/render/bvh.cpp:53-89)."""
        out = []
        for o, (m, _) in zip([o for o in self.document.objects if o.visible], self.matrices):
            mesh = self.document.meshes[o.mesh]
            p = mesh.positions[mesh.corner_positions].astype(F32)  # (T,3,3)
            w = ((m[0] * p[..., 0:1] + m[1] * p[..., 1:2]) + (m[2] * p[..., 2:3] + m[3] * F32(1)))
            out.append(w[..., :3].astype(F32))
        return np.concatenate(out) if out else np.zeros((0, 3, 3), F32)


# ---- procedural geometry ---------------------------------------------------------------------

def quad_mesh(corners, normal=None) -> MeshData:
    """Two triangles (0,1,2) and (0,2,3) over four corners; normal from the winding."""
    p = np.asarray(corners, dtype=F32)
    if normal is None:
        n = np.cross(p[1] - p[0], p[2] - p[0]).astype(np.float64)
        normal = n / np.linalg.norm(n)
    normal = np.asarray(normal, dtype=F32)
    idx = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32)
    normals = np.broadcast_to(normal, (2, 3, 3)).astype(F32)
    uvs = np.array([[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]], dtype=F32)
    return MeshData(p, idx, normals, uvs)


def box_mesh(size=(1.0, 1.0, 1.0)) -> MeshData:
    """Axis-aligned box centred on the origin, 12 outward-wound triangles, flat normals."""
    sx, sy, sz = (F32(v) * F32(0.5) for v in size)
    faces = [  # (normal, four corners counter-clockwise seen from outside)
        ((1, 0, 0), [(sx, -sy, sz), (sx, -sy, -sz), (sx, sy, -sz), (sx, sy, sz)]),
        ((-1, 0, 0), [(-sx, -sy, -sz), (-sx, -sy, sz), (-sx, sy, sz), (-sx, sy, -sz)]),
        ((0, 1, 0), [(-sx, sy, sz), (sx, sy, sz), (sx, sy, -sz), (-sx, sy, -sz)]),
        ((0, -1, 0), [(-sx, -sy, -sz), (sx, -sy, -sz), (sx, -sy, sz), (-sx, -sy, sz)]),
        ((0, 0, 1), [(-sx, -sy, sz), (sx, -sy, sz), (sx, sy, sz), (-sx, sy, sz)]),
        ((0, 0, -1), [(sx, -sy, -sz), (-sx, -sy, -sz), (-sx, sy, -sz), (sx, sy, -sz)]),
    ]
    positions, idx, normals = [], [], []
    for f, (n, quad) in enumerate(faces):
        base = 4 * f
        positions += quad
        idx += [[base, base + 1, base + 2], [base, base + 2, base + 3]]
        normals += [[n, n, n], [n, n, n]]
    return MeshData(np.asarray(positions, F32), np.asarray(idx, np.uint32),
                    np.asarray(normals, F32), np.zeros((12, 3, 2), F32))


def icosphere(subdivisions: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20 * 4^subdivisions outward-wound triangles (float64 vertices)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
         (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    vertices = np.asarray(v, dtype=np.float64)
    vertices /= np.linalg.norm(vertices, axis=1, keepdims=True)
    faces = np.asarray(f, dtype=np.int64)
    for _ in range(subdivisions):
        edges = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        unique, inverse = np.unique(key, axis=0, return_inverse=True)
        mid = vertices[unique[:, 0]] + vertices[unique[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = vertices.shape[0]
        vertices = np.concatenate([vertices, mid])
        n = faces.shape[0]
        inverse = inverse.reshape(-1)
        m01, m12, m20 = (inverse[:n] + base, inverse[n:2 * n] + base, inverse[2 * n:] + base)
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        faces = np.concatenate([np.stack([a, m01, m20], 1), np.stack([b, m12, m01], 1),
                                np.stack([c, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return vertices, faces


def _hash3(ix, iy, iz, seed):
    """Integer lattice hash to [-1, 1] (own mixing, 32-bit arithmetic)."""
    h = (ix.astype(np.uint32) * np.uint32(0x8DA6B343)) ^ (iy.astype(np.uint32) * np.uint32(0xD8163841)) \
        ^ (iz.astype(np.uint32) * np.uint32(0xCB1AB31F)) ^ np.uint32(seed * 0x9E3779B1 & 0xFFFFFFFF)
    h ^= h >> np.uint32(15)
    h *= np.uint32(0x2C1B3C6D)
    h ^= h >> np.uint32(12)
    h *= np.uint32(0x297A2D39)
    h ^= h >> np.uint32(15)
    return (h.astype(np.float32) * F32(1.0 / 4294967295.0)) * F32(2) - F32(1)


def value_noise(points: np.ndarray, seed: int, frequency: float = 3.0) -> np.ndarray:
    """FP32 3D value noise: lattice values from _hash3, smoothstep-weighted trilinear blend."""
    p = points.astype(F32) * F32(frequency)
    cell = np.floor(p)
    f = p - cell
    w = f * f * (F32(3) - F32(2) * f)
    ci = cell.astype(np.int64)
    result = np.zeros(points.shape[0], dtype=F32)
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                val = _hash3(ci[:, 0] + dx, ci[:, 1] + dy, ci[:, 2] + dz, seed)
                wx = w[:, 0] if dx else F32(1) - w[:, 0]
                wy = w[:, 1] if dy else F32(1) - w[:, 1]
                wz = w[:, 2] if dz else F32(1) - w[:, 2]
                result += (wx * wy * wz * val).astype(F32)
    return result


def displaced_icosphere(subdivisions: int, seed: int, amplitude: float = 0.1) -> MeshData:
    """Icosphere with FP32 radial value-noise displacement and smooth vertex normals."""
    v64, faces = icosphere(subdivisions)
    v = v64.astype(F32)
    radius = F32(1) + F32(amplitude) * value_noise(v, seed)
    positions = (v * radius[:, None]).astype(F32)
    tri = positions[faces]
    face_n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]).astype(np.float64)
    vn = np.zeros((positions.shape[0], 3), np.float64)
    for k in range(3):
        np.add.at(vn, faces[:, k], face_n)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True)
    normals = vn.astype(F32)[faces]
    return MeshData(positions, faces.astype(np.uint32), normals, None)


# ---- workloads ---------------------------------------------------------------------------------

def cornell_box() -> SceneDocument:
    """The 36-triangle Cornell box: 5 wall quads of a unit box, two rotated boxes and a 0.25^2
    single-sided ceiling light with radiance (17, 12, 4); pinhole camera with a 40 degree field
    of view at the open front, looking at the box centre; black environment."""
    doc = SceneDocument()
    doc.camera = Camera(position=(0.0, 0.5, 1.87), target=(0.0, 0.5, 0.0), up=(0.0, 1.0, 0.0),
                        vertical_fov_degrees=40.0, near_plane=0.05, far_plane=100.0)
    doc.environment = (0.0, 0.0, 0.0)
    doc.materials = [
        Material("diffuse", (0.725, 0.71, 0.68)),   # 0 white walls
        Material("diffuse", (0.63, 0.065, 0.05)),   # 1 left, red
        Material("diffuse", (0.14, 0.45, 0.09)),    # 2 right, green
        Material("diffuse", (0.725, 0.725, 0.725)), # 3 boxes
        Material("diffuse", (0.78, 0.78, 0.78), emission=(17.0, 12.0, 4.0),
                 double_sided=False),               # 4 light
    ]
    h = 0.5
    walls = {
        "floor": ([(-h, 0, h), (h, 0, h), (h, 0, -h), (-h, 0, -h)], 0),
        "ceiling": ([(-h, 1, -h), (h, 1, -h), (h, 1, h), (-h, 1, h)], 0),
        "back": ([(-h, 0, -h), (h, 0, -h), (h, 1, -h), (-h, 1, -h)], 0),
        "left": ([(-h, 0, h), (-h, 0, -h), (-h, 1, -h), (-h, 1, h)], 1),
        "right": ([(h, 0, -h), (h, 0, h), (h, 1, h), (h, 1, -h)], 2),
    }
    for corners, material in walls.values():
        doc.meshes.append(quad_mesh(corners))
        doc.objects.append(SceneObject(len(doc.meshes) - 1, material))
    doc.meshes.append(box_mesh((0.3, 0.3, 0.3)))
    doc.objects.append(SceneObject(len(doc.meshes) - 1, 3,
                                   Transform((0.17, 0.15, 0.12), (0.0, -18.0, 0.0))))
    doc.meshes.append(box_mesh((0.3, 0.6, 0.3)))
    doc.objects.append(SceneObject(len(doc.meshes) - 1, 3,
                                   Transform((-0.17, 0.3, -0.15), (0.0, 15.0, 0.0))))
    q = 0.125
    doc.meshes.append(quad_mesh([(-q, 0.998, -q), (q, 0.998, -q), (q, 0.998, q), (-q, 0.998, q)]))
    doc.objects.append(SceneObject(len(doc.meshes) - 1, 4))
    return doc


def random_material(rng: np.random.Generator) -> Material:
    """Uniform over diffuse (albedo U[.1,.9]^3), GGX metal (roughness U[.05,.5], F0 colour
    U[.5,1]^3), mirror (colour 0.9) and glass (IOR 1.5)."""
    choice = int(rng.integers(0, 4))
    if choice == 0:
        return Material("diffuse", tuple(rng.uniform(0.1, 0.9, 3).tolist()))
    if choice == 1:
        return Material("conductor", tuple(rng.uniform(0.5, 1.0, 3).tolist()),
                        roughness=float(rng.uniform(0.05, 0.5)))
    if choice == 2:
        return Material("mirror", (0.9, 0.9, 0.9))
    return Material("dielectric", (1.0, 1.0, 1.0), ior=1.5)


def sphere_field(count: int, extent: float, seed: int, subdivisions: int = 4,
                 variants: int | None = None, amplitude: float = 0.1) -> SceneDocument:
    """`count` displaced icospheres placed uniformly in an extent^3 box above a ground quad.

    Each sphere has scale U[0.2, 1.5], a random orientation and a material from
    ``random_material``. ``variants`` limits the number of distinct displaced meshes (each
    sphere picks one); None gives every sphere its own noise seed."""
    rng = np.random.default_rng(seed)
    doc = SceneDocument()
    doc.environment = (1.0, 1.0, 1.0)
    doc.directional_lights = [DirectionalLight((-1.0, -2.0, -1.0), (1.0, 0.95, 0.85), 3.0)]
    half = extent / 2
    doc.camera = Camera(position=(0.0, half, half + 10.0), target=(0.0, half, 0.0),
                        up=(0.0, 1.0, 0.0), vertical_fov_degrees=45.0, near_plane=0.05,
                        far_plane=10.0 * extent, aperture_radius=0.05, focus_distance=10.0)
    doc.materials.append(Material("diffuse", (0.5, 0.5, 0.5)))
    g = 10 * extent
    doc.meshes.append(quad_mesh([(-g, 0, g), (g, 0, g), (g, 0, -g), (-g, 0, -g)]))
    doc.objects.append(SceneObject(0, 0))
    mesh_count = count if variants is None else variants
    first_mesh = len(doc.meshes)
    for k in range(mesh_count):
        doc.meshes.append(displaced_icosphere(subdivisions, seed * 7919 + k, amplitude))
    for k in range(count):
        scale = float(rng.uniform(0.2, 1.5))
        center = (float(rng.uniform(-half, half)), float(rng.uniform(0.0, extent)),
                  float(rng.uniform(-half, half)))
        rotation = tuple(rng.uniform(0.0, 360.0, 3).tolist())
        doc.materials.append(random_material(rng))
        mesh = first_mesh + (k if variants is None else int(rng.integers(0, variants)))
        doc.objects.append(SceneObject(mesh, len(doc.materials) - 1,
                                       Transform(center, rotation, (scale, scale, scale))))
    return doc


def large_scene(seed: int = 2) -> SceneDocument:
    """About 1M triangles: 200 displaced 4-subdivision icospheres (5,120 triangles each) in a
    20^3 box on a ground quad; constant environment 1 plus one directional light; thin lens with
    aperture 0.05 and focus distance 10."""
    return sphere_field(200, 20.0, seed, subdivisions=4)


def stress_scene(seed: int = 5, count: int = 4000, variants: int = 64) -> SceneDocument:
    """About 20M triangles: 4,000 displaced icospheres in a 50^3 box inside one homogeneous
    medium (sigma_a = (0.01, 0.02, 0.03), sigma_s = 0.1, g = 0)."""
    doc = sphere_field(count, 50.0, seed, subdivisions=4, variants=variants)
    doc.media = [MediumRegion((-26.0, -1.0, -26.0), (26.0, 51.0, 26.0),
                              (0.01, 0.02, 0.03), (0.1, 0.1, 0.1), 0.0)]
    return doc


_PER_SPHERE = {0: 20, 1: 80, 2: 320, 3: 1280, 4: 5120}


def _job_spheres(triangles: int) -> tuple[int, int]:
    """Subdivision level and sphere count of a job scene of about `triangles` triangles."""
    budget = max(0, triangles - 36)
    level = 3 if budget < 200_000 else 4
    return level, max(1, budget // _PER_SPHERE[level])


def job_scene_triangles(triangles: int) -> int:
    """The exact triangle count job_scene(triangles, seed) builds (any seed)."""
    level, n = _job_spheres(triangles)
    return 36 + n * _PER_SPHERE[level]


def job_scene(triangles: int, seed: int) -> SceneDocument:
    """A Cornell shell filled with displaced icospheres up to about `triangles` triangles
    (the uneven job table's scenes)."""
    rng = np.random.default_rng(seed)
    doc = cornell_box()
    level, n = _job_spheres(triangles)
    variants = min(n, 8)
    first = len(doc.meshes)
    for k in range(variants):
        doc.meshes.append(displaced_icosphere(level, seed * 31 + k, 0.1))
    radius = 0.35 / max(1.0, n ** (1.0 / 3.0))
    for k in range(n):
        doc.materials.append(random_material(rng))
        c = (float(rng.uniform(-0.4, 0.4)), float(rng.uniform(0.1, 0.9)),
             float(rng.uniform(-0.4, 0.4)))
        doc.objects.append(SceneObject(first + int(rng.integers(0, variants)),
                                       len(doc.materials) - 1,
                                       Transform(c, tuple(rng.uniform(0, 360, 3).tolist()),
                                                 (radius, radius, radius))))
    return doc


def job_table(count: int = 256, seed: int = 3) -> list[dict]:
    """The uneven job mix of the batching and serving workloads, seeded: triangle count
    log-uniform in [10k, 500k], square resolution with pixel count log-uniform in
    [128^2, 1024^2], samples per pixel log-uniform in [4, 256], maximum depth uniform in
    {4, ..., 12}, render seed per job."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(count):
        triangles = int(round(np.exp(rng.uniform(np.log(10_000), np.log(500_000)))))
        side = int(round(np.exp(rng.uniform(np.log(128), np.log(1024)))))
        spp = int(round(np.exp(rng.uniform(np.log(4), np.log(256)))))
        depth = int(rng.integers(4, 13))
        jobs.append({"triangles": triangles, "width": side, "height": side,
                     "samples_per_pixel": spp, "maximum_depth": depth,
                     "scene_seed": seed * 100_003 + i, "render_seed": i + 1})
    return jobs
