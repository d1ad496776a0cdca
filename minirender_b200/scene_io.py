"""Scene JSON v1 and Wavefront OBJ ingestion, so the reference's own scene files render directly.

``load_scene(path)`` follows ``load_scene`` (src/assets/scene_io.cpp:45-160): the same keys,
defaults and validation, meshes loaded from OBJ files relative to the scene file, objects,
materials and meshes referenced by id. ``load_obj(path)`` follows ``load_obj``
(src/assets/obj_loader.cpp:14-92): positions shared, one normal and uv per triangle corner, unit
corner normals from ``vn`` or else the triangle's geometric normal, degenerate triangles and zero
normals rejected.

The reference parses OBJ text with tinyobjloader v2.0.0rc13 (cmake/Dependencies.cmake:36-38),
which is not in the reference tree. Its published behaviour is restated here for what the
reference's scenes use: ``v``/``vn``/``vt`` records, 1-based and negative (relative) indices,
``v``, ``v/t``, ``v//n`` and ``v/t/n`` face corners, and triangulation of a quad along its
shorter diagonal (corners 0-2 when strictly shorter than 1-3: triangles 0,1,2 and 0,2,3; else
0,1,3 and 1,2,3). Faces of more than four corners are split as a fan from the first corner, which
matches tinyobjloader for convex polygons. Groups, objects, smoothing and material libraries carry
no geometry and are ignored.

Textures (src/assets/scene_io.cpp:111-124): the "textures" table's images are decoded by
``image_io.read_texture`` (PNG at any bit depth, EXR, Radiance HDR) with their "encoding" ("srgb"
converts 8/16-bit samples to linear; EXR and HDR must be "linear"); materials reference them by id
("base_color_texture", "normal_texture" with "normal_scale" and "normal_flip_y", "texture_filter")
and so does "environment_map" ("texture", "strength", "rotation_degrees"). A normal map must be a
linear texture (src/scene/scene.cpp:295-301). Cloth and subsurface materials load and are rejected
when the scene is created, as the C ABI documents.
"""

from __future__ import annotations

import json
import os

import numpy as np

from .image_io import read_texture, write_exr
from .scene import (Camera, DirectionalLight, Material, MediumRegion, MeshData, SceneDocument,
                    SceneObject, TextureData, Transform)

F32 = np.float32
MATERIAL_KINDS = ("diffuse", "conductor", "mirror", "dielectric", "cloth", "subsurface")
MAXIMUM_MEDIUM_REGIONS = 32


def _index(token: str, count: int, what: str) -> int:
    i = int(token)
    if i < 0:
        i = count + i  # relative to the records read so far
    else:
        i -= 1
    if i < 0 or i >= count:
        raise ValueError(f"OBJ has an invalid {what} index")
    return i


def _triangulate(corners, positions):
    n = len(corners)
    if n < 3:
        raise ValueError("OBJ face has fewer than three corners")
    if n == 3:
        return [tuple(corners)]
    if n == 4:
        p = [positions[c[0]] for c in corners]
        e02 = p[2] - p[0]
        e13 = p[3] - p[1]
        if float(np.dot(e02, e02)) < float(np.dot(e13, e13)):
            return [(corners[0], corners[1], corners[2]), (corners[0], corners[2], corners[3])]
        return [(corners[0], corners[1], corners[3]), (corners[1], corners[2], corners[3])]
    return [(corners[0], corners[k], corners[k + 1]) for k in range(1, n - 1)]


def load_obj(path: str) -> MeshData:
    """MeshData of an OBJ file (load_obj, src/assets/obj_loader.cpp:14-92)."""
    positions, normals, uvs, faces = [], [], [], []
    with open(path, "r", encoding="utf-8", errors="replace") as f:
        for line in f:
            fields = line.split("#", 1)[0].split()
            if not fields:
                continue
            tag = fields[0]
            if tag == "v":
                positions.append(np.array([float(x) for x in fields[1:4]], F32))
            elif tag == "vn":
                normals.append(np.array([float(x) for x in fields[1:4]], F32))
            elif tag == "vt":
                uvs.append(np.array([float(x) for x in fields[1:3]], F32))
            elif tag == "f":
                corners = []
                for token in fields[1:]:
                    parts = token.split("/")
                    v = _index(parts[0], len(positions), "vertex")
                    t = _index(parts[1], len(uvs), "UV") if len(parts) > 1 and parts[1] else -1
                    n = _index(parts[2], len(normals), "normal") if len(parts) > 2 and parts[2] else -1
                    corners.append((v, t, n))
                faces.append(corners)
    if not positions:
        raise ValueError("OBJ has no positions")
    pos = np.stack(positions)
    corner_positions, corner_normals, corner_uvs = [], [], []
    for face in faces:
        for tri in _triangulate(face, pos):
            a, b, c = (pos[k[0]] for k in tri)
            cross = np.cross((b - a).astype(F32), (c - a).astype(F32)).astype(F32)
            length = F32(np.sqrt(F32(np.dot(cross, cross))))
            if not (length > F32(1e-10)):
                raise ValueError("OBJ has a degenerate triangle")
            geometric = (cross / length).astype(F32)
            tri_normals, tri_uvs = [], []
            for (_, t, n) in tri:
                if n >= 0:
                    normal = normals[n]
                    nl = F32(np.sqrt(F32(np.dot(normal, normal))))
                    if not (nl > F32(1e-10)):
                        raise ValueError("OBJ normal is zero")
                    tri_normals.append((normal / nl).astype(F32))
                else:
                    tri_normals.append(geometric)
                tri_uvs.append(uvs[t] if t >= 0 else np.zeros(2, F32))
            corner_positions.append([k[0] for k in tri])
            corner_normals.append(tri_normals)
            corner_uvs.append(tri_uvs)
    if not corner_positions:
        raise ValueError("OBJ has no faces")
    mesh = MeshData(pos, np.asarray(corner_positions, np.uint32),
                    np.asarray(corner_normals, F32), np.asarray(corner_uvs, F32))
    mesh.validate()
    return mesh


def _vector3(value, what: str = "vector") -> tuple:
    if not isinstance(value, list) or len(value) != 3:
        raise ValueError(f"Expected a three-component {what}")
    return tuple(float(F32(x)) for x in value)


def _double3(value) -> tuple:
    if not isinstance(value, list) or len(value) != 3:
        raise ValueError("Medium vector requires three numbers")
    return tuple(float(x) for x in value)


def load_scene(path: str) -> SceneDocument:
    """SceneDocument of a scene JSON v1 file (load_scene, src/assets/scene_io.cpp:45-160)."""
    try:
        with open(path, "r", encoding="utf-8") as f:
            data = json.load(f)
        version = data["version"]
        if not isinstance(version, int) or isinstance(version, bool) or version != 1:
            raise ValueError("Unsupported scene version")
        directory = os.path.dirname(os.path.abspath(path))
        doc = SceneDocument()
        cam = data["camera"]
        doc.camera = Camera(position=_vector3(cam["position"]), target=_vector3(cam["target"]),
                            up=_vector3(cam["up"]),
                            vertical_fov_degrees=float(F32(cam["vertical_fov"])),
                            near_plane=float(F32(cam["near"])), far_plane=float(F32(cam["far"])),
                            aperture_radius=float(F32(cam.get("aperture_radius", 0.0))),
                            focus_distance=float(F32(cam.get("focus_distance", 4.0))))
        doc.environment = _vector3(data["environment"])
        if "media" in data:
            media = data["media"]
            if not isinstance(media, list) or len(media) > MAXIMUM_MEDIUM_REGIONS:
                raise ValueError("Media must be an array of at most 32 regions")
            doc.media = [MediumRegion(_double3(m["minimum"]), _double3(m["maximum"]),
                                      _double3(m["absorption"]), _double3(m["scattering"]),
                                      float(m["anisotropy"]), bool(m.get("enabled", True)))
                         for m in media]
        texture_index = {}
        for t in data.get("textures", []):
            encoding = t.get("encoding", "srgb")
            if encoding not in ("srgb", "linear"):
                raise ValueError("Unknown texture encoding")
            if t["id"] in texture_index:
                raise ValueError(f"Duplicate texture id '{t['id']}'")
            texture_index[t["id"]] = len(doc.textures)
            doc.textures.append(TextureData(read_texture(os.path.join(directory, t["source"]),
                                                         encoding == "linear"),
                                            encoding == "linear"))

        def texture(name, what):
            if not name:
                return None
            if name not in texture_index:
                raise ValueError(f"{what} references missing texture: {name}")
            return texture_index[name]

        environment = data.get("environment_map", {})
        doc.environment_texture = texture(environment.get("texture", ""), "Environment")
        doc.environment_strength = float(F32(environment.get("strength", 1.0)))
        doc.environment_rotation_degrees = float(F32(environment.get("rotation_degrees", 0.0)))
        material_index = {}
        for m in data["materials"]:
            kind = m["kind"]
            if kind not in MATERIAL_KINDS:
                raise ValueError(f"Unknown material kind '{kind}'")
            texture_filter = m.get("texture_filter", "trilinear")
            if texture_filter not in ("nearest", "bilinear", "trilinear"):
                raise ValueError(f"Unknown texture filter: {texture_filter}")
            normal = texture(m.get("normal_texture", ""), "Material")
            if normal is not None and not doc.textures[normal].linear:
                raise ValueError("Normal map must reference a linear texture")
            material_index[m["id"]] = len(doc.materials)
            doc.materials.append(Material(kind, _vector3(m["base_color"]),
                                          _vector3(m.get("emission", [0, 0, 0])),
                                          float(F32(m.get("roughness", 0.35))),
                                          float(F32(m.get("ior", 1.5))),
                                          bool(m.get("double_sided", True)),
                                          texture(m.get("base_color_texture", ""), "Material"),
                                          texture_filter, normal,
                                          float(F32(m.get("normal_scale", 1.0))),
                                          bool(m.get("normal_flip_y", False))))
        mesh_index = {}
        for m in data["meshes"]:
            mesh_index[m["id"]] = len(doc.meshes)
            doc.meshes.append(load_obj(os.path.join(directory, m["source"])))
        for o in data["objects"]:
            if o["mesh"] not in mesh_index:
                raise ValueError(f"Object '{o['id']}' references a missing mesh")
            if o["material"] not in material_index:
                raise ValueError(f"Object '{o['id']}' references a missing material")
            t = o["transform"]
            doc.objects.append(SceneObject(mesh_index[o["mesh"]], material_index[o["material"]],
                                           Transform(_vector3(t["translation"]),
                                                     _vector3(t["rotation"]),
                                                     _vector3(t["scale"])),
                                           bool(o.get("visible", True))))
        for light in data["directional_lights"]:
            doc.directional_lights.append(DirectionalLight(_vector3(light["direction"]),
                                                           _vector3(light["color"]),
                                                           float(F32(light["intensity"]))))
        return doc
    except (KeyError, TypeError, ValueError, OSError) as error:
        message = f"missing key {error}" if isinstance(error, KeyError) else str(error)
        raise ValueError(f"Scene {path}: {message}") from error


def _fmt(v) -> str:
    return "%.9g" % float(v)  # float32 round-trips through 9 significant digits


def save_obj(mesh: MeshData, path: str):
    """Writes a MeshData as OBJ triangles with one vt and vn per corner (load_obj reads it back
    exactly)."""
    mesh.validate()
    uvs = mesh.corner_uvs if mesh.corner_uvs is not None else np.zeros(
        (mesh.triangle_count, 3, 2), F32)
    lines = ["# minirender_b200 mesh"]
    lines += ["v %s %s %s" % tuple(_fmt(x) for x in p) for p in mesh.positions]
    lines += ["vt %s %s" % tuple(_fmt(x) for x in uv) for uv in uvs.reshape(-1, 2)]
    lines += ["vn %s %s %s" % tuple(_fmt(x) for x in n) for n in mesh.corner_normals.reshape(-1, 3)]
    for t, corners in enumerate(mesh.corner_positions):
        lines.append("f " + " ".join(f"{int(p) + 1}/{3 * t + k + 1}/{3 * t + k + 1}"
                                     for k, p in enumerate(corners)))
    with open(path, "w", encoding="utf-8") as f:
        f.write("\n".join(lines) + "\n")


def _material_json(k: int, m: Material) -> dict:
    out = {"id": f"material_{k}", "kind": m.kind, "base_color": list(m.base_color),
           "emission": list(m.emission), "roughness": m.roughness, "ior": m.ior,
           "double_sided": bool(m.double_sided), "texture_filter": m.texture_filter,
           "normal_scale": m.normal_scale, "normal_flip_y": bool(m.normal_flip_y)}
    if m.base_color_texture is not None:
        out["base_color_texture"] = f"texture_{m.base_color_texture}"
    if m.normal_texture is not None:
        out["normal_texture"] = f"texture_{m.normal_texture}"
    return out


def save_scene(doc: SceneDocument, path: str):
    """Writes a SceneDocument as scene JSON v1 with one OBJ file per mesh beside it
    (mesh_<k>.obj); load_scene reads it back."""
    directory = os.path.dirname(os.path.abspath(path))
    stem = os.path.splitext(os.path.basename(path))[0]
    meshes = []
    for k, mesh in enumerate(doc.meshes):
        name = f"{stem}_mesh_{k}.obj"
        save_obj(mesh, os.path.join(directory, name))
        meshes.append({"id": f"mesh_{k}", "source": name})
    c = doc.camera
    data = {
        "version": 1,
        "camera": {"position": list(c.position), "target": list(c.target), "up": list(c.up),
                   "vertical_fov": c.vertical_fov_degrees, "near": c.near_plane,
                   "far": c.far_plane, "aperture_radius": c.aperture_radius,
                   "focus_distance": c.focus_distance},
        "environment": list(doc.environment),
        "materials": [_material_json(k, m) for k, m in enumerate(doc.materials)],
        "meshes": meshes,
        "objects": [{"id": f"object_{k}", "mesh": f"mesh_{o.mesh}",
                     "material": f"material_{o.material}", "visible": bool(o.visible),
                     "transform": {"translation": list(o.transform.translation),
                                   "rotation": list(o.transform.rotation_degrees),
                                   "scale": list(o.transform.scale)}}
                    for k, o in enumerate(doc.objects)],
        "directional_lights": [{"id": f"light_{k}", "direction": list(l.direction),
                                "color": list(l.color), "intensity": l.intensity}
                               for k, l in enumerate(doc.directional_lights)],
    }
    if doc.textures:
        data["textures"] = []
        for k, t in enumerate(doc.textures):
            name = f"{stem}_texture_{k}.exr"  # linear float: the decoded texels round-trip exactly
            write_exr(os.path.join(directory, name), t.rgb)
            data["textures"].append({"id": f"texture_{k}", "source": name, "encoding": "linear"})
    if doc.environment_texture is not None:
        data["environment_map"] = {"texture": f"texture_{doc.environment_texture}",
                                   "strength": doc.environment_strength,
                                   "rotation_degrees": doc.environment_rotation_degrees}
    if doc.media:
        data["media"] = [{"id": f"medium_{k}", "minimum": list(m.minimum),
                          "maximum": list(m.maximum), "absorption": list(m.absorption),
                          "scattering": list(m.scattering), "anisotropy": m.anisotropy,
                          "enabled": bool(m.enabled)} for k, m in enumerate(doc.media)]
    with open(path, "w", encoding="utf-8") as f:
        json.dump(data, f, indent=1)
