"""JSON scene files and frame checkpoints in the reference's format, without Qt.

The reference reads and writes scenes with OptixSceneLoader::readJSON / writeJSON
(OptixSceneLoader.cpp:31-180) and its classes' readJSON methods: an "Integrator", a "Background", a
"Camera", a "Lights" array and a "Geometries" array of OBJ files with a position, a scale, rotations and
a material ({"mtl_name": <shader name>, "mtl_parameters": {...}}), plus "frame_count" and "buffer_path"
for a saved frame (OptixScene::saveScene / loadBuffer, OptixScene.cpp:200-298: the float4 accumulation
buffer as raw native floats next to the JSON file).  ``load_json_scene`` builds a SceneData from such a
file; ``save_checkpoint`` / ``load_checkpoint`` write and restore a render's accumulation buffer and
frame count so that rendering resumes where it stopped.

Relative paths in the file are resolved against ``base_dir`` (default: the JSON file's directory); the
reference resolves them against its build directory.  Parameters left out keep the reference classes'
defaults.  Geometry transforms are M = T(position) R_z R_y R_x R(angle, axis) S(scale)
(Geometry.cpp:286-291) applied to the vertices on the host, normals by the inverse transpose.
Integrator "DepthTracer" and the normal / flat / anisotropic materials are outside this path and raise.
"""
import json
import math
import os

import numpy as np

from . import _native as nat
from . import scene as sc

MATERIAL_NAMES = {  # materialNames, structs.h:227-239
    "diffuse_shader": sc.DIFFUSE_SHADER, "transparent_shader": sc.TRANSPARENT_SHADER,
    "rough_transparent_shader": sc.ROUGH_TRANSPARENT_SHADER, "metallic_shader": sc.METALLIC_SHADER,
    "translucent_shader": sc.TRANSLUCENT_SHADER, "rough_translucent_shader": sc.ROUGH_TRANSLUCENT_SHADER,
    "lambertian_interface_shader": sc.LAMBERTIAN_INTERFACE_SHADER, "rough_diffuse_shader": sc.ROUGH_DIFFUSE_SHADER,
}


def _v3(x):
    return tuple(float(v) for v in x[:3])


def rotation_matrix(angle_deg, axis):
    """Rotation by angle_deg about the unit vector `axis` (right-handed, Rodrigues)."""
    a = np.asarray(axis, np.float64)
    n = np.linalg.norm(a)
    x, y, z = (a / n) if n > 0 else (0.0, 1.0, 0.0)
    t = float(np.float32(angle_deg) * np.float32(math.pi) / np.float32(180.0))
    c, s = math.cos(t), math.sin(t)
    k = 1.0 - c
    return np.array([[k * x * x + c, k * x * y - s * z, k * x * z + s * y],
                     [k * x * y + s * z, k * y * y + c, k * y * z - s * x],
                     [k * x * z - s * y, k * y * z + s * x, k * z * z + c]], np.float64)


def geometry_transform(p):
    """3x3 linear part and translation of a geometry's parameters (Geometry.cpp:92-130, :286-291)."""
    R = np.eye(3)
    if "rotation" in p:
        r = p["rotation"]
        R = rotation_matrix(r[0], r[1:4])
    Rx = rotation_matrix(p["x_rotation"], (1, 0, 0)) if "x_rotation" in p else np.eye(3)
    Ry = rotation_matrix(p["y_rotation"], (0, 1, 0)) if "y_rotation" in p else np.eye(3)
    Rz = rotation_matrix(p["z_rotation"], (0, 0, 1)) if "z_rotation" in p else np.eye(3)
    S = np.diag(np.asarray(p.get("scale", (1.0, 1.0, 1.0)), np.float64)[:3])
    return Rz @ Ry @ Rx @ R @ S, np.asarray(p.get("position", (0.0, 0.0, 0.0)), np.float64)[:3]


def _transform_mesh(m, A, t):
    pos = (m.positions.astype(np.float64) @ A.T + t).astype(np.float32)
    nrm = None
    if m.normals is not None:
        nrm = (m.normals.astype(np.float64) @ np.linalg.inv(A)).astype(np.float32)  # inverse transpose, row vectors
    return sc.Mesh(pos, m.vindex, m.material, nrm, m.nindex)


def material_from_json(obj, unsupported=None):
    """A material from {"mtl_name", "mtl_parameters"} (each class's loadFromJSON).  A shader outside the
    path tracer (normal_shader, flat_shader, anisotropic_structure_shader) raises, or is replaced by
    `unsupported` when one is given."""
    name = obj.get("mtl_name", "diffuse_shader")
    p = obj.get("mtl_parameters", {})
    if name not in MATERIAL_NAMES:
        if unsupported is not None:
            return unsupported
        raise ValueError("material %r is outside the path tracer (supported: %s)" % (name, ", ".join(MATERIAL_NAMES)))
    kind = MATERIAL_NAMES[name]
    if kind == sc.DIFFUSE_SHADER:
        return sc.DiffuseMaterial(_v3(p.get("diffuse_color", (0.8, 0.8, 0.8))))
    if kind == sc.METALLIC_SHADER:
        m = sc.MetallicMaterial()
        re = p.get("real_ior", [c[0] for c in m.ior])
        im = p.get("imaginary_ior", [c[1] for c in m.ior])
        m.setIor(tuple((float(re[k]), float(im[k])) for k in range(3)))
        if "roughness" in p:
            m.setRoughness(p["roughness"][:2])
        m.setMicrofacetModel(p.get("microfacet_model", m.microfacet_model))
        m.setNormalDistribution(p.get("normal_distribution", m.normal_distribution))
        return m
    if kind == sc.ROUGH_TRANSPARENT_SHADER:
        m = sc.RoughTransparentMaterial()
        r = p.get("roughness", m.roughness)
        return sc.RoughTransparentMaterial(ior=p.get("ior", m.ior), roughness=r[0] if isinstance(r, (list, tuple)) else r,
                                           glass_absorption=_v3(p.get("glass_absorption", m.glass_absorption)),
                                           microfacet_model=p.get("microfacet_model", m.microfacet_model),
                                           normal_distribution=p.get("normal_distribution", m.normal_distribution))
    if kind == sc.TRANSPARENT_SHADER:
        return sc.TransparentMaterial(ior=p.get("ior", 1.3), glass_absorption=_v3(p.get("glass_absorption", (0.0, 0.0, 0.0))))
    if kind == sc.LAMBERTIAN_INTERFACE_SHADER:
        return sc.LambertianInterfaceMaterial(color=_v3(p.get("diffuse_color", (1.0, 1.0, 1.0))), ior=p.get("ior", 1.3))
    if kind == sc.ROUGH_DIFFUSE_SHADER:
        m = sc.RoughDiffuseMaterial()
        return sc.RoughDiffuseMaterial(color=_v3(p.get("diffuse_color", m.color)), ior=p.get("ior", m.ior),
                                       roughness=tuple(p.get("roughness", m.roughness))[:2],
                                       microfacet_model=p.get("microfacet_model", m.microfacet_model),
                                       normal_distribution=p.get("normal_distribution", m.normal_distribution))
    cls = sc.TranslucentMaterial if kind == sc.TRANSLUCENT_SHADER else sc.RoughTranslucentMaterial
    kw = {}
    for key in ("scattering", "absorption", "meancosine"):
        if key in p:
            kw[key] = _v3(p[key])
    for key in ("ior", "scale", "dipole_model"):
        if key in p:
            kw[key] = p[key]
    if cls is sc.RoughTranslucentMaterial:
        for key in ("microfacet_model", "normal_distribution"):
            if key in p:
                kw[key] = p[key]
        if "roughness" in p:
            kw["roughness"] = tuple(p["roughness"])[:2]
    return cls(**kw)


def _light_from_json(obj, base_dir):
    kind = obj.get("type", "")
    p = obj.get("parameters", {})
    rad = _v3(p.get("radiance", (1.0, 1.0, 1.0)))
    k = kind.lower()
    if k == "pointlight":
        return sc.PointLight(_v3(p.get("position", (0.0, 0.0, 0.0))), rad)
    if k == "directionallight":
        return sc.DirectionalLight(_v3(p.get("direction", (0.0, -1.0, 0.0))), rad)
    if k == "diskarealight":
        return sc.DiskAreaLight(_v3(p.get("position", (0.0, 0.0, 0.0))), rad, p.get("radius", 1.0), p.get("theta", 0.0), p.get("phi", 0.0))
    if k == "sphericallight":
        return sc.SphericalLight(_v3(p.get("position", (0.0, 0.0, 0.0))), rad, p.get("radius", 0.05))
    if k == "trianglesarealight":  # an OBJ mesh as emitter (TriangleAreaLight::readJSON, Light.cpp:149-220)
        A, t = geometry_transform(p)
        meshes = sc.load_obj(os.path.join(base_dir, p["path"]))
        pos, idx = [], []
        base = 0
        for m in meshes:
            tm = _transform_mesh(m, A, t)
            pos.append(tm.positions)
            idx.append(tm.vindex + base)
            base += len(tm.positions)
        return sc.TriangleAreaLight(np.concatenate(pos), np.concatenate(idx), rad)
    raise ValueError("unsupported light type %r" % kind)


class JsonScene:
    """A scene read from a JSON file: `data` (SceneData), the saved `frame_count` and the absolute path
    of the saved accumulation buffer (`buffer_path`, or None)."""

    def __init__(self, data, frame_count, buffer_path, document, path):
        self.data, self.frame_count, self.buffer_path = data, frame_count, buffer_path
        self.document, self.path = document, path


def load_json_scene(path, base_dir=None, rr_start_depth=0, unsupported_material=None):
    """OptixSceneLoader::readJSON (OptixSceneLoader.cpp:105-180) into a SceneData."""
    with open(path) as f:
        doc = json.load(f)
    base_dir = base_dir or os.path.dirname(os.path.abspath(path))
    ip = doc.get("Integrator", {})
    if ip.get("type", "PathTracer").lower() != "pathtracer":
        raise ValueError("integrator %r is outside the path tracer" % ip.get("type"))
    p = ip.get("parameters", {})
    integrator = sc.PathTracer(max_depth=p.get("max_depth", 50), scene_epsilon=p.get("scene_epsilon", 1e-4),
                               exception_color=_v3(p.get("exception_color", (1.0, 0.0, 0.0))), rr_start_depth=rr_start_depth)
    cp = doc.get("Camera", {}).get("parameters", {})
    w, h = int(cp.get("width", 512)), int(cp.get("height", 512))
    camera = sc.PinholeCamera(eye=_v3(cp.get("eye", (0.0, 0.0, 0.0))), lookat=_v3(cp.get("lookat", (0.0, 0.0, -1.0))),
                              up=_v3(cp.get("up", (0.0, 1.0, 0.0))), vfov=cp.get("vfov", 60.0), width=w, height=h,
                              patch_origin=tuple(cp.get("patch_origin", (0, 0))), patch_dims=tuple(cp.get("patch_dims", (w, h))))
    bg = doc.get("Background", {})
    bp = bg.get("parameters", {})
    if bg.get("type", "ConstantBackground").lower() == "envmapbackground" and "path" in bp:
        background = sc.EnvMapBackground(path=os.path.join(base_dir, bp["path"]))
    else:
        background = sc.ConstantBackground(_v3(bp.get("background_color", (1.0, 1.0, 1.0))))
    meshes = []
    for g in doc.get("Geometries", []):
        if g.get("type", "obj").lower() != "obj":
            raise ValueError("geometry type %r is not supported" % g.get("type"))
        gp = g.get("parameters", {})
        A, t = geometry_transform(gp)
        mat = material_from_json(gp["material"], unsupported_material) if "material" in gp else None
        for m in sc.load_obj(os.path.join(base_dir, gp["path"]), material=mat):
            meshes.append(_transform_mesh(m, A, t))
    lights = [_light_from_json(L, base_dir) for L in doc.get("Lights", [])]
    data = sc.SceneData(integrator, camera, background, meshes, lights)
    buffer_path = os.path.join(base_dir, doc["buffer_path"]) if "buffer_path" in doc else None
    return JsonScene(data, int(doc.get("frame_count", 0)), buffer_path, doc, path)


def save_checkpoint(renderer, json_path, document):
    """OptixScene::saveScene (OptixScene.cpp:200-232): writes the scene document to `json_path` itself,
    with "frame_count" (the frames rendered so far) and "buffer_path" (a .raw file of width * height
    float4 beside it, written from the context's accumulation buffer).  `document` is the scene's JSON
    document (a JsonScene or its `document` dict), so that the saved file reloads as a complete scene
    through load_json_scene, as the reference's saved scenes do."""
    if isinstance(document, JsonScene):
        document = document.document
    if not isinstance(document, dict) or not document:
        raise ValueError("save_checkpoint needs the scene document (JsonScene.document) so that the file reloads as a scene")
    raw = os.path.splitext(json_path)[0] + ".raw"
    img = renderer.readback()
    np.ascontiguousarray(img, np.float32).tofile(raw)
    doc = dict(document)
    doc["frame_count"] = int(renderer.frame)
    doc["buffer_path"] = os.path.basename(raw)
    with open(json_path, "w") as f:
        json.dump(doc, f, indent=1)
    return json_path


def load_checkpoint(renderer, json_path):
    """OptixScene::loadScene / loadBuffer (OptixScene.cpp:235-298): restores the accumulation buffer and
    the frame count, so the next render continues the running mean at frame `frame_count`."""
    with open(json_path) as f:
        doc = json.load(f)
    raw = os.path.join(os.path.dirname(os.path.abspath(json_path)), doc["buffer_path"])
    W, H = renderer.data.camera.width, renderer.data.camera.height
    img = np.fromfile(raw, np.float32)
    if img.size != W * H * 4:
        raise ValueError("%s holds %d floats, the camera needs %d" % (raw, img.size, W * H * 4))
    frames = int(doc.get("frame_count", 0))
    nat.call("pt_set_accumulation", renderer.ctx, img.ctypes.data, frames)
    renderer.frame = frames
    return frames
