"""Scene-object API of the reference, over the C ABI.

The reference's host classes write OptiX variables; these write the same parameters through
include/orf_b200.h.  Class and setter names follow the reference (Integrator.h, Camera.h,
Background.h, Light.h, Material.h); ``Renderer`` plays the part of OptixScene (OptixScene.h) and
its ``renderScene`` mirrors OptixScene::renderScene (OptixScene.cpp:139-168): one frame per call,
`frame` incremented, the result folded into the running mean.

Invalid parameters raise ``PtError`` (status PT_INVALID_ARG) from the native library, which checks
every value before any device work.
"""
import ctypes
import math
import os

import numpy as np

from . import _native as nat

# ---------------------------------------------------------------- enums (structs.h)
DIFFUSE_SHADER = 0
TRANSPARENT_SHADER = 2
ROUGH_TRANSPARENT_SHADER = 3
METALLIC_SHADER = 4
TRANSLUCENT_SHADER = 5
ROUGH_TRANSLUCENT_SHADER = 6
LAMBERTIAN_INTERFACE_SHADER = 7
ROUGH_DIFFUSE_SHADER = 9
AREA_LIGHT_MATERIAL = 100
STANDARD_DIPOLE, DIRECTIONAL_DIPOLE = 0, 1
WALTER_MODEL, VISIBLE_NORMALS_MODEL, MULTISCATTERING_MODEL = 0, 1, 2
BECKMANN_DISTRIBUTION, GGX_DISTRIBUTION = 0, 1
POINT_LIGHT, DIRECTIONAL_LIGHT, TRIANGLES_AREA_LIGHT, DISK_LIGHT, SPHERICAL_LIGHT = 0, 1, 2, 3, 4


class DiffuseParams(ctypes.Structure):
    _fields_ = [("diffuse_color", ctypes.c_float * 3)]


class MetallicParams(ctypes.Structure):
    _fields_ = [("ior", ctypes.c_double * 6), ("roughness", ctypes.c_float * 2), ("microfacet_model", ctypes.c_uint32),
                ("normal_distribution", ctypes.c_uint32)]


class RoughTransparentParams(ctypes.Structure):
    _fields_ = [("ior", ctypes.c_float), ("roughness", ctypes.c_float), ("glass_absorption", ctypes.c_float * 3),
                ("microfacet_model", ctypes.c_uint32), ("normal_distribution", ctypes.c_uint32)]


class TransparentParams(ctypes.Structure):
    _fields_ = [("ior", ctypes.c_float), ("glass_absorption", ctypes.c_float * 3)]


class LambertianInterfaceParams(ctypes.Structure):
    _fields_ = [("diffuse_color", ctypes.c_float * 3), ("ior", ctypes.c_float)]


class RoughDiffuseParams(ctypes.Structure):
    _fields_ = [("diffuse_color", ctypes.c_float * 3), ("ior", ctypes.c_float), ("roughness", ctypes.c_float * 2),
                ("microfacet_model", ctypes.c_uint32), ("normal_distribution", ctypes.c_uint32)]


class AreaLightParams(ctypes.Structure):
    _fields_ = [("radiance", ctypes.c_float * 3)]


class TranslucentParams(ctypes.Structure):
    _fields_ = [("scattering", ctypes.c_float * 3), ("absorption", ctypes.c_float * 3), ("meancosine", ctypes.c_float * 3),
                ("ior", ctypes.c_float), ("scale", ctypes.c_float), ("dipole_model", ctypes.c_uint32)]


class BuildInfo(ctypes.Structure):
    """pt_build_info: the acceleration structure of the last pt_build."""
    _fields_ = [("builder", ctypes.c_uint32), ("n_triangles", ctypes.c_uint32), ("bvh2_nodes", ctypes.c_uint32), ("bvh2_depth", ctypes.c_uint32),
                ("wide_nodes", ctypes.c_uint32), ("wide_depth", ctypes.c_uint32), ("build_ms", ctypes.c_float), ("device_ms", ctypes.c_float),
                ("sah_cost", ctypes.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class MicrofacetBatch(ctypes.Structure):
    """pt_microfacet_batch: one batch of multiscattering-walk / conductor-Fresnel queries."""
    _fields_ = [("op", ctypes.c_uint32), ("normal_distribution", ctypes.c_uint32), ("normal", ctypes.c_float * 3), ("eta", ctypes.c_float),
                ("ior", ctypes.c_double * 6), ("rho", ctypes.c_float * 3)]


MSQ_OPS = {"dielectric_eval": 0, "dielectric_sample": 1, "conductor_eval": 2, "conductor_sample": 3, "diffuse_eval": 4,
           "diffuse_sample": 5, "conductor_fresnel": 6, "visible_normal": 7}


class RoughTranslucentParams(ctypes.Structure):
    _fields_ = [("scattering", ctypes.c_float * 3), ("absorption", ctypes.c_float * 3), ("meancosine", ctypes.c_float * 3),
                ("ior", ctypes.c_float), ("scale", ctypes.c_float), ("dipole_model", ctypes.c_uint32), ("roughness", ctypes.c_float * 2),
                ("microfacet_model", ctypes.c_uint32), ("normal_distribution", ctypes.c_uint32)]


# ScatteringMaterialProperties (structs.h:116-144, 260 bytes) and PositionSample (:105-114, 80 bytes).
SCATTERING_PROPERTIES_DTYPE = np.dtype([(name, "<f4", 3) if name not in ("relative_ior", "mean_transport") else (name, "<f4")
                                        for name in ("relative_ior", "ior_real", "ior_imag", "absorption", "scattering", "meancosine",
                                                     "extinction", "reducedExtinction", "deltaEddExtinction", "D", "transport", "C_phi",
                                                     "C_phi_inv", "C_E", "A", "albedo", "reducedAlbedo", "de", "three_D", "two_A_de",
                                                     "global_coeff", "one_over_three_ext", "mean_transport")])
POSITION_SAMPLE_DTYPE = np.dtype([("pos", "<f4", 3), ("dir", "<f4", 3), ("normal", "<f4", 3), ("L", "<f4", 3), ("transmitted", "<f4", 3),
                                  ("weight", "<f4", 3), ("padding", "<f4", 2)])
assert SCATTERING_PROPERTIES_DTYPE.itemsize == 260 and POSITION_SAMPLE_DTYPE.itemsize == 80


class RenderStats(ctypes.Structure):
    _fields_ = [("path_samples", ctypes.c_uint64), ("segments", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("capped_walks", ctypes.c_uint64), ("clamped_indices", ctypes.c_uint64), ("gpu_ms", ctypes.c_float),
                ("extend_ms", ctypes.c_float), ("extend_launches", ctypes.c_uint32), ("kernel_launches", ctypes.c_uint32),
                ("dipole_gathers", ctypes.c_uint64), ("dipole_pairs", ctypes.c_uint64), ("gather_overflows", ctypes.c_uint64),
                ("gather_ms", ctypes.c_float)]


# LightStruct (40 B) and TriangleLight (92 B), structs.h:42-103, as numpy record types.
LIGHT_DTYPE = np.dtype([("light_type", "<u4"), ("emitted_radiance", "<f4", 3), ("p", "<f4", 3), ("padding", "<f4", 3)])
TRIANGLE_LIGHT_DTYPE = np.dtype([("v0", "<f4", 3), ("v1", "<f4", 3), ("v2", "<f4", 3), ("n0", "<f4", 3), ("n1", "<f4", 3),
                                 ("n2", "<f4", 3), ("has_normals", "<u4"), ("emission", "<f4", 3), ("area", "<f4")])
assert LIGHT_DTYPE.itemsize == 40 and TRIANGLE_LIGHT_DTYPE.itemsize == 92


def _f3(v):
    return (ctypes.c_float * 3)(*[float(x) for x in v])


# ---------------------------------------------------------------- Integrator.h
class PathTracer:
    """PathTracer (Integrator.cpp:6-24 defaults: max_depth 50, scene_epsilon 1e-4, red exception)."""

    def __init__(self, max_depth=50, scene_epsilon=1e-4, exception_color=(1.0, 0.0, 0.0), rr_start_depth=0):
        self.max_depth = int(max_depth)
        self.scene_epsilon = float(scene_epsilon)
        self.exception_color = tuple(exception_color)
        self.rr_start_depth = int(rr_start_depth)

    def setMaxDepth(self, d):
        self.max_depth = int(d)

    def setSceneEpsilon(self, e):
        self.scene_epsilon = float(e)

    def setExceptionColor(self, c):
        self.exception_color = tuple(c)

    def getMaxDepth(self):
        return self.max_depth

    def getSceneEpsilon(self):
        return self.scene_epsilon


# ---------------------------------------------------------------- Camera.h
class PinholeCamera:
    """PinholeCamera: eye / lookat / up / vfov -> U, V, W as PinholeCamera::calculateCameraVariables
    (Camera.cpp:83-103): W = lookat - eye (not normalised), U = |W| tan(vfov/2) aspect * unit(W x up),
    V = |W| tan(vfov/2) * unit(U x W)."""

    def __init__(self, eye, lookat, up, vfov, width, height, patch_origin=(0, 0), patch_dims=None):
        self.eye = np.asarray(eye, np.float32)
        self.lookat = np.asarray(lookat, np.float32)
        self.up = np.asarray(up, np.float32)
        self.vfov = float(vfov)
        self.width = int(width)
        self.height = int(height)
        self.patch_origin = tuple(int(x) for x in patch_origin)
        self.patch_dims = tuple(int(x) for x in (patch_dims or (width, height)))
        self.calculateCameraVariables()

    def calculateCameraVariables(self):
        W = (self.lookat - self.eye).astype(np.float32)
        wlen = np.float32(np.linalg.norm(W.astype(np.float64)))
        U = np.cross(W.astype(np.float64), self.up.astype(np.float64))
        U = (U / np.linalg.norm(U)).astype(np.float32)
        V = np.cross(U.astype(np.float64), W.astype(np.float64))
        V = (V / np.linalg.norm(V)).astype(np.float32)
        vlen = np.float32(wlen * np.float32(math.tan(0.5 * self.vfov * math.pi / 180.0)))
        V = (V * vlen).astype(np.float32)
        ulen = np.float32(vlen * np.float32(self.width / self.height))
        U = (U * ulen).astype(np.float32)
        self.U, self.V, self.W = U, V, W

    def setEye(self, e):
        self.eye = np.asarray(e, np.float32)
        self.calculateCameraVariables()

    def setLookat(self, l):
        self.lookat = np.asarray(l, np.float32)
        self.calculateCameraVariables()

    def setUp(self, u):
        self.up = np.asarray(u, np.float32)
        self.calculateCameraVariables()

    def setFov(self, f):
        self.vfov = float(f)
        self.calculateCameraVariables()

    def resizeCamera(self, width, height):
        self.width, self.height = int(width), int(height)
        self.patch_dims = (self.width, self.height)
        self.calculateCameraVariables()


# ---------------------------------------------------------------- Background.h
class ConstantBackground:
    def __init__(self, background_color=(1.0, 1.0, 1.0)):
        self.background_color = tuple(background_color)

    def setBackgroundColor(self, c):
        self.background_color = tuple(c)


def read_hdr(path):
    """A Radiance RGBE file decoded on the host (pt_hdr_read): float4 texels [H, W, 4], row 0 = the file's
    last scanline, as loadHDRTexture orients it (HDRLoader.cpp:225-290)."""
    w, h = ctypes.c_uint32(), ctypes.c_uint32()
    nat.call("pt_hdr_read", os.fsencode(path), None, 0, ctypes.byref(w), ctypes.byref(h))
    out = np.empty((h.value, w.value, 4), np.float32)
    nat.call("pt_hdr_read", os.fsencode(path), out.ctypes.data, out.size, ctypes.byref(w), ctypes.byref(h))
    return out


class EnvMapBackground:
    """EnvMapBackground (Background.cpp:57-69): float4 texels [H, W, 4], row 0 at v = 0, or a Radiance
    .hdr file given by `path` (the reference's loadTexture path), which the renderer uploads as RGBE and
    expands on the device (pt_set_envmap_hdr); `rgba` then holds the same texels decoded on the host."""

    def __init__(self, rgba=None, path=None):
        self.path = None if path is None else os.fspath(path)
        if self.path is not None:
            rgba = read_hdr(self.path)
        self.rgba = np.ascontiguousarray(rgba, np.float32)
        assert self.rgba.ndim == 3 and self.rgba.shape[2] == 4


class EnvMapLight:
    """The environment map as a light in light_buffer (light_type 5, sampled with
    sample_environment of Envmap.h:66-98): diffuse next-event estimation picks it like any light."""


# ---------------------------------------------------------------- Material.h
class _Textured:
    """Optional per-texel parameter: a texture [H, W, C] read at the nearest texel of a cube map around
    `texture_center` (pt_material_set_texture)."""
    texture = None
    texture_center = (0.0, 0.0, 0.0)

    def setTexture(self, texture, center=(0.0, 0.0, 0.0)):
        self.texture = None if texture is None else np.ascontiguousarray(texture, np.float32)
        self.texture_center = tuple(float(x) for x in center)


class DiffuseMaterial(_Textured):
    """diffuse_color; setTexture(albedo [H, W, 3], center) makes it per texel."""
    type = DIFFUSE_SHADER

    def __init__(self, color=(0.8, 0.8, 0.8)):
        self.color = tuple(color)

    def params(self):
        return DiffuseParams(_f3(self.color))

    def setColor(self, c):
        self.color = tuple(c)


class MetallicMaterial(_Textured):
    """Conductor with complex IOR per RGB (MyComplex3); defaults of MetallicMaterial.cpp:7-26
    (gold, roughness 0.1, Walter model, Beckmann distribution).  setTexture(roughness [H, W], center)
    makes the (isotropic) roughness per texel."""
    type = METALLIC_SHADER
    GOLD = ((0.170265, 3.01893), (0.511516, 2.44734), (1.47544, 1.87263))  # Material.h:328

    def __init__(self, ior=GOLD, roughness=(0.1, 0.1), microfacet_model=WALTER_MODEL, normal_distribution=BECKMANN_DISTRIBUTION):
        self.ior = tuple(tuple(float(x) for x in c) for c in ior)
        self.roughness = tuple(float(x) for x in roughness)
        self.microfacet_model = int(microfacet_model)
        self.normal_distribution = int(normal_distribution)

    def params(self):
        flat = [v for c in self.ior for v in c]
        return MetallicParams((ctypes.c_double * 6)(*flat), (ctypes.c_float * 2)(*self.roughness), self.microfacet_model,
                              self.normal_distribution)

    def setIor(self, ior):
        self.ior = tuple(tuple(float(x) for x in c) for c in ior)

    def setRoughness(self, r):
        self.roughness = tuple(float(x) for x in r)

    def setMicrofacetModel(self, m):
        self.microfacet_model = int(m)

    def setNormalDistribution(self, d):
        self.normal_distribution = int(d)


class RoughTransparentMaterial:
    """Rough dielectric; defaults of RoughTransparentMaterial.cpp:7-28 (ior 1.3, roughness 0.1,
    no absorption, Walter model, Beckmann distribution)."""
    type = ROUGH_TRANSPARENT_SHADER

    def __init__(self, ior=1.3, roughness=0.1, glass_absorption=(0.0, 0.0, 0.0), microfacet_model=WALTER_MODEL,
                 normal_distribution=BECKMANN_DISTRIBUTION):
        self.ior = float(ior)
        self.roughness = float(roughness)
        self.glass_absorption = tuple(glass_absorption)
        self.microfacet_model = int(microfacet_model)
        self.normal_distribution = int(normal_distribution)

    def params(self):
        return RoughTransparentParams(self.ior, self.roughness, _f3(self.glass_absorption), self.microfacet_model,
                                      self.normal_distribution)


class TransparentMaterial:
    """Smooth glass (TransparentMaterial.cpp:7-20, shader transparent_shader.cu): mtl["ior"] and
    mtl["glass_absorption"]; defaults ior 1.3, no absorption."""
    type = TRANSPARENT_SHADER

    def __init__(self, ior=1.3, glass_absorption=(0.0, 0.0, 0.0)):
        self.ior = float(ior)
        self.glass_absorption = tuple(float(x) for x in glass_absorption)

    def params(self):
        return TransparentParams(self.ior, _f3(self.glass_absorption))

    def setIor(self, i):
        self.ior = float(i)

    def setAbsorption(self, a):
        self.glass_absorption = tuple(float(x) for x in a)


class LambertianInterfaceMaterial:
    """Lambertian base under a smooth dielectric interface (LambertianInterfaceMaterial.cpp:7-20,
    shader lambertian_interface_shader.cu): mtl["diffuse_color"], mtl["ior"]; defaults 1 and 1.3."""
    type = LAMBERTIAN_INTERFACE_SHADER

    def __init__(self, color=(1.0, 1.0, 1.0), ior=1.3):
        self.color = tuple(float(x) for x in color)
        self.ior = float(ior)

    def params(self):
        return LambertianInterfaceParams(_f3(self.color), self.ior)

    def setColor(self, c):
        self.color = tuple(float(x) for x in c)

    def setIor(self, i):
        self.ior = float(i)


class RoughDiffuseMaterial:
    """Lambertian base under a rough dielectric interface (RoughDiffuseMaterial.cpp:7-28, shader
    rough_diffuse_shader.cu): mtl["diffuse_color"], mtl["ior"], mtl["roughness"],
    mtl["normal_distribution"], mtl["microfacet_model"]; defaults 1, 1.3, (0.1, 0.1), Beckmann, Walter."""
    type = ROUGH_DIFFUSE_SHADER

    def __init__(self, color=(1.0, 1.0, 1.0), ior=1.3, roughness=(0.1, 0.1), microfacet_model=WALTER_MODEL,
                 normal_distribution=BECKMANN_DISTRIBUTION):
        self.color = tuple(float(x) for x in color)
        self.ior = float(ior)
        self.roughness = tuple(float(x) for x in roughness)
        self.microfacet_model = int(microfacet_model)
        self.normal_distribution = int(normal_distribution)

    def params(self):
        return RoughDiffuseParams(_f3(self.color), self.ior, (ctypes.c_float * 2)(*self.roughness), self.microfacet_model,
                                  self.normal_distribution)

    def setColor(self, c):
        self.color = tuple(float(x) for x in c)

    def setIor(self, i):
        self.ior = float(i)

    def setRoughness(self, r):
        self.roughness = tuple(float(x) for x in r)

    def setMicrofacetModel(self, m):
        self.microfacet_model = int(m)

    def setNormalDistribution(self, d):
        self.normal_distribution = int(d)


class TranslucentMaterial:
    """Smooth translucent surface with the dipole BSSRDF (TranslucentMaterial.cpp, shader
    subsurface_scattering_shader.cu).  Coefficients per RGB channel in 1/mm, scaled by `scale` to
    scene units; defaults: the "Apple" entry of getDefaultMaterial (TranslucentMaterial.cpp:245-250),
    scale 100, standard dipole (:7-19)."""
    type = TRANSLUCENT_SHADER

    def __init__(self, scattering=(2.29, 2.39, 1.97), absorption=(0.0030, 0.0034, 0.0046), meancosine=(0.0, 0.0, 0.0), ior=1.3,
                 scale=100.0, dipole_model=STANDARD_DIPOLE):
        self.scattering = tuple(float(x) for x in scattering)
        self.absorption = tuple(float(x) for x in absorption)
        self.meancosine = tuple(float(x) for x in meancosine)
        self.ior = float(ior)
        self.scale = float(scale)
        self.dipole_model = int(dipole_model)

    def params(self):
        return TranslucentParams(_f3(self.scattering), _f3(self.absorption), _f3(self.meancosine), self.ior, self.scale, self.dipole_model)

    def setIor(self, i):
        self.ior = float(i)

    def setScale(self, s):
        self.scale = float(s)

    def setAbsorption(self, a):
        self.absorption = tuple(float(x) for x in a)

    def setScattering(self, s):
        self.scattering = tuple(float(x) for x in s)

    def setMeanCosine(self, m):
        self.meancosine = tuple(float(x) for x in m)

    def setDipoleModel(self, m):
        self.dipole_model = int(m)


class RoughTranslucentMaterial(TranslucentMaterial):
    """Rough translucent surface (RoughTranslucentMaterial.cpp, shader rough_subsurface_scattering_shader.cu):
    the dipole BSSRDF behind a rough dielectric boundary with mtl["roughness"], mtl["microfacet_model"]
    and mtl["normal_distribution"] (defaults: roughness 0.1, Walter model, Beckmann distribution)."""
    type = ROUGH_TRANSLUCENT_SHADER

    def __init__(self, roughness=(0.1, 0.1), microfacet_model=WALTER_MODEL, normal_distribution=BECKMANN_DISTRIBUTION, **kw):
        super().__init__(**kw)
        self.roughness = tuple(float(x) for x in roughness)
        self.microfacet_model = int(microfacet_model)
        self.normal_distribution = int(normal_distribution)

    def params(self):
        return RoughTranslucentParams(_f3(self.scattering), _f3(self.absorption), _f3(self.meancosine), self.ior, self.scale, self.dipole_model,
                                      (ctypes.c_float * 2)(*self.roughness), self.microfacet_model, self.normal_distribution)

    def setRoughness(self, r):
        self.roughness = tuple(float(x) for x in r)


class AreaLightMaterial:
    """The emitter program TriangleAreaLight attaches to its geometry (arealight_shader.cu)."""
    type = AREA_LIGHT_MATERIAL

    def __init__(self, radiance):
        self.radiance = tuple(radiance)

    def params(self):
        return AreaLightParams(_f3(self.radiance))


# ---------------------------------------------------------------- Light.h
class TriangleAreaLight:
    """TriangleAreaLight: an emitting triangle mesh.  Produces its LightStruct (triangle_count /
    buffer_start_idx / buffer_end_idx stored as float, structs.h:66-74), its TriangleLight records
    (area = 0.5 |(v1-v0) x (v2-v0)|, Light.cpp:286-297) and the emitter geometry."""

    def __init__(self, positions, vindex, radiance):
        self.positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        self.vindex = np.ascontiguousarray(vindex, np.int32).reshape(-1, 3)
        self.radiance = tuple(float(x) for x in radiance)

    def triangle_records(self):
        recs = np.zeros(len(self.vindex), TRIANGLE_LIGHT_DTYPE)
        for k, (a, b, c) in enumerate(self.vindex):
            v0, v1, v2 = self.positions[a], self.positions[b], self.positions[c]
            recs[k]["v0"], recs[k]["v1"], recs[k]["v2"] = v0, v1, v2
            recs[k]["has_normals"] = 0
            recs[k]["emission"] = self.radiance
            perp = np.cross((v1 - v0).astype(np.float32), (v2 - v0).astype(np.float32)).astype(np.float32)
            recs[k]["area"] = np.float32(0.5 * float(np.sqrt(np.float32(np.dot(perp, perp)))))
        return recs


class PointLight:
    def __init__(self, position, radiance):
        self.position, self.radiance = tuple(position), tuple(radiance)


class DirectionalLight:
    def __init__(self, direction, radiance):
        self.direction, self.radiance = tuple(direction), tuple(radiance)


class DiskAreaLight:
    """DiskAreaLight (Light.cpp:370-503): a one-sided emitting disk at `position` with `radius`, facing
    the normal (sin theta sin phi, cos theta, sin theta cos phi) for theta / phi in degrees; defaults
    of the reference's constructor.  Sampled for next-event estimation (LightSampler.h:73-100) and
    intersected as analytic geometry (disk_mesh.cu) with the area-light emitter program."""

    def __init__(self, position=(0.0, 0.0, 0.0), radiance=(1.0, 1.0, 1.0), radius=1.0, theta=0.0, phi=0.0):
        self.position = tuple(float(x) for x in position)
        self.radiance = tuple(float(x) for x in radiance)
        self.radius = float(radius)
        self.theta = float(theta)
        self.phi = float(phi)

    def setPosition(self, p):
        self.position = tuple(float(x) for x in p)

    def setRadiance(self, r):
        self.radiance = tuple(float(x) for x in r)

    def setRadius(self, r):
        self.radius = float(r)

    def setNormal(self, theta, phi):
        self.theta, self.phi = float(theta), float(phi)


class SphericalLight:
    """SphericalLight (Light.cpp:505-610): an emitting sphere (default radius 0.05), sampled on the
    hemisphere facing the shaded point (LightSampler.h:103-141) and intersected as analytic geometry
    (sphere_mesh.cu) with the area-light emitter program."""

    def __init__(self, position=(0.0, 0.0, 0.0), radiance=(1.0, 1.0, 1.0), radius=0.05):
        self.position = tuple(float(x) for x in position)
        self.radiance = tuple(float(x) for x in radiance)
        self.radius = float(radius)

    def setPosition(self, p):
        self.position = tuple(float(x) for x in p)

    def setRadiance(self, r):
        self.radiance = tuple(float(x) for x in r)

    def setRadius(self, r):
        self.radius = float(r)


def light_buffers(lights):
    """light_buffer and triangle_light_buffer for a list of lights (OptixSceneLoader.cpp:284-347)."""
    ls = np.zeros(len(lights), LIGHT_DTYPE)
    tri_recs = []
    start = 0
    for k, L in enumerate(lights):
        if isinstance(L, TriangleAreaLight):
            recs = L.triangle_records()
            ls[k]["light_type"] = TRIANGLES_AREA_LIGHT
            ls[k]["emitted_radiance"] = L.radiance
            ls[k]["p"] = (float(len(recs)), float(start), float(start + len(recs) - 1))
            tri_recs.append(recs)
            start += len(recs)
        elif isinstance(L, PointLight):
            ls[k]["light_type"] = POINT_LIGHT
            ls[k]["emitted_radiance"] = L.radiance
            ls[k]["p"] = L.position
        elif isinstance(L, EnvMapLight):
            ls[k]["light_type"] = 5
            ls[k]["emitted_radiance"] = (1.0, 1.0, 1.0)
        elif isinstance(L, DiskAreaLight):  # DiskLightStruct: position, radius, phi, theta (structs.h:76-84)
            ls[k]["light_type"] = DISK_LIGHT
            ls[k]["emitted_radiance"] = L.radiance
            ls[k]["p"] = L.position
            ls[k]["padding"] = (L.radius, L.phi, L.theta)
        elif isinstance(L, SphericalLight):  # SphericalLightStruct: position, radius (structs.h:86-93)
            ls[k]["light_type"] = SPHERICAL_LIGHT
            ls[k]["emitted_radiance"] = L.radiance
            ls[k]["p"] = L.position
            ls[k]["padding"] = (L.radius, 0.0, 0.0)
        elif isinstance(L, DirectionalLight):
            ls[k]["light_type"] = DIRECTIONAL_LIGHT
            ls[k]["emitted_radiance"] = L.radiance
            d = np.asarray(L.direction, np.float32)
            ls[k]["p"] = d / np.float32(np.linalg.norm(d))
        else:
            raise TypeError("unsupported light %r" % (L,))
    tris = np.concatenate(tri_recs) if tri_recs else np.zeros(0, TRIANGLE_LIGHT_DTYPE)
    return ls, tris


class Mesh:
    """A triangle mesh with one material (the OBJGeometry buffers of ObjLoader.cpp:278-373)."""

    def __init__(self, positions, vindex, material, normals=None, nindex=None):
        self.positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        self.vindex = np.ascontiguousarray(vindex, np.int32).reshape(-1, 3)
        self.normals = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        self.nindex = None if nindex is None else np.ascontiguousarray(nindex, np.int32).reshape(-1, 3)
        self.material = material


class ObjGroup(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 128), ("material", ctypes.c_char * 128), ("first_triangle", ctypes.c_uint32),
                ("n_triangles", ctypes.c_uint32), ("diffuse", ctypes.c_float * 3), ("has_diffuse", ctypes.c_int32)]


def load_obj(path, material=None, materials=None):
    """The groups of a Wavefront OBJ file (pt_obj_read: glm's reader as ObjLoader flattens it) as Meshes:
    one per non-empty group, sharing the file's vertex and normal arrays.  A group's material is
    materials[<usemtl name>] if given, else `material`, else a DiffuseMaterial of the group's Kd."""
    obj = ctypes.c_void_p()
    nat.call("pt_obj_read", os.fsencode(path), ctypes.byref(obj))
    try:
        info = (ctypes.c_uint32 * 5)()
        nat.call("pt_obj_get_info", obj, info)
        nv, nn, nt, ntri, ng = list(info)
        pos = np.zeros((nv, 3), np.float32)
        nrm = np.zeros((max(nn, 1), 3), np.float32)
        vidx = np.zeros((ntri, 3), np.int32)
        nidx = np.zeros((ntri, 3), np.int32)
        nat.call("pt_obj_get_arrays", obj, pos.ctypes.data, nrm.ctypes.data if nn else None, None, vidx.ctypes.data, nidx.ctypes.data,
                 None, None)
        meshes = []
        for k in range(ng):
            g = ObjGroup()
            nat.call("pt_obj_get_group", obj, k, ctypes.byref(g))
            name = g.material.decode()
            mat = (materials or {}).get(name) or material or DiffuseMaterial(tuple(g.diffuse))
            tri = slice(g.first_triangle, g.first_triangle + g.n_triangles)
            ni = nidx[tri]
            meshes.append(Mesh(pos, vidx[tri], mat, nrm if nn and np.all(ni >= 0) else None, ni if nn and np.all(ni >= 0) else None))
        return meshes
    finally:
        nat.call("pt_obj_free", obj)


# ---------------------------------------------------------------- scene flattening
class SceneData:
    """Everything a render needs, flattened in one fixed order that the GPU context and the CPU
    oracle both use: materials are numbered in order of first use (meshes first, then the emitter
    materials of TriangleAreaLights); triangles follow mesh order, then the lights' emitter meshes."""

    def __init__(self, integrator, camera, background, meshes, lights, probe_samples=500):
        self.integrator, self.camera, self.background = integrator, camera, background
        self.probe_samples = int(probe_samples)  # context["samples"] (OptixSceneLoader.cpp:11-17)
        self.lights = list(lights)
        self.meshes = list(meshes)
        for L in self.lights:
            if isinstance(L, TriangleAreaLight):
                self.meshes.append(Mesh(L.positions, L.vindex, AreaLightMaterial(L.radiance)))
        self.materials = []
        index = {}
        self.mesh_material = []
        for m in self.meshes:
            if id(m.material) not in index:
                index[id(m.material)] = len(self.materials)
                self.materials.append(m.material)
            self.mesh_material.append(index[id(m.material)])
        self.light_buffer, self.triangle_light_buffer = light_buffers(self.lights)

    def translucent_objects(self):
        """(material index, first triangle, triangle count) of every mesh with a translucent material,
        in mesh order (OptixSceneLoader::computeTranslucentGeometries)."""
        out, first = [], 0
        for m, mid in zip(self.meshes, self.mesh_material):
            if getattr(m.material, "type", None) in (TRANSLUCENT_SHADER, ROUGH_TRANSLUCENT_SHADER):
                out.append((mid, first, len(m.vindex)))
            first += len(m.vindex)
        return out

    @property
    def n_triangles(self):
        return sum(len(m.vindex) for m in self.meshes)

    def flat_triangles(self):
        """(tri_pos [T,9] float32, tri_info [T,4] int32, normals [N,3] float32) as pt_mesh_add stores them."""
        pos, info, nrm = [], [], []
        nbase = 0
        for m, mid in zip(self.meshes, self.mesh_material):
            pos.append(m.positions[m.vindex].reshape(-1, 9))
            inf = np.full((len(m.vindex), 4), -1, np.int32)
            inf[:, 3] = mid
            if m.normals is not None:
                ok = np.all(m.nindex >= 0, axis=1)
                inf[ok, :3] = m.nindex[ok] + nbase
                nrm.append(m.normals)
                nbase += len(m.normals)
            info.append(inf)
        normals = np.concatenate(nrm).astype(np.float32) if nrm else np.zeros((0, 3), np.float32)
        return np.ascontiguousarray(np.concatenate(pos), np.float32), np.ascontiguousarray(np.concatenate(info)), normals


# ---------------------------------------------------------------- OptixScene
class Renderer:
    """Owns a pt_ctx and plays the part of OptixScene: scene setup, build, renderScene()."""

    def __init__(self, data, device=0, max_paths_in_flight=None, build_options=None):
        self.data = data
        self.integrator, self.camera, self.background = data.integrator, data.camera, data.background
        self.frame = 0
        ctx = ctypes.c_void_p()
        nat.check(nat.lib().pt_context_create(device, ctypes.byref(ctx)), "pt_context_create")
        self.ctx = ctx
        if max_paths_in_flight:
            nat.call("pt_set_max_paths_in_flight", self.ctx, int(max_paths_in_flight))
        self.material_ids = {}
        for k, mat in enumerate(data.materials):
            mid = ctypes.c_uint32()
            p = mat.params()
            nat.call("pt_material_create", self.ctx, mat.type, ctypes.byref(p), ctypes.sizeof(p), ctypes.byref(mid))
            assert mid.value == k
            self.material_ids[id(mat)] = k
        self.apply_integrator()
        self.apply_camera()
        self.apply_background()
        nat.call("pt_set_probe_count", self.ctx, data.probe_samples)
        self.texture_ids = {}
        for k, mat in enumerate(data.materials):
            tex = getattr(mat, "texture", None)
            if tex is not None:
                ch = 1 if tex.ndim == 2 else tex.shape[2]
                tid = ctypes.c_uint32()
                nat.call("pt_texture_create", self.ctx, tex.ctypes.data, tex.shape[1], tex.shape[0], ch, ctypes.byref(tid))
                nat.call("pt_material_set_texture", self.ctx, k, tid.value, _f3(mat.texture_center))
                self.texture_ids[id(mat)] = tid.value
        for m, mid in zip(data.meshes, data.mesh_material):
            nn = 0 if m.normals is None else len(m.normals)
            first = ctypes.c_uint32()
            nat.call("pt_mesh_add", self.ctx, m.positions.ctypes.data, len(m.positions), m.vindex.ctypes.data, len(m.vindex),
                     None if m.normals is None else m.normals.ctypes.data, nn,
                     None if m.nindex is None else m.nindex.ctypes.data, mid, ctypes.byref(first))
        lb, tb = data.light_buffer, data.triangle_light_buffer
        nat.call("pt_lights_upload", self.ctx, lb.ctypes.data if len(lb) else None, len(lb), tb.ctypes.data if len(tb) else None, len(tb))
        for name, value in (build_options or {}).items():
            nat.call("pt_set_option", self.ctx, name.encode(), int(value))
        nat.call("pt_build", self.ctx)

    def rebuild(self, **options):
        """Set build options (e.g. bvh_builder=1) and rebuild the acceleration structure (pt_build)."""
        for name, value in options.items():
            nat.call("pt_set_option", self.ctx, name.encode(), int(value))
        nat.call("pt_build", self.ctx)

    def set_option(self, name, value):
        """A launch option or mode of pt_set_option (e.g. "overlap", "refill", "bin_items")."""
        nat.call("pt_set_option", self.ctx, name.encode(), int(value))

    def build_info(self):
        """pt_build_info of the last build (SAH cost included)."""
        b = BuildInfo()
        nat.call("pt_get_build_info", self.ctx, ctypes.byref(b))
        return b

    def update_material(self, mat):
        """Push changed parameters of a material already in the scene."""
        p = mat.params()
        nat.call("pt_material_update", self.ctx, self.material_ids[id(mat)], ctypes.byref(p), ctypes.sizeof(p))

    def apply_integrator(self):
        I = self.integrator
        nat.call("pt_set_integrator", self.ctx, I.max_depth, I.scene_epsilon, _f3(I.exception_color), I.rr_start_depth)

    def apply_camera(self):
        C = self.camera
        nat.call("pt_set_camera", self.ctx, _f3(C.eye), _f3(C.U), _f3(C.V), _f3(C.W), C.width, C.height,
                 (ctypes.c_uint32 * 2)(*C.patch_origin), (ctypes.c_uint32 * 2)(*C.patch_dims))
        self.frame = 0

    def apply_background(self):
        if isinstance(self.background, EnvMapBackground) and self.background.path is not None:
            nat.call("pt_set_envmap_hdr", self.ctx, os.fsencode(self.background.path))
        elif isinstance(self.background, EnvMapBackground):
            e = self.background.rgba
            nat.call("pt_set_envmap", self.ctx, e.ctypes.data, e.shape[1], e.shape[0])
        else:
            nat.call("pt_set_background_constant", self.ctx, _f3(self.background.background_color))

    def envmap_tables(self):
        H, W = self.background.rgba.shape[:2]
        out = [np.empty(H, np.float32), np.empty(H, np.float32), np.empty((H, W), np.float32), np.empty((H, W), np.float32)]
        nat.call("pt_get_envmap_tables", self.ctx, *[o.ctypes.data for o in out])
        return out

    def probes(self):
        """The PositionSample records of the last frame rendered (object-major)."""
        n = ctypes.c_uint64()
        nat.call("pt_get_probes", self.ctx, None, 0, ctypes.byref(n))
        out = np.zeros(n.value, POSITION_SAMPLE_DTYPE)
        if n.value:
            nat.call("pt_get_probes", self.ctx, out.ctypes.data, n.value, ctypes.byref(n))
        return out

    def scattering_properties(self, mat):
        out = np.zeros(1, SCATTERING_PROPERTIES_DTYPE)
        nat.call("pt_get_scattering_properties", self.ctx, self.material_ids[id(mat)], out.ctypes.data)
        return out[0]

    def renderScene(self):
        """One frame, as OptixScene::renderScene: frame++ and one integrator pass."""
        nat.call("pt_render_frames", self.ctx, self.frame, 1)
        self.frame += 1

    def render(self, n_frames):
        """n_frames more frames folded into the running mean (one wavefront launch group)."""
        nat.call("pt_render_frames", self.ctx, self.frame, int(n_frames))
        self.frame += int(n_frames)

    def readback(self):
        out = np.empty((self.camera.height, self.camera.width, 4), np.float32)
        nat.call("pt_readback", self.ctx, out.ctypes.data)
        return out

    def stats(self):
        s = RenderStats()
        nat.call("pt_get_render_stats", self.ctx, ctypes.byref(s))
        return s

    def sync(self):
        nat.call("pt_sync", self.ctx)

    def stream(self):
        return nat.lib().pt_context_stream(self.ctx)

    def close(self):
        if getattr(self, "ctx", None):
            nat.lib().pt_context_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- batches (no counterpart in the reference)
class TuneResult(ctypes.Structure):
    _fields_ = [("extend_mode", ctypes.c_int32), ("refill", ctypes.c_int32), ("max_paths_in_flight", ctypes.c_uint64),
                ("best_mpaths_per_s", ctypes.c_float), ("trials", ctypes.c_uint32), ("bin_items", ctypes.c_uint32)]


class Batch:
    """Several Renderers rendered by one wavefront pass (pt_batch_*): each render traces the next
    `frames` frames of every scene; the launch sequence is captured once in a CUDA graph."""

    def __init__(self, renderers, frames, device=0):
        b = ctypes.c_void_p()
        nat.call("pt_batch_create", device, ctypes.byref(b))
        self.b = b
        self.renderers = list(renderers)
        self.frames = [int(f) for f in frames]
        for R, f in zip(self.renderers, self.frames):
            nat.call("pt_batch_add", self.b, R.ctx, f)

    def set_option(self, name, value):
        nat.call("pt_batch_set_option", self.b, name.encode(), int(value))

    def _sync_frames(self):
        for R in self.renderers:
            n = ctypes.c_uint32()
            nat.call("pt_get_next_frame", R.ctx, ctypes.byref(n))
            R.frame = n.value

    def render(self):
        nat.call("pt_batch_render", self.b)
        self._sync_frames()

    def render_sequential(self):
        nat.call("pt_batch_render_sequential", self.b)
        self._sync_frames()

    def autotune(self, frames_per_trial=1):
        r = TuneResult()
        nat.call("pt_batch_autotune", self.b, int(frames_per_trial), ctypes.byref(r))
        self._sync_frames()
        return r

    def stats(self):
        s = RenderStats()
        nat.call("pt_batch_get_stats", self.b, ctypes.byref(s))
        return s

    def stream(self):
        return nat.lib().pt_batch_stream(self.b)

    def close(self):
        if getattr(self, "b", None):
            nat.lib().pt_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
