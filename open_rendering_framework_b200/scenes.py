"""Procedural scenes of the benchmark configurations (synthetic stand-ins: the reference ships no
benchmark scenes, and its demo scene depends on assets that are not in the repository).

single_scene(): the single-scene render -- a closed box of 12 triangles (diffuse, albedo 0.7), an
icosphere subdivided 6 times (81,920 triangles, radius 0.3) of GGX conductor with alpha 0.2 and
complex IOR R = 0.2+3.9i, G = 0.55+3.15i, B = 0.9+2.4i (the (0.2,0.9)-(3.9,2.4) range read as
red/blue endpoints, green in between), an icosphere subdivided 5 times (20,480 triangles, radius
0.3) of rough dielectric (Beckmann, alpha 0.1, eta 1.5), and one 0.25 x 0.25 quad light of radiance
15 under the ceiling; 512 x 512, max depth 8, Russian roulette from depth 3.  The placement is fixed:
box [-1,1]^3, camera at (0, 0, 0.9) looking down -z with a 60 degree vertical field of view,
conductor sphere at (-0.45, -0.7, -0.3), dielectric sphere at (0.45, -0.7, 0.1), light at y = 0.99.
"""
import numpy as np

from . import scene as sc


def icosphere(subdiv, radius=1.0, center=(0.0, 0.0, 0.0)):
    """Icosahedron subdivided `subdiv` times (20 * 4^subdiv triangles), projected to the sphere,
    with per-vertex normals (positions, vindex, normals, nindex)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
             (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
             (8, 6, 7), (9, 8, 1)]
    V = np.array(verts, np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array(faces, np.int64)
    for _ in range(subdiv):
        edges = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        mids = V[uniq[:, 0]] + V[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = len(V)
        V = np.concatenate([V, mids])
        m = inv.reshape(3, -1).T + base  # midpoint of edges (0,1), (1,2), (2,0) per face
        a, b, c = F[:, 0], F[:, 1], F[:, 2]
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        F = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)])
    normals = V.astype(np.float32)
    pos = (V * radius + np.asarray(center, np.float64)).astype(np.float32)
    vi = F.astype(np.int32)
    return pos, vi, normals, vi.copy()


def box(lo=(-1.0, -1.0, -1.0), hi=(1.0, 1.0, 1.0)):
    """A closed box of 12 triangles (no vertex normals: the geometric normal is used)."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    P = np.array([(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0), (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)], np.float32)
    quads = [(0, 1, 2, 3), (5, 4, 7, 6), (4, 0, 3, 7), (1, 5, 6, 2), (4, 5, 1, 0), (3, 2, 6, 7)]
    tris = []
    for a, b, c, d in quads:
        tris += [(a, b, c), (a, c, d)]
    return P, np.array(tris, np.int32)


def quad_light(center, size, y_down=True):
    """A horizontal square of 2 triangles facing -y (the emitter test of arealight_shader.cu is
    front-facing against the geometric normal cross(v1-v0, v2-v0))."""
    cx, cy, cz = center
    h = size / 2.0
    P = np.array([(cx - h, cy, cz - h), (cx + h, cy, cz - h), (cx + h, cy, cz + h), (cx - h, cy, cz + h)], np.float32)
    idx = np.array([(0, 1, 2), (0, 2, 3)], np.int32) if y_down else np.array([(0, 2, 1), (0, 3, 2)], np.int32)
    return P, idx


def single_scene(width=512, height=512, metal_subdiv=6, glass_subdiv=5, max_depth=8, rr_start_depth=3,
                 metal_model=sc.WALTER_MODEL, glass_model=sc.WALTER_MODEL):
    integrator = sc.PathTracer(max_depth=max_depth, scene_epsilon=1e-4, rr_start_depth=rr_start_depth)
    camera = sc.PinholeCamera(eye=(0.0, 0.0, 0.9), lookat=(0.0, 0.0, -1.0), up=(0.0, 1.0, 0.0), vfov=60.0, width=width, height=height)
    background = sc.ConstantBackground((0.0, 0.0, 0.0))
    diffuse = sc.DiffuseMaterial((0.7, 0.7, 0.7))
    metal = sc.MetallicMaterial(ior=((0.2, 3.9), (0.55, 3.15), (0.9, 2.4)), roughness=(0.2, 0.2), microfacet_model=metal_model,
                                normal_distribution=sc.GGX_DISTRIBUTION)
    glass = sc.RoughTransparentMaterial(ior=1.5, roughness=0.1, glass_absorption=(0.0, 0.0, 0.0), microfacet_model=glass_model,
                                        normal_distribution=sc.BECKMANN_DISTRIBUTION)
    bp, bi = box()
    mp, mi, mn, mni = icosphere(metal_subdiv, 0.3, (-0.45, -0.7, -0.3))
    gp, gi, gn, gni = icosphere(glass_subdiv, 0.3, (0.45, -0.7, 0.1))
    meshes = [sc.Mesh(bp, bi, diffuse), sc.Mesh(mp, mi, metal, mn, mni), sc.Mesh(gp, gi, glass, gn, gni)]
    lp, li = quad_light((0.0, 0.99, 0.0), 0.25)
    lights = [sc.TriangleAreaLight(lp, li, (15.0, 15.0, 15.0))]
    return sc.SceneData(integrator, camera, background, meshes, lights)


def layered_scene(width=64, height=64, subdiv=3, max_depth=8, rr_start_depth=0, rough_model=sc.WALTER_MODEL,
                  rough_distribution=sc.BECKMANN_DISTRIBUTION):
    """The remaining material programs side by side in the diffuse box under the quad light: a Lambertian
    base under a smooth interface (lambertian_interface_shader.cu), one under a rough interface
    (rough_diffuse_shader.cu, with the given microfacet model and distribution) and a smooth glass
    sphere with absorption (transparent_shader.cu)."""
    integrator = sc.PathTracer(max_depth=max_depth, scene_epsilon=1e-4, rr_start_depth=rr_start_depth)
    camera = sc.PinholeCamera(eye=(0.0, 0.0, 0.9), lookat=(0.0, 0.0, -1.0), up=(0.0, 1.0, 0.0), vfov=60.0, width=width, height=height)
    background = sc.ConstantBackground((0.0, 0.0, 0.0))
    diffuse = sc.DiffuseMaterial((0.7, 0.7, 0.7))
    lamb = sc.LambertianInterfaceMaterial(color=(0.8, 0.3, 0.2), ior=1.5)
    rough = sc.RoughDiffuseMaterial(color=(0.2, 0.6, 0.8), ior=1.4, roughness=(0.3, 0.3), microfacet_model=rough_model,
                                    normal_distribution=rough_distribution)
    glass = sc.TransparentMaterial(ior=1.5, glass_absorption=(0.5, 0.2, 0.1))
    bp, bi = box()
    ap, ai, an, ani = icosphere(subdiv, 0.28, (-0.48, -0.45, -0.45))
    rp, ri, rn, rni = icosphere(subdiv, 0.28, (0.08, -0.45, -0.6))
    gp, gi, gn, gni = icosphere(subdiv, 0.25, (0.45, -0.4, -0.2))
    meshes = [sc.Mesh(bp, bi, diffuse), sc.Mesh(ap, ai, lamb, an, ani), sc.Mesh(rp, ri, rough, rn, rni), sc.Mesh(gp, gi, glass, gn, gni)]
    lp, li = quad_light((0.0, 0.99, 0.0), 0.25)
    lights = [sc.TriangleAreaLight(lp, li, (15.0, 15.0, 15.0))]
    return sc.SceneData(integrator, camera, background, meshes, lights)


def analytic_light_scene(width=64, height=64, subdiv=3, max_depth=8, rr_start_depth=0):
    """The diffuse box lit by a DiskAreaLight under the ceiling (radius 0.2, facing down: theta 180)
    and a SphericalLight (radius 0.08) above a GGX conductor sphere and a Lambertian-interface sphere;
    both lights are seen by camera rays through their analytic geometry (disk_mesh.cu, sphere_mesh.cu)
    and block shadow rays."""
    integrator = sc.PathTracer(max_depth=max_depth, scene_epsilon=1e-4, rr_start_depth=rr_start_depth)
    camera = sc.PinholeCamera(eye=(0.0, 0.0, 0.9), lookat=(0.0, 0.0, -1.0), up=(0.0, 1.0, 0.0), vfov=60.0, width=width, height=height)
    background = sc.ConstantBackground((0.0, 0.0, 0.0))
    diffuse = sc.DiffuseMaterial((0.7, 0.7, 0.7))
    metal = sc.MetallicMaterial(ior=((0.2, 3.9), (0.55, 3.15), (0.9, 2.4)), roughness=(0.15, 0.15), microfacet_model=sc.VISIBLE_NORMALS_MODEL,
                                normal_distribution=sc.GGX_DISTRIBUTION)
    lamb = sc.LambertianInterfaceMaterial(color=(0.3, 0.7, 0.3), ior=1.5)
    bp, bi = box()
    mp, mi, mn, mni = icosphere(subdiv, 0.28, (-0.4, -0.45, -0.5))
    ap, ai, an, ani = icosphere(subdiv, 0.25, (0.4, -0.5, -0.3))
    meshes = [sc.Mesh(bp, bi, diffuse), sc.Mesh(mp, mi, metal, mn, mni), sc.Mesh(ap, ai, lamb, an, ani)]
    lights = [sc.DiskAreaLight(position=(0.0, 0.95, -0.3), radiance=(6.0, 6.0, 5.5), radius=0.2, theta=180.0, phi=0.0),
              sc.SphericalLight(position=(0.1, 0.1, -0.6), radiance=(20.0, 14.0, 8.0), radius=0.08)]
    return sc.SceneData(integrator, camera, background, meshes, lights)


def open_lights_scene(width=64, height=64, subdiv=3, max_depth=8, rr_start_depth=0):
    """An open scene (no enclosing box: a 6 x 6 diffuse floor quad under a black background) lit by a
    DirectionalLight and a PointLight (LightSampler.h:20-37): a diffuse icosphere, a GGX conductor
    icosphere and a Lambertian-interface icosphere on the floor, so that the lights' shadow rays reach
    the light (a directional light's to infinity) or are blocked by the spheres."""
    integrator = sc.PathTracer(max_depth=max_depth, scene_epsilon=1e-4, rr_start_depth=rr_start_depth)
    camera = sc.PinholeCamera(eye=(0.0, 0.6, 1.6), lookat=(0.0, -0.2, 0.0), up=(0.0, 1.0, 0.0), vfov=50.0, width=width, height=height)
    background = sc.ConstantBackground((0.0, 0.0, 0.0))
    floor = sc.DiffuseMaterial((0.6, 0.6, 0.6))
    diffuse = sc.DiffuseMaterial((0.8, 0.3, 0.2))
    metal = sc.MetallicMaterial(ior=((0.2, 3.9), (0.55, 3.15), (0.9, 2.4)), roughness=(0.2, 0.2), microfacet_model=sc.WALTER_MODEL,
                                normal_distribution=sc.GGX_DISTRIBUTION)
    lamb = sc.LambertianInterfaceMaterial(color=(0.2, 0.4, 0.8), ior=1.5)
    fp_ = np.array([(-3, -0.5, -3), (3, -0.5, -3), (3, -0.5, 3), (-3, -0.5, 3)], np.float32)
    fi = np.array([(0, 2, 1), (0, 3, 2)], np.int32)
    dp, di, dn, dni = icosphere(subdiv, 0.25, (-0.5, -0.25, -0.2))
    mp, mi, mn, mni = icosphere(subdiv, 0.25, (0.0, -0.25, -0.5))
    lp, li, ln, lni = icosphere(subdiv, 0.25, (0.5, -0.25, -0.1))
    meshes = [sc.Mesh(fp_, fi, floor), sc.Mesh(dp, di, diffuse, dn, dni), sc.Mesh(mp, mi, metal, mn, mni), sc.Mesh(lp, li, lamb, ln, lni)]
    d = np.array([-0.4, -1.0, -0.3])
    d /= np.linalg.norm(d)
    lights = [sc.DirectionalLight(direction=tuple(d), radiance=(2.5, 2.4, 2.2)), sc.PointLight(position=(0.6, 1.2, 0.8), radiance=(4.0, 3.0, 2.0))]
    return sc.SceneData(integrator, camera, background, meshes, lights)


def sky_envmap(width=2048, height=1024, sun_dir=(0.35, 0.55, 0.45), sun_peak=5.0e4, sun_sigma_deg=1.0):
    """Procedural equirectangular sky in the reference's mapping (envmap.h: u = (atan2(x, z) + pi) / 2pi,
    v = 1 - acos(y) / pi): a vertical gradient from horizon to zenith, a darker ground, and a Gaussian sun
    lobe of the given peak radiance and angular width.  float4 texels [H, W, 4], row 0 at v = 0."""
    u = (np.arange(width, dtype=np.float64) + 0.5) / width
    v = (np.arange(height, dtype=np.float64) + 0.5) / height
    theta = (1.0 - v)[:, None] * np.pi
    phi = (2.0 * u - 1.0)[None, :] * np.pi
    d = np.stack([np.sin(theta) * np.sin(phi), np.cos(theta) * np.ones_like(phi), np.sin(theta) * np.cos(phi)], -1)
    y = d[..., 1:2]
    horizon = np.array([0.85, 0.9, 1.0])
    zenith = np.array([0.15, 0.35, 0.85])
    ground = np.array([0.25, 0.22, 0.2])
    sky = np.where(y >= 0, horizon + (zenith - horizon) * np.sqrt(np.clip(y, 0, 1)), ground)
    s = np.asarray(sun_dir, np.float64)
    s /= np.linalg.norm(s)
    ang = np.arccos(np.clip(np.tensordot(d, s, axes=([2], [0])), -1, 1))
    sig = np.radians(sun_sigma_deg)
    sun = sun_peak * np.exp(-0.5 * (ang / sig) ** 2)[..., None] * np.array([1.0, 0.95, 0.85])
    rgb = sky + sun
    out = np.concatenate([rgb, np.ones(rgb.shape[:2] + (1,))], -1).astype(np.float32)
    return np.ascontiguousarray(out)


def env_scene(width=256, height=256, env_w=256, env_h=128, metal_subdiv=3, glass_subdiv=2, env_as_light=True, max_depth=6):
    """Open scene lit only by the procedural sky (no box): a diffuse floor quad, a conductor and a
    dielectric sphere; the environment map is both the miss radiance and (optionally) a light."""
    integrator = sc.PathTracer(max_depth=max_depth, scene_epsilon=1e-4)
    camera = sc.PinholeCamera(eye=(0.0, 0.3, 2.2), lookat=(0.0, -0.3, 0.0), up=(0.0, 1.0, 0.0), vfov=45.0, width=width, height=height)
    background = sc.EnvMapBackground(sky_envmap(env_w, env_h, sun_peak=5.0e4, sun_sigma_deg=4.0))
    floor = sc.DiffuseMaterial((0.6, 0.6, 0.55))
    metal = sc.MetallicMaterial(ior=((0.2, 3.9), (0.55, 3.15), (0.9, 2.4)), roughness=(0.2, 0.2), normal_distribution=sc.GGX_DISTRIBUTION)
    glass = sc.RoughTransparentMaterial(ior=1.5, roughness=0.1, normal_distribution=sc.BECKMANN_DISTRIBUTION)
    fp_ = np.array([(-3, -1, -3), (3, -1, -3), (3, -1, 3), (-3, -1, 3)], np.float32)
    fi = np.array([(0, 2, 1), (0, 3, 2)], np.int32)
    mp, mi, mn, mni = icosphere(metal_subdiv, 0.5, (-0.6, -0.5, 0.0))
    gp, gi, gn, gni = icosphere(glass_subdiv, 0.5, (0.6, -0.5, 0.2))
    meshes = [sc.Mesh(fp_, fi, floor), sc.Mesh(mp, mi, metal, mn, mni), sc.Mesh(gp, gi, glass, gn, gni)]
    lights = [sc.EnvMapLight()] if env_as_light else []
    return sc.SceneData(integrator, camera, background, meshes, lights)


def value_noise3(p, seed, cells=4.0):
    """Seeded 3-D value noise in [-1, 1]: random values on an integer lattice (cells per unit),
    trilinearly interpolated with a smoothstep fade.  p: [N, 3]."""
    rng = np.random.default_rng(seed)
    n = 64
    table = rng.uniform(-1.0, 1.0, size=(n, n, n))
    q = (np.asarray(p, np.float64) + 8.0) * cells
    i0 = np.floor(q).astype(np.int64)
    f = q - i0
    f = f * f * (3.0 - 2.0 * f)
    out = np.zeros(len(q))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * (f[:, 2] if dz else 1 - f[:, 2])
                out += w * table[(i0[:, 0] + dx) % n, (i0[:, 1] + dy) % n, (i0[:, 2] + dz) % n]
    return out


def jittered_icosphere(subdiv, radius=1.0, center=(0.0, 0.0, 0.0), amplitude=0.02, seed=0):
    """icosphere() with every vertex moved along its radius by value noise of the given relative
    amplitude (2% of the radius by default); vertex normals are the area-weighted face normals."""
    pos, vi, _, _ = icosphere(subdiv, 1.0)
    d = pos.astype(np.float64)
    r = 1.0 + amplitude * value_noise3(d, seed)
    P = d * r[:, None] * radius + np.asarray(center, np.float64)
    fn = np.cross(P[vi[:, 1]] - P[vi[:, 0]], P[vi[:, 2]] - P[vi[:, 0]])
    N = np.zeros_like(P)
    for k in range(3):
        np.add.at(N, vi[:, k], fn)
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    return P.astype(np.float32), vi, N.astype(np.float32), vi.copy()


def dipole_coefficients(seed):
    """Per-RGB reduced scattering sigma_s' ~ U[0.5, 3] /mm and absorption sigma_a ~ U[0.001, 0.05] /mm
    (mean cosine 0, so sigma_s = sigma_s')."""
    rng = np.random.default_rng(seed)
    return tuple(rng.uniform(0.5, 3.0, 3)), tuple(rng.uniform(0.001, 0.05, 3))


def subsurface_scene(width=1024, height=1024, subdiv=7, probe_samples=4096, env_w=2048, env_h=1024, seed=3, dipole_model=sc.STANDARD_DIPOLE,
                     max_depth=8, scale=100.0):
    """The subsurface configuration: a translucent icosphere subdivided `subdiv` times (7: 327,680
    triangles), radius 0.5, vertices jittered by 2% value noise, dipole BSSRDF with seeded
    coefficients in 1/mm and eta 1.3, scaled by `scale` (100: one scene unit is 100 mm, so the sphere
    is 10 cm across), `probe_samples` probe points per frame; lit by the procedural sky (gradient
    plus a Gaussian sun lobe of peak 5e4) as background and as the only light."""
    integrator = sc.PathTracer(max_depth=max_depth, scene_epsilon=1e-4)
    camera = sc.PinholeCamera(eye=(0.0, 0.35, 2.0), lookat=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), vfov=36.0, width=width, height=height)
    background = sc.EnvMapBackground(sky_envmap(env_w, env_h, sun_peak=5.0e4, sun_sigma_deg=1.0 if env_w >= 1024 else 6.0))
    sigma_s, sigma_a = dipole_coefficients(seed)
    mat = sc.TranslucentMaterial(scattering=sigma_s, absorption=sigma_a, meancosine=(0.0, 0.0, 0.0), ior=1.3, scale=scale,
                                 dipole_model=dipole_model)
    p, i, n, ni = jittered_icosphere(subdiv, 0.5, (0.0, 0.0, 0.0), 0.02, seed)
    meshes = [sc.Mesh(p, i, mat, n, ni)]
    return sc.SceneData(integrator, camera, background, meshes, [sc.EnvMapLight()], probe_samples=probe_samples)


def translucent_box_scene(width=64, height=64, subdiv=3, probe_samples=64, dipole_model=sc.STANDARD_DIPOLE, max_depth=6, two_objects=False,
                          rough=None):
    """A small closed scene for parity checks: the diffuse box, a translucent icosphere (and
    optionally a second translucent object with its own material), a quad light.  rough =
    (roughness, microfacet model, normal distribution) makes the icosphere a rough translucent one."""
    integrator = sc.PathTracer(max_depth=max_depth, scene_epsilon=1e-4)
    camera = sc.PinholeCamera(eye=(0.0, 0.0, 0.9), lookat=(0.0, 0.0, -1.0), up=(0.0, 1.0, 0.0), vfov=60.0, width=width, height=height)
    background = sc.ConstantBackground((0.0, 0.0, 0.0))
    diffuse = sc.DiffuseMaterial((0.7, 0.7, 0.7))
    kw = dict(scattering=(0.74, 0.88, 1.01), absorption=(0.032, 0.17, 0.48), ior=1.3, scale=10.0, dipole_model=dipole_model)
    if rough is None:
        skin = sc.TranslucentMaterial(**kw)
    else:
        skin = sc.RoughTranslucentMaterial(roughness=(rough[0], rough[0]), microfacet_model=rough[1], normal_distribution=rough[2], **kw)
    bp, bi = box()
    p, i, n, ni = jittered_icosphere(subdiv, 0.35, (-0.2, -0.6, -0.2), 0.02, 1)
    meshes = [sc.Mesh(bp, bi, diffuse), sc.Mesh(p, i, skin, n, ni)]
    if two_objects:
        marble = sc.TranslucentMaterial(scattering=(2.19, 2.62, 3.00), absorption=(0.0021, 0.0041, 0.0071), ior=1.5, scale=10.0,
                                        dipole_model=dipole_model)
        q, j, m, mj = icosphere(max(1, subdiv - 1), 0.25, (0.45, -0.7, 0.1))
        meshes.append(sc.Mesh(q, j, marble, m, mj))
    lp, li = quad_light((0.0, 0.99, 0.0), 0.5)
    lights = [sc.TriangleAreaLight(lp, li, (15.0, 15.0, 15.0))]
    return sc.SceneData(integrator, camera, background, meshes, lights, probe_samples=probe_samples)


def heightfield(n, extent=1.2, height=0.15, y0=-0.35, seed=0):
    """An n x n grid of quads (2 n^2 triangles) over [-extent/2, extent/2]^2 at y0 + height * value
    noise, with per-vertex normals from central differences."""
    t = np.linspace(-extent / 2, extent / 2, n + 1)
    X, Z = np.meshgrid(t, t, indexing="ij")
    P = np.stack([X.ravel(), np.zeros(X.size), Z.ravel()], 1)
    H = height * value_noise3(P * 1.5, seed, cells=2.0).reshape(n + 1, n + 1)
    Y = y0 + H
    dx = np.gradient(Y, t, axis=0)
    dz = np.gradient(Y, t, axis=1)
    N = np.stack([-dx, np.ones_like(Y), -dz], -1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    pos = np.stack([X, Y, Z], -1).reshape(-1, 3).astype(np.float32)
    idx = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1)
    a, b, c, d = idx[:-1, :-1].ravel(), idx[1:, :-1].ravel(), idx[1:, 1:].ravel(), idx[:-1, 1:].ravel()
    tris = np.concatenate([np.stack([a, c, b], 1), np.stack([a, d, c], 1)]).astype(np.int32)
    return pos, tris, N.reshape(-1, 3).astype(np.float32), tris.copy()


BATCH_MATERIALS = ("diffuse", "ggx", "beckmann", "rough_dielectric", "dipole")


def batch_scene(k, seed=0, size_scale=1.0, spp_scale=1.0, env_w=128, env_h=64, probe_samples=500):
    """Scene k of the batched configuration: a seeded mesh (an icosphere at the subdivision nearest a
    log-uniform [1e3, 5e5] triangle count, or a heightfield grid of that size), a material drawn
    uniformly from diffuse / GGX conductor / Beckmann conductor / rough dielectric / dipole, a
    resolution from {128, 256, 512, 1024}^2 and a log-uniform spp in [4, 256]; lit by a procedural sky
    (background and light).  Dipole scenes use the reference's default of 500 probes per frame
    (SAMPLES_FRAME, OptixSceneLoader.cpp:11).  size_scale / spp_scale shrink the resolution and spp
    (tests)."""
    rng = np.random.default_rng([seed, k])
    tris = float(np.exp(rng.uniform(np.log(1e3), np.log(5e5))))
    res = int(rng.choice([128, 256, 512, 1024]))
    spp = int(round(np.exp(rng.uniform(np.log(4), np.log(256)))))
    kind = BATCH_MATERIALS[int(rng.integers(0, 5))]
    use_grid = bool(rng.integers(0, 2))
    res = max(8, int(res * size_scale))
    spp = max(1, int(round(spp * spp_scale)))
    if kind == "diffuse":
        mat = sc.DiffuseMaterial(tuple(rng.uniform(0.3, 0.9, 3)))
    elif kind == "ggx":
        mat = sc.MetallicMaterial(ior=((0.2, 3.9), (0.55, 3.15), (0.9, 2.4)), roughness=(0.2, 0.2), microfacet_model=sc.VISIBLE_NORMALS_MODEL,
                                  normal_distribution=sc.GGX_DISTRIBUTION)
    elif kind == "beckmann":
        mat = sc.MetallicMaterial(roughness=(0.15, 0.15), microfacet_model=sc.WALTER_MODEL, normal_distribution=sc.BECKMANN_DISTRIBUTION)
    elif kind == "rough_dielectric":
        mat = sc.RoughTransparentMaterial(ior=1.5, roughness=0.1, microfacet_model=sc.WALTER_MODEL, normal_distribution=sc.BECKMANN_DISTRIBUTION)
    else:
        s_, a_ = dipole_coefficients(seed * 1000 + k)
        mat = sc.TranslucentMaterial(scattering=s_, absorption=a_, ior=1.3, scale=100.0)
    if use_grid:
        n = max(4, int(round((tris / 2) ** 0.5)))
        p, i, nn, ni = heightfield(n, seed=seed * 1000 + k)
    else:
        sub = int(np.clip(round(np.log(tris / 20.0) / np.log(4.0)), 2, 7))
        p, i, nn, ni = jittered_icosphere(sub, 0.4, (0.0, 0.0, 0.0), 0.02, seed * 1000 + k)
    floor = sc.DiffuseMaterial((0.5, 0.5, 0.5))
    fp_ = np.array([(-4, -0.45, -4), (4, -0.45, -4), (4, -0.45, 4), (-4, -0.45, 4)], np.float32)
    fi = np.array([(0, 2, 1), (0, 3, 2)], np.int32)
    az = rng.uniform(0, 2 * np.pi)
    eye = (2.0 * np.sin(az), 0.8, 2.0 * np.cos(az))
    camera = sc.PinholeCamera(eye=eye, lookat=(0.0, -0.1, 0.0), up=(0.0, 1.0, 0.0), vfov=40.0, width=res, height=res)
    background = sc.EnvMapBackground(sky_envmap(env_w, env_h, sun_peak=5.0e4 if env_w >= 1024 else 2.0e3, sun_sigma_deg=6.0))
    integrator = sc.PathTracer(max_depth=8, scene_epsilon=1e-4, rr_start_depth=3)
    meshes = [sc.Mesh(p, i, mat, nn, ni), sc.Mesh(fp_, fi, floor)]
    data = sc.SceneData(integrator, camera, background, meshes, [sc.EnvMapLight()], probe_samples=probe_samples)
    return data, spp, {"triangles": int(len(i)), "mesh": "grid" if use_grid else "icosphere", "material": kind, "resolution": res, "spp": spp}


def batch_scenes(n=64, seed=0, size_scale=1.0, spp_scale=1.0, **kw):
    """The n scenes of the batched configuration: [(SceneData, spp, description)]."""
    return [batch_scene(k, seed, size_scale, spp_scale, **kw) for k in range(n)]


def inverse_scene(width=256, height=256, subdiv=5, tex_res=256, seed=0, max_depth=6, probe_samples=500, scale=10.0):
    """The differentiable configuration: the single-scene geometry with both icospheres at `subdiv`
    subdivisions -- the diffuse box carries an albedo texture (tex_res^2 x 3, cube map around the box
    center), the GGX conductor sphere a roughness texture (tex_res^2, cube map around its center), and
    the second sphere is a translucent material (standard dipole) whose sigma_a and sigma_s' per RGB
    (1/mm, scaled by `scale` to scene units) are parameters; max depth 6, Russian roulette from depth 3.
    Every parameter is drawn from a seeded U[0.1, 0.9]."""
    rng = np.random.default_rng(seed)
    integrator = sc.PathTracer(max_depth=max_depth, scene_epsilon=1e-4, rr_start_depth=3)
    camera = sc.PinholeCamera(eye=(0.0, 0.0, 0.9), lookat=(0.0, 0.0, -1.0), up=(0.0, 1.0, 0.0), vfov=60.0, width=width, height=height)
    background = sc.ConstantBackground((0.0, 0.0, 0.0))
    diffuse = sc.DiffuseMaterial((0.7, 0.7, 0.7))
    diffuse.setTexture(rng.uniform(0.1, 0.9, (tex_res, tex_res, 3)).astype(np.float32), (0.0, 0.0, 0.0))
    metal_center = (-0.45, -0.7, -0.3)
    metal = sc.MetallicMaterial(ior=((0.2, 3.9), (0.55, 3.15), (0.9, 2.4)), roughness=(0.2, 0.2), microfacet_model=sc.WALTER_MODEL,
                                normal_distribution=sc.GGX_DISTRIBUTION)
    metal.setTexture(rng.uniform(0.1, 0.9, (tex_res, tex_res)).astype(np.float32), metal_center)
    sig = rng.uniform(0.1, 0.9, 6)
    trans = sc.TranslucentMaterial(scattering=tuple(sig[3:]), absorption=tuple(sig[:3]), meancosine=(0.0, 0.0, 0.0), ior=1.3, scale=scale)
    bp, bi = box()
    mp, mi, mn, mni = icosphere(subdiv, 0.3, metal_center)
    tp, ti, tn, tni = icosphere(subdiv, 0.3, (0.45, -0.7, 0.1))
    meshes = [sc.Mesh(bp, bi, diffuse), sc.Mesh(mp, mi, metal, mn, mni), sc.Mesh(tp, ti, trans, tn, tni)]
    lp, li = quad_light((0.0, 0.99, 0.0), 0.25)
    lights = [sc.TriangleAreaLight(lp, li, (15.0, 15.0, 15.0))]
    data = sc.SceneData(integrator, camera, background, meshes, lights, probe_samples=probe_samples)
    return data, (diffuse, metal, trans)
