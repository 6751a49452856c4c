"""Test infrastructure (oracle only): ctypes bindings for the two CPU oracles.

* ``ref()``  -> oracle/_ref/libref_oracle.so: the reference's own device-math headers compiled for
  the host (built from the reference sources by oracle/Makefile; the built file travels with the
  repository).  ``None`` when it was never built.
* ``orc()``  -> oracle/liboracle.so: the oracle restatement (FP32 bit-identical to ``ref()``, FP64
  instantiations, CPU path tracer).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use this module;
the product never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libref_oracle.so")
ORC_SO = os.path.join(HERE, "liboracle.so")

_ref = None
_orc = None

F = ctypes.c_float
D = ctypes.c_double
U = ctypes.c_uint
L = ctypes.c_long
I = ctypes.c_int
P = ctypes.c_void_p


def fp(a):
    """Pointer to a contiguous numpy array's data."""
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(P)


def build():
    """Build both oracle libraries (the reference one only where the reference sources exist)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def _sig(lib, name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            return None
        lib = ctypes.CDLL(REF_SO)
        _sig(lib, "ref_tea16", U, [U, U])
        _sig(lib, "ref_rnd_tea_stream", U, [U, P, L])
        _sig(lib, "ref_rnd_lcg_stream", U, [U, P, L])
        _sig(lib, "ref_rnd_md5_stream", None, [P, P, P, L])
        _sig(lib, "ref_md5_u2", None, [U, U, U, P])
        _sig(lib, "ref_erfinv", D, [D])
        _sig(lib, "ref_bsdf_queries", None, [L, L, L, P, P, F, P, P, P, P])
        _sig(lib, "ref_sample_visible_normal", None, [P, P, F, F, F, F, U, P])
        _sig(lib, "ref_eval_visible_normal", F, [P, P, P, F, F, U])
        _sig(lib, "ref_sample_normal", None, [P, F, F, F, U, P])
        _sig(lib, "ref_masking_G1", F, [P, P, P, F, U])
        _sig(lib, "ref_masking_G1_aniso", F, [P, P, P, F, F, U])
        _sig(lib, "ref_eval_bsdf", F, [P, P, P, F, F, U])
        _sig(lib, "ref_fresnel_R_vec", F, [P, P, F])
        _sig(lib, "ref_fresnel_complex", None, [P, P, P, P])
        _sig(lib, "ref_complex_recip", None, [P, P])
        _sig(lib, "ref_ms_dielectric_eval", F, [P, P, P, F, F, F, P, U, U])
        _sig(lib, "ref_ms_dielectric_sample", None, [P, P, F, F, F, P, P, U, P])
        _sig(lib, "ref_ms_conductor_eval", None, [P, P, P, P, F, F, P, U, U, P])
        _sig(lib, "ref_ms_conductor_sample", None, [P, P, P, F, F, P, P, U, P, P])
        _sig(lib, "ref_ms_diffuse_eval", None, [P, P, P, F, F, P, U, P, U, P])
        _sig(lib, "ref_ms_diffuse_sample", None, [P, P, F, F, P, P, P, U, P, P])
        _sig(lib, "ref_sample_cosine_weighted", None, [P, P, P])
        _sig(lib, "ref_sample_barycentric", None, [P, P])
        _sig(lib, "ref_create_onb", None, [P, P, P])
        _sig(lib, "ref_set_light_buffers", None, [P, L, P, L])
        _sig(lib, "ref_direct_illumination", None, [P, L, P, P, P, P])
        _sig(lib, "ref_set_envmap", None, [P, I, I, P, P, P, P])
        _sig(lib, "ref_env_lookup", None, [P, P])
        _sig(lib, "ref_sample_environment", None, [P, P, P, P])
        _sig(lib, "ref_set_scattering_properties", None, [P, L])
        _sig(lib, "ref_dipole_bssrdf", None, [F, P])
        _sig(lib, "ref_dirpole_bssrdf", None, [P, P, P, P, P, P])
        _sig(lib, "ref_bssrdf_queries", None, [U, L, P, P])
        _sig(lib, "ref_microfacet_queries", None, [U, U, P, F, P, P, L, P, P, P, P, P, P, P])
        _sig(lib, "ref_C_phi", F, [F])
        _sig(lib, "ref_C_E", F, [F])
        _sig(lib, "ref_sizeof", I, [ctypes.c_char_p])
        _sig(lib, "ref_oob_reads", ctypes.c_ulonglong, [])
        _ref = lib
    return _ref


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_SO):
            raise RuntimeError("oracle/liboracle.so is not built (run oracle/Makefile)")
        lib = ctypes.CDLL(ORC_SO)
        _sig(lib, "orc_tea16", U, [U, U])
        _sig(lib, "orc_rnd_tea_stream", U, [U, P, L])
        _sig(lib, "orc_rnd_lcg_stream", U, [U, P, L])
        _sig(lib, "orc_rnd_md5_stream", None, [P, P, P, L])
        _sig(lib, "orc_md5_u2", None, [U, U, P])
        _sig(lib, "orc_erfinv", D, [D])
        _sig(lib, "orc_bsdf_queries_f", None, [L, L, L, P, P, F, P, P, P, P, I])
        _sig(lib, "orc_bsdf_queries_d", None, [L, L, L, P, P, F, P, P, P, P, I])
        _sig(lib, "orc_c1_make_inputs", None, [L, L, P, P])
        _sig(lib, "orc_sample_visible_normal_f", None, [P, P, F, F, F, F, U, P])
        _sig(lib, "orc_sample_visible_normal_d", None, [P, P, F, F, F, F, U, P])
        _sig(lib, "orc_eval_visible_normal_f", F, [P, P, P, F, F, U])
        _sig(lib, "orc_sample_normal_f", None, [P, F, F, F, U, P])
        _sig(lib, "orc_masking_G1_f", F, [P, P, P, F, U])
        _sig(lib, "orc_masking_G1_aniso_f", F, [P, P, P, F, F, U])
        _sig(lib, "orc_eval_bsdf_f", F, [P, P, P, F, F, U])
        _sig(lib, "orc_eval_bsdf_d", D, [P, P, P, F, F, U])
        _sig(lib, "orc_fresnel_R_vec_f", F, [P, P, F])
        _sig(lib, "orc_fresnel_complex_f", None, [P, P, P, P])
        _sig(lib, "orc_fresnel_complex_d", None, [P, P, P, P])
        _sig(lib, "orc_complex_recip_f", None, [P, P])
        _sig(lib, "orc_ms_dielectric_eval_f", F, [P, P, P, F, F, F, P, U, U])
        _sig(lib, "orc_ms_dielectric_eval_d", D, [P, P, P, F, F, F, P, U, U])
        _sig(lib, "orc_ms_dielectric_sample_f", None, [P, P, F, F, F, P, P, U, P])
        _sig(lib, "orc_ms_conductor_eval_f", None, [P, P, P, P, F, F, P, U, U, P])
        _sig(lib, "orc_ms_conductor_sample_f", None, [P, P, P, F, F, P, P, U, P, P])
        _sig(lib, "orc_ms_diffuse_eval_f", None, [P, P, P, F, F, P, U, P, U, P])
        _sig(lib, "orc_ms_diffuse_sample_f", None, [P, P, F, F, P, P, P, U, P, P])
        _sig(lib, "orc_sample_cosine_weighted_f", None, [P, P, P])
        _sig(lib, "orc_sample_barycentric_f", None, [P, P])
        _sig(lib, "orc_create_onb_f", None, [P, P, P])
        _sig(lib, "orc_direct_illumination_f", None, [P, P, L, P, L, L, P, P, P, P])
        _sig(lib, "orc_microfacet_queries_f", None, [U, U, P, F, P, P, L, P, P, P, P, P, P, P, I])
        _sig(lib, "orc_microfacet_queries_d", None, [U, U, P, F, P, P, L, P, P, P, P, P, P, P, I])
        _sig(lib, "orc_bsdf_given_m_f", None, [L, P, P, P, F, P, P, P, P, P])
        _sig(lib, "orc_C_phi_f", F, [F])
        _sig(lib, "orc_C_E_f", F, [F])
        _orc = lib
    return _orc


def c1_inputs(n, first=0):
    """Synthetic BSDF-query inputs (SoA wo[3][n], alpha[n]) from the oracle's generator."""
    wo = np.empty((3, n), np.float32)
    alpha = np.empty(n, np.float32)
    orc().orc_c1_make_inputs(n, first, fp(wo), fp(alpha))
    return wo, alpha


def bsdf_queries(n, first, n_ggx_below, wo, alpha, eta=1.0 / 1.5, fp64=False, threads=1, which="orc"):
    """Run the config-1 query batch on the CPU: returns (wi[3][n], f, pdf, F)."""
    dt = np.float64 if fp64 else np.float32
    wi = np.empty((3, n), dt)
    f = np.empty(n, dt)
    pdf = np.empty(n, dt)
    F_ = np.empty(n, dt)
    if which == "ref":
        assert not fp64
        ref().ref_bsdf_queries(n, first, n_ggx_below, fp(wo), fp(alpha), eta, fp(wi), fp(f), fp(pdf), fp(F_))
    elif fp64:
        orc().orc_bsdf_queries_d(n, first, n_ggx_below, fp(wo), fp(alpha), eta, fp(wi), fp(f), fp(pdf), fp(F_), threads)
    else:
        orc().orc_bsdf_queries_f(n, first, n_ggx_below, fp(wo), fp(alpha), eta, fp(wi), fp(f), fp(pdf), fp(F_), threads)
    return wi, f, pdf, F_


# ---------------------------------------------------------------- CPU path tracer (orc_trace.cpp)
def _trace_sigs(lib):
    if getattr(lib, "_trace_bound", False):
        return
    _sig(lib, "orc_scene_create", P, [P, P, U, P, U, P, P, P, P, P, U, P, U, P, U, P, U, U, P, I, F, I, P])
    _sig(lib, "orc_scene_destroy", None, [P])
    _sig(lib, "orc_render", L, [P, U, U, U, U, P, P, I])
    _sig(lib, "orc_capped", L, [P])
    _sig(lib, "orc_trace_batch", None, [P, P, L, I, P, P, P, P])
    _sig(lib, "orc_scene_set_env", None, [P, P, I, I])
    _sig(lib, "orc_env_tables", None, [P, P, P, P, P])
    _sig(lib, "orc_env_query", None, [P, P, L, P, P, L, P, P])
    _sig(lib, "orc_scene_set_translucent", None, [P, U, P, U])
    _sig(lib, "orc_scene_add_translucent_object", None, [P, U, U, U])
    _sig(lib, "orc_scene_set_samples", None, [P, U])
    _sig(lib, "orc_scene_set_texture", None, [P, U, P, U, U, U, P])
    _sig(lib, "orc_cube_texel", U, [P, P, U, U])
    _sig(lib, "orc_scene_record", None, [P, I])
    _sig(lib, "orc_scene_set_translucent_raw", None, [P, U, P, P, P, D, D])
    _sig(lib, "orc_tape_stats", None, [P, P])
    _sig(lib, "orc_tape_eval", None, [P, P, P, P, P, P, P, I])
    _sig(lib, "orc_scene_probes", L, [P, P])
    _sig(lib, "orc_compute_coefficients", None, [P, P, P, F, F, P])
    _sig(lib, "orc_dipole_bssrdf", None, [P, F, P])
    _sig(lib, "orc_dirpole_bssrdf", None, [P, P, P, P, P, P, P])
    _sig(lib, "orc_bssrdf_queries_f", None, [P, P, P, F, F, U, L, P, P, I])
    _sig(lib, "orc_bssrdf_queries_d", None, [P, P, P, F, F, U, L, P, P, I])
    lib._trace_bound = True


def compute_coefficients(mat):
    """TranslucentMaterial::computeCoefficients restated (260-byte ScatteringMaterialProperties)."""
    lib = orc()
    _trace_sigs(lib)
    out = np.zeros(65, np.float32)
    a = np.asarray(mat.absorption, np.float32)
    s = np.asarray(mat.scattering, np.float32)
    g = np.asarray(mat.meancosine, np.float32)
    lib.orc_compute_coefficients(fp(a), fp(s), fp(g), mat.ior, mat.scale, fp(out))
    return out


def dipole_bssrdf(props, dist, which="orc"):
    out = np.empty(3, np.float32)
    props = np.ascontiguousarray(props, np.float32)
    if which == "ref":
        ref().ref_set_scattering_properties(fp(props), 260)
        ref().ref_dipole_bssrdf(dist, fp(out))
    else:
        lib = orc()
        _trace_sigs(lib)
        lib.orc_dipole_bssrdf(fp(props), dist, fp(out))
    return out


def dirpole_bssrdf(props, xi, ni, w12, xo, no, which="orc"):
    out = np.empty(3, np.float32)
    props = np.ascontiguousarray(props, np.float32)
    args = [np.ascontiguousarray(v, np.float32) for v in (xi, ni, w12, xo, no)]
    if which == "ref":
        ref().ref_set_scattering_properties(fp(props), 260)
        ref().ref_dirpole_bssrdf(*[fp(a) for a in args], fp(out))
    else:
        lib = orc()
        _trace_sigs(lib)
        lib.orc_dirpole_bssrdf(fp(props), *[fp(a) for a in args], fp(out))
    return out


class OracleScene:
    """The CPU restatement of the reference's recursive path tracer over a SceneData
    (open_rendering_framework_b200.scene) flattened exactly as the GPU context stores it."""

    def __init__(self, data):
        lib = orc()
        _trace_sigs(lib)
        self.lib = lib
        self.data = data
        tri_pos, tri_info, normals = data.flat_triangles()
        n_m = len(data.materials)
        mtype = np.zeros(n_m, np.uint32)
        mmodel = np.zeros(n_m, np.uint32)
        mdist = np.zeros(n_m, np.uint32)
        mab = np.zeros((n_m, 8), np.float32)
        mior = np.zeros((n_m, 6), np.float64)
        for k, m in enumerate(data.materials):
            mtype[k] = m.type
            name = type(m).__name__
            if name == "DiffuseMaterial":
                mab[k, :3] = m.color
            elif name == "MetallicMaterial":
                mmodel[k], mdist[k] = m.microfacet_model, m.normal_distribution
                mab[k, :2] = m.roughness
                mior[k] = [v for c in m.ior for v in c]
            elif name == "RoughTransparentMaterial":
                mmodel[k], mdist[k] = m.microfacet_model, m.normal_distribution
                mab[k, 0], mab[k, 1] = m.ior, m.roughness
                mab[k, 4:7] = m.glass_absorption
            elif name == "AreaLightMaterial":
                mab[k, :3] = m.radiance
            elif name == "TransparentMaterial":
                mab[k, 0] = m.ior
                mab[k, 4:7] = m.glass_absorption
            elif name == "LambertianInterfaceMaterial":
                mab[k, :3] = m.color
                mab[k, 3] = m.ior
            elif name == "RoughDiffuseMaterial":
                mmodel[k], mdist[k] = m.microfacet_model, m.normal_distribution
                mab[k, :3] = m.color
                mab[k, 3] = m.ior
                mab[k, 5:7] = m.roughness
            elif name == "TranslucentMaterial":
                pass
            elif name == "RoughTranslucentMaterial":
                mmodel[k], mdist[k] = m.microfacet_model, m.normal_distribution
                mab[k, :2] = m.roughness
            else:
                raise TypeError(name)
        C = data.camera
        cam = np.concatenate([C.eye, C.U, C.V, C.W]).astype(np.float32)
        patch = np.array(list(C.patch_origin) + list(C.patch_dims), np.uint32)
        I_ = data.integrator
        bg = np.asarray(getattr(data.background, "background_color", (0.0, 0.0, 0.0)), np.float32)
        # keep every buffer alive for the scene's lifetime
        self._keep = [tri_pos, tri_info, normals, mtype, mmodel, mdist, mab, mior, cam, patch, bg,
                      np.ascontiguousarray(data.light_buffer), np.ascontiguousarray(data.triangle_light_buffer)]
        lb, tb = self._keep[-2], self._keep[-1]
        self.h = lib.orc_scene_create(fp(tri_pos), fp(tri_info), len(tri_pos), fp(normals) if len(normals) else None, len(normals),
                                      fp(mtype), fp(mmodel), fp(mdist), fp(mab), fp(mior), n_m,
                                      fp(lb) if len(lb) else None, len(lb), fp(tb) if len(tb) else None, len(tb),
                                      fp(cam), C.width, C.height, fp(patch), I_.max_depth, I_.scene_epsilon, I_.rr_start_depth, fp(bg))
        self.tex_of_material = {}
        for k, m in enumerate(data.materials):
            if type(m).__name__ in ("TranslucentMaterial", "RoughTranslucentMaterial"):
                props = compute_coefficients(m)
                self._keep.append(props)
                lib.orc_scene_set_translucent(self.h, k, fp(props), m.dipole_model)
                g = np.asarray(m.meancosine, np.float64)
                sa = np.asarray(m.absorption, np.float32).astype(np.float64)
                ssr = np.asarray(m.scattering, np.float32).astype(np.float64) * (1.0 - g)
                lib.orc_scene_set_translucent_raw(self.h, k, fp(sa), fp(ssr), fp(g), float(np.float32(m.ior)), float(np.float32(m.scale)))
        for k, m in enumerate(data.materials):
            tex = getattr(m, "texture", None)
            if tex is not None:
                tex = np.ascontiguousarray(tex, np.float32)
                center = np.asarray(m.texture_center, np.float32)
                self._keep += [tex, center]
                ch = 1 if tex.ndim == 2 else tex.shape[2]
                self.tex_of_material[k] = len(self.tex_of_material)
                lib.orc_scene_set_texture(self.h, k, fp(tex), tex.shape[1], tex.shape[0], ch, fp(center))
        for mid, first, n in data.translucent_objects():
            lib.orc_scene_add_translucent_object(self.h, mid, first, n)
        lib.orc_scene_set_samples(self.h, getattr(data, "probe_samples", 500))
        env = getattr(data.background, "rgba", None)
        if env is not None:
            env = np.ascontiguousarray(env, np.float32)
            self._keep.append(env)
            lib.orc_scene_set_env(self.h, fp(env), env.shape[1], env.shape[0])

    def render(self, first_frame, n_frames, accum=None, p_begin=0, p_end=None, path_radiance=False, threads=1):
        """Runs the CPU tracer; returns (accum [H,W,4] or None, per-path radiance [F,P,3] or None)."""
        W, H = self.data.camera.width, self.data.camera.height
        p_end = W * H if p_end is None else p_end
        pr = np.zeros((n_frames, p_end - p_begin, 3), np.float32) if path_radiance else None
        if accum is not None:
            accum = np.ascontiguousarray(accum, np.float32)
        self.lib.orc_render(self.h, first_frame, n_frames, p_begin, p_end, fp(pr) if pr is not None else None,
                            fp(accum) if accum is not None else None, threads)
        self._tape_range = (p_begin, p_end)
        return accum, pr

    # ---- path tapes (FP64 re-evaluation of the recorded paths; adjoint checks)
    def record(self, on=True):
        self.lib.orc_scene_record(self.h, 1 if on else 0)

    def tape_stats(self):
        out = np.zeros(3, np.int64)
        self.lib.orc_tape_stats(self.h, fp(out))
        return tuple(int(x) for x in out)

    def param_layout(self, materials):
        """(offsets per texture id, offsets per material, size) for parameters of the given materials:
        a textured material contributes its texture, a translucent one its 6 sigmas."""
        n_tex = len(self.tex_of_material)
        tex_off = np.full(max(1, n_tex), -1, np.int64)
        mat_off = np.full(max(1, len(self.data.materials)), -1, np.int64)
        off = 0
        for m in materials:
            k = self.data.materials.index(m)
            if k in self.tex_of_material:
                tex_off[self.tex_of_material[k]] = off
                off += m.texture.size
            else:
                mat_off[k] = off
                off += 6
        return tex_off, mat_off, off

    def tape_eval(self, P, tex_off, mat_off, dimg=None, threads=8):
        """FP64 image [npix, 3] of the recorded paths at parameters P; with dimg, also the FP64
        gradient of the loss whose image gradient is dimg ([npix, 3])."""
        P = np.ascontiguousarray(P, np.float64)
        npix = self._tape_npix()
        img = np.zeros((npix, 3), np.float64)
        grad = None
        if dimg is not None:
            dimg = np.ascontiguousarray(dimg, np.float64)
            grad = np.zeros_like(P)
        self.lib.orc_tape_eval(self.h, fp(P), fp(tex_off), fp(mat_off), fp(img), fp(dimg) if dimg is not None else None,
                               fp(grad) if grad is not None else None, threads)
        return img, grad

    def _tape_npix(self):
        return self._tape_range[1] - self._tape_range[0]

    def probes(self):
        """PositionSample records of the last frame rendered, as raw float32 [n, 20]."""
        n = self.lib.orc_scene_probes(self.h, None)
        out = np.zeros((n, 20), np.float32)
        if n:
            self.lib.orc_scene_probes(self.h, fp(out))
        return out

    def env_tables(self):
        H, W = self.data.background.rgba.shape[:2]
        mpdf, mcdf = np.empty(H, np.float32), np.empty(H, np.float32)
        cpdf, ccdf = np.empty((H, W), np.float32), np.empty((H, W), np.float32)
        self.lib.orc_env_tables(self.h, fp(mpdf), fp(mcdf), fp(cpdf), fp(ccdf))
        return mpdf, mcdf, cpdf, ccdf

    def env_query(self, dirs, seeds):
        dirs = np.ascontiguousarray(dirs, np.float32)
        seeds = np.ascontiguousarray(seeds, np.uint32).copy()
        looked = np.empty_like(dirs)
        sd = np.empty((len(seeds), 3), np.float32)
        sL = np.empty((len(seeds), 3), np.float32)
        self.lib.orc_env_query(self.h, fp(dirs), len(dirs), fp(looked), fp(seeds), len(seeds), fp(sd), fp(sL))
        return looked, seeds, sd, sL

    def trace(self, rays8, brute=False):
        """Closest and any hit for rays [n,8] = (origin, tmin, dir, tmax)."""
        rays8 = np.ascontiguousarray(rays8, np.float32)
        n = len(rays8)
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        bary = np.empty((n, 2), np.float32)
        anyh = np.empty(n, np.int32)
        self.lib.orc_trace_batch(self.h, fp(rays8), n, 1 if brute else 0, fp(prim), fp(t), fp(bary), fp(anyh))
        return prim, t, bary, anyh

    def close(self):
        if getattr(self, "h", None):
            self.lib.orc_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bssrdf_queries(params, model, inputs, fp64=False, which="orc", threads=1):
    """A batch of BSSRDF values S[3][n] of one translucent material.  params: (absorption[3],
    scattering[3], meancosine[3], ior, scale) as pt_translucent_params holds them; model 0 (standard
    dipole) takes inputs = dist[n], model 1 (directional) inputs = [15][n] (xi, ni, w12, xo, no).
    which="ref" runs the reference's own dipoles compiled for the host on the FP32 coefficients of
    the restatement (bit-identical to TranslucentMaterial::computeCoefficients); fp64 derives the
    coefficients and evaluates in double."""
    sa, ss, g, ior, scale = params
    sa, ss, g = (np.ascontiguousarray(v, np.float32) for v in (sa, ss, g))
    inputs = np.ascontiguousarray(inputs, np.float32)
    n = inputs.shape[-1]
    if which == "ref":
        assert not fp64
        lib = orc()
        _trace_sigs(lib)
        props = np.zeros(65, np.float32)
        lib.orc_compute_coefficients(fp(sa), fp(ss), fp(g), ior, scale, fp(props))
        out = np.empty((3, n), np.float32)
        ref().ref_set_scattering_properties(fp(props), 260)
        ref().ref_bssrdf_queries(model, n, fp(inputs), fp(out))
        return out
    lib = orc()
    _trace_sigs(lib)
    out = np.empty((3, n), np.float64 if fp64 else np.float32)
    f = lib.orc_bssrdf_queries_d if fp64 else lib.orc_bssrdf_queries_f
    f(fp(sa), fp(ss), fp(g), ior, scale, model, n, fp(inputs), fp(out), threads)
    return out


MF_OPS = {"dielectric_eval": 0, "dielectric_sample": 1, "conductor_eval": 2, "conductor_sample": 3, "diffuse_eval": 4,
          "diffuse_sample": 5, "conductor_fresnel": 6, "visible_normal": 7}


def microfacet_queries(op, dist, wi, wo, alpha, seed, order, normal=(0.0, 0.0, 1.0), eta=1.0 / 1.5, ior=(1.0, 0.0) * 3,
                       rho=(1.0, 1.0, 1.0), fp64=False, which="orc", threads=1):
    """A batch of multiscattering-walk / conductor-Fresnel queries (see orc_microfacet_queries_f):
    returns (out[3][n], weight[3][n], seed after, order after)."""
    op = MF_OPS[op] if isinstance(op, str) else int(op)
    wi = np.ascontiguousarray(wi, np.float32)
    wo = np.ascontiguousarray(wo, np.float32)
    alpha = np.ascontiguousarray(alpha, np.float32)
    seed = np.ascontiguousarray(seed, np.uint32).copy()
    order = np.ascontiguousarray(order, np.uint32).copy()
    n = alpha.size
    n3 = np.asarray(normal, np.float32)
    ior6 = np.asarray(ior, np.float64).reshape(6)
    rho3 = np.asarray(rho, np.float32)
    dt = np.float64 if fp64 else np.float32
    out = np.zeros((3, n), dt)
    weight = np.zeros((3, n), dt)
    if which == "ref":
        assert not fp64
        ref().ref_microfacet_queries(op, dist, fp(n3), eta, fp(ior6), fp(rho3), n, fp(wi), fp(wo), fp(alpha), fp(seed), fp(order),
                                     fp(out), fp(weight))
    else:
        f = orc().orc_microfacet_queries_d if fp64 else orc().orc_microfacet_queries_f
        f(op, dist, fp(n3), eta, fp(ior6), fp(rho3), n, fp(wi), fp(wo), fp(alpha), fp(seed), fp(order), fp(out), fp(weight), threads)
    return out, weight, seed, order
