"""Pins the oracle restatement (oracle/liboracle.so) to the reference.

Every check is bit-exact in FP32: the restatement keeps the reference's operation order and its
float/double promotions, and both are built with g++ without contraction.  The vectors in
tests/golden/ref_math.npz were produced by the reference's own headers compiled for the host
(tests/golden/make_golden.py); where that compiled reference is present it is also checked
directly on fresh inputs.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle_ctypes as oc

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_math.npz"))


def bits_equal(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    same = a.view(np.uint32) == b.view(np.uint32)
    return bool(np.all(same | (np.isnan(a) & np.isnan(b))))


def test_tea16_golden():
    O = oc.orc()
    got = np.array([O.orc_tea16(int(a), int(b)) for a, b in GOLD["tea16_in"]], np.uint32)
    assert np.array_equal(got, GOLD["tea16_out"])
    assert O.orc_tea16(12345, 0) == 0x5DF0BA3F


@pytest.mark.parametrize("kind", ["tea", "lcg"])
def test_rng_stream_golden(kind):
    O = oc.orc()
    fn = O.orc_rnd_tea_stream if kind == "tea" else O.orc_rnd_lcg_stream
    for k, s in enumerate(GOLD["rng_seeds"]):
        row = np.empty(32, np.float32)
        fin = fn(int(s), oc.fp(row), 32)
        assert fin == GOLD["rng_%s_final" % kind][k]
        assert bits_equal(row, GOLD["rng_%s" % kind][k])


def test_md5_stream_golden():
    O = oc.orc()
    seeds = GOLD["rng_seeds"]
    for k in range(64):
        x = ctypes.c_uint(int(seeds[k]))
        y = ctypes.c_uint(int(seeds[(k + 1) % 64]))
        row = np.empty(32, np.float32)
        O.orc_rnd_md5_stream(ctypes.byref(x), ctypes.byref(y), oc.fp(row), 32)
        assert bits_equal(row, GOLD["rng_md5"][k])
        assert (x.value, y.value) == tuple(GOLD["rng_md5_final"][k])


def test_c1_inputs_and_queries_golden():
    n = GOLD["c1_alpha"].size
    wo, alpha = oc.c1_inputs(n)
    assert bits_equal(wo, GOLD["c1_wo"]) and bits_equal(alpha, GOLD["c1_alpha"])
    wi, f, pdf, F = oc.bsdf_queries(n, 0, n // 2, wo, alpha)
    assert bits_equal(wi, GOLD["c1_wi"])
    assert bits_equal(f, GOLD["c1_f"])
    assert bits_equal(pdf, GOLD["c1_pdf"])
    assert bits_equal(F, GOLD["c1_F"])


def test_multiscatter_golden():
    O = oc.orc()
    nrm = np.array([0, 0, 1], np.float32)
    inv = GOLD["cond_eta"]
    rho = GOLD["ms_rho"]
    for k in range(GOLD["ms_alpha"].size):
        wi, wo, a, d = GOLD["ms_wi"][k], GOLD["ms_wo"][k], float(GOLD["ms_alpha"][k]), int(GOLD["ms_dist"][k])
        s = ctypes.c_uint(int(GOLD["ms_seed"][k]))
        v = O.orc_ms_dielectric_eval_f(oc.fp(wi), oc.fp(wo), oc.fp(nrm), 1.0 / 1.5, a, a, ctypes.byref(s), 0, d)
        assert bits_equal(np.float32(v), GOLD["ms_diel"][k]) and s.value == GOLD["ms_diel_seed"][k], k
        wo_up = np.abs(wo).astype(np.float32)
        s = ctypes.c_uint(int(GOLD["ms_seed"][k]))
        out = np.empty(3, np.float32)
        O.orc_ms_conductor_eval_f(oc.fp(wi), oc.fp(wo_up), oc.fp(nrm), oc.fp(inv), a, a, ctypes.byref(s), 0, d, oc.fp(out))
        assert bits_equal(out, GOLD["ms_cond"][k]) and s.value == GOLD["ms_cond_seed"][k], k
        s = ctypes.c_uint(int(GOLD["ms_seed"][k]))
        O.orc_ms_diffuse_eval_f(oc.fp(wi), oc.fp(wo_up), oc.fp(nrm), a, a, ctypes.byref(s), 0, oc.fp(rho), d, oc.fp(out))
        assert bits_equal(out, GOLD["ms_diff"][k]) and s.value == GOLD["ms_diff_seed"][k], k


def test_conductor_fresnel_golden():
    O = oc.orc()
    inv = np.empty(6, np.float64)
    O.orc_complex_recip_f(oc.fp(GOLD["cond_ior"]), oc.fp(inv))
    assert np.array_equal(inv, GOLD["cond_eta"])
    for k in range(GOLD["fc_wi"].shape[0]):
        out = np.empty(3, np.float32)
        O.orc_fresnel_complex_f(oc.fp(GOLD["fc_wi"][k]), oc.fp(GOLD["fc_m"][k]), oc.fp(inv), oc.fp(out))
        assert bits_equal(out, GOLD["fc_out"][k]), k


@pytest.mark.skipif(oc.ref() is None, reason="compiled reference (oracle/_ref) not built")
def test_fresh_queries_against_compiled_reference():
    n = 1 << 15
    wo, alpha = oc.c1_inputs(n, first=12345)
    for n_ggx in (n, 0):
        a = oc.bsdf_queries(n, 12345, 12345 + n_ggx, wo, alpha, which="ref")
        b = oc.bsdf_queries(n, 12345, 12345 + n_ggx, wo, alpha)
        for x, y in zip(a, b):
            assert bits_equal(x, y)


@pytest.mark.skipif(oc.ref() is None, reason="compiled reference (oracle/_ref) not built")
def test_fresh_pieces_against_compiled_reference():
    R, O = oc.ref(), oc.orc()
    rng = np.random.default_rng(7)
    for _ in range(2000):
        n = rng.normal(size=3).astype(np.float32)
        n /= np.linalg.norm(n)
        n = n.astype(np.float32)
        v = rng.normal(size=3).astype(np.float32)
        v = (v / np.linalg.norm(v)).astype(np.float32)
        m = rng.normal(size=3).astype(np.float32)
        m = (m / np.linalg.norm(m)).astype(np.float32)
        a = np.float32(rng.uniform(0.02, 1.0))
        z1, z2 = np.float32(rng.uniform()), np.float32(rng.uniform())
        for d in (0, 1):
            o1, o2 = np.empty(3, np.float32), np.empty(3, np.float32)
            R.ref_sample_normal(oc.fp(n), z1, z2, a, d, oc.fp(o1))
            O.orc_sample_normal_f(oc.fp(n), z1, z2, a, d, oc.fp(o2))
            assert bits_equal(o1, o2)
            R.ref_sample_visible_normal(oc.fp(v), oc.fp(n), a, a, z1, z2, d, oc.fp(o1))
            O.orc_sample_visible_normal_f(oc.fp(v), oc.fp(n), a, a, z1, z2, d, oc.fp(o2))
            assert bits_equal(o1, o2)
            assert bits_equal(np.float32(R.ref_masking_G1(oc.fp(v), oc.fp(m), oc.fp(n), a, d)),
                              np.float32(O.orc_masking_G1_f(oc.fp(v), oc.fp(m), oc.fp(n), a, d)))
            assert bits_equal(np.float32(R.ref_masking_G1_aniso(oc.fp(v), oc.fp(m), oc.fp(n), a, a, d)),
                              np.float32(O.orc_masking_G1_aniso_f(oc.fp(v), oc.fp(m), oc.fp(n), a, a, d)))
            assert bits_equal(np.float32(R.ref_eval_visible_normal(oc.fp(v), oc.fp(m), oc.fp(n), a, a, d)),
                              np.float32(O.orc_eval_visible_normal_f(oc.fp(v), oc.fp(m), oc.fp(n), a, a, d)))
            assert bits_equal(np.float32(R.ref_eval_bsdf(oc.fp(v), oc.fp(m), oc.fp(n), a, np.float32(1 / 1.5), d)),
                              np.float32(O.orc_eval_bsdf_f(oc.fp(v), oc.fp(m), oc.fp(n), a, np.float32(1 / 1.5), d)))
        s1 = ctypes.c_uint(int(rng.integers(0, 2**32)))
        s2 = ctypes.c_uint(s1.value)
        o1, o2 = np.empty(3, np.float32), np.empty(3, np.float32)
        R.ref_sample_cosine_weighted(oc.fp(n), ctypes.byref(s1), oc.fp(o1))
        O.orc_sample_cosine_weighted_f(oc.fp(n), ctypes.byref(s2), oc.fp(o2))
        assert bits_equal(o1, o2) and s1.value == s2.value


def test_env_lookup_and_sampling_golden():
    from open_rendering_framework_b200 import scenes

    data = scenes.env_scene(8, 8, env_w=64, env_h=32)
    data.background.rgba = GOLD["env_map"]
    O = oc.OracleScene(data)
    mp, mc, cp, cc = O.env_tables()
    # the oracle's CDF build is the one the golden sampling vectors were made with
    for a, b in ((mp, "env_mpdf"), (mc, "env_mcdf"), (cp, "env_cpdf"), (cc, "env_ccdf")):
        assert bits_equal(a, GOLD[b])
    looked, fin, sdir, sL = O.env_query(GOLD["env_dirs"], GOLD["env_seeds"])
    assert bits_equal(looked, GOLD["env_looked"])
    assert bits_equal(sdir, GOLD["env_sdir"]) and bits_equal(sL, GOLD["env_sL"])
    assert np.array_equal(fin, GOLD["env_sfin"])


def test_env_tables_are_valid_distributions():
    from open_rendering_framework_b200 import scenes

    data = scenes.env_scene(8, 8, env_w=128, env_h=64)
    mp, mc, cp, cc = oc.OracleScene(data).env_tables()
    assert mc[-1] == 1.0 and cc[-1, -1] == 1.0
    assert np.all(np.diff(mc) >= 0) and np.all(np.diff(cc, axis=1) >= -1e-6)
    # marginal pdf integrates to 1 over rows, each conditional pdf to 1 over its row
    assert abs(mp.mean() - 1.0) < 1e-4
    assert np.allclose(cp.mean(axis=1), 1.0, atol=1e-4)


def test_dipoles_golden():
    """Standard and directional dipole of the restatement against the reference's outputs."""
    P = GOLD["dip_props"]
    for k in range(P.shape[0]):
        for j in range(GOLD["dip_dist"].size):
            assert bits_equal(oc.dipole_bssrdf(P[k], GOLD["dip_dist"][j]), GOLD["dip_std"][k, j]), (k, j)
            got = oc.dirpole_bssrdf(P[k], GOLD["dip_xi"][j], GOLD["dip_ni"][j], GOLD["dip_w12"][j], GOLD["dip_xo"][j], GOLD["dip_no"][j])
            assert bits_equal(got, GOLD["dip_dir"][k, j]), (k, j)


def test_scattering_properties_derivation():
    """computeCoefficients restated: the fixture's properties are reproduced bit for bit and obey
    the definitions (D = 1/(3 sigma_t'), sigma_tr = sqrt(sigma_a / D), A = (1 - C_E) / (2 C_phi))."""
    from open_rendering_framework_b200 import scene as sc, scenes

    for seed in range(4):
        s_, a_ = scenes.dipole_coefficients(seed)
        p = oc.compute_coefficients(sc.TranslucentMaterial(scattering=s_, absorption=a_, ior=1.3 + 0.1 * seed, scale=100.0))
        assert bits_equal(p, GOLD["dip_props"][seed])
        rec = p.view(sc.SCATTERING_PROPERTIES_DTYPE)[0]
        np.testing.assert_allclose(rec["D"], 1.0 / (3.0 * rec["reducedExtinction"]), rtol=1e-6)
        np.testing.assert_allclose(rec["transport"], np.sqrt(rec["absorption"] / rec["D"]), rtol=1e-6)
        np.testing.assert_allclose(rec["A"], (1.0 - rec["C_E"]) / (2.0 * rec["C_phi"]), rtol=1e-6)
        np.testing.assert_allclose(rec["absorption"], np.float32(a_) * np.float32(100.0), rtol=1e-7)


@pytest.mark.skipif(oc.ref() is None, reason="compiled reference (oracle/_ref) not built")
def test_fresh_dipoles_against_compiled_reference():
    from open_rendering_framework_b200 import scene as sc, scenes

    rng = np.random.default_rng(11)
    for seed in (5, 6):
        s_, a_ = scenes.dipole_coefficients(seed)
        P = oc.compute_coefficients(sc.TranslucentMaterial(scattering=s_, absorption=a_, meancosine=(0.3, 0.2, 0.1), ior=1.4, scale=30.0))
        for _ in range(500):
            d = np.float32(rng.uniform(0.0, 1.0))
            assert bits_equal(oc.dipole_bssrdf(P, d), oc.dipole_bssrdf(P, d, which="ref"))
            v = [rng.normal(size=3).astype(np.float32) for _ in range(5)]
            args = (v[0] * 0.2, v[1] / np.linalg.norm(v[1]), v[2] / np.linalg.norm(v[2]), v[3] * 0.2, v[4] / np.linalg.norm(v[4]))
            assert bits_equal(oc.dirpole_bssrdf(P, *args), oc.dirpole_bssrdf(P, *args, which="ref"))


def test_translucent_oracle_is_deterministic_and_well_formed():
    """The CPU restatement's probe pass and gathers give the same probes and image whatever the
    thread count (probe paths never read the probe set being built), and the probes are sane:
    unit normals, 0 <= T12 <= 1, L >= 0."""
    from open_rendering_framework_b200 import scenes

    data = scenes.translucent_box_scene(24, 24, subdiv=2, probe_samples=48, two_objects=True)
    out = []
    for threads in (1, 6):
        O = oc.OracleScene(data)
        acc, _ = O.render(0, 2, accum=np.zeros((24, 24, 4), np.float32), threads=threads)
        out.append((acc, O.probes()))
    assert bits_equal(out[0][0], out[1][0]) and bits_equal(out[0][1], out[1][1])
    pr = out[0][1]
    assert pr.shape == (96, 20)
    np.testing.assert_allclose(np.linalg.norm(pr[:, 6:9], axis=1), 1.0, atol=1e-5)
    assert np.all((pr[:, 15:18] >= 0) & (pr[:, 15:18] <= 1)) and np.all(pr[:, 9:12] >= 0)
    assert np.any(pr[:, 9:12] > 0)


def test_tape_gradient_matches_fp64_central_differences():
    """The FP64 path-tape gradient (the adjoint's reference) against FP64 central differences of the
    loss: albedo texels (next-event estimates and bounce weights), GGX roughness texels and the six
    dipole sigmas (Beer transmittance and dipole gathers)."""
    from open_rendering_framework_b200 import scenes

    data, (dif, met, tr) = scenes.inverse_scene(16, 16, subdiv=2, tex_res=18, probe_samples=24, seed=1)
    O = oc.OracleScene(data)
    O.record(True)
    acc, _ = O.render(0, 3, accum=np.zeros((16, 16, 4), np.float32), threads=4)
    tex_off, mat_off, n = O.param_layout([dif, met, tr])
    P = np.concatenate([dif.texture.ravel(), met.texture.ravel(), np.asarray(tr.absorption, np.float32),
                        np.asarray(tr.scattering, np.float32)]).astype(np.float64)
    img, _ = O.tape_eval(P, tex_off, mat_off)
    # the tape re-evaluates the rendered image
    assert np.max(np.abs(img - acc[..., :3].reshape(-1, 3)) / np.maximum(np.abs(acc[..., :3].reshape(-1, 3)), 1e-6)) < 1e-3
    target = img * 0.5 + 0.01
    _, g = O.tape_eval(P, tex_off, mat_off, dimg=2.0 * (img - target))

    def loss(Pv):
        im, _ = O.tape_eval(Pv, tex_off, mat_off)
        return np.sum((im - target) ** 2)

    nz = np.nonzero(g)[0]
    n_alb = dif.texture.size
    alb = nz[nz < n_alb]
    rgh = nz[(nz >= n_alb) & (nz < n - 6)]
    assert len(alb) > 10 and len(rgh) > 5
    rng = np.random.default_rng(2)
    pick = list(rng.choice(alb, 8, replace=False)) + list(rng.choice(rgh, 5, replace=False)) + list(range(n - 6, n))
    for i in pick:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += 1e-4
        Pm[i] -= 1e-4
        fd = (loss(Pp) - loss(Pm)) / 2e-4
        assert abs(fd - g[i]) <= 1e-5 * abs(fd) + 1e-12, (i, fd, g[i])
