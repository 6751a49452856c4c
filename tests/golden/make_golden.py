"""Generate the golden vectors in tests/golden/ref_math.npz from the reference itself.

The reference has no tests or fixtures of its own, so its own device-math headers, compiled for
the host from the reference sources (oracle/_ref/libref_oracle.so, built by oracle/Makefile),
produce the vectors.  Inputs are seeded numpy draws; every output is whatever the reference code
returns for them.  Run from the repository root:  python tests/golden/make_golden.py
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle_ctypes as oc  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_math.npz")


def unit_vectors(rng, n, upper=True):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    if upper:
        v[:, 2] = np.abs(v[:, 2]) + 1e-3
        v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v.astype(np.float32)


def main():
    R = oc.ref()
    if R is None:
        raise SystemExit("oracle/_ref/libref_oracle.so is not built (needs the reference sources)")
    rng = np.random.default_rng(20261203)
    g = {}

    # RNG streams (random.h): 64 seeds x 32 draws each.
    seeds = rng.integers(0, 2**32, size=64, dtype=np.uint64).astype(np.uint32)
    g["rng_seeds"] = seeds
    for kind, fn in (("tea", R.ref_rnd_tea_stream), ("lcg", R.ref_rnd_lcg_stream)):
        out = np.empty((64, 32), np.float32)
        fin = np.empty(64, np.uint32)
        for k, s in enumerate(seeds):
            row = np.empty(32, np.float32)
            fin[k] = fn(int(s), oc.fp(row), 32)
            out[k] = row
        g["rng_%s" % kind] = out
        g["rng_%s_final" % kind] = fin
    md5 = np.empty((64, 32), np.float32)
    md5_final = np.empty((64, 2), np.uint32)
    for k in range(64):
        x = ctypes.c_uint(int(seeds[k]))
        y = ctypes.c_uint(int(seeds[(k + 1) % 64]))
        row = np.empty(32, np.float32)
        R.ref_rnd_md5_stream(ctypes.byref(x), ctypes.byref(y), oc.fp(row), 32)
        md5[k] = row
        md5_final[k] = (x.value, y.value)
    g["rng_md5"] = md5
    g["rng_md5_final"] = md5_final
    tea_ab = rng.integers(0, 2**32, size=(256, 2), dtype=np.uint64).astype(np.uint32)
    g["tea16_in"] = tea_ab
    g["tea16_out"] = np.array([R.ref_tea16(int(a), int(b)) for a, b in tea_ab], np.uint32)

    # Config-1 BSDF queries: 4096 queries, first half GGX, from the synthetic generator.
    n = 4096
    wo, alpha = oc.c1_inputs(n)
    wi, f, pdf, F = oc.bsdf_queries(n, 0, n // 2, wo, alpha, which="ref")
    g.update(c1_wo=wo, c1_alpha=alpha, c1_wi=wi, c1_f=f, c1_pdf=pdf, c1_F=F)

    # Multiscattering walks (Microfacet.h:95-177), shading normal +z, both distributions.
    m = 256
    nrm = np.array([0, 0, 1], np.float32)
    ms_wi = unit_vectors(rng, m)
    ms_wo = unit_vectors(rng, m, upper=False)
    ms_alpha = rng.uniform(0.05, 1.0, m).astype(np.float32)
    ms_seed = rng.integers(0, 2**32, size=m, dtype=np.uint64).astype(np.uint32)
    ms_dist = (np.arange(m) % 2).astype(np.uint32)
    eta6 = np.array([0.2, 3.9, 0.55, 3.15, 0.9, 2.4], np.float64)
    inv = np.empty(6, np.float64)
    R.ref_complex_recip(oc.fp(eta6), oc.fp(inv))
    g.update(ms_wi=ms_wi, ms_wo=ms_wo, ms_alpha=ms_alpha, ms_seed=ms_seed, ms_dist=ms_dist, cond_ior=eta6, cond_eta=inv)
    diel = np.empty(m, np.float32)
    diel_seed = np.empty(m, np.uint32)
    cond = np.empty((m, 3), np.float32)
    cond_seed = np.empty(m, np.uint32)
    diff = np.empty((m, 3), np.float32)
    diff_seed = np.empty(m, np.uint32)
    rho = np.array([0.7, 0.5, 0.3], np.float32)
    for k in range(m):
        s = ctypes.c_uint(int(ms_seed[k]))
        diel[k] = R.ref_ms_dielectric_eval(oc.fp(ms_wi[k]), oc.fp(ms_wo[k]), oc.fp(nrm), 1.0 / 1.5, ms_alpha[k], ms_alpha[k],
                                           ctypes.byref(s), 0, int(ms_dist[k]))
        diel_seed[k] = s.value
        s = ctypes.c_uint(int(ms_seed[k]))
        out = np.empty(3, np.float32)
        R.ref_ms_conductor_eval(oc.fp(ms_wi[k]), oc.fp(np.abs(ms_wo[k]).astype(np.float32)), oc.fp(nrm), oc.fp(inv), ms_alpha[k], ms_alpha[k],
                                ctypes.byref(s), 0, int(ms_dist[k]), oc.fp(out))
        cond[k] = out
        cond_seed[k] = s.value
        s = ctypes.c_uint(int(ms_seed[k]))
        R.ref_ms_diffuse_eval(oc.fp(ms_wi[k]), oc.fp(np.abs(ms_wo[k]).astype(np.float32)), oc.fp(nrm), ms_alpha[k], ms_alpha[k],
                              ctypes.byref(s), 0, oc.fp(rho), int(ms_dist[k]), oc.fp(out))
        diff[k] = out
        diff_seed[k] = s.value
    g.update(ms_diel=diel, ms_diel_seed=diel_seed, ms_cond=cond, ms_cond_seed=cond_seed, ms_diff=diff, ms_diff_seed=diff_seed,
             ms_rho=rho)

    # Conductor Fresnel with complex IOR (Fresnel.h:78-91).
    fw = unit_vectors(rng, m)
    fm = unit_vectors(rng, m)
    fc = np.empty((m, 3), np.float32)
    for k in range(m):
        out = np.empty(3, np.float32)
        R.ref_fresnel_complex(oc.fp(fw[k]), oc.fp(fm[k]), oc.fp(inv), oc.fp(out))
        fc[k] = out
    g.update(fc_wi=fw, fc_m=fm, fc_out=fc)

    # Environment map lookup and importance sampling (Envmap.h:57-98) on a small procedural map, with
    # the CDF tables built by the oracle restatement of env_cameras.cu (that program is not compiled by
    # the reference build, so its restatement is checked for self-consistency in the tests instead).
    from open_rendering_framework_b200 import scenes

    env = scenes.sky_envmap(64, 32, sun_peak=5.0e4, sun_sigma_deg=8.0)
    data = scenes.env_scene(8, 8, env_w=64, env_h=32)
    data.background.rgba = env
    O = oc.OracleScene(data)
    mp, mc, cp, cc = O.env_tables()
    R.ref_set_envmap(oc.fp(env), env.shape[1], env.shape[0], oc.fp(mp), oc.fp(mc), oc.fp(cp), oc.fp(cc))
    dirs = unit_vectors(rng, 256, upper=False)
    seeds = rng.integers(0, 2**32, size=256, dtype=np.uint64).astype(np.uint32)
    looked = np.empty((256, 3), np.float32)
    sdir = np.empty((256, 3), np.float32)
    sL = np.empty((256, 3), np.float32)
    sfin = np.empty(256, np.uint32)
    pos = np.zeros(3, np.float32)
    for k in range(256):
        R.ref_env_lookup(oc.fp(dirs[k]), oc.fp(looked[k]))
        s_ = ctypes.c_uint(int(seeds[k]))
        R.ref_sample_environment(oc.fp(pos), ctypes.byref(s_), oc.fp(sdir[k]), oc.fp(sL[k]))
        sfin[k] = s_.value
    g.update(env_map=env, env_mpdf=mp, env_mcdf=mc, env_cpdf=cp, env_ccdf=cc, env_dirs=dirs, env_looked=looked, env_seeds=seeds,
             env_sdir=sdir, env_sL=sL, env_sfin=sfin)

    # Dipole BSSRDFs (dipoles/standard_dipole.h, dipoles/directional_dipole.h) on scattering
    # properties from the restatement of TranslucentMaterial::computeCoefficients (that file needs Qt
    # and is not compiled; the derived properties are pinned by the dipoles' outputs).
    from open_rendering_framework_b200 import scene as sc

    r2 = np.random.default_rng(20261204)
    props = []
    for seed in range(4):
        s_, a_ = scenes.dipole_coefficients(seed)
        props.append(oc.compute_coefficients(sc.TranslucentMaterial(scattering=s_, absorption=a_, ior=1.3 + 0.1 * seed, scale=100.0)))
    props = np.stack(props)
    nd = 256
    dist = r2.uniform(0.0, 0.5, nd).astype(np.float32)
    dist[:8] = 0.0
    dp = np.empty((4, nd, 3), np.float32)
    xi = (r2.normal(size=(nd, 3)) * 0.3).astype(np.float32)
    xo = (r2.normal(size=(nd, 3)) * 0.3).astype(np.float32)
    xo[:4] = xi[:4]
    ni, no, w12 = unit_vectors(r2, nd, False), unit_vectors(r2, nd, False), unit_vectors(r2, nd, False)
    dd = np.empty((4, nd, 3), np.float32)
    for k in range(4):
        for j in range(nd):
            dp[k, j] = oc.dipole_bssrdf(props[k], dist[j], which="ref")
            dd[k, j] = oc.dirpole_bssrdf(props[k], xi[j], ni[j], w12[j], xo[j], no[j], which="ref")
    g.update(dip_props=props, dip_dist=dist, dip_std=dp, dip_xi=xi, dip_xo=xo, dip_ni=ni, dip_no=no, dip_w12=w12, dip_dir=dd)

    np.savez_compressed(OUT, **g)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
