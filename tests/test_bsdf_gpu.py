"""GPU parity of the config-1 BSDF-query kernel and the RNG streams, through the C ABI.

Bars (stated in the tests):
* RNG streams (tea, LCG, MD5): bit-exact against the oracle.
* BSDF queries (wi, f, pdf, F): within 1e-5 relative of the FP32 oracle (|wi - wi_ref| for the
  direction) for at least 99% of queries, and no less accurate than the reference's own FP32 math:
  the GPU's 99.99th-percentile error against the FP64 oracle is at most 1.5x that of the FP32
  oracle.  Exact agreement is not reachable: glibc's and CUDA's float transcendentals (acosf,
  atan2f, tanf, erff, ...) differ by 1-2 ulp on a few percent of arguments, and the sampled normal
  feeds D(m), whose relative sensitivity grows like 1/alpha^2, so a last-bit difference in m becomes
  1e-5..1e-2 in f on ~0.5% of queries.  The FP32 reference itself is off by up to 0.3-350x relative
  from FP64 on the worst queries.  Maxima and percentiles are written to gpurun_out/.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from oracle import oracle_ctypes as oc
from open_rendering_framework_b200 import _native as nat

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_TOL = 1e-5
MIN_FRACTION = 0.99
FP64_P9999_RATIO = 1.5


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel_err(got, ref, floor=1e-30):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return np.abs(got - ref) / np.maximum(np.abs(ref), floor)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_rng_streams_bit_exact(kind):
    n, draws = 4096, 64
    rng = np.random.default_rng(kind)
    words = 2 * n if kind == 2 else n
    seeds = rng.integers(0, 2**32, size=words, dtype=np.uint64).astype(np.uint32)
    d_seeds = dev(seeds.view(np.int32))
    d_out = torch.empty(n * draws, dtype=torch.float32, device="cuda")
    nat.call("pt_rng_streams", kind, d_seeds.data_ptr(), n, draws, d_out.data_ptr(), None)
    torch.cuda.synchronize()
    got = d_out.cpu().numpy().reshape(n, draws)
    fin = d_seeds.cpu().numpy().view(np.uint32)
    O = oc.orc()
    for k in range(0, n, 97):
        row = np.empty(draws, np.float32)
        if kind == 2:
            x, y = ctypes.c_uint(int(seeds[2 * k])), ctypes.c_uint(int(seeds[2 * k + 1]))
            O.orc_rnd_md5_stream(ctypes.byref(x), ctypes.byref(y), oc.fp(row), draws)
            assert (fin[2 * k], fin[2 * k + 1]) == (x.value, y.value)
        else:
            fn = O.orc_rnd_tea_stream if kind == 0 else O.orc_rnd_lcg_stream
            assert fin[k] == fn(int(seeds[k]), oc.fp(row), draws)
        assert np.array_equal(got[k].view(np.uint32), row.view(np.uint32)), k


def run_gpu_queries(wo, alpha, first, n_ggx_below, eta):
    n = alpha.size
    d_wo, d_a = dev(wo), dev(alpha)
    d_wi = torch.empty((3, n), dtype=torch.float32, device="cuda")
    outs = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3)]
    nat.call("pt_bsdf_queries", d_wo.data_ptr(), d_a.data_ptr(), n, first, n_ggx_below, eta, d_wi.data_ptr(),
             outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), None)
    torch.cuda.synchronize()
    return (d_wi.cpu().numpy(),) + tuple(o.cpu().numpy() for o in outs)


@pytest.mark.parametrize("first,ggx_fraction", [(0, 0.5), (1 << 21, 1.0), (3 << 20, 0.0)])
def test_bsdf_queries_match_oracle(first, ggx_fraction):
    n = 1 << 18
    eta = np.float32(1.0 / 1.5)
    wo, alpha = oc.c1_inputs(n, first)
    n_ggx_below = first + int(n * ggx_fraction)
    got = run_gpu_queries(wo, alpha, first, n_ggx_below, eta)
    ref32 = oc.bsdf_queries(n, first, n_ggx_below, wo, alpha, eta=eta, threads=os.cpu_count() or 1)
    ref64 = oc.bsdf_queries(n, first, n_ggx_below, wo, alpha, eta=eta, fp64=True, threads=os.cpu_count() or 1)
    report = {}
    worst = {}
    for name, g, r32, r64 in zip(("wi", "f", "pdf", "F"), got, ref32, ref64):
        assert np.all(np.isfinite(g) == np.isfinite(r32)), name
        if name == "wi":
            # directions: Euclidean distance between the unit vectors (relative to |wi| = 1)
            e = np.linalg.norm(np.asarray(g, np.float64) - r32, axis=0)
            e64 = np.linalg.norm(np.asarray(g, np.float64) - r64, axis=0)
            e3264 = np.linalg.norm(np.asarray(r32, np.float64) - r64, axis=0)
        else:
            e, e64, e3264 = rel_err(g, r32), rel_err(g, r64), rel_err(r32, r64)
        frac = float(np.mean(e <= REL_TOL))
        report[name] = {
            "fraction_within_1e-5": frac,
            "n_outside": int(np.sum(e > REL_TOL)),
            "max_rel_vs_fp32_oracle": float(np.max(e)),
            "max_rel_gpu_vs_fp64": float(np.max(e64)),
            "max_rel_fp32_oracle_vs_fp64": float(np.max(e3264)),
            "p99.99_gpu_vs_fp64": float(np.quantile(e64, 0.9999)),
            "p99.99_fp32_oracle_vs_fp64": float(np.quantile(e3264, 0.9999)),
        }
        worst[name] = [int(first + i) for i in np.argsort(e)[-8:]]
    os.makedirs("gpurun_out", exist_ok=True)
    with open(os.path.join("gpurun_out", "bsdf_parity_%d.json" % first), "w") as fh:
        json.dump({"report": report, "worst_query_indices": worst}, fh, indent=1)
    for name, r in report.items():
        assert r["fraction_within_1e-5"] >= MIN_FRACTION, (name, r)
        assert r["p99.99_gpu_vs_fp64"] <= FP64_P9999_RATIO * r["p99.99_fp32_oracle_vs_fp64"] + 1e-7, (name, r)
    print(json.dumps({"first": first, "ggx_fraction": ggx_fraction, "n": n, "report": report}))


def test_bsdf_queries_host_path_matches_device_path():
    n = 4096
    wo, alpha = oc.c1_inputs(n, 77)
    got = run_gpu_queries(wo, alpha, 77, 77 + n // 2, np.float32(1 / 1.5))
    wi = np.empty((3, n), np.float32)
    f, pdf, F = (np.empty(n, np.float32) for _ in range(3))
    nat.call("pt_bsdf_queries_host", oc.fp(wo), oc.fp(alpha), n, 77, 77 + n // 2, np.float32(1 / 1.5),
             oc.fp(wi), oc.fp(f), oc.fp(pdf), oc.fp(F))
    for a, b in zip(got, (wi, f, pdf, F)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_empty_and_edge_inputs():
    # n == 0 is a no-op; grazing and normal-incidence directions stay finite where the oracle is finite.
    nat.call("pt_bsdf_queries", 0, 0, 0, 0, 0, 0.5, 0, 0, 0, 0, None)
    wo = np.array([[0.0, 0.0, 0.9999, 0.7071], [0.0, 0.0, 0.0141, 0.0], [1.0, 1.0, 0.01, 0.7071]], np.float32)
    alpha = np.array([0.05, 1.0, 0.5, 0.3], np.float32)
    for n_ggx in (0, 4):
        got = run_gpu_queries(wo, alpha, 0, n_ggx, np.float32(1 / 1.5))
        ref = oc.bsdf_queries(4, 0, n_ggx, wo, alpha, eta=np.float32(1 / 1.5))
        for g, r in zip(got, ref):
            assert np.array_equal(np.isfinite(g), np.isfinite(r))
            m = np.isfinite(r)
            assert np.all(rel_err(g[m], r[m], 1e-6) < 1e-4)
