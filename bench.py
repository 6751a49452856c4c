"""Benchmark: Mpath-samples/s of the single-scene wavefront render on one B200 (per GPU replica), with the
metric's other two arms -- the 64-scene batch and forward + adjoint -- in the same default line.

Workload (one step, default --workload single_scene): 512 x 512 pixels x 64 camera samples (frames)
of the procedural single scene (box of 12 diffuse triangles, 81,920-triangle GGX conductor
icosphere, 20,480-triangle Beckmann dielectric icosphere, 0.25 x 0.25 quad light of radiance 15),
max depth 8, Russian roulette from depth 3 -- 16,777,216 path samples per step, traced as one
wavefront launch group.

The default line (single scene, one GPU) also carries `batched` and `fwd_adjoint` objects (the two
workloads below, each device-timed with its own `e2e`) and, for each arm, the relMSE of its image against
a 16x-spp render of the same scene (frames after the measured ones, so the two are independent).  Its
`roofline` is the extend kernel's instruction-issue roofline: warp instructions per traced segment from
the committed ncu record (profiles/k_extend_single_scene_ncu.csv) times the segments of a live-timed
render, against one warp instruction per clock per SM sub-partition at the sampled SM clock; the HBM
view (56 algorithmic bytes per segment) sits beside it.

--workload build: the BVH builders -- the subsurface mesh (327,680 triangles) and the 64 batch meshes,
host binned SAH vs the device LBVH (option bvh_builder), in ms per million triangles, and the
single-scene render over each tree.

--workload batched: 64 seeded procedural scenes (icospheres or heightfields of 1e3-5e5 triangles,
diffuse / GGX / Beckmann / rough-dielectric / dipole materials, 128^2-1024^2 pixels, 4-256 spp,
procedural sky light) rendered as one batch: one step = one batch render of every scene's spp, one
CUDA-graph launch, with the engine options from the autotuner.  The same frames rendered scene after
scene through single-scene passes (the plain path) are timed beside it (`plain`).

--workload adjoint: the differentiable configuration -- the single-scene geometry at 5 subdivisions
with a 256^2 x 3 albedo texture on the box, a 256^2 GGX roughness texture on the conductor sphere and
a dipole sphere whose sigma_a / sigma_s' are parameters (all seeded U[0.1, 0.9]), 256 x 256 x 64 spp,
depth 6; L2 loss against a target rendered at 1024 spp from other seeded parameters.  One step = the
differentiable forward render + the path-replay adjoint; `forward` reports the forward alone.

--workload bsdf: the batched BSDF-query configuration -- 2^22 FP32 queries per step (first half GGX,
second half Beckmann), alpha ~ U[0.05,1], cos(theta_o) ~ U[0.01,1], (u1,u2) from tea<16> seeded by
the query index, dielectric eta 1.5; per query the sampled visible normal's reflection wi, the
Walter BSDF value, the pdf and the Fresnel term.  Unit: M queries/s.  Its CPU baseline is the
reference's own Microfacet/Fresnel headers compiled for the host (oracle/_ref), on all host cores.

--workload ingest: the scene readers -- one step reads a 2048 x 1024 run-length-encoded .hdr sky into
the environment map (pt_set_envmap_hdr: host parse, device RGBE expansion, CDF build) and a
327,680-triangle OBJ icosphere with normals (pt_obj_read + arrays), both written from seeded data.
Unit: MB/s of file bytes.  Its reference arm times the reference's own HDRLoader and glm readers
compiled for the host (oracle/_ref/libref_io.so) on the same files.

--workload subsurface: 1024 x 1024 pixels x 256 frames (--spp) of the translucent scene: a
327,680-triangle jittered icosphere with the dipole BSSRDF (standard; --dipole directional), 4,096
probes per frame (2^20 over the 256 frames), lit by a 2048 x 1024 procedural sky with a sun lobe of
peak 5e4 as background and light.  Its dominant kernel is the dipole gather, which is bound by
integer issue (one MD5 hash per (gather, probe) pair), so its line reports pair evaluations per
second instead of a memory roofline.

Arms
  --impl ours (default): the CUDA path through the C ABI.  `value` is device-timed (CUDA events
      on the render stream, barrier + synchronize on both sides, max over ranks); `e2e` times the
      public API with host buffers: per step a camera + material update (H2D), the render, and the
      float4 image read back into pinned host memory (D2H).
  --impl reference: the reference's path tracer has no CPU build (OptiX), so its CPU restatement
      (oracle/orc/orc_trace.cpp: path_tracer.cu and the shaders, recursive, the reference's math)
      runs on all host cores over a bounded sample of the same workload.

Multi-GPU: the path shards by scene/frames with no exchange step, so N GPUs run N independent
replicas (weak scaling); value = all ranks' path samples / max-over-ranks time.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpath-samples/s plain vs batched vs fwd+adjoint on 1 B200 at equal image relMSE"
UNIT = "Mpath-samples/s"
WORKLOAD = ("single-scene render 512x512, 64 spp, max depth 8, Russian roulette from depth 3: 12-triangle diffuse box, "
            "81,920-triangle GGX conductor icosphere, 20,480-triangle Beckmann rough-dielectric icosphere, quad light")
EXTEND_BYTES_PER_SEGMENT = 56  # queue id 4 + ray 32 + hit record 16 + material-queue append 4
GATHER_INSTR_PER_PAIR = 256    # thread instructions per (gather, probe) pair of k_gather, from its ncu capture


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="single_scene", choices=["single_scene", "subsurface", "batched", "adjoint", "bsdf", "ingest", "build", "queries"])
    ap.add_argument("--queries", type=int, default=1 << 22, help="bsdf and queries workloads: queries per step / launch")
    ap.add_argument("--scenes", type=int, default=64, help="batched workload: number of scenes")
    ap.add_argument("--spp", type=int, default=None, help="frames per step (default 64, subsurface 256)")
    ap.add_argument("--width", type=int, default=None)
    ap.add_argument("--height", type=int, default=None)
    ap.add_argument("--dipole", default="standard", choices=["standard", "directional"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-arms", action="store_true", help="single scene: skip the batched and forward+adjoint arms and the relMSE")
    return ap.parse_args()


SUBSURFACE = ("subsurface render 1024x1024, 256 spp, max depth 8: 327,680-triangle icosphere jittered by 2%% value noise, %s dipole "
              "BSSRDF with seeded sigma_s' ~ U[0.5,3]/mm and sigma_a ~ U[0.001,0.05]/mm per RGB, eta 1.3, 4,096 probes per frame "
              "(2^20 over 256 frames); 2048x1024 procedural sky + Gaussian sun lobe (peak 5e4) as background and importance-sampled light")


def workload(args):
    """(scene data, frames per step, description) of the selected workload."""
    from open_rendering_framework_b200 import scene as sc
    from open_rendering_framework_b200 import scenes

    if args.workload == "adjoint":
        w = args.width or 256
        data, _ = scenes.inverse_scene(w, w, subdiv=5, tex_res=256, seed=0)
        return data, args.spp or 64, ADJOINT
    if args.workload == "subsurface":
        w, h = args.width or 1024, args.height or 1024
        model = sc.DIRECTIONAL_DIPOLE if args.dipole == "directional" else sc.STANDARD_DIPOLE
        data = scenes.subsurface_scene(w, h, subdiv=7, probe_samples=4096, env_w=2048, env_h=1024, dipole_model=model)
        desc = SUBSURFACE % args.dipole
        if (w, h) != (1024, 1024):
            desc += " (resized to %dx%d)" % (w, h)
        return data, args.spp or 256, desc
    w, h = args.width or 512, args.height or 512
    desc = WORKLOAD if (w, h) == (512, 512) else WORKLOAD + " (resized to %dx%d)" % (w, h)
    return scenes.single_scene(width=w, height=h), args.spp or 64, desc


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_record(name):
    """Totals per metric over the launches of a committed ncu record under profiles/ (the tool's CSV:
    either one row per (launch, metric) from `--csv --log-file`, or one row per launch from
    `ncu -i ... --page raw --csv`), and the `# key: value` header lines above it.  None if absent."""
    import csv

    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    header, rows = {}, []
    with open(path) as fh:
        for line in fh:
            if line.startswith("#"):
                if ":" in line:
                    k, v = line[1:].split(":", 1)
                    header[k.strip()] = v.strip()
                continue
            rows.append(line)
    table = list(csv.reader(rows))
    if len(table) < 2:
        return None
    head = table[0]
    totals, launches = {}, set()
    num = lambda x: float(x.replace(",", ""))
    if "Metric Name" in head:
        k_id, k_name, k_val = head.index("ID"), head.index("Metric Name"), head.index("Metric Value")
        for r in table[1:]:
            if len(r) == len(head):
                launches.add(r[k_id])
                totals[r[k_name]] = totals.get(r[k_name], 0.0) + num(r[k_val])
    else:
        first = head.index("CC") + 1
        for r in table[2:]:  # row 1 holds the units
            if len(r) != len(head):
                continue
            launches.add(r[head.index("ID")])
            for k in range(first, len(head)):
                totals[head[k]] = totals.get(head[k], 0.0) + num(r[k])
    return {"totals": totals, "launches": len(launches), "header": header}


def extend_capture_record():
    """Per-segment figures of the extend kernel from its committed ncu record
    (profiles/k_extend_single_scene_ncu.csv: the raw ncu rows of every k_extend_persistent launch of the
    first render of the capture command, preceded by '#' lines that give the segments those launches
    traced, from the same command's JSON line).  Returns {"warp_inst_per_segment",
    "thread_inst_per_warp_inst", "dram_bytes_per_segment", "segments", "launches"} or None."""
    rec = ncu_record("k_extend_single_scene_ncu.csv")
    if not rec or "segments" not in rec["header"]:
        return None
    segments = float(rec["header"]["segments"].split()[0].replace(",", ""))
    t = rec["totals"]
    warp = t.get("smsp__inst_executed.sum", 0.0)
    if warp <= 0 or segments <= 0:
        return None
    dram = t["dram__bytes_read.sum"] + t["dram__bytes_write.sum"]
    return {"warp_inst_per_segment": warp / segments, "thread_inst_per_warp_inst": t["smsp__thread_inst_executed.sum"] / warp,
            "dram_bytes_per_segment": dram / segments, "segments": segments, "launches": rec["launches"]}


def bsdf_capture_record():
    """Per-query figures of the BSDF-query kernels from their committed ncu record
    (profiles/k_bsdf_queries_c1_ncu.csv: both launches of one step, the query count in its header)."""
    rec = ncu_record("k_bsdf_queries_c1_ncu.csv")
    if not rec or "queries" not in rec["header"]:
        return None
    q = float(rec["header"]["queries"])
    t = rec["totals"]
    return {"warp_inst_per_query": t["smsp__inst_executed.sum"] / q,
            "dram_bytes_per_query": (t["dram__bytes_read.sum"] + t["dram__bytes_write.sum"]) / q, "launches": rec["launches"]}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        # the timed region starts once the sampler is live (its first row has arrived)
        t0 = time.perf_counter()
        while self.proc and not self.rows and self.proc.poll() is None and time.perf_counter() - t0 < 3.0:
            time.sleep(0.02)
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "", 1).isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def max_over_ranks(x, world, device="cuda"):
    """The largest of the ranks' values of x: one all-reduce (MAX) that every rank makes at the same
    point (a multi-GPU time is the slowest rank's).  One rank: x itself."""
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, world, steps, seconds_max):
    """Whole-job throughput of independent replicas, in millions of units per second: the units all
    ranks processed over the slowest rank's time."""
    return world * steps * units_per_rank / seconds_max / 1e6


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def cpu_baseline_sample(data, target_s=12.0, threads=None):
    """Times the CPU restatement of the reference tracer on a bounded sample of the workload."""
    from oracle import oracle_ctypes as oc

    threads = threads or os.cpu_count() or 1
    O = oc.OracleScene(data)
    W = data.camera.width
    # calibrate on a small band, then size the sample for ~target_s seconds
    rows = 4
    mid = data.camera.height // 2 - rows // 2
    t0 = time.perf_counter()
    O.render(0, 1, p_begin=W * mid, p_end=W * (mid + rows), threads=threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    rate = rows * W / dt
    n_paths = int(min(max(rate * target_s, W), W * data.camera.height * 64))
    frames = max(1, min(64, n_paths // (W * 32)))
    if data.translucent_objects():
        frames = max(1, min(4, frames))  # every frame also runs the probe pass
    band = max(1, min(data.camera.height, n_paths // (W * frames)))
    p0 = W * max(0, (data.camera.height - band) // 2)
    t0 = time.perf_counter()
    O.render(0, frames, p_begin=p0, p_end=p0 + W * band, threads=threads)
    dt = time.perf_counter() - t0
    samples = W * band * frames
    O.close()
    return {"value": samples / dt / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%d rows x %d px x %d spp (%d path samples) of the same scene, CPU restatement of the reference's "
                      "recursive path tracer (path_tracer.cu + shaders, its own math; probe pass included), %d threads, %.1f s" % (
                          band, W, frames, samples, threads, dt)}


def run_reference_batched(args):
    """Reference arm of the batched workload: the CPU restatement on a bounded sample of each step's
    work -- step k renders 8 rows through the middle of scene k mod n at one sample per pixel."""
    from oracle import oracle_ctypes as oc
    from open_rendering_framework_b200 import scenes

    S = scenes.batch_scenes(args.scenes, seed=0)
    threads = os.cpu_count() or 1
    band = 8
    total, samples = 0.0, 0
    for k in range(args.warmup + args.steps):
        data = S[k % len(S)][0]
        O = oc.OracleScene(data)
        W, H = data.camera.width, data.camera.height
        p0 = W * max(0, H // 2 - band // 2)
        t0 = time.perf_counter()
        O.render(0, 1, p_begin=p0, p_end=p0 + W * band, threads=threads)
        dt = time.perf_counter() - t0
        O.close()
        if k >= args.warmup:
            total += dt
            samples += W * band
    value = samples / total / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total * 1e3 / max(1, args.steps), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": BATCHED % len(S), "sample_per_step": "8 rows x 1 spp of scene (step mod %d)" % len(S)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "8 rows x 1 spp of one scene per step, scenes in order; CPU restatement of the reference's "
                                   "recursive tracer (probe pass included), all host cores"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


BSDF = ("batched BSDF queries: %d FP32 queries per step, first half GGX and second half Beckmann, alpha ~ U[0.05,1], "
        "cos(theta_o) ~ U[0.01,1], (u1,u2) from tea<16> seeded by the query index, dielectric eta 1.5; outputs the sampled "
        "wi, the Walter BSDF value, the pdf and the Fresnel term")
BSDF_BYTES_PER_QUERY = 40  # in: wo 12 + alpha 4; out: wi 12 + f 4 + pdf 4 + F 4


def bsdf_cpu_sample(n_max, target_s=10.0, threads=None):
    """Times the reference's own Microfacet/Fresnel headers compiled for the host (oracle/_ref) on the
    same query batch, over all host cores (one ctypes call per thread and contiguous chunk of query
    indices; ctypes releases the GIL).  The sample takes equal numbers of queries from the GGX half
    and the Beckmann half of the batch.  Falls back to the oracle restatement if the compiled
    reference is absent."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle_ctypes as oc

    threads = threads or os.cpu_count() or 1
    kind = "reference" if oc.ref() is not None else "port"
    which = "ref" if kind == "reference" else "orc"

    def run(n_half):
        jobs = []
        per = max(1, (n_half + threads - 1) // threads)
        for base in (0, n_max // 2):
            for t in range(threads):
                first = base + t * per
                cnt = min(per, base + n_half - first)
                if cnt <= 0:
                    break
                wo, alpha = oc.c1_inputs(cnt, first)
                jobs.append((first, cnt, wo, alpha))
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=threads) as ex:
            list(ex.map(lambda j: oc.bsdf_queries(j[1], j[0], n_max // 2, j[2], j[3], which=which), jobs))
        return time.perf_counter() - t0, sum(j[1] for j in jobs)

    dt, done = run(min(n_max // 2, 1 << 14))
    rate = done / max(dt, 1e-3)
    dt, done = run(int(min(n_max // 2, max(1 << 14, rate * target_s / 2))))
    return {"value": done / dt / 1e6, "unit": "M queries/s", "cores": threads, "kind": kind,
            "sample": "%d queries (half from each distribution's range of the %d-query batch), %s, %d threads, %.1f s" % (
                done, n_max, "the reference's Microfacet/Fresnel headers compiled for the host with g++ -O2, no fast-math"
                if kind == "reference" else "the oracle restatement of the reference's math", threads, dt)}


def run_bsdf(args, world, rank, local):
    import torch

    from open_rendering_framework_b200 import _native as nat

    torch.cuda.set_device(local)
    n = args.queries
    L = nat.lib()
    wo = np.empty((3, n), np.float32)
    alpha = np.empty(n, np.float32)
    nat.call("pt_c1_make_inputs", n, 0, wo.ctypes.data, alpha.ctypes.data)
    dev = torch.device("cuda", local)
    d_wo = torch.from_numpy(wo).to(dev)
    d_a = torch.from_numpy(alpha).to(dev)
    d_wi = torch.empty((3, n), dtype=torch.float32, device=dev)
    d_f, d_pdf, d_F = (torch.empty(n, dtype=torch.float32, device=dev) for _ in range(3))
    stream = torch.cuda.current_stream(dev)
    sh = ctypes.c_void_p(stream.cuda_stream)

    def launch():
        nat.call("pt_bsdf_queries", d_wo.data_ptr(), d_a.data_ptr(), n, 0, n // 2, 1.0 / 1.5, d_wi.data_ptr(), d_f.data_ptr(),
                 d_pdf.data_ptr(), d_F.data_ptr(), sh)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    for _ in range(max(3, args.warmup)):
        launch()
    torch.cuda.synchronize()
    barrier()
    launches0 = L.pt_kernel_launch_count()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clocks:
        evs[0].record(stream)
        for k in range(args.steps):
            launch()
            evs[k + 1].record(stream)
        torch.cuda.synchronize()
    launches = L.pt_kernel_launch_count() - launches0
    ms = evs[0].elapsed_time(evs[-1])
    barrier()
    t_max = max_over_ranks(ms, world, dev)
    ms_max = t_max
    value = replica_throughput(n, world, args.steps, ms_max * 1e-3)

    # end to end: host buffers through pt_bsdf_queries_host (H2D of wo and alpha, the kernel, D2H of
    # wi, f, pdf and F, synchronous) from pinned host memory
    h_wo = torch.from_numpy(wo).pin_memory()
    h_a = torch.from_numpy(alpha).pin_memory()
    h_wi = torch.empty((3, n), dtype=torch.float32).pin_memory()
    h_f, h_pdf, h_F = (torch.empty(n, dtype=torch.float32).pin_memory() for _ in range(3))

    def host_call():
        nat.call("pt_bsdf_queries_host", h_wo.data_ptr(), h_a.data_ptr(), n, 0, n // 2, 1.0 / 1.5, h_wi.data_ptr(), h_f.data_ptr(),
                 h_pdf.data_ptr(), h_F.data_ptr())

    host_call()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        host_call()
    e2e_s = time.perf_counter() - t0
    t_max = max_over_ranks(e2e_s, world, dev)
    e2e_value = replica_throughput(n, world, args.steps, t_max)
    same = bool(torch.equal(h_f, d_f.cpu()) and torch.equal(h_wi, d_wi.cpu()))

    peak, peak_kind = load_peaks()
    launch_ms = ms_max / args.steps
    achieved = BSDF_BYTES_PER_QUERY * n / (launch_ms * 1e-3) / 1e9
    rec = bsdf_capture_record()
    sm_mhz = clocks.summary().get("sm_mhz") or 1965.0
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    issue_peak = n_sm * 4 * sm_mhz * 1e6 / 1e9
    issue_achieved = rec["warp_inst_per_query"] * n / (launch_ms * 1e-3) / 1e9 if rec else None
    line = {
        "metric": "M BSDF queries/s (batched BSDF queries on 1 B200)", "value": value, "unit": "M queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": launch_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": BSDF % n, "queries_per_step": n, "parallelism": "replicas (one independent batch per GPU)",
                   "l2": "inputs + outputs of %.0f MB per step, larger than L2" % (BSDF_BYTES_PER_QUERY * n / 1e6)},
        "e2e": {"value": e2e_value, "unit": "M queries/s", "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 24 * n,
                "what": "pt_bsdf_queries_host from pinned host buffers (copies in, kernels, copies out in chunks of 2^19 queries on two streams; synchronous)",
                "identical_to_device_path": same},
        "roofline": {"bound": "issue", "kernel": "k_bsdf_queries (GGX and Beckmann launches of one step)",
                     "achieved": issue_achieved, "peak": issue_peak, "unit": "G warp instructions/s",
                     "frac": issue_achieved / issue_peak if issue_achieved else None,
                     "peak_source": "1 warp instruction / clock / SM sub-partition x 4 x %d SMs x median SM clock %.0f MHz" % (n_sm, sm_mhz),
                     "warp_instructions_per_query": rec["warp_inst_per_query"] if rec else None,
                     "traffic": rec["dram_bytes_per_query"] * n if rec else None,
                     "traffic_unit": "DRAM bytes per step (ncu record of the same launch size, profiles/k_bsdf_queries_c1_ncu.csv)",
                     "hbm": {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                             "algorithmic_bytes_per_query": BSDF_BYTES_PER_QUERY},
                     "note": "the kernels are bound by instruction issue (16-round TEA, transcendentals, the Beckmann Newton loop and "
                             "double erfinv), not by their 40 algorithmic bytes per query"},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = bsdf_cpu_sample(n)
        one = bsdf_cpu_sample(n, target_s=2.0, threads=1)
        line["cpu_baseline"]["one_core"] = {"value": one["value"], "unit": one["unit"], "sample": one["sample"]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference_bsdf(args):
    """Reference arm of the bsdf workload: the reference's headers compiled for the host, all host
    cores, each step a bounded sample of the query batch."""
    n = args.queries
    for _ in range(max(0, min(args.warmup, 1))):
        bsdf_cpu_sample(n, target_s=1.0)
    vals, secs = [], 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        s = bsdf_cpu_sample(n, target_s=4.0)
        secs += time.perf_counter() - t0
        vals.append(s["value"])
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "M BSDF queries/s (batched BSDF queries on 1 B200)", "value": value, "unit": "M queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": BSDF % n, "sample_per_step": s["sample"]},
        "cpu_baseline": dict(s, value=value),
        "e2e": {"value": value, "unit": "M queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


INGEST = ("scene readers: a 2048x1024 run-length-encoded RGBE sky (.hdr) into the environment map and a 327,680-triangle "
          "icosphere OBJ with vertex normals (v//n faces), written from seeded data")


def ingest_files(directory):
    """The .hdr and .obj files of the ingest workload (written once per run)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import io_samples

    from open_rendering_framework_b200 import scenes

    hdr = os.path.join(directory, "sky.hdr")
    sky = scenes.sky_envmap(2048, 1024)
    with open(hdr, "wb") as f:
        f.write(io_samples.hdr_bytes(io_samples.rgbe_from_float(sky[::-1, :, :3]), rle=True))
    pos, idx, nrm, nidx = scenes.icosphere(7, 1.0)
    obj = os.path.join(directory, "sphere.obj")
    with open(obj, "w") as f:
        f.write("".join("v %.7g %.7g %.7g\n" % tuple(p) for p in pos))
        f.write("".join("vn %.7g %.7g %.7g\n" % tuple(n) for n in nrm))
        f.write("".join("f %d//%d %d//%d %d//%d\n" % (a + 1, x + 1, b + 1, y + 1, c + 1, z + 1) for (a, b, c), (x, y, z) in zip(idx, nidx)))
    return hdr, obj


def run_ingest(args, world, rank, local):
    import tempfile

    import torch

    from open_rendering_framework_b200 import _native as nat
    from open_rendering_framework_b200 import scene as sc

    torch.cuda.set_device(local)
    with tempfile.TemporaryDirectory() as d:
        hdr, obj = ingest_files(d)
        nbytes = os.path.getsize(hdr) + os.path.getsize(obj)
        R = sc.Renderer(__import__("open_rendering_framework_b200.scenes", fromlist=["x"]).single_scene(width=16, height=16, metal_subdiv=1,
                                                                                                       glass_subdiv=1), device=local)
        L = nat.lib()

        def step():
            nat.call("pt_set_envmap_hdr", R.ctx, hdr.encode())
            m = ctypes.c_void_p()
            nat.call("pt_obj_read", obj.encode(), ctypes.byref(m))
            info = (ctypes.c_uint32 * 5)()
            nat.call("pt_obj_get_info", m, info)
            pos = np.empty(3 * info[0], np.float32)
            nrm = np.empty(3 * info[1], np.float32)
            vi = np.empty(3 * info[3], np.int32)
            ni = np.empty(3 * info[3], np.int32)
            nat.call("pt_obj_get_arrays", m, pos.ctypes.data, nrm.ctypes.data, None, vi.ctypes.data, ni.ctypes.data, None, None)
            nat.call("pt_obj_free", m)

        for _ in range(max(3, args.warmup)):
            step()
        torch.cuda.synchronize()
        launches0 = L.pt_kernel_launch_count()
        with ClockSampler(local) as clocks:
            t0 = time.perf_counter()
            for _ in range(args.steps):
                step()
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
        launches = L.pt_kernel_launch_count() - launches0
        R.close()
        value = args.steps * nbytes / dt / 1e6
        line = {
            "metric": "MB/s of scene files read (ingest)", "value": value, "unit": "MB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8/f32", "data": "synthetic",
            "config": {"workload": INGEST, "bytes_per_step": nbytes},
            "e2e": {"value": value, "unit": "MB/s", "h2d_bytes_per_step": 2048 * 1024 * 4, "d2h_bytes_per_step": 0,
                    "what": "file bytes read from the page cache through the C ABI, device decode and CDF build included"},
            "gpu_launches": int(launches), "clocks": clocks.summary(),
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = ingest_reference(hdr, obj, nbytes, 3)
        print(json.dumps(line), flush=True)


def ingest_reference(hdr, obj, nbytes, reps):
    """The reference's HDRLoader (loadHDRTexture) and glmReadOBJ compiled for the host, on the same files."""
    lib = os.path.join(ROOT, "oracle", "_ref", "libref_io.so")
    if not os.path.exists(lib):
        return {"value": None, "unit": "MB/s", "cores": 1, "kind": "reference", "sample": "oracle/_ref/libref_io.so not built"}
    L = ctypes.CDLL(lib)
    w, h = ctypes.c_uint(), ctypes.c_uint()
    buf = np.empty(4 * 2048 * 1024, np.float32)
    counts = (ctypes.c_uint * 5)()
    t0 = time.perf_counter()
    for _ in range(reps):
        L.ref_hdr_load(hdr.encode(), buf.ctypes.data_as(ctypes.c_void_p), ctypes.c_ulong(buf.size), ctypes.byref(w), ctypes.byref(h))
        L.ref_obj_load(obj.encode(), counts, *([None] * 8), 0)
    dt = time.perf_counter() - t0
    return {"value": reps * nbytes / dt / 1e6, "unit": "MB/s", "cores": 1, "kind": "reference",
            "sample": "%d reads of both files by HDRLoader.cpp + glm.cpp compiled for the host (one thread, as in the reference)" % reps}


def run_reference_ingest(args):
    import tempfile

    with tempfile.TemporaryDirectory() as d:
        hdr, obj = ingest_files(d)
        nbytes = os.path.getsize(hdr) + os.path.getsize(obj)
        ingest_reference(hdr, obj, nbytes, 1)
        s = ingest_reference(hdr, obj, nbytes, max(1, args.steps))
    line = {"impl": "reference", "metric": "MB/s of scene files read (ingest)", "value": s["value"], "unit": "MB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": nbytes / (s["value"] or 1) / 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/f32", "data": "synthetic", "config": {"workload": INGEST},
            "cpu_baseline": s, "e2e": {"value": s["value"], "unit": "MB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


QUERIES = ("per-query entries: %d queries per launch of the dipole BSSRDF of one translucent material (the subsurface "
           "configuration's seeded coefficients, eta 1.3, scale 100; standard dipole on distances log-uniform over 1e-3..30 mean "
           "free paths, directional dipole on point pairs of a sphere of 50 mean free paths with random incoming directions; FP32 "
           "and FP64) and of the multiscattering walks and the conductor Fresnel (GGX and Beckmann, alpha ~ U[0.1, 0.9], upper-"
           "hemisphere directions, the single-scene conductor's complex IOR)")
MSQ_OPS = ["dielectric_eval", "dielectric_sample", "conductor_eval", "conductor_sample", "diffuse_eval", "diffuse_sample",
           "conductor_fresnel", "visible_normal"]


def query_inputs(n, seed=0):
    """Seeded inputs of the per-query workload: the material, the standard dipole's distances, the
    directional dipole's 15 x n rows, and the microfacet walks' wi, wo, alpha."""
    import numpy as np

    from open_rendering_framework_b200 import scenes

    rng = np.random.default_rng(seed)
    sigma_s, sigma_a = scenes.dipole_coefficients(3)
    params = (np.float32(sigma_a), np.float32(sigma_s), np.zeros(3, np.float32), 1.3, 100.0)
    mfp = 1.0 / float(params[4] * (np.min(params[1]) + np.min(params[0])))
    dist = (mfp * np.exp(rng.uniform(np.log(1e-3), np.log(30.0), n))).astype(np.float32)

    def unit(m):
        v = rng.normal(size=(m, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    Rs = 50.0 * mfp
    ni = unit(n)
    t = np.cross(ni, unit(n))
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    ang = dist / Rs
    no = ni * np.cos(ang)[:, None] + t * np.sin(ang)[:, None]
    w12 = unit(n)
    w12 = np.where((np.sum(w12 * ni, axis=1) > 0)[:, None], -w12, w12)
    geo = np.concatenate([(Rs * ni).T, ni.T, w12.T, (Rs * no).T, no.T]).astype(np.float32)
    up = lambda v: np.where(v[:, 2:3] < 0, v * np.array([1, 1, -1]), v)
    wi = up(unit(n)).T.astype(np.float32)
    wo = up(unit(n)).T.astype(np.float32)
    alpha = rng.uniform(0.1, 0.9, n).astype(np.float32)
    return params, dist, geo, np.ascontiguousarray(wi), np.ascontiguousarray(wo), alpha


def run_queries(args, world, rank, local):
    """Throughput of the per-query entries (pt_bssrdf_queries in FP32 and FP64, pt_microfacet_queries for
    every operation and both distributions) at a launch size larger than L2, device-resident inputs."""
    import ctypes

    import numpy as np
    import torch

    from open_rendering_framework_b200 import _native as nat
    from open_rendering_framework_b200 import scene as sc

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.queries
    params, dist, geo, wi, wo, alpha = query_inputs(n)
    tp = sc.TranslucentParams((ctypes.c_float * 3)(*params[1]), (ctypes.c_float * 3)(*params[0]), (ctypes.c_float * 3)(*params[2]),
                              params[3], params[4], sc.STANDARD_DIPOLE)
    d_dist, d_geo = torch.from_numpy(dist).to(dev), torch.from_numpy(geo).to(dev)
    d_wi, d_wo, d_alpha = torch.from_numpy(wi).to(dev), torch.from_numpy(wo).to(dev), torch.from_numpy(alpha).to(dev)
    d_seed = torch.arange(n, dtype=torch.int32, device=dev)
    d_order = torch.zeros(n, dtype=torch.int32, device=dev)
    out32 = torch.empty((3, n), dtype=torch.float32, device=dev)
    out64 = torch.empty((3, n), dtype=torch.float64, device=dev)
    weight = torch.empty((3, n), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    launches = [0]

    def bssrdf(model, precision, d_in):
        tp.dipole_model = model
        nat.call("pt_bssrdf_queries", ctypes.byref(tp), precision, d_in.data_ptr(), n, (out64 if precision else out32).data_ptr(), sp)
        launches[0] += 1

    def walk(op, distn):
        b = sc.MicrofacetBatch()
        b.op, b.normal_distribution = op, distn
        b.normal[:] = [0.0, 0.0, 1.0]
        b.eta = 1.0 / 1.5
        b.ior[:] = [0.2, 3.9, 0.55, 3.15, 0.9, 2.4]
        b.rho[:] = [0.7, 0.7, 0.7]
        d_order.zero_()
        nat.call("pt_microfacet_queries", ctypes.byref(b), d_wi.data_ptr(), d_wo.data_ptr(), d_alpha.data_ptr(), d_seed.data_ptr(),
                 d_order.data_ptr(), n, out32.data_ptr(), weight.data_ptr(), sp)
        launches[0] += 1

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    peak, peak_kind = load_peaks()
    with ClockSampler(local) as clocks:
        per_op = {}
        for model, name, d_in, in_bytes in ((sc.STANDARD_DIPOLE, "standard", d_dist, 4), (sc.DIRECTIONAL_DIPOLE, "directional", d_geo, 60)):
            for precision, out_bytes in ((0, 12), (1, 24)):
                ms = timed(lambda: bssrdf(model, precision, d_in))
                per_op["bssrdf_%s_%s" % (name, "fp64" if precision else "fp32")] = {
                    "m_queries_per_s": n / (ms * 1e-3) / 1e6, "ms": ms,
                    "hbm_gb_s": (in_bytes + out_bytes) * n / (ms * 1e-3) / 1e9}
        for distn, dname in ((sc.GGX_DISTRIBUTION, "ggx"), (sc.BECKMANN_DISTRIBUTION, "beckmann")):
            for op, oname in enumerate(MSQ_OPS):
                ms = timed(lambda: walk(op, distn))
                per_op["%s_%s" % (oname, dname)] = {"m_queries_per_s": n / (ms * 1e-3) / 1e6, "ms": ms}
        # end to end: the directional dipole from pinned host rows, values read back, every step
        h_geo = torch.from_numpy(geo).pin_memory()
        h_out = torch.empty((3, n), dtype=torch.float32).pin_memory()

        def e2e_step():
            d_geo.copy_(h_geo, non_blocking=True)
            bssrdf(sc.DIRECTIONAL_DIPOLE, 0, d_geo)
            h_out.copy_(out32, non_blocking=True)

        e2e_ms = timed(e2e_step)
    head = per_op["bssrdf_directional_fp32"]
    rec = ncu_record("k_bssrdf_queries_ncu.csv")
    sm_mhz = clocks.summary().get("sm_mhz") or 1965.0
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    issue_peak = n_sm * 4 * sm_mhz * 1e6 / 1e9
    per_q = rec["totals"]["smsp__inst_executed.sum"] / float(rec["header"]["queries"]) if rec and "queries" in rec["header"] else None
    issue_achieved = per_q * n / (head["ms"] * 1e-3) / 1e9 if per_q else None
    issue_roofline = {
        "bound": "issue", "kernel": "k_bssrdf_directional (FP32)", "achieved": issue_achieved, "peak": issue_peak,
        "unit": "G warp instructions/s", "frac": issue_achieved / issue_peak if issue_achieved else None,
        "peak_source": "1 warp instruction / clock / SM sub-partition x 4 x %d SMs x median SM clock %.0f MHz" % (n_sm, sm_mhz),
        "warp_instructions_per_query": per_q,
        "traffic": ((rec["totals"]["dram__bytes_read.sum"] + rec["totals"]["dram__bytes_write.sum"]) / float(rec["header"]["queries"]) * n)
        if per_q else None,
        "traffic_unit": "DRAM bytes per launch (ncu record of the same launch size, profiles/k_bssrdf_queries_ncu.csv)",
        "hbm": {"achieved": head["hbm_gb_s"], "peak": peak, "unit": "GB/s", "frac": head["hbm_gb_s"] / peak, "peak_source": peak_kind,
                "algorithmic_bytes_per_query": 72}}
    line = {
        "metric": "M queries/s (per-query BSSRDF and microfacet-walk entries on 1 B200)", "value": head["m_queries_per_s"],
        "unit": "M queries/s", "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": head["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": QUERIES % n, "headline": "the directional dipole in FP32 (the per-pair term of the subsurface gathers)",
                   "l2": "inputs + outputs of %.0f MB per directional launch, larger than L2" % (72 * n / 1e6)},
        "per_op": per_op,
        "e2e": {"value": n / (e2e_ms * 1e-3) / 1e6, "unit": "M queries/s", "h2d_bytes_per_step": 60 * n, "d2h_bytes_per_step": 12 * n,
                "what": "the directional dipole from pinned host rows, values copied back, every step"},
        "roofline": issue_roofline,
        "gpu_launches": launches[0],
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle_ctypes as oc

        threads = os.cpu_count() or 1
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < 3.0:  # whole passes over the batch's rows for about three seconds
            oc.bssrdf_queries(params, 1, geo, which="ref", threads=threads)
            done += n
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": done / dt / 1e6, "unit": "M queries/s", "cores": threads, "kind": "reference",
                                "sample": "%d directional-dipole queries (passes over the %d-query batch), the reference's "
                                          "dipoles/directional_dipole.h compiled for the host, %d threads, %.1f s" % (done, n, threads, dt)}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference_queries(args):
    """Reference arm of the queries workload: the reference's directional dipole (dipoles/
    directional_dipole.h) compiled for the host, all host cores, on the same query rows (each step a
    pass over a bounded slice of them)."""
    from oracle import oracle_ctypes as oc

    params, dist, geo, wi, wo, alpha = query_inputs(args.queries)
    threads = os.cpu_count() or 1
    m = min(args.queries, 1 << 21)
    for _ in range(max(0, min(args.warmup, 1))):
        oc.bssrdf_queries(params, 1, geo[:, :m], which="ref", threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oc.bssrdf_queries(params, 1, geo[:, :m], which="ref", threads=threads)
    dt = time.perf_counter() - t0
    value = m * args.steps / dt / 1e6
    sample = "%d directional-dipole queries per step, the reference's dipoles/directional_dipole.h compiled for the host, %d threads" % (
        m, threads)
    print(json.dumps({
        "impl": "reference", "metric": "M queries/s (per-query BSSRDF and microfacet-walk entries on 1 B200)", "value": value,
        "unit": "M queries/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": QUERIES % args.queries, "sample_per_step": sample},
        "cpu_baseline": {"value": value, "unit": "M queries/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "M queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def run_reference(args, world, rank):
    from open_rendering_framework_b200 import scenes

    if rank != 0:
        return
    if args.workload == "batched":
        return run_reference_batched(args)
    if args.workload == "bsdf":
        return run_reference_bsdf(args)
    if args.workload == "ingest":
        return run_reference_ingest(args)
    if args.workload == "queries":
        return run_reference_queries(args)
    if args.workload == "build":
        print(json.dumps({"impl": "reference", "unavailable": "the reference builds its BVH inside OptiX (Trbvh / Sbvh, "
                                                              "OptixSceneLoader.cpp:136), which has no CPU build and is not on this box"}), flush=True)
        return
    data, _, desc = workload(args)
    from oracle import oracle_ctypes as oc

    threads = os.cpu_count() or 1
    O = oc.OracleScene(data)
    W, H = data.camera.width, data.camera.height
    band = 16  # rows per step: each step is a bounded sample (16 rows x 8 spp; 1 spp for the subsurface scene)
    frames = 8 if args.workload == "single_scene" else 1
    p0 = W * (H // 2 - band // 2)
    for _ in range(max(0, args.warmup)):
        O.render(0, 1, p_begin=p0, p_end=p0 + W * 2, threads=threads)
    t0 = time.perf_counter()
    for k in range(args.steps):
        O.render(k * frames, frames, p_begin=p0, p_end=p0 + W * band, threads=threads)
    dt = time.perf_counter() - t0
    samples = args.steps * W * band * frames
    value = samples / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(1, args.steps), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "sample_per_step": "%d rows x %d px x %d spp" % (band, W, frames)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "%d rows x %d px x %d spp per step; the reference's OptiX tracer has no CPU build, so its "
                                   "CPU restatement (path_tracer.cu + shaders, the reference's math) runs on all host cores" % (
                                       band, W, frames)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    O.close()


BATCHED = ("batched render of %d seeded procedural scenes in one pass (CUDA graph): meshes log-uniform over 1e3-5e5 triangles "
           "(jittered icospheres or value-noise heightfields) on a diffuse floor, materials uniform over diffuse / GGX conductor / "
           "Beckmann conductor / Beckmann rough dielectric / dipole (500 probes per frame, the reference's default), resolutions from {128,256,512,1024}^2, "
           "spp log-uniform over 4-256, 128x64 procedural sky as background and light, max depth 8, Russian roulette from depth 3")


def rel_mse(img, ref):
    """Mean over pixels and channels of (I - I_ref)^2 / (I_ref^2 + 1e-2)."""
    img = np.asarray(img, np.float64)[..., :3]
    ref = np.asarray(ref, np.float64)[..., :3]
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def reference_image(R, spp, factor=16):
    """The same scene at factor x spp from frames [spp, spp + factor*spp), independent of the frames
    0..spp-1 of the measured image: rendered into a cleared accumulation buffer starting at frame spp,
    whose running mean then holds sum / (spp + factor*spp), rescaled to the mean of those frames."""
    from open_rendering_framework_b200 import _native as nat

    R.apply_camera()
    n = factor * spp
    nat.call("pt_render_frames", R.ctx, spp, n)
    R.frame = spp + n
    img = R.readback().astype(np.float64)
    return img * ((spp + n) / n)


def batched_roofline(st, clocks, local):
    """Roofline of the batched pass's dominant kernel from a profiled pass's render stats: the dipole
    gather against the INT32 issue bound (thread instructions per pair from the gather's ncu capture),
    or the extend kernel's HBM view (its algorithmic bytes per segment over its live time); the other
    kernel's figures ride along."""
    import torch

    sm_mhz = clocks.summary().get("sm_mhz") or 1965.0
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    peak, peak_kind = load_peaks()
    ext_s, gat_s = st.extend_ms * 1e-3, st.gather_ms * 1e-3
    hbm = st.segments * EXTEND_BYTES_PER_SEGMENT / ext_s / 1e9 if ext_s > 0 else None
    extend = {"bound": "hbm", "kernel": "k_extend_persistent (closest-hit traversal + material class record)",
              "achieved": hbm, "peak": peak, "unit": "GB/s", "frac": hbm / peak if hbm else None, "peak_source": peak_kind,
              "algorithmic_bytes_per_segment": EXTEND_BYTES_PER_SEGMENT, "traffic": None,
              "extend_share_of_pass": st.extend_ms / st.gpu_ms if st.gpu_ms else None,
              "segments_per_path": st.segments / max(1, st.path_samples)}
    alu_peak = n_sm * 64 * sm_mhz * 1e6 / GATHER_INSTR_PER_PAIR / 1e9
    pairs = st.dipole_pairs / gat_s / 1e9 if gat_s > 0 else None
    gather = {"bound": "alu", "kernel": "k_gather (dipole gathers: one MD5 draw per (gather, probe) pair)",
              "achieved": pairs, "peak": alu_peak, "unit": "Gpair/s", "frac": pairs / alu_peak if pairs else None,
              "peak_source": "INT32 pipe: 64 lanes/clk/SM x SMs x median SM clock / %d thread instructions per pair "
                             "(ncu capture of the subsurface configuration's gather)" % GATHER_INSTR_PER_PAIR,
              "traffic": None, "gather_share_of_pass": st.gather_ms / st.gpu_ms if st.gpu_ms else None,
              "pairs_per_gather": st.dipole_pairs / max(1, st.dipole_gathers)}
    if st.gather_ms > st.extend_ms:
        gather["extend"] = extend
        out = gather
    else:
        extend["gather"] = gather
        out = extend
    out["timing"] = ("CUDA events around every extend and gather launch of one profiled batch pass "
                     "(no graph, in-order schedule); pass time %.1f ms" % st.gpu_ms)
    return out


def measure_batched(args, world, local, relmse=True):
    """The batched configuration (64 seeded scenes in one pass from a CUDA graph): device-timed
    throughput, the same frames scene after scene (plain), the reference's launch pattern, the
    end-to-end figure, and the images' relMSE against 16x-spp references."""
    import torch

    from open_rendering_framework_b200 import _native as nat
    from open_rendering_framework_b200 import scene as sc
    from open_rendering_framework_b200 import scenes

    torch.cuda.set_device(local)
    # each rank renders its own copy of the batch (replicas: per-rank work fixed, weak scaling)
    S = scenes.batch_scenes(args.scenes, seed=0)
    Rs = [sc.Renderer(d, device=local) for d, _, _ in S]
    spp = [p for _, p, _ in S]
    B = sc.Batch(Rs, spp, device=local)
    stream = torch.cuda.ExternalStream(B.stream())
    path_samples = sum(d.camera.width * d.camera.height * p for d, p, _ in S)
    tune = B.autotune(frames_per_trial=4)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    for _ in range(max(3, args.warmup)):
        B.render()
    torch.cuda.synchronize()
    barrier()
    L = nat.lib()
    launches0 = L.pt_kernel_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            B.render()
        e1.record(stream)
        torch.cuda.synchronize()
    launches = L.pt_kernel_launch_count() - launches0
    ms_max = max_over_ranks(e0.elapsed_time(e1), world, "cuda")
    value = replica_throughput(path_samples, world, args.steps, ms_max * 1e-3)
    # the plain path: the same frames, scene after scene, each by its own single-scene pass
    B.render_sequential()
    torch.cuda.synchronize()
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    B.render_sequential()
    p1.record(stream)
    torch.cuda.synchronize()
    plain = path_samples / (p0.elapsed_time(p1) * 1e-3) / 1e6
    # the reference's launch pattern: one pass per frame per scene (OptixScene::renderScene launches the
    # integrator once per frame, OptixScene.cpp:139-168), scene after scene; each context has its own
    # stream, so this one is timed on the host between device synchronisations
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    for R, f in zip(Rs, spp):
        for _ in range(f):
            R.renderScene()
    for R in Rs:
        R.sync()
    torch.cuda.synchronize()
    plain_per_frame = path_samples / (time.perf_counter() - w0) / 1e6
    B._sync_frames()
    # end to end: per step every scene's camera and materials set from the host (which also clears
    # every accumulation buffer), the batch render of frames 0..spp-1, and every image read back into
    # pinned host memory
    imgs = [torch.empty((d.camera.height, d.camera.width, 4), dtype=torch.float32, pin_memory=True) for d, _, _ in S]
    h2d = sum(ctypes.sizeof(m.params()) for d, _, _ in S for m in d.materials) + 12 * 4 * len(S)
    d2h = sum(im.numel() * 4 for im in imgs)

    def e2e_step():
        for R in Rs:
            R.apply_camera()
            for m in R.data.materials:
                R.update_material(m)
        B.render()
        for R, im in zip(Rs, imgs):
            nat.call("pt_readback", R.ctx, im.data_ptr())

    e2e_step()
    torch.cuda.synchronize()
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    f1.record(stream)
    torch.cuda.synchronize()
    t_max = max_over_ranks(f0.elapsed_time(f1), world, "cuda")
    e2e_value = replica_throughput(path_samples, world, args.steps, t_max * 1e-3)
    st = B.stats()
    # ---- roofline of the batch's dominant kernel, from one more pass without the graph and with CUDA
    # events around every extend and gather launch (in-order schedule, as the single-scene profile)
    B.set_option("use_graph", 0)
    B.set_option("profile", 1)
    B.render()
    pst = B.stats()
    B.set_option("profile", 0)
    B.set_option("use_graph", 1)
    roofline = batched_roofline(pst, clocks, local)
    kinds = {}
    for _, p, info in S:
        kinds[info["material"]] = kinds.get(info["material"], 0) + 1
    out = {
        "value": value, "unit": UNIT, "ms_per_step": ms_max / args.steps, "steps": args.steps, "warmup": max(3, args.warmup),
        "workload": BATCHED % len(S), "path_samples_per_step": path_samples, "scenes": len(S), "materials": kinds,
        "timing": "CUDA events on the batch stream around the graph launches",
        "plain_same_frames": {"value": plain, "unit": UNIT, "what": "the same frames rendered scene after scene by single-scene passes"},
        "batched_over_plain_same_frames": value / plain,
        "plain_per_frame": {"value": plain_per_frame, "unit": UNIT,
                            "what": "the same frames rendered one pass per frame per scene, scene after scene (the "
                                    "reference's launch pattern), host-timed between device synchronisations"},
        "batched_over_plain_per_frame": value / plain_per_frame,
        "autotune": {"extend_mode": tune.extend_mode, "refill": tune.refill, "max_paths_in_flight": tune.max_paths_in_flight,
                     "bin_items": tune.bin_items, "trials": tune.trials, "best_calibration_mpaths_per_s": tune.best_mpaths_per_s},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": roofline,
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "stats": {"segments_per_path": st.segments / max(1, st.path_samples), "dipole_gathers": st.dipole_gathers,
                  "dipole_pairs": st.dipole_pairs},
        "l2": "inputs larger than L2: %.1f GB of path state per chunk" % (tune.max_paths_in_flight * 178 / 1e9),
    }
    if relmse:
        # relMSE of each scene's batched image (frames 0..spp-1, the e2e step's) against its 16x-spp
        # reference, frames [spp, 17 spp): one more batched pass over the same scenes (the scene contexts
        # hold no wavefront buffers of their own; the batch engine's are shared), each accumulation
        # cleared with its next frame set to spp (pt_set_accumulation), the running mean rescaled to the
        # mean of those frames.  The plain path renders bit-identical images (tests/test_batch_gpu.py),
        # so its relMSE on the same frames is the same number.
        t0 = time.perf_counter()
        imgs_np = [im.numpy().copy() for im in imgs]
        B2 = sc.Batch(Rs, [16 * p for p in spp], device=local)
        for R, p in zip(Rs, spp):
            zeros = np.zeros((R.data.camera.height, R.data.camera.width, 4), np.float32)
            nat.call("pt_set_accumulation", R.ctx, zeros.ctypes.data, p)
        B2.render()
        errs = []
        for R, im, p in zip(Rs, imgs_np, spp):
            ref = R.readback().astype(np.float64) * (17.0 / 16.0)
            errs.append(rel_mse(im, ref))
        B2.close()
        by_mat = {}
        for (_, p, info), e in zip(S, errs):
            by_mat.setdefault(info["material"], []).append(e)
        out["relmse_vs_16x_spp"] = {"median_over_scenes": float(np.median(errs)), "mean_over_scenes": float(np.mean(errs)),
                                    "max_over_scenes": float(np.max(errs)),
                                    "median_by_material": {k: float(np.median(v)) for k, v in sorted(by_mat.items())},
                                    "note": "Monte Carlo error of the low-spp frames: largest for glossy conductors and "
                                            "rough dielectrics at a few spp, which pick up the sun by BSDF sampling",
                                    "per_scene": [float(e) for e in errs], "reference": "frames [spp, 17 spp) of each scene",
                                    "plain_same_frames": "identical (bit-identical images)", "seconds": time.perf_counter() - t0}
    B.close()
    for R in Rs:
        R.close()
    return out


def run_batched(args, world, rank, local):
    m = measure_batched(args, world, local)
    line = {
        "metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": m["warmup"],
        "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": m["workload"], "path_samples_per_step": m["path_samples_per_step"], "scenes": m["scenes"],
                   "materials": m["materials"], "parallelism": "replicas (one independent batch per GPU)", "l2": m["l2"]},
        "e2e": m["e2e"], "gpu_launches": m["gpu_launches"], "clocks": m["clocks"],
        "roofline": m["roofline"],
    }
    for k in ("plain_same_frames", "batched_over_plain_same_frames", "plain_per_frame", "batched_over_plain_per_frame", "autotune", "stats",
              "relmse_vs_16x_spp"):
        if k in m:
            line[k] = m[k]
    if rank == 0:
        print(json.dumps(line), flush=True)


ADJOINT = ("inverse rendering 256x256, 64 spp, depth 6, RR from depth 3: 12-triangle box with a 256x256x3 albedo texture, "
           "5-subdivision GGX conductor icosphere with a 256x256 roughness texture, 5-subdivision standard-dipole icosphere "
           "(sigma_a, sigma_s' per RGB, 500 probes per frame), quad light; parameters seeded U[0.1,0.9]; L2 loss against a "
           "1024-spp target from other seeded parameters; forward + path-replay adjoint per step")


def adjoint_roofline(fst, ast, clocks, local):
    """Roofline of the forward + adjoint arm's dominant kernel from one profiled step (the forward
    pass's and the adjoint pass's render stats): a dipole gather against the INT32 issue bound, or the
    extend kernel's HBM view.  The bound uses the forward gather's thread instructions per pair (ncu);
    the adjoint gather adds the derivatives of its accepted pairs, so its fraction is a lower bound."""
    import torch

    sm_mhz = clocks.summary().get("sm_mhz") or 1965.0
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    peak, peak_kind = load_peaks()
    total = fst.gpu_ms + ast.gpu_ms
    parts = {"forward_extend": fst.extend_ms, "forward_gather": fst.gather_ms, "adjoint_extend": ast.extend_ms,
             "adjoint_gather": ast.gather_ms}
    shares = {k: (v / total if total else None) for k, v in parts.items()}
    top = max(parts, key=parts.get)
    if top.endswith("gather"):
        s = fst if top.startswith("forward") else ast
        alu_peak = n_sm * 64 * sm_mhz * 1e6 / GATHER_INSTR_PER_PAIR / 1e9
        achieved = s.dipole_pairs / (s.gather_ms * 1e-3) / 1e9 if s.gather_ms else None
        kernel = "k_gather (forward dipole gathers)" if top.startswith("forward") else \
            "k_gather_adjoint (the adjoint pass's dipole gathers: the MD5 chain replayed, derivatives of accepted pairs)"
        out = {"bound": "alu", "kernel": kernel, "achieved": achieved, "peak": alu_peak, "unit": "Gpair/s",
               "frac": achieved / alu_peak if achieved else None,
               "peak_source": "INT32 pipe: 64 lanes/clk/SM x SMs x median SM clock / %d thread instructions per pair of the "
                              "forward gather (ncu)%s" % (GATHER_INSTR_PER_PAIR, "" if top.startswith("forward") else
                                                          "; the adjoint gather does more per pair, so frac is a lower bound"),
               "traffic": None, "pairs_per_gather": s.dipole_pairs / max(1, s.dipole_gathers)}
    else:
        s = fst if top.startswith("forward") else ast
        hbm = s.segments * EXTEND_BYTES_PER_SEGMENT / (s.extend_ms * 1e-3) / 1e9 if s.extend_ms else None
        out = {"bound": "hbm", "kernel": "k_extend_persistent (%s pass)" % top.split("_")[0], "achieved": hbm, "peak": peak,
               "unit": "GB/s", "frac": hbm / peak if hbm else None, "peak_source": peak_kind,
               "algorithmic_bytes_per_segment": EXTEND_BYTES_PER_SEGMENT, "traffic": None}
    out["shares_of_forward_plus_adjoint"] = shares
    out["timing"] = ("CUDA events around every extend and gather launch of one profiled forward + adjoint step (in-order "
                     "schedule); forward %.2f ms, adjoint %.2f ms" % (fst.gpu_ms, ast.gpu_ms))
    return out


def measure_adjoint(args, local, relmse=True, spp=None, width=None):
    """The differentiable configuration: forward (differentiable) render + path-replay adjoint per
    step, device-timed per phase; the end-to-end figure through the torch.autograd.Function; the
    forward image's relMSE against a 16x-spp reference."""
    import torch

    from open_rendering_framework_b200 import diff
    from open_rendering_framework_b200 import scene as sc
    from open_rendering_framework_b200 import scenes

    torch.cuda.set_device(local)
    W = width or 256
    spp = spp or 64
    data, (dif, met, tr) = scenes.inverse_scene(W, W, subdiv=5, tex_res=256, seed=0)
    tdata, _ = scenes.inverse_scene(W, W, subdiv=5, tex_res=256, seed=1)
    T = sc.Renderer(tdata, device=local)
    T.render(1024)
    target = torch.from_numpy(T.readback()[..., :3].copy()).cuda()
    T.close()
    DS = diff.DiffScene(data, dif, met, tr, device=local)
    albedo = torch.from_numpy(dif.texture.copy()).cuda().requires_grad_()
    rough = torch.from_numpy(met.texture.copy()).cuda().requires_grad_()
    sigma = torch.tensor(list(tr.absorption) + list(tr.scattering), dtype=torch.float32, device="cuda").requires_grad_()
    path_samples = W * W * spp
    last = {}

    def step():
        for t in (albedo, rough, sigma):
            t.grad = None
        img = diff.render(DS, spp, albedo, rough, sigma)
        fst = DS.stats()
        loss = ((img - target) ** 2).sum()
        loss.backward()
        ast = DS.stats()
        last["img"] = img
        return float(loss.item()), fst, ast

    for _ in range(max(3, args.warmup)):
        step()
    fwd_ms, adj_ms, seg, gathers, launches = 0.0, 0.0, 0, 0, 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        e0.record()
        for _ in range(args.steps):
            loss, fst, ast = step()
            fwd_ms += fst.gpu_ms
            adj_ms += ast.gpu_ms
            seg += fst.segments
            gathers += fst.dipole_gathers
            launches += fst.kernel_launches + ast.kernel_launches
        e1.record()
        torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    dev_ms = fwd_ms + adj_ms
    g = [albedo.grad, rough.grad, sigma.grad]
    out = {
        "value": args.steps * path_samples / (dev_ms * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": dev_ms / args.steps, "steps": args.steps,
        "warmup": max(3, args.warmup), "workload": ADJOINT, "path_samples_per_step": path_samples,
        "parameters": int(sum(t.numel() for t in g)),
        "timing": "device time of the forward and adjoint launches (CUDA events on the scene stream)",
        "forward": {"value": args.steps * path_samples / (fwd_ms * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": fwd_ms / args.steps},
        "adjoint_ms_per_step": adj_ms / args.steps,
        "fwd_plus_adjoint_over_forward": dev_ms / fwd_ms,
        "target_fwd_plus_adjoint_le_3x_forward": bool(dev_ms / fwd_ms <= 3.0),
        "e2e": {"value": args.steps * path_samples / (e2e_ms * 1e-3) / 1e6, "unit": UNIT, "h2d_bytes_per_step": 6 * 4 + 64,
                "d2h_bytes_per_step": 4 + 24, "what": "torch.autograd.Function forward + loss + backward, host sigma update and loss read-back"},
        "loss": loss,
        "grad_norms": [float(t.norm().item()) for t in g],
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "stats": {"segments_per_path": seg / (args.steps * path_samples), "dipole_gathers_per_step": gathers / args.steps},
        "l2": "per-path forward state of %.2f GB re-read by the adjoint" % (path_samples * 16 * 8 / 1e9),
    }
    # ---- roofline of the arm's dominant kernel: one more step with CUDA events around every extend and
    # gather launch of its forward and adjoint passes
    from open_rendering_framework_b200 import _native as nat

    nat.call("pt_set_profiling", DS.R.ctx, 1)
    _, pf, pa = step()
    nat.call("pt_set_profiling", DS.R.ctx, 0)
    out["roofline"] = adjoint_roofline(pf, pa, clocks, local)
    if relmse:
        img = last["img"].detach().cpu().numpy()
        ref = reference_image(DS.R, spp)
        out["relmse_vs_16x_spp"] = {"forward_image": rel_mse(img, ref), "reference": "frames [64, 1088) of the same scene and parameters"}
    DS.close()
    return out


def run_adjoint(args, world, rank, local):
    m = measure_adjoint(args, local, spp=args.spp, width=args.width)
    line = {
        "metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": m["warmup"],
        "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": m["workload"], "path_samples_per_step": m["path_samples_per_step"], "parameters": m["parameters"],
                   "l2": m["l2"]},
        "e2e": m["e2e"], "roofline": m["roofline"], "gpu_launches": m["gpu_launches"], "clocks": m["clocks"],
    }
    for k in ("forward", "adjoint_ms_per_step", "fwd_plus_adjoint_over_forward", "target_fwd_plus_adjoint_le_3x_forward", "loss",
              "grad_norms", "stats", "relmse_vs_16x_spp"):
        line[k] = m[k]
    print(json.dumps(line), flush=True)


BUILD = ("BVH build: the subsurface configuration's 327,680-triangle jittered icosphere and the 64 meshes of the batched "
         "configuration (1e3-5e5 triangles each), host binned-SAH builder vs device LBVH builder (option bvh_builder); "
         "the single-scene render (512x512, 64 spp) traced over each builder's tree")


def run_build(args, world, rank, local):
    """Milliseconds per million triangles of the device LBVH builder (Morton codes, radix sort, Karras
    hierarchy, SAH leaves, 4-wide collapse, all on the device) against the host binned-SAH builder,
    and the single-scene render speed over each tree (the trees' quality)."""
    import torch

    from open_rendering_framework_b200 import scene as sc
    from open_rendering_framework_b200 import scenes

    torch.cuda.set_device(local)
    reps = max(3, args.steps)

    def build_times(data, builder):
        R = sc.Renderer(data, device=local, build_options={"bvh_builder": builder})
        for _ in range(max(1, args.warmup)):
            R.rebuild(bvh_builder=builder)
        ms, dev = [], []
        for _ in range(reps):
            R.rebuild(bvh_builder=builder)
            b = R.build_info()
            ms.append(b.build_ms)
            dev.append(b.device_ms)
        info = R.build_info().as_dict()
        R.close()
        return statistics.median(ms), statistics.median(dev), info

    with ClockSampler(local) as clocks:
        c3 = scenes.subsurface_scene(64, 64)  # the mesh is what is built; a small camera keeps set-up cheap
        c3_host = build_times(c3, 0)
        c3_dev = build_times(c3, 1)
        S = scenes.batch_scenes(args.scenes, seed=0, size_scale=1 / 16)
        tot_tris = sum(d.n_triangles for d, _, _ in S)
        c4 = {0: [0.0, 0.0], 1: [0.0, 0.0]}
        for d, _, _ in S:
            for b in (0, 1):
                ms, dev, _ = build_times(d, b)
                c4[b][0] += ms
                c4[b][1] += dev
        # the trees' quality: the single-scene render over each
        render = {}
        data = scenes.single_scene()
        for b in (0, 1):
            R = sc.Renderer(data, device=local, build_options={"bvh_builder": b})
            for _ in range(max(1, args.warmup)):
                R.render(64)
            stream = torch.cuda.ExternalStream(R.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            n = max(3, args.steps // 2)
            for _ in range(n):
                R.render(64)
            e1.record(stream)
            torch.cuda.synchronize()
            render[b] = {"value": n * 512 * 512 * 64 / (e0.elapsed_time(e1) * 1e-3) / 1e6, "unit": UNIT, "sah_cost": R.build_info().sah_cost,
                         "build": R.build_info().as_dict()}
            R.close()
    n3 = c3_dev[2]["n_triangles"]
    per_m = lambda ms, n: ms / (n / 1e6)
    line = {
        "metric": "ms per million triangles (BVH build, device LBVH)", "value": per_m(c3_dev[0], n3), "unit": "ms/Mtri", "n_gpus": 1,
        "steps": reps, "warmup": max(1, args.warmup), "ms_per_step": c3_dev[0], "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": BUILD, "triangles": n3, "batch_meshes": len(S), "batch_triangles": tot_tris},
        "subsurface_mesh": {"device": {"ms": c3_dev[0], "device_ms": c3_dev[1], "ms_per_mtri": per_m(c3_dev[0], n3), "tree": c3_dev[2]},
                            "host": {"ms": c3_host[0], "ms_per_mtri": per_m(c3_host[0], n3), "tree": c3_host[2]},
                            "host_over_device": c3_host[0] / c3_dev[0]},
        "batch_meshes": {"device": {"ms": c4[1][0], "device_ms": c4[1][1], "ms_per_mtri": per_m(c4[1][0], tot_tris)},
                         "host": {"ms": c4[0][0], "ms_per_mtri": per_m(c4[0][0], tot_tris)}, "host_over_device": c4[0][0] / c4[1][0]},
        "single_scene_render": {"host_tree": render[0], "device_tree": render[1], "device_over_host": render[1]["value"] / render[0]["value"]},
        "e2e": {"value": per_m(c3_dev[0], n3), "unit": "ms/Mtri", "h2d_bytes_per_step": 36 * n3, "d2h_bytes_per_step": 0,
                "what": "pt_build's BVH step through the C ABI from the host triangle list (upload included)"},
        "cpu_baseline": {"value": per_m(c3_host[0], n3), "unit": "ms/Mtri", "cores": os.cpu_count() or 1, "kind": "port",
                         "sample": "the library's host binned-SAH builder on the same mesh (the reference's OptiX builders cannot run here)"},
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch

    from open_rendering_framework_b200 import _native as nat
    from open_rendering_framework_b200 import scene as sc
    from open_rendering_framework_b200 import scenes

    torch.cuda.set_device(local)
    data, spp, desc = workload(args)
    R = sc.Renderer(data, device=local)
    stream = torch.cuda.ExternalStream(R.stream())
    width, height = data.camera.width, data.camera.height
    path_samples = width * height * spp

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    # ---- device-timed steps
    first_render = None
    for k in range(args.warmup):
        R.render(spp)
        if k == 0:
            s0 = R.stats()  # the first render's extend launches are what the committed ncu record captures
            first_render = {"segments": int(s0.segments), "extend_launches": int(s0.extend_launches), "frames": [0, spp]}
    R.sync()
    barrier()
    torch.cuda.synchronize()
    L = nat.lib()
    launches0 = L.pt_kernel_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            R.render(spp)
        e1.record(stream)
        torch.cuda.synchronize()
    launches = L.pt_kernel_launch_count() - launches0
    ms = e0.elapsed_time(e1)
    barrier()
    t_max = max_over_ranks(ms, world, "cuda")
    ms_max = t_max
    value = replica_throughput(path_samples, world, args.steps, ms_max * 1e-3)

    # ---- end-to-end through the public API with host buffers
    img_host = torch.empty((height, width, 4), dtype=torch.float32, pin_memory=True)
    mats = [m for m in data.materials]
    h2d = sum(ctypes.sizeof(m.params()) for m in mats)
    d2h = img_host.numel() * 4
    for _ in range(2):
        R.apply_camera()
        for m in mats:
            R.update_material(m)
        R.render(spp)
        nat.call("pt_readback", R.ctx, img_host.data_ptr())
    barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        R.apply_camera()           # camera variables (and a cleared accumulation buffer)
        for m in mats:             # material parameters, copied host -> device
            R.update_material(m)
        R.render(spp)
        nat.call("pt_readback", R.ctx, img_host.data_ptr())  # float4 image -> pinned host memory
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)
    t_max = max_over_ranks(e2e_ms, world, "cuda")
    e2e_value = replica_throughput(path_samples, world, args.steps, t_max * 1e-3)

    # ---- image error of this arm: the e2e step's image (frames 0..spp-1) against a 16x-spp reference
    relmse = None
    if args.workload == "single_scene" and not args.no_arms:
        img = img_host.numpy().copy()
        relmse = {"value": rel_mse(img, reference_image(R, spp)), "reference": "frames [%d, %d) of the same scene" % (spp, 17 * spp)}

    # ---- roofline of the dominant kernel (closest-hit extend), from a separately profiled render
    nat.call("pt_set_profiling", R.ctx, 1)
    R.render(spp)
    st = R.stats()
    nat.call("pt_set_profiling", R.ctx, 0)
    peak, peak_kind = load_peaks()
    ext_s = st.extend_ms * 1e-3
    launches_ext = max(1, st.extend_launches)
    # HBM view: algorithmic bytes of one launch / that launch's average duration == the totals' ratio
    hbm_achieved = st.segments * EXTEND_BYTES_PER_SEGMENT / ext_s / 1e9 if ext_s > 0 else None
    rec = extend_capture_record()
    hbm = {"achieved": hbm_achieved, "peak": peak, "unit": "GB/s", "frac": hbm_achieved / peak if hbm_achieved else None,
           "peak_source": peak_kind, "algorithmic_bytes_per_segment": EXTEND_BYTES_PER_SEGMENT,
           "traffic": rec["dram_bytes_per_segment"] * st.segments / launches_ext if rec else None,
           "traffic_unit": "DRAM bytes per launch (ncu record of the same kernel, scaled by the segments a launch traces)"}
    # issue view: warp instructions per segment (ncu record) x segments / extend time, against one warp
    # instruction per clock per SM sub-partition (4 per SM) at the sampled SM clock
    sm_mhz = clocks.summary().get("sm_mhz") or 1965.0
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    issue_peak = n_sm * 4 * sm_mhz * 1e6 / 1e9
    issue_achieved = rec["warp_inst_per_segment"] * st.segments / ext_s / 1e9 if (rec and ext_s > 0) else None
    roofline = {"bound": "issue", "kernel": "k_extend_persistent (closest-hit traversal + material class record)",
                "achieved": issue_achieved, "peak": issue_peak, "unit": "G warp instructions/s",
                "frac": issue_achieved / issue_peak if issue_achieved else None,
                "peak_source": "1 warp instruction / clock / SM sub-partition x 4 x %d SMs x median SM clock %.0f MHz" % (n_sm, sm_mhz),
                "warp_instructions_per_segment": rec["warp_inst_per_segment"] if rec else None,
                "threads_per_warp_instruction": rec["thread_inst_per_warp_inst"] if rec else None,
                "traffic": hbm["traffic"], "traffic_unit": hbm["traffic_unit"],
                "hbm": hbm,
                "extend_ms_per_launch": st.extend_ms / launches_ext,
                "extend_share_of_render": st.extend_ms / st.gpu_ms if st.gpu_ms else None,
                "segments_per_path": st.segments / st.path_samples, "shadow_rays_per_path": st.shadow_rays / st.path_samples,
                "giga_rays_per_s": (st.segments + st.shadow_rays) / (st.gpu_ms * 1e-3) / 1e9,
                "record": "profiles/k_extend_single_scene_ncu.csv" if rec else None}
    if args.workload == "subsurface":
        # integer-issue bound: 64 INT32 lanes per clock per SM at the sampled SM clock, divided by the
        # thread instructions one pair takes (ncu capture of k_gather)
        sm_mhz = clocks.summary().get("sm_mhz") or 1965.0
        alu_peak = torch.cuda.get_device_properties(local).multi_processor_count * 64 * sm_mhz * 1e6 / GATHER_INSTR_PER_PAIR / 1e9
        achieved_g = st.dipole_pairs / (st.gather_ms * 1e-3) / 1e9 if st.gather_ms else None
        roofline = {"bound": "alu", "kernel": "k_gather (dipole gathers: one MD5 draw per (gather, probe) pair)",
                    "achieved": achieved_g, "unit": "Gpair/s", "peak": alu_peak,
                    "peak_source": "INT32 pipe: 64 lanes/clk/SM x SMs x median SM clock / %d thread instructions per pair (ncu)" %
                                   GATHER_INSTR_PER_PAIR,
                    "frac": achieved_g / alu_peak if achieved_g else None, "traffic": None,
                    "gather_share_of_render": st.gather_ms / st.gpu_ms if st.gpu_ms else None,
                    "pairs_per_gather": st.dipole_pairs / max(1, st.dipole_gathers),
                    "gathers_per_path": st.dipole_gathers / st.path_samples,
                    "probe_bytes_per_pair": 16, "extend": roofline}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": desc, "path_samples_per_step": path_samples, "parallelism": "replicas (one independent render per GPU)",
                   "l2": "inputs larger than L2: per-path wavefront state of %.1f GB per step" % (path_samples * 176 / 1e9)},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": roofline,
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "stats": {"capped_walks": st.capped_walks, "clamped_indices": st.clamped_indices, "dipole_gathers": st.dipole_gathers,
                  "dipole_pairs": st.dipole_pairs, "first_render": first_render},
    }
    if relmse:
        line["relmse_vs_16x_spp"] = relmse
    R.close()
    if args.workload == "single_scene" and world == 1 and not args.no_arms:
        # the metric's other two arms on the same GPU: the 64-scene batch and forward + adjoint
        line["batched"] = measure_batched(args, world, local)
        line["fwd_adjoint"] = measure_adjoint(args, local)
        line["arms"] = ("value = plain single-scene arm; batched = the 64-scene batch in one CUDA-graph pass; fwd_adjoint = the "
                        "differentiable configuration (forward + path-replay adjoint); each carries its own e2e and its image relMSE "
                        "against a 16x-spp reference of the same scene")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(data)
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "batched":
            run_batched(args, world, rank, local)
        elif args.workload == "bsdf":
            run_bsdf(args, world, rank, local)
        elif args.workload == "ingest":
            if rank == 0:
                run_ingest(args, world, rank, local)
        elif args.workload == "adjoint":
            if rank == 0:
                run_adjoint(args, world, rank, local)
        elif args.workload == "build":
            if rank == 0:
                run_build(args, world, rank, local)
        elif args.workload == "queries":
            run_queries(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
